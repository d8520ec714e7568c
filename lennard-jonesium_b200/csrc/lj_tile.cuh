// lj_tile.cuh -- the mixed-precision pair kernel over shared-memory tiles of
// neighbour cells, and the list build that feeds it.
//
// Atoms are stored in list-cell order (z fastest), so the cells of one (x, y)
// column are contiguous in memory.  A tile is a run of `len` consecutive cells
// of one column, z0 .. z0 + len - 1; its atoms' neighbours all lie in the
// window of 9 columns x (len + 2) cells around it.  One block of the pair
// kernel owns one tile: it copies the FP32 cell-local coordinates of every
// window atom into shared memory once (coalesced loads of at most 18
// contiguous slot ranges), with the x and y offset of the window column
// already added, then each thread runs its home atoms' neighbour lists
// against shared memory instead of gathering from L1/L2.
//
// The list entries of this path are 16 bits: the atom's position in its
// tile's staging array (14 bits) and the z offset of its stencil cell
// (2 bits, dz + 1).  The entry order (stencil cell, then slot) and the
// candidate test are those of build_list_warp_kernel, so the pair set and the
// FP32 summation order are unchanged; the separation is
//     s_x = xl_i - (xl_j + dx a_x),  s_y likewise,  s_z = (xl_i - xl_j) - dz a_z
// with xl the cell-local coordinates of the FP32 path (lj_mixed.cuh).  A tile
// whose window holds more atoms than the shared-memory capacity (very dense
// or strongly clustered systems) is not staged: its block reads the same
// entries through the slot map from global memory instead.
#pragma once

#include "lj_mixed.cuh"

namespace ljb {

constexpr int kTileMaxRun = 8;                      // cells per tile, at most
constexpr int kTileMaxWin = 9 * (kTileMaxRun + 2);  // window cells per tile (90)
constexpr int kTileThreads = 128;
constexpr unsigned kTileIdxBits = 14;
constexpr unsigned kTileIdxMask = (1u << kTileIdxBits) - 1u;
constexpr int kTileMaxStaged = (int)kTileIdxMask;   // window atoms of a tile; index T is the ghost
constexpr int kTilePieces = 18;                     // <= 2 contiguous slot ranges per window column
constexpr int kTileMaxSmemAtoms = 13824;            // staging slots that fit 227 KB of shared memory

struct TileGeom {
    int nruns;    // tiles per (x, y) column
    int cap;      // window atoms that fit the shared-memory staging array
    float a[3];   // list-cell edges
};

struct TilePiece {
    int base, end;  // staging indices [base, end)
    int slot;       // slot of the staging index base
    float ox, oy;   // x and y offset of the window column
};

// Tile r of a column: cells [z0, z0 + len).
__host__ __device__ inline void tile_run(int r, int nz, int nruns, int& z0, int& len) {
    z0 = (int)(((long long)r * nz) / nruns);
    len = (int)(((long long)(r + 1) * nz) / nruns) - z0;
}

__device__ inline int tile_run_of(int cz, int nz, int nruns) {
    int r = (int)(((long long)cz * nruns) / nz);
    int z0, len;
    for (int it = 0; it < 4; ++it) {  // r is at most one or two tiles off
        tile_run(r, nz, nruns, z0, len);
        if (cz < z0) --r;
        else if (cz >= z0 + len) ++r;
        else break;
    }
    return r;
}

// Window cell w (0 .. len + 1, z = z0 - 1 + w) of window column k (0 .. 8,
// x offset k / 3 - 1, y offset k % 3 - 1), periodic.
__device__ inline int tile_window_cell(const Grid& g, int cx, int cy, int z0, int k, int w) {
    int x = cx + k / 3 - 1, y = cy + k % 3 - 1, z = z0 - 1 + w;
    x += x < 0 ? g.n[0] : (x >= g.n[0] ? -g.n[0] : 0);
    y += y < 0 ? g.n[1] : (y >= g.n[1] ? -g.n[1] : 0);
    z += z < 0 ? g.n[2] : (z >= g.n[2] ? -g.n[2] : 0);
    return g.flat(x, y, z);
}

// One warp: wb[e] = staging index of window cell e = k (len + 2) + w (the
// exclusive prefix of the window cells' atom counts); wb[9 (len + 2)] = total.
__device__ inline void tile_window_scan(const Grid& g, const int* __restrict__ start, int cx, int cy, int z0,
                                        int len, int* wb) {
    int lane = threadIdx.x & 31;
    int W = len + 2, nw = 9 * W;
    int c[3];
    int s = 0;
#pragma unroll
    for (int u = 0; u < 3; ++u) {
        int e = 3 * lane + u;
        c[u] = 0;
        if (e < nw) {
            int cell = tile_window_cell(g, cx, cy, z0, e / W, e % W);
            c[u] = start[cell + 1] - start[cell];
        }
        s += c[u];
    }
    int incl = s;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    int ex = incl - s;
#pragma unroll
    for (int u = 0; u < 3; ++u) {
        int e = 3 * lane + u;
        if (e < nw) wb[e] = ex;
        ex += c[u];
    }
    if (lane == 31) wb[nw] = incl;
    __syncwarp();
}

// ---------------------------------------------------------------------------
// List build for the tiled kernel: build_list_warp_kernel's candidate loop,
// writing 16-bit entries, 8 to a 16-byte group, groups stored [g][N].
// ---------------------------------------------------------------------------
__device__ __forceinline__ void append_entry16(unsigned short (&grp)[8], int& n, int cap, unsigned entry,
                                               uint4* __restrict__ nbr8, size_t N, int i) {
    if (n < cap) {
        grp[n & 7] = (unsigned short)entry;
        if ((n & 7) == 7) nbr8[(size_t)(n >> 3) * N + i] = *reinterpret_cast<const uint4*>(grp);
    }
    ++n;
}

static __global__ void __launch_bounds__(32 * kBuildWarps)
build_list_tile_kernel(int N, const float4* __restrict__ posf, Grid g, const int* __restrict__ start, float3 Lf,
                       float cut2, int cap, int nruns, uint4* __restrict__ nbr8, int* __restrict__ cnt, Scalars* sc,
                       Gate gate) {
    if (!gate.open()) return;
    __shared__ __align__(16) float cxs[kBuildWarps][3][32];
    __shared__ __align__(16) unsigned short grp_s[kBuildWarps][32][8];
    __shared__ int wb_s[kBuildWarps][kTileMaxWin + 1];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int c = blockIdx.x * kBuildWarps + warp;
    int ncell = g.ncell();
    int wmax = 0, tmax = 0;
    unsigned short(&grp)[8] = grp_s[warp][lane];
    if (c < ncell) {
        int ca = c / (g.n[1] * g.n[2]), cb = (c / g.n[2]) % g.n[1], cc = c % g.n[2];
        int r = tile_run_of(cc, g.n[2], nruns);
        int z0, len;
        tile_run(r, g.n[2], nruns, z0, len);
        int* wb = wb_s[warp];
        tile_window_scan(g, start, ca, cb, z0, len, wb);
        int W = len + 2, T = wb[9 * W], h = cc - z0;
        tmax = T;
        int hs = start[c], he = start[c + 1];
        for (int h0 = hs; h0 < he; h0 += 32) {
            int i = h0 + lane;
            bool own = i < he;
            float4 xi = own ? posf[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            int n = 0;
            for (int a = -1; a <= 1; ++a) {
                int na = ca + a, ia = na < 0 ? -1 : (na >= g.n[0] ? 1 : 0);
                na -= ia * g.n[0];
                for (int b = -1; b <= 1; ++b) {
                    int nb = cb + b, ib = nb < 0 ? -1 : (nb >= g.n[1] ? 1 : 0);
                    nb -= ib * g.n[1];
                    int k = (a + 1) * 3 + (b + 1);
                    for (int d = -1; d <= 1; ++d) {
                        int nc = cc + d, ic = nc < 0 ? -1 : (nc >= g.n[2] ? 1 : 0);
                        nc -= ic * g.n[2];
                        int cell = g.flat(na, nb, nc);
                        float2 sx = make_float2(xi.x - ia * Lf.x, xi.x - ia * Lf.x);
                        float2 sy = make_float2(xi.y - ib * Lf.y, xi.y - ib * Lf.y);
                        float2 sz = make_float2(xi.z - ic * Lf.z, xi.z - ic * Lf.z);
                        int js = start[cell], je = start[cell + 1];
                        // staging index of slot j: wbase + j; dz code in the top 2 bits
                        unsigned wbase = (unsigned)(wb[k * W + h + d + 1] - js);
                        unsigned code = (unsigned)(d + 1) << kTileIdxBits;
                        for (int j0 = js; j0 < je; j0 += 32) {
                            int cntj = min(32, je - j0);
                            __syncwarp();
                            float4 q = lane < cntj ? posf[j0 + lane] : make_float4(1e18f, 1e18f, 1e18f, 0.f);
                            cxs[warp][0][lane] = -q.x;
                            cxs[warp][1][lane] = -q.y;
                            cxs[warp][2][lane] = -q.z;
                            __syncwarp();
                            unsigned mask = 0;
                            for (int t = 0; t < cntj; t += 2) {
                                float2 qx = *reinterpret_cast<const float2*>(&cxs[warp][0][t]);
                                float2 qy = *reinterpret_cast<const float2*>(&cxs[warp][1][t]);
                                float2 qz = *reinterpret_cast<const float2*>(&cxs[warp][2][t]);
                                float2 dx = __fadd2_rn(sx, qx), dy = __fadd2_rn(sy, qy), dz = __fadd2_rn(sz, qz);
                                float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
                                mask |= (r2.x < cut2 ? 1u : 0u) << t;
                                mask |= (r2.y < cut2 ? 2u : 0u) << t;
                            }
                            if (cntj < 32) mask &= (1u << cntj) - 1u;
                            unsigned self = (unsigned)(i - j0);
                            if (self < 32u) mask &= ~(1u << self);
                            if (!own) mask = 0;
                            while (mask) {
                                int t = __ffs(mask) - 1;
                                mask &= mask - 1;
                                append_entry16(grp, n, cap, ((wbase + (unsigned)(j0 + t)) & kTileIdxMask) | code,
                                               nbr8, N, i);
                            }
                        }
                    }
                }
            }
            if (own) {
                int m = n < cap ? n : cap;
                cnt[i] = m;
                if (m & 7) {  // pad the last group with the tile's ghost (index T, no z offset)
                    unsigned ghost = ((unsigned)T & kTileIdxMask) | (1u << kTileIdxBits);
                    for (int q = m & 7; q < 8; ++q) grp[q] = (unsigned short)ghost;
                    nbr8[(size_t)(m >> 3) * N + i] = *reinterpret_cast<const uint4*>(grp);
                }
                wmax = max(wmax, n);
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        wmax = max(wmax, __shfl_down_sync(0xffffffffu, wmax, off));
        tmax = max(tmax, __shfl_down_sync(0xffffffffu, tmax, off));
    }
    if (lane == 0 && c < ncell) {
        atomicMax(&sc->max_count, wmax);
        atomicMax(&sc->max_staged, tmax);
        // more than 14 bits of staging index: the entries cannot address the window
        if (wmax > cap || tmax > kTileMaxStaged) atomicExch(&sc->overflow, 1);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd((unsigned long long*)&sc->builds, 1ull);
}

// ---------------------------------------------------------------------------
// The tiled pair kernel.
// ---------------------------------------------------------------------------

// 16-byte asynchronous copy global -> shared (cp.async, L2 only), and the wait
// for this thread's outstanding copies.
__device__ __forceinline__ void cp_async16(float4* smem, const float4* gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Window atom `idx` straight from global memory (tiles whose window exceeds
// the staging array).
__device__ __forceinline__ float4 tile_fetch_global(const float4* __restrict__ posl, const TilePiece* pieces,
                                                    unsigned idx, int T) {
    if ((int)idx >= T) return make_float4(1e18f, 1e18f, 1e18f, 0.f);
    int p = 0;
    while (p < kTilePieces - 1 && (int)idx >= pieces[p].end) ++p;
    TilePiece pc = pieces[p];
    float4 q = posl[pc.slot + ((int)idx - pc.base)];
    return make_float4(q.x + pc.ox, q.y + pc.oy, q.z, 0.f);
}

template <bool STAGED>
__device__ __forceinline__ void tile_group(const uint4 grp, const float4 xi, const float4* __restrict__ stage,
                                           const float4* __restrict__ posl, const TilePiece* pieces, int T,
                                           const MixedParams& mp, float az, float& cx, float& cy, float& cz,
                                           float& cv, float& cw) {
    const unsigned w[4] = {grp.x, grp.y, grp.z, grp.w};
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
        unsigned e[4] = {w[2 * hh] & 0xffffu, w[2 * hh] >> 16, w[2 * hh + 1] & 0xffffu, w[2 * hh + 1] >> 16};
        float4 q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            q[u] = STAGED ? stage[min(e[u] & kTileIdxMask, (unsigned)T)]
                          : tile_fetch_global(posl, pieces, e[u] & kTileIdxMask, T);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            // dz + 1 in {0, 1, 2} -> exactly -1, 0, 1 (8388608 + k is exact in FP32)
            float t = __int_as_float(0x4b000000 | (e[u] >> kTileIdxBits)) - 8388609.0f;
            float dx = xi.x - q[u].x;
            float dy = xi.y - q[u].y;
            float dz = fmaf(-t, az, xi.z - q[u].z);
            float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            bool hit = r2 < mp.rc2;
            float ir2 = rcp_approx(r2);
            float ir6 = ir2 * ir2 * ir2;
            float x = r2 * mp.inv_rc2;
            float V = fmaf(4.f * ir6, ir6 - 1.f, fmaf(mp.beta, x - 1.f, mp.alpha));
            float W = fmaf(24.f * ir6, fmaf(2.f, ir6, -1.f), -2.f * mp.beta * x);
            float f = hit ? W * ir2 : 0.f;
            cx = fmaf(f, dx, cx);
            cy = fmaf(f, dy, cy);
            cz = fmaf(f, dz, cz);
            cv += hit ? V : 0.f;
            cw += hit ? W : 0.f;
        }
    }
}

template <bool KICK, bool STAGED>
__device__ __forceinline__ void tile_home_atoms(int N, int hs, int he, const float4* __restrict__ posl, Soa s,
                                                const uint4* __restrict__ nbr8, const int* __restrict__ cnt,
                                                const float4* __restrict__ stage, const TilePiece* pieces, int T,
                                                const PairParams& pp, const MixedParams& mp, float az,
                                                double (&acc)[4]) {
    for (int i = hs + (int)threadIdx.x; i < he; i += kTileThreads) {
        const float4 xi = posl[i];
        double fx = 0, fy = 0, fz = 0, pe = 0, w = 0;
        int ng = (cnt[i] + 7) >> 3;
        uint4 cur = ng > 0 ? __ldcs(&nbr8[i]) : make_uint4(0, 0, 0, 0);
        for (int gi = 0; gi < ng; ++gi) {
            uint4 nxt = gi + 1 < ng ? __ldcs(&nbr8[(size_t)(gi + 1) * N + i]) : cur;
            // one group = 8 neighbours summed in FP32, then added in FP64
            float cx = 0.f, cy = 0.f, cz = 0.f, cv = 0.f, cw = 0.f;
            tile_group<STAGED>(cur, xi, stage, posl, pieces, T, mp, az, cx, cy, cz, cv, cw);
            fx += (double)cx;
            fy += (double)cy;
            fz += (double)cz;
            pe += (double)cv;
            w += (double)cw;
            cur = nxt;
        }
        s.at(FX, i) = fx;
        s.at(FY, i) = fy;
        s.at(FZ, i) = fz;
        acc[1] += pe;
        acc[2] += w;
        if (KICK) {
            double f3[3] = {fx, fy, fz};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double v = kick(s.at(VX + k, i), f3[k], pp.dt);
                s.at(VX + k, i) = v;
                acc[0] = fma(v, v, acc[0]);
                double d = s.at(DX + k, i);
                acc[3] = fma(d, d, acc[3]);
            }
        }
    }
}

// One block per tile.  Dynamic shared memory: (tg.cap + 1) float4 staging
// slots (the last one for the ghost).  Partial sums per block as in the
// other pair kernels: {sum v^2, 2 PE, 2 W, sum d^2}.
template <bool KICK>
static __global__ void __launch_bounds__(kTileThreads, 4)
force_mixed_tile_kernel(int N, const float4* __restrict__ posl, Soa s, const uint4* __restrict__ nbr8,
                        const int* __restrict__ cnt, const int* __restrict__ start, Grid g, TileGeom tg,
                        PairParams pp, MixedParams mp, double* __restrict__ partials) {
    extern __shared__ float4 stage[];
    __shared__ int wb[kTileMaxWin + 1];
    __shared__ TilePiece pieces[kTilePieces];
    int r = blockIdx.x % tg.nruns, col = blockIdx.x / tg.nruns;
    int cx = col / g.n[1], cy = col % g.n[1];
    int z0, len;
    tile_run(r, g.n[2], tg.nruns, z0, len);
    int W = len + 2;
    if (threadIdx.x < 32) tile_window_scan(g, start, cx, cy, z0, len, wb);
    __syncthreads();
    int T = wb[9 * W];
    if (threadIdx.x < kTilePieces) {
        // window column k in two pieces split where z wraps (the first or the
        // last window cell); a column that does not wrap has an empty second piece
        int k = threadIdx.x >> 1, part = threadIdx.x & 1;
        int ws = z0 == 0 ? 1 : (z0 + len == g.n[2] ? len + 1 : W);
        int wlo = part ? ws : 0, whi = part ? W : ws;
        TilePiece p;
        p.base = wb[k * W + wlo];
        p.end = wb[k * W + whi];
        p.slot = wlo < whi ? start[tile_window_cell(g, cx, cy, z0, k, wlo)] : 0;
        p.ox = (float)(k / 3 - 1) * tg.a[0];
        p.oy = (float)(k % 3 - 1) * tg.a[1];
        pieces[threadIdx.x] = p;
    }
    __syncthreads();
    bool staged = T <= tg.cap;
    if (staged) {
        // all of this thread's window atoms in flight at once (asynchronous
        // 16-byte global -> shared copies), then the column offsets in place
        int p = 0;
        for (int idx = threadIdx.x; idx < T; idx += kTileThreads) {
            while (p < kTilePieces - 1 && idx >= pieces[p].end) ++p;
            cp_async16(&stage[idx], &posl[pieces[p].slot + (idx - pieces[p].base)]);
        }
        cp_async_wait_all();
        p = 0;
        for (int idx = threadIdx.x; idx < T; idx += kTileThreads) {
            while (p < kTilePieces - 1 && idx >= pieces[p].end) ++p;
            float4 q = stage[idx];
            stage[idx] = make_float4(q.x + pieces[p].ox, q.y + pieces[p].oy, q.z, 0.f);
        }
        if (threadIdx.x == 0) stage[T] = make_float4(1e18f, 1e18f, 1e18f, 0.f);
    }
    __syncthreads();
    int hs = start[g.flat(cx, cy, z0)], he = start[g.flat(cx, cy, z0 + len - 1) + 1];
    double acc[4] = {0, 0, 0, 0};
    if (staged)
        tile_home_atoms<KICK, true>(N, hs, he, posl, s, nbr8, cnt, stage, pieces, T, pp, mp, tg.a[2], acc);
    else
        tile_home_atoms<KICK, false>(N, hs, he, posl, s, nbr8, cnt, stage, pieces, T, pp, mp, tg.a[2], acc);
    block_sum<4, kTileThreads>(acc);
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; ++q) partials[(size_t)blockIdx.x * 4 + q] = acc[q];
}

}  // namespace ljb
