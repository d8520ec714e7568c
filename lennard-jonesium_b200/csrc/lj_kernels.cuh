// lj_kernels.cuh -- kernels of the single-system engine (FP64 drop-in path and
// the shared binning / neighbour-list machinery).
//
// Device layout (HBM), all in cell-sorted slot order and re-sorted at every
// neighbour-list build:
//   pos   double4[N]       x, y, z, 0 -- gathered by neighbours, one 32-byte sector each
//   soa   double[9][N]     vx vy vz | dx dy dz (displacement) | fx fy fz, coalesced per atom
//   ids   int[N]           slot -> atom id (the reference's column index)
//   bd    double[3][N]     displacement at the last list build (skin criterion)
//   nbr   uint32[cap][N]   neighbour list, transposed so entry k of all atoms is contiguous;
//                          slot in the low 27 bits, a 5-bit code above it
//   cnt   int[N]           neighbour count
#pragma once

#include "lj_common.cuh"

namespace ljb {

enum SoaField { VX = 0, VY, VZ, DX, DY, DZ, FX, FY, FZ, SOA_FIELDS };

struct Soa {
    double* p;
    int N;
    __device__ __forceinline__ double& at(int f, int i) const { return p[(size_t)f * N + i]; }
};

// Rebuild gate: evaluated identically by every kernel of the rebuild chain.
struct Gate {
    const Scalars* sc;
    double thresh2;  // rebuild when max |d - d_build|^2 exceeds this
    int always;      // small-box / zero-skin mode: rebuild every step
    __device__ __forceinline__ bool open() const {
        if (always || sc->need_rebuild) return true;
        return __longlong_as_double((long long)sc->max_disp2) > thresh2;
    }
};

// ---------------------------------------------------------------------------
// Integration: integrator.cpp:62-88, first half (kick, drift, displacement, wrap)
// ---------------------------------------------------------------------------
template <bool PERIODIC, bool TRACK, bool LOCAL>
static __global__ void __launch_bounds__(kThreads)
kick_drift_kernel(int N, const double4* pos, double4* pos_out, Soa s, const double* __restrict__ bd,
                  const double* __restrict__ bx, float4* __restrict__ posl, PairParams pp, Scalars* sc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    if (i < N) {
        double4 x = pos[i];
        double xs[3] = {x.x, x.y, x.z};
        float l[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double v = kick(s.at(VX + k, i), s.at(FX + k, i), pp.dt);
            double inc = __dmul_rn(v, pp.dt);
            double xn = __dadd_rn(xs[k], inc);
            double dn = __dadd_rn(s.at(DX + k, i), inc);
            if (PERIODIC) xn = wrap(xn, pp.L[k]);
            s.at(VX + k, i) = v;
            s.at(DX + k, i) = dn;
            xs[k] = xn;
            if (TRACK || LOCAL) {
                double e = dn - bd[(size_t)k * N + i];
                m = fma(e, e, m);
                // mixed path: cell-local FP32 coordinate xl = bx + (d - d_build)
                if (LOCAL) l[k] = (float)(bx[(size_t)k * N + i] + e);
            }
        }
        pos_out[i] = make_double4(xs[0], xs[1], xs[2], 0.0);
        if (LOCAL) posl[i] = make_float4(l[0], l[1], l[2], 0.f);
    }
    if (TRACK) {
        m = warp_max(m);
        if ((threadIdx.x & 31) == 0 && m > 0.0)
            atomicMax(&sc->max_disp2, (unsigned long long)__double_as_longlong(m));
    }
}

// Second half kick without a force calculation (LJ_FORCE_NONE), with the
// measurement partial sums.
static __global__ void __launch_bounds__(kThreads)
kick_measure_kernel(int N, Soa s, double dt, int do_kick, double* __restrict__ partials) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0, 0, 0, 0};
    if (i < N) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double v = s.at(VX + k, i);
            if (do_kick) {
                v = kick(v, s.at(FX + k, i), dt);
                s.at(VX + k, i) = v;
            }
            acc[0] = fma(v, v, acc[0]);
            double d = s.at(DX + k, i);
            acc[3] = fma(d, d, acc[3]);
        }
    }
    block_sum<4, kThreads>(acc);
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; ++q) partials[(size_t)blockIdx.x * 4 + q] = acc[q];
}

// ---------------------------------------------------------------------------
// Cell binning (counting sort): particle_pair_filter.cpp:141-154
// ---------------------------------------------------------------------------
template <bool GATED>
static __global__ void __launch_bounds__(kThreads)
bin_count_kernel(int N, const double4* __restrict__ pos, Grid g, int* __restrict__ cell_of,
                 int* __restrict__ rank, int* __restrict__ count, Gate gate) {
    if (GATED && !gate.open()) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double4 x = pos[i];
    int c = g.flat(cell_coord(x.x, g.ratio[0], g.n[0]), cell_coord(x.y, g.ratio[1], g.n[1]),
                   cell_coord(x.z, g.ratio[2], g.n[2]));
    cell_of[i] = c;
    rank[i] = atomicAdd(&count[c], 1);
}

// Exclusive scan of count[0..n) into start[0..n]: tile sums, scan of tile sums, apply.
template <bool GATED>
static __global__ void __launch_bounds__(1024)
scan_reduce_kernel(const int* __restrict__ count, int n, int* __restrict__ tile_sums, Gate gate) {
    if (GATED && !gate.open()) return;
    int base = blockIdx.x * kScanTile + threadIdx.x * 4;
    int s = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) s += base + q < n ? count[base + q] : 0;
    __shared__ int tot;
    block_exclusive_scan<1024>(s, &tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

template <bool GATED>
static __global__ void __launch_bounds__(1024)
scan_tiles_kernel(int* __restrict__ tile_sums, int ntiles, Gate gate) {
    if (GATED && !gate.open()) return;
    int x = threadIdx.x < ntiles ? tile_sums[threadIdx.x] : 0;
    __shared__ int tot;
    int ex = block_exclusive_scan<1024>(x, &tot);
    if (threadIdx.x < ntiles) tile_sums[threadIdx.x] = ex;
}

template <bool GATED>
static __global__ void __launch_bounds__(1024)
scan_apply_kernel(int* __restrict__ count, int n, const int* __restrict__ tile_sums,
                  int* __restrict__ start, Gate gate) {
    if (GATED && !gate.open()) return;
    int base = blockIdx.x * kScanTile + threadIdx.x * 4;
    int c[4];
    int s = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        c[q] = base + q < n ? count[base + q] : 0;
        s += c[q];
    }
    __shared__ int tot;
    int ex = block_exclusive_scan<1024>(s, &tot) + tile_sums[blockIdx.x];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (base + q < n) {
            start[base + q] = ex;
            count[base + q] = 0;  // ready for the next binning
        }
        ex += c[q];
    }
    if (base < n && base + 4 >= n) start[n] = ex;
}

template <bool GATED>
static __global__ void __launch_bounds__(kThreads)
scatter_kernel(int N, const int* __restrict__ cell_of, const int* __restrict__ rank,
               const int* __restrict__ start, int* __restrict__ order, Gate gate) {
    if (GATED && !gate.open()) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    order[start[cell_of[i]] + rank[i]] = i;
}

// Order each cell's members by their previous slot.  Slots come from the last
// sort, so the order is a fixed function of the trajectory and every run is
// bit-reproducible without reading atom ids.  (The reference's own cell
// contents, ascending atom id, are produced by lj_gpu_debug_cells.)
// One warp per cell: cells of up to 32 atoms are sorted in registers by a
// bitonic network over warp shuffles; larger cells (rare) by one lane.
constexpr int kSortWarps = 4;

template <bool GATED>
static __global__ void __launch_bounds__(32 * kSortWarps)
cell_sort_kernel(int ncell, const int* __restrict__ start, int* __restrict__ order, Gate gate) {
    if (GATED && !gate.open()) return;
    int lane = threadIdx.x & 31;
    int c = blockIdx.x * kSortWarps + (threadIdx.x >> 5);
    if (c >= ncell) return;
    int b = start[c], e = start[c + 1], n = e - b;
    if (n <= 1) return;
    if (n <= 32) {
        int v = lane < n ? order[b + lane] : 0x7fffffff;
#pragma unroll
        for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                int o = __shfl_xor_sync(0xffffffffu, v, j);
                bool up = (lane & k) == 0, lower = (lane & j) == 0;
                v = (lower == up) ? min(v, o) : max(v, o);
            }
        if (lane < n) order[b + lane] = v;
        return;
    }
    if (lane == 0)
        for (int k = b + 1; k < e; ++k) {
            int v = order[k], q = k - 1;
            while (q >= b && order[q] > v) {
                order[q + 1] = order[q];
                --q;
            }
            order[q + 1] = v;
        }
}

// Gather the state into sorted order (into the scratch copies).
static __global__ void __launch_bounds__(kThreads)
gather_kernel(int N, const int* __restrict__ order, const double4* __restrict__ pos,
              double4* __restrict__ pos_out, Soa s, Soa s_out, const int* __restrict__ ids,
              int* __restrict__ ids_out, double* __restrict__ bd, Gate gate) {
    if (!gate.open()) return;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    int o = order[k];
    pos_out[k] = pos[o];
#pragma unroll
    for (int f = 0; f < SOA_FIELDS; ++f) s_out.at(f, k) = s.at(f, o);
    ids_out[k] = ids[o];
#pragma unroll
    for (int q = 0; q < 3; ++q) bd[(size_t)q * N + k] = s.at(DX + q, o);
}

// Copy the sorted state back and write the FP32 position copy used by the list build.
static __global__ void __launch_bounds__(kThreads)
copy_back_kernel(int N, const double4* __restrict__ pos_in, double4* __restrict__ pos, Soa s_in,
                 Soa s, const int* __restrict__ ids_in, int* __restrict__ ids, float4* __restrict__ posf,
                 Gate gate) {
    if (!gate.open()) return;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    double4 x = pos_in[k];
    pos[k] = x;
    posf[k] = make_float4((float)x.x, (float)x.y, (float)x.z, 0.f);
#pragma unroll
    for (int f = 0; f < SOA_FIELDS; ++f) s.at(f, k) = s_in.at(f, k);
    ids[k] = ids_in[k];
}

// Neighbour list over the 27-cell stencil of the list grid.
//
// Layout: groups of 4 entries, group g of atom i at nbr4[g * N + i] (one 16-byte
// load per group, coalesced across a warp); the tail of the last group is
// padded with the ghost slot N, which sits far outside every box.  An entry
// holds the slot in its low 27 bits and a 5-bit code above: the lattice image
// in SMALL mode (grids under 3 cells per axis, rebuilt every step), otherwise
// the stencil offset (the pair kernels recompute the minimum image each step).
//
// The candidate test runs in FP32 on box coordinates against a radius widened
// by 8 * L * 2^-24, so the list is a superset of the FP64 pair set; the pair
// kernels apply the exact test.
template <bool SMALL>
static __global__ void __launch_bounds__(kThreads)
build_list_kernel(int N, const double4* __restrict__ pos, const float4* __restrict__ posf, Grid g,
                  const int* __restrict__ start,
                  float3 Lf, float cut2, int cap, uint4* __restrict__ nbr4,
                  int* __restrict__ cnt, Scalars* sc, Gate gate) {
    if (!gate.open()) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = 0;
    unsigned* nbr = reinterpret_cast<unsigned*>(nbr4);
    if (i < N) {
        float4 xi = posf[i];
        // the home cell comes from the FP64 position, exactly as the binning placed the atom
        double4 xd = pos[i];
        int ci[3] = {cell_coord(xd.x, g.ratio[0], g.n[0]), cell_coord(xd.y, g.ratio[1], g.n[1]),
                     cell_coord(xd.z, g.ratio[2], g.n[2])};
        for (int a = -1; a <= 1; ++a) {
            int na = ci[0] + a, ia = na < 0 ? -1 : (na >= g.n[0] ? 1 : 0);
            na -= ia * g.n[0];
            for (int b = -1; b <= 1; ++b) {
                int nb = ci[1] + b, ib = nb < 0 ? -1 : (nb >= g.n[1] ? 1 : 0);
                nb -= ib * g.n[1];
                for (int c = -1; c <= 1; ++c) {
                    int nc = ci[2] + c, ic = nc < 0 ? -1 : (nc >= g.n[2] ? 1 : 0);
                    nc -= ic * g.n[2];
                    int cell = g.flat(na, nb, nc);
                    float sx = ia * Lf.x, sy = ib * Lf.y, sz = ic * Lf.z;
                    unsigned code = SMALL ? offset_code(ia, ib, ic) : offset_code(a, b, c);
                    int e = start[cell + 1];
                    for (int j = start[cell]; j < e; ++j) {
                        float4 xj = posf[j];
                        float dx = (xi.x - xj.x) - sx;
                        float dy = (xi.y - xj.y) - sy;
                        float dz = (xi.z - xj.z) - sz;
                        if (fmaf(dz, dz, fmaf(dy, dy, dx * dx)) < cut2 && j != i) {
                            if (n < cap) nbr[((size_t)(n >> 2) * N + i) * 4 + (n & 3)] = make_entry((unsigned)j, code);
                            ++n;
                        }
                    }
                }
            }
        }
        int m = n < cap ? n : cap;
        cnt[i] = m;
        for (int k = m; k < ((m + 3) & ~3); ++k)  // ghost padding (code 13: no image, no offset)
            nbr[((size_t)(k >> 2) * N + i) * 4 + (k & 3)] = make_entry((unsigned)N, kGhostCode);
    }
    // block max of n -> sc->max_count; overflow flag
    int m = n;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&sc->max_count, m);
        if (m > cap) atomicExch(&sc->overflow, 1);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd((unsigned long long*)&sc->builds, 1ull);
}

// Warp-per-cell list build for grids of >= 3 cells per axis (the minimum-image
// form).  One warp owns one list cell: lanes hold the cell's atoms (in chunks of
// 32).  Atoms are stored cell by cell with z fastest, so the three stencil
// cells z - 1, z, z + 1 of each of the 9 stencil columns are one contiguous
// slot range (two where the column wraps in z).  The warp walks each range in
// chunks of 32 candidates staged in shared memory (one coalesced load, stored
// negated as separate x / y / z rows); every lane tests the staged candidates
// through broadcast reads, two per instruction with Blackwell's packed FP32x2
// add / multiply / fma, in unrolled blocks of 8 that only set bits of a hit
// mask.  The masks of up to kBuildRecords chunks are kept in shared memory
// (with the entry of each chunk's first candidate and the candidates from
// which the code's z offset steps up) and then appended in one loop over all
// their set bits: the warp runs as many append rounds as its busiest lane has
// hits (a warp-uniform count), instead of the busiest lane's hits in every
// chunk added up.  In a round every lane with hits left appends one entry,
// first moving on to its next record with hits when its current mask is empty
// (a per-lane bit set of the records with hits, so the walk takes no divergent
// loop), and writes the entry with one 4-byte store through a pointer stepped
// per append.  Entries, their order (stencil cell, then slot) and the
// candidate radius are those of build_list_kernel<false>.  The per-cell body,
// build_cell_lists, also serves the batched engine's list build.
constexpr int kBuildWarps = 4;
constexpr int kBuildRecords = 24;  // <= 32: bits of a lane's record set

// Shared memory of one list-building warp: the staged candidates and the
// chunk records waiting to be appended (per chunk: the entry of its first
// candidate, and the candidate indices within the chunk from which the z
// offset of the code is one and two steps up -- INT_MAX: none).
struct __align__(16) BuildSmem {
    float cxs[3][32];
    unsigned rec_mask[kBuildRecords][32];
    int4 rec_meta[kBuildRecords];
};

// One warp builds the lists of the atoms of list cell (ca, cb, cc) of grid g
// (>= 3 cells per axis).  `start` holds the slot ranges of the grid's cells
// (slots are global: N is the list stride and the ghost slot).  Returns the
// largest list length of the warp's lanes (before the capacity cut).
__device__ __forceinline__ int build_cell_lists(int ca, int cb, int cc, const Grid& g, const int* __restrict__ start,
                                                const float4* __restrict__ posf, float3 Lf, float cut2, int cap,
                                                uint4* __restrict__ nbr4, int* __restrict__ cnt, int N,
                                                BuildSmem& sm, int lane) {
    int wmax = 0;
    unsigned* const list = reinterpret_cast<unsigned*>(nbr4);  // entry q of group g of slot i: (g*N + i)*4 + q
    int nz = g.n[2];
    // the column's z cells d = -1, 0, 1 as at most two contiguous pieces,
    // split where the column wraps (each piece has one z image)
    int npc = 1, pd0[2] = {-1, 0}, pd1[2] = {1, 1}, pic[2] = {0, 0};
    if (cc == 0) {
        npc = 2; pd0[0] = -1; pd1[0] = -1; pic[0] = -1; pd0[1] = 0; pd1[1] = 1; pic[1] = 0;
    } else if (cc == nz - 1) {
        npc = 2; pd0[0] = -1; pd1[0] = 0; pic[0] = 0; pd0[1] = 1; pd1[1] = 1; pic[1] = 1;
    }
    const float2 mcut2 = make_float2(-cut2, -cut2);
    const int c = g.flat(ca, cb, cc);
    int hs = start[c], he = start[c + 1];
    for (int h0 = hs; h0 < he; h0 += 32) {
        int i = h0 + lane;
        bool own = i < he;
        float4 xi = own ? posf[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        int n = 0;
        int nrec = 0;     // chunk records waiting to be appended (warp-uniform)
        unsigned ne = 0;  // this lane's waiting records with hits (bit k: record k)
        int pend = 0;     // this lane's hits in the waiting records
        // append the hits of the recorded chunks in order, one per lane and
        // round, for as many rounds as the busiest lane has hits
        auto flush = [&]() {
            __syncwarp();
            int rounds = __reduce_max_sync(0xffffffffu, pend);
            unsigned m = 0;
            int4 meta = make_int4(0, 0, INT_MAX, INT_MAX);
            // the entry slot of this lane's next entry, stepped per append
            // (entry q + 1 of a group, or entry 0 of the next group N*4 - 3 on)
            unsigned* p = list + ((size_t)(n >> 2) * N + i) * 4 + (n & 3);
            const size_t next_group = (size_t)N * 4 - 3;
            for (int r = 0; r < rounds; ++r) {
                if (m == 0 && ne != 0) {
                    int k = __ffs(ne) - 1;
                    ne &= ne - 1;
                    m = sm.rec_mask[k][lane];
                    meta = sm.rec_meta[k];
                }
                if (m != 0) {
                    int t = __clz(m);
                    m ^= 0x80000000u >> t;
                    // entry of candidate j0 + t: the record's first entry plus t slots,
                    // plus one z step of the code per cell boundary passed
                    unsigned e = (unsigned)meta.x + ((unsigned)t << kCodeBits) + (t >= meta.y ? 16u : 0u) +
                                 (t >= meta.z ? 16u : 0u);
                    if (n < cap) *p = e;
                    p += (n & 3) == 3 ? next_group : 1;
                    ++n;
                }
            }
            __syncwarp();
            nrec = 0;
            pend = 0;
        };
        for (int a = -1; a <= 1; ++a) {
            int na = ca + a, ia = na < 0 ? -1 : (na >= g.n[0] ? 1 : 0);
            na -= ia * g.n[0];
            for (int b = -1; b <= 1; ++b) {
                int nb = cb + b, ib = nb < 0 ? -1 : (nb >= g.n[1] ? 1 : 0);
                nb -= ib * g.n[1];
                int col = g.flat(na, nb, 0);
                // slot where the d = 0 and d = 1 cells of this column begin
                int s0 = start[col + cc], s1 = start[col + (cc + 1 == nz ? 0 : cc + 1)];
                float2 sx = make_float2(xi.x - ia * Lf.x, xi.x - ia * Lf.x);
                float2 sy = make_float2(xi.y - ib * Lf.y, xi.y - ib * Lf.y);
                for (int pc = 0; pc < npc; ++pc) {
                    int zlo = cc + pd0[pc], zhi = cc + pd1[pc];
                    zlo += zlo < 0 ? nz : (zlo >= nz ? -nz : 0);
                    zhi += zhi < 0 ? nz : (zhi >= nz ? -nz : 0);
                    int js = start[col + zlo], je = start[col + zhi + 1];
                    float2 sz = make_float2(xi.z - pic[pc] * Lf.z, xi.z - pic[pc] * Lf.z);
                    for (int j0 = js; j0 < je; j0 += 32) {
                        int cntj = min(32, je - j0);
                        __syncwarp();
                        float4 q = lane < cntj ? posf[j0 + lane] : make_float4(1e18f, 1e18f, 1e18f, 0.f);
                        sm.cxs[0][lane] = -q.x;
                        sm.cxs[1][lane] = -q.y;
                        sm.cxs[2][lane] = -q.z;
                        __syncwarp();
                        unsigned mask = 0;
                        // the four blocks of 8 unrolled, cut short past the range
#pragma unroll
                        for (int t0 = 0; t0 < 32; t0 += 8) {
                            if (t0 >= cntj) break;
                            // r2 < cut2 exactly when r2 - cut2 is negative: its sign bit
                            // is shifted into `sub`, first candidate highest
                            unsigned sub = 0;
#pragma unroll
                            for (int t = 0; t < 8; t += 4) {
                                float4 qx = *reinterpret_cast<const float4*>(&sm.cxs[0][t0 + t]);
                                float4 qy = *reinterpret_cast<const float4*>(&sm.cxs[1][t0 + t]);
                                float4 qz = *reinterpret_cast<const float4*>(&sm.cxs[2][t0 + t]);
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                    float2 px = h ? make_float2(qx.z, qx.w) : make_float2(qx.x, qx.y);
                                    float2 py = h ? make_float2(qy.z, qy.w) : make_float2(qy.x, qy.y);
                                    float2 pz = h ? make_float2(qz.z, qz.w) : make_float2(qz.x, qz.y);
                                    float2 dx = __fadd2_rn(sx, px), dy = __fadd2_rn(sy, py), dz = __fadd2_rn(sz, pz);
                                    float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
                                    float2 sg = __fadd2_rn(r2, mcut2);
                                    sub = __funnelshift_l(__float_as_uint(sg.x), sub, 1);
                                    sub = __funnelshift_l(__float_as_uint(sg.y), sub, 1);
                                }
                            }
                            mask |= sub << (24 - t0);  // candidate t at bit 31 - t
                        }
                        if (cntj < 32) mask &= ~(0xffffffffu >> cntj);  // fillers past the range
                        unsigned self = (unsigned)(i - j0);
                        if (self < 32u) mask &= ~(0x80000000u >> self);
                        if (!own) mask = 0;
                        if (__any_sync(0xffffffffu, mask != 0u)) {
                            sm.rec_mask[nrec][lane] = mask;
                            ne |= (mask != 0u ? 1u : 0u) << nrec;
                            pend += __popc(mask);
                            if (lane == 0) {
                                // the piece's z offsets: slot j lies in the cell
                                // d = pd0 + (j >= s0 if the piece holds d = 0) + ...
                                int dl = pd0[pc], dh = pd1[pc];
                                sm.rec_meta[nrec] =
                                    make_int4((int)make_entry((unsigned)j0, offset_code(a, b, dl)),
                                              dl < 0 && dh >= 0 ? s0 - j0 : INT_MAX,
                                              dl < 1 && dh >= 1 ? s1 - j0 : INT_MAX, 0);
                            }
                            if (++nrec == kBuildRecords) flush();
                        }
                    }
                }
            }
        }
        if (nrec) flush();
        if (own) {
            int m = n < cap ? n : cap;
            cnt[i] = m;
            for (int k = m; k < ((m + 3) & ~3); ++k)  // pad the last group with the ghost slot
                list[((size_t)(k >> 2) * N + i) * 4 + (k & 3)] = make_entry((unsigned)N, kGhostCode);
            wmax = max(wmax, n);
        }
    }
    return wmax;
}

static __global__ void __launch_bounds__(32 * kBuildWarps)
build_list_warp_kernel(int N, const double4* __restrict__ pos, const float4* __restrict__ posf, Grid g,
                       const int* __restrict__ start, float3 Lf, float cut2, int cap,
                       uint4* __restrict__ nbr4, int* __restrict__ cnt, Scalars* sc, Gate gate) {
    if (!gate.open()) return;
    __shared__ BuildSmem bs[kBuildWarps];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int c = blockIdx.x * kBuildWarps + warp;
    int ncell = g.ncell();
    int wmax = 0;
    if (c < ncell)
        wmax = build_cell_lists(c / (g.n[1] * g.n[2]), (c / g.n[2]) % g.n[1], c % g.n[2], g, start, posf, Lf, cut2,
                                cap, nbr4, cnt, N, bs[warp], lane);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) wmax = max(wmax, __shfl_down_sync(0xffffffffu, wmax, off));
    if (lane == 0 && c < ncell) {
        atomicMax(&sc->max_count, wmax);
        if (wmax > cap) atomicExch(&sc->overflow, 1);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd((unsigned long long*)&sc->builds, 1ull);
}

// ---------------------------------------------------------------------------
// FP64 pair force: full shell over the neighbour list (each atom sums its own
// row, so per-atom sums are deterministic and need no atomics), LJ spline of
// lennard_jones_force.cpp:107-119.  KICK fuses the second half kick
// (integrator.cpp:82) and the measurement partial sums into the epilogue.
//
// The loop runs over groups of 4 neighbours: the next group's indices are
// loaded (streaming, evict-first) while the current group's 4 positions are
// gathered and its 4 pairs evaluated without branches, the cutoff applied as a
// select.  That keeps several independent memory requests in flight per warp.
// ---------------------------------------------------------------------------
enum { KIND_LJ = 1, KIND_CONST = 2 };

// Fusion of the next step's first half kick and drift into the pair kernel's
// epilogue (kick_drift_kernel's arithmetic, in the same order): the new
// positions go to the other position buffer, which no pair kernel of this
// step reads.
struct Fuse {
    double4* pos_next;        // nullptr: no fusion
    float4* posl_next;        // mixed path: next step's cell-local coordinates
    const double4* pos;       // this step's positions (the mixed kernel reads FP32 copies)
    const double* bd;         // displacement at the last list build
    const double* bx;         // mixed path: cell-local position at the last list build
    Scalars* sc;
    int track, local, periodic;
};

// Second half kick (integrator.cpp:82) with the measurement partials and, when
// fused, the next step's first half kick, drift, displacement and periodic
// wrap (integrator.cpp:70-78).  Returns |d - d_build|^2 for the rebuild test.
__device__ __forceinline__ double step_epilogue(int N, int i, Soa s, const double4 x, const double (&f3)[3],
                                                const PairParams& pp, const Fuse& fz, double (&acc)[4]) {
    double xs[3] = {x.x, x.y, x.z};
    float l[3] = {0.f, 0.f, 0.f};
    double m = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double v = kick(s.at(VX + k, i), f3[k], pp.dt);
        acc[0] = fma(v, v, acc[0]);
        double d = s.at(DX + k, i);
        acc[3] = fma(d, d, acc[3]);
        if (fz.pos_next) {
            v = kick(v, f3[k], pp.dt);
            double inc = __dmul_rn(v, pp.dt);
            double xn = __dadd_rn(xs[k], inc);
            double dn = __dadd_rn(d, inc);
            if (fz.periodic) xn = wrap(xn, pp.L[k]);
            s.at(DX + k, i) = dn;
            xs[k] = xn;
            if (fz.track || fz.local) {
                double e = dn - fz.bd[(size_t)k * N + i];
                m = fma(e, e, m);
                if (fz.local) l[k] = (float)(fz.bx[(size_t)k * N + i] + e);
            }
        }
        s.at(VX + k, i) = v;
    }
    if (fz.pos_next) {
        fz.pos_next[i] = make_double4(xs[0], xs[1], xs[2], 0.0);
        if (fz.local) fz.posl_next[i] = make_float4(l[0], l[1], l[2], 0.f);
    }
    return fz.track ? m : 0.0;
}

// Warp max of the fused displacement into the next step's rebuild criterion.
__device__ __forceinline__ void fused_track(const Fuse& fz, double m) {
    if (fz.pos_next && fz.track) {
        m = warp_max(m);
        if ((threadIdx.x & 31) == 0 && m > 0.0)
            atomicMax(&fz.sc->max_disp2_next, (unsigned long long)__double_as_longlong(m));
    }
}

// One 32-byte position in a single 256-bit load (sm_100 ld.global.v4.f64;
// positions are double4 in cudaMalloc'd arrays, so always 32-byte aligned).
__device__ __forceinline__ double4 ld_pos(const double4* p) {
    double4 r;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
    return r;
}

// 1/x: the hardware's approximate FP64 reciprocal refined by one third-order
// (Householder) step y <- y (1 + e + e^2), e = 1 - x y: the seed's ~2^-20
// relative error cubes to ~2^-60, below the last bit of the result, in three
// dependent FMAs where two Newton-Raphson steps need four.
__device__ __forceinline__ double rcp_nr(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
}

template <bool SMALL>
__device__ __forceinline__ void separation(const double4& xi, const double4& xj, unsigned e, bool near,
                                           const PairParams& pp, double& dx, double& dy, double& dz) {
    dx = __dsub_rn(xi.x, xj.x);
    dy = __dsub_rn(xi.y, xj.y);
    dz = __dsub_rn(xi.z, xj.z);
    if (SMALL) {
        int ia = entry_axis(e, 0), ib = entry_axis(e, 1), ic = entry_axis(e, 2);
        dx = __dsub_rn(dx, ia * pp.L[0]);
        dy = __dsub_rn(dy, ib * pp.L[1]);
        dz = __dsub_rn(dz, ic * pp.L[2]);
    } else if (near) {
        // minimum image; identical to the reference's stencil image for every
        // pair inside the cutoff (the list grid has >= 3 cells per axis)
        if ((__double2hiint(dx) & 0x7fffffff) > pp.halfL_hi[0]) dx = __dsub_rn(dx, copysign(pp.L[0], dx));
        if ((__double2hiint(dy) & 0x7fffffff) > pp.halfL_hi[1]) dy = __dsub_rn(dy, copysign(pp.L[1], dy));
        if ((__double2hiint(dz) & 0x7fffffff) > pp.halfL_hi[2]) dz = __dsub_rn(dz, copysign(pp.L[2], dz));
    }
}

template <int KIND>
__device__ __forceinline__ void pair_fp64(const PairParams& pp, double r2, double& f, double& V, double& W) {
    if (KIND == KIND_LJ) {
        bool hit = r2 < pp.rc2;
        double ir2 = rcp_nr(r2);
        double ir6 = ir2 * ir2 * ir2;
        double x = r2 * pp.inv_rc2;
        double v = fma(4.0 * ir6, ir6 - 1.0, fma(pp.beta, x - 1.0, pp.alpha));
        double w = fma(24.0 * ir6, fma(2.0, ir6, -1.0), -2.0 * pp.beta * x);
        f = hit ? w * ir2 : 0.0;
        V = hit ? v : 0.0;
        W = hit ? w : 0.0;
    } else {
        // tests/cpp/mock/constant_short_range_force.cpp:35-53
        double norm = sqrt(r2);
        bool hit = r2 < pp.rc2 && norm < pp.rc;
        V = hit ? pp.strength * (pp.rc - norm) : 0.0;
        W = hit ? pp.strength * norm : 0.0;
        f = hit ? W / (norm * norm) : 0.0;
    }
}

// LJ spline pairs of one atom (lennard_jones_force.cpp:107-119) accumulated as
// the force plus power sums: with u = r^-6 and x = r^2 / rc^2 the pair terms
// are V = 4u(u - 1) + beta x + (alpha - beta) and W = u(48u - 24) - 2 beta x,
// so the atom's energy and virial follow from sum u^2, sum u, sum r^2 and the
// pair count, formed once per atom, instead of V and W per pair; the force
// magnitude over r is W / r^2 = u(48u - 24) r^-2 - 2 beta / rc^2 (22 instead of
// 28 FP64 operations per pair).  Pairs at or beyond the cutoff add nothing.
struct LjSums {
    double fx = 0, fy = 0, fz = 0, su2 = 0, su = 0, sr2 = 0;
    int nh = 0;
};

__device__ __forceinline__ void lj_accumulate(const PairParams& pp, double dx, double dy, double dz, LjSums& a) {
    const double wq = -2.0 * pp.beta * pp.inv_rc2;
    double r2 = norm2(dx, dy, dz);
    bool hit = r2 < pp.rc2;
    double ir2 = rcp_nr(r2);
    double u = ir2 * ir2 * ir2;
    double f = hit ? fma(u * fma(48.0, u, -24.0), ir2, wq) : 0.0;  // W / r^2 = u(48u - 24) r^-2 + wq
    double uh = hit ? u : 0.0;
    a.su2 = fma(uh, uh, a.su2);
    a.su += uh;
    a.sr2 += hit ? r2 : 0.0;
    a.nh += hit ? 1 : 0;
    a.fx = fma(f, dx, a.fx);
    a.fy = fma(f, dy, a.fy);
    a.fz = fma(f, dz, a.fz);
}

// The atom's sum of pair energies and of pair virials (each pair counted in
// both of its atoms' rows, halved by the finalize).
__device__ __forceinline__ void lj_energy(const PairParams& pp, const LjSums& a, double& pe, double& w) {
    const double bq = pp.beta * pp.inv_rc2, abq = pp.alpha - pp.beta, wq = -2.0 * pp.beta * pp.inv_rc2;
    pe = fma(4.0, a.su2 - a.su, fma(bq, a.sr2, abq * (double)a.nh));
    w = fma(48.0, a.su2, fma(-24.0, a.su, wq * a.sr2));
}

// Occupancy bound: 768 resident threads' worth of blocks per SM caps the kernel
// at 80 registers (no spills); it is latency-bound on the neighbour gathers,
// and 24 resident warps per SM measured ~12 % faster than 16 at 114 registers.
template <int KIND, bool SMALL, bool KICK, int BS = kThreads>
static __global__ void __launch_bounds__(BS, 768 / BS)
force_fp64_kernel(int N, const double4* __restrict__ pos, Soa s, const uint4* __restrict__ nbr4,
                  const int* __restrict__ cnt, PairParams pp, double* __restrict__ partials, Fuse fu) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0, 0, 0, 0};  // sum v^2, sum pe_i, sum w_i, sum d^2
    double m = 0.0;
    if (i < N) {
        const double4 xi = pos[i];
        bool near = !(xi.x >= pp.near_lo && xi.x < pp.near_hi[0] && xi.y >= pp.near_lo &&
                      xi.y < pp.near_hi[1] && xi.z >= pp.near_lo && xi.z < pp.near_hi[2]);
        LjSums a;        // KIND_LJ
        double pe = 0, w = 0;  // KIND_CONST
        // list indices stream from HBM: two groups in flight ahead of the two
        // being evaluated
        int ng = (cnt[i] + 3) >> 2;
        const uint4* lp = nbr4 + i;
        const uint4 z4 = make_uint4(0u, 0u, 0u, 0u);
        uint4 A = ng > 0 ? __ldcs(lp) : z4;
        uint4 B = ng > 1 ? __ldcs(lp + (size_t)N) : z4;
        auto group = [&](const uint4 grp) {
            const unsigned e[4] = {grp.x, grp.y, grp.z, grp.w};
            double4 q[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) q[u] = ld_pos(pos + entry_slot(e[u]));
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                double dx, dy, dz;
                separation<SMALL>(xi, q[u], e[u], near, pp, dx, dy, dz);
                if (KIND == KIND_LJ) {
                    lj_accumulate(pp, dx, dy, dz, a);
                } else {
                    double f, V, W;
                    pair_fp64<KIND>(pp, norm2(dx, dy, dz), f, V, W);
                    a.fx = fma(f, dx, a.fx);
                    a.fy = fma(f, dy, a.fy);
                    a.fz = fma(f, dz, a.fz);
                    pe += V;
                    w += W;
                }
            }
        };
        for (int g = 0; g < ng; g += 2) {
            uint4 C = g + 2 < ng ? __ldcs(lp + (size_t)(g + 2) * N) : z4;
            uint4 D = g + 3 < ng ? __ldcs(lp + (size_t)(g + 3) * N) : z4;
            group(A);
            if (g + 1 < ng) group(B);
            A = C;
            B = D;
        }
        if (KIND == KIND_LJ) lj_energy(pp, a, pe, w);
        s.at(FX, i) = a.fx;
        s.at(FY, i) = a.fy;
        s.at(FZ, i) = a.fz;
        acc[1] = pe;
        acc[2] = w;
        if (KICK) {
            const double f3[3] = {a.fx, a.fy, a.fz};
            m = step_epilogue(N, i, s, xi, f3, pp, fu, acc);
        }
    }
    if (KICK) fused_track(fu, m);
    block_sum<4, BS>(acc);
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; ++q) partials[(size_t)blockIdx.x * 4 + q] = acc[q];
}

// ---------------------------------------------------------------------------
// Step finalisation: sum the per-block partials in a fixed order and publish
// ThermodynamicMeasurement::Result (measurements.hpp:59-70).
// mode 0: after a step (t += dt); 1: after a force evaluation (PE, W only);
// 2: measurement of the current state.
// ---------------------------------------------------------------------------
// Step graphs: the finalize of a step also takes the next step's rebuild
// decision (the conditional handle of the next step's rebuild node), saving
// that step a one-thread launch.
struct NextStep {
    Gate gate;
    cudaGraphConditionalHandle h;
    int set;  // 0: no next step in this graph
};

static __global__ void __launch_bounds__(1024)
finalize_kernel(const double* __restrict__ partials, int nblocks, int N, double dt, int mode,
                int forces_valid, Scalars* sc, double* __restrict__ ring, int ring_cap, NextStep next) {
    // thread 0 loads the scalars it updates before the reduction, so that those
    // loads overlap the partials' instead of following one another at the end
    // (only this kernel changes them while it runs)
    double t0 = 0, pe0 = 0, vir0 = 0;
    long long steps0 = 0, rebuilds0 = 0;
    unsigned long long md2_0 = 0, md2_next = 0;
    int need0 = 0;
    if (threadIdx.x == 0) {
        t0 = sc->t;
        pe0 = sc->pe;
        vir0 = sc->vir;
        steps0 = sc->steps;
        rebuilds0 = sc->graph_rebuilds;
        md2_0 = sc->max_disp2;
        md2_next = sc->max_disp2_next;
        need0 = sc->need_rebuild;
    }
    // each thread sums blocks tid, tid + 1024, ... in that order; eight blocks'
    // partials (32-byte loads) are in flight at a time
    double acc[4] = {0, 0, 0, 0};
    const double4* p4 = reinterpret_cast<const double4*>(partials);
    for (int b0 = threadIdx.x; b0 < nblocks; b0 += 8 * 1024) {
        double4 t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            int b = b0 + u * 1024;
            t[u] = b < nblocks ? p4[b] : make_double4(0.0, 0.0, 0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (b0 + u * 1024 < nblocks) {
                acc[0] += t[u].x;
                acc[1] += t[u].y;
                acc[2] += t[u].z;
                acc[3] += t[u].w;
            }
        }
    }
    block_sum<4, 1024>(acc);
    if (threadIdx.x == 0) {
        double pe = pe0, vir = vir0, t = t0;
        if (forces_valid) {
            pe = 0.5 * acc[1];
            vir = 0.5 * acc[2];
            sc->pe = pe;
            sc->vir = vir;
        }
        // a step's record goes to ring slot (step index mod ring_cap); the extra
        // slot ring_cap holds single measurements
        double* out = ring + 7 * (size_t)(mode == 0 ? (int)(steps0 % ring_cap) : ring_cap);
        if (mode == 0) {
            t = t0 + dt;  // integrator.cpp:85
            sc->t = t;
            sc->steps = steps0 + 1;
        }
        if (mode != 1) {
            double ke = 0.5 * acc[0];
            double rec[7];
            rec[0] = t;
            rec[1] = ke;
            rec[2] = pe;
            rec[3] = pe + ke;
            rec[4] = vir;
            rec[5] = (2. / 3.) * ke / (double)N;
            rec[6] = acc[3] / (double)N;
            for (int q = 0; q < 7; ++q) out[q] = rec[q];
            if (!isfinite(ke) || !isfinite(pe) || !isfinite(vir)) sc->nonfinite = 1;
        } else if (!isfinite(pe) || !isfinite(vir)) {
            sc->nonfinite = 1;
        }
        unsigned long long md2 = md2_0;
        int need = need0;
        if (mode != 2) {  // a measurement changes nothing that a rebuild depends on
            // the next step's displacement (a fused epilogue's, else 0 for kick_drift)
            md2 = md2_next;
            need = 0;
            sc->max_disp2 = md2;
            sc->max_disp2_next = 0ull;
            sc->need_rebuild = 0;
        }
        if (next.set) {
            // next.gate.open() on the values just written
            bool open = next.gate.always || need || __longlong_as_double((long long)md2) > next.gate.thresh2;
            if (open) sc->graph_rebuilds = rebuilds0 + 1;
            cudaGraphSetConditional(next.h, open ? 1u : 0u);
        }
    }
}

// ThermodynamicAnalyzer::result (analyzers.cpp:44-159) over the last W step
// records of a record ring, one block per system: record k of the window
// (k = 0 oldest) of system s sits at ring + 7 * (slot(k) * nsys + s) with
// slot(k) = (last - (W - 1) + k) mod ring_cap.  Two passes as
// tools::MovingSample::statistics (moving_sample.hpp:107-188): the means, then
// the Bessel-corrected variance of T and the covariance of (t, MSD); each sum
// is a fixed-order block reduction.
constexpr int kStatsThreads = 256;

static __global__ void __launch_bounds__(kStatsThreads)
window_stats_kernel(const double* __restrict__ ring, int ring_cap, int nsys, long long last, int W,
                    const int* __restrict__ natoms, const double* __restrict__ density, double* __restrict__ out) {
    int s = blockIdx.x;
    auto rec = [&](int k) {
        long long step = last - (W - 1) + k;
        int slot = (int)(((step % ring_cap) + ring_cap) % ring_cap);
        return ring + 7 * ((size_t)slot * nsys + s);
    };
    // pass 1: sums of T, TE, W, t, MSD
    double a[5] = {0, 0, 0, 0, 0};
    for (int k = threadIdx.x; k < W; k += kStatsThreads) {
        const double* r = rec(k);
        a[0] += r[5];
        a[1] += r[3];
        a[2] += r[4];
        a[3] += r[0];
        a[4] += r[6];
    }
    block_sum<5, kStatsThreads>(a);
    __shared__ double mean[5];
    if (threadIdx.x == 0)
        for (int q = 0; q < 5; ++q) mean[q] = a[q] / (double)W;
    __syncthreads();
    // pass 2: sum (T - <T>)^2, (t - <t>)(MSD - <MSD>), (t - <t>)^2
    double c[3] = {0, 0, 0};
    for (int k = threadIdx.x; k < W; k += kStatsThreads) {
        const double* r = rec(k);
        double dT = r[5] - mean[0], dt = r[0] - mean[3], dm = r[6] - mean[4];
        c[0] += dT * dT;
        c[1] += dt * dm;
        c[2] += dt * dt;
    }
    block_sum<3, kStatsThreads>(c);
    if (threadIdx.x == 0) {
        double N = (double)natoms[s], rho = density[s];
        double T = mean[0];
        double varT = c[0] / (double)(W - 1);
        double* o = out + 6 * (size_t)s;
        o[0] = T;
        o[1] = rho;
        o[2] = mean[1];
        o[3] = rho * (T + mean[2] / (3.0 * N));
        o[4] = (3. / 2.) / (1 - (3. / 2.) * N * (varT / (T * T)));
        o[5] = (1. / 6.) * ((c[1] / (double)(W - 1)) / (c[2] / (double)(W - 1)));
    }
}

// Graph step: decide on the device whether the rebuild subgraph runs this step.
static __global__ void decide_rebuild_kernel(Gate gate, cudaGraphConditionalHandle h, Scalars* sc) {
    bool open = gate.open();
    if (open) sc->graph_rebuilds += 1;
    cudaGraphSetConditional(h, open ? 1u : 0u);
}

static __global__ void __launch_bounds__(kThreads)
scale_kernel(int N, Soa s, double factor) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
#pragma unroll
    for (int k = 0; k < 3; ++k) s.at(VX + k, i) = __dmul_rn(s.at(VX + k, i), factor);
}

// set_temperature (transformations.cpp:94-116): the factor is computed on the
// device from the KE of the record written by the preceding measurement.
static __global__ void set_temperature_factor_kernel(const double* rec, double target, double* factor) {
    *factor = sqrt(target / rec[5]);
}

static __global__ void __launch_bounds__(kThreads)
scale_from_device_kernel(int N, Soa s, const double* __restrict__ factor) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double f = *factor;
#pragma unroll
    for (int k = 0; k < 3; ++k) s.at(VX + k, i) = __dmul_rn(s.at(VX + k, i), f);
}

// ---------------------------------------------------------------------------
// Host <-> device layout conversion (atom-id order <-> sorted slots)
// ---------------------------------------------------------------------------
static __global__ void unpack_kernel(int N, const double* __restrict__ in, int stride, int field,
                              double4* __restrict__ pos, Soa s, int* __restrict__ ids) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double* p = in + (size_t)i * stride;
    if (field < 0) {
        pos[i] = make_double4(p[0], p[1], p[2], 0.0);
        ids[i] = i;
    } else {
        for (int k = 0; k < 3; ++k) s.at(field + k, i) = p[k];
    }
}

static __global__ void pack_kernel(int N, double* __restrict__ out, int stride, int field,
                            const double4* __restrict__ pos, Soa s, const int* __restrict__ ids) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    double* p = out + (size_t)ids[k] * stride;
    double v[3];
    if (field < 0) {
        double4 x = pos[k];
        v[0] = x.x; v[1] = x.y; v[2] = x.z;
    } else {
        for (int q = 0; q < 3; ++q) v[q] = s.at(field + q, k);
    }
    for (int q = 0; q < 3; ++q) p[q] = v[q];
    if (stride == 4) p[3] = 0.0;
}

// Reference binning for the debug API: cell of each atom id, and members as ids.
static __global__ void debug_members_kernel(int N, const int* __restrict__ cell_of_slot,
                                     const int* __restrict__ rank, const int* __restrict__ start,
                                     const int* __restrict__ ids, int* __restrict__ members,
                                     int* __restrict__ cell_of_id) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    members[start[cell_of_slot[k]] + rank[k]] = ids[k];
    cell_of_id[ids[k]] = cell_of_slot[k];
}

static __global__ void sort_members_kernel(int ncell, const int* __restrict__ start, int* __restrict__ m) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    for (int k = start[c] + 1; k < start[c + 1]; ++k) {
        int v = m[k], q = k - 1;
        while (q >= start[c] && m[q] > v) {
            m[q + 1] = m[q];
            --q;
        }
        m[q + 1] = v;
    }
}

// The in-cutoff pair set as seen by the force kernel (i < j by id).
template <bool SMALL>
static __global__ void debug_pairs_kernel(int N, const double4* __restrict__ pos,
                                   const uint4* __restrict__ nbr4, const int* __restrict__ cnt,
                                   const int* __restrict__ ids, PairParams pp, long long cap,
                                   int* oi, int* oj, int* oimg, double* or2,
                                   unsigned long long* counter) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double4 xi = pos[i];
    const unsigned* nbr = reinterpret_cast<const unsigned*>(nbr4);
    for (int k = 0; k < cnt[i]; ++k) {
        unsigned e = nbr[((size_t)(k >> 2) * N + i) * 4 + (k & 3)];
        int j = (int)entry_slot(e);
        if (ids[i] >= ids[j]) continue;
        double4 xj = pos[j];
        double d[3] = {__dsub_rn(xi.x, xj.x), __dsub_rn(xi.y, xj.y), __dsub_rn(xi.z, xj.z)};
        int img[3] = {0, 0, 0};
        if (SMALL) {
            for (int q = 0; q < 3; ++q) img[q] = entry_axis(e, q);
        } else {
            for (int q = 0; q < 3; ++q)
                if ((__double2hiint(d[q]) & 0x7fffffff) > pp.halfL_hi[q]) img[q] = d[q] > 0 ? 1 : -1;
        }
        for (int q = 0; q < 3; ++q) d[q] = __dsub_rn(d[q], img[q] * pp.L[q]);
        double r2 = norm2(d[0], d[1], d[2]);
        if (r2 < pp.rc2) {
            unsigned long long slot = atomicAdd(counter, 1ull);
            if ((long long)slot < cap) {
                oi[slot] = ids[i];
                oj[slot] = ids[j];
                oimg[slot] = image_code(img[0], img[1], img[2]);
                or2[slot] = r2;
            }
        }
    }
}

}  // namespace ljb
