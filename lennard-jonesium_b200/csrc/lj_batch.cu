// lj_batch.cu -- many independent systems of uneven size in one launch per
// kernel: the batched engine behind run_sweep (a grid of (T, rho) runs).
//
// Packed system table.  The atoms of all systems are concatenated (system s
// owns slots [atom_off_s, atom_off_s + N_s)), and so are their list-cell grids
// (cells [cell_off_s, cell_off_s + ncell_s)).  Each per-atom kernel runs over a
// block table in which every block belongs to one system and covers the same
// 128 atoms as block j of that system run alone; every cell belongs to one
// system.  Rebuilds are gated per system by its own skin criterion, the cell
// scan is segmented per system, and each system's records come from its own
// blocks' partial sums in the single-system order.  A batched run therefore
// reproduces, bit for bit, the same systems run one at a time through
// lj_gpu_* (tests/test_gpu_batch.py checks this).
//
// One step = kick_drift -> decide (per-system rebuild flags + graph conditional)
// -> IF(rebuild chain) -> force(+kick) -> finalize (one block per system), and
// lj_batch_step launches whole CUDA graphs of several such steps.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lj_gpu.h"
#include "lj_kernels.cuh"

using namespace ljb;

double list_skin(double requested, double Lmin, double rc);

namespace {

struct SysDev {
    int atom_off, natoms;
    int cell_off, ncell;
    int blk_off, nblk;    // blocks of kThreads atoms (integration, measurement)
    int fblk_off, nfblk;  // blocks of the pair kernel (force_block atoms)
    Grid grid;
    PairParams pp;
    double thresh2;  // rebuild when max |d - d_build|^2 exceeds this
    int always;      // zero skin: rebuild every step
    float cut2;      // FP32 list radius^2 (widened past FP32 rounding)
    float3 Lf;
};

struct SysState {
    double t, pe, vir;
    unsigned long long max_disp2;
    int need_rebuild;
    int rebuild;  // decided for this step
    int active;
    int pad;
    long long builds, steps;
};

struct BatchFlags {
    int overflow, nonfinite, any_rebuild, slot;  // slot: ring slot of the current step
    long long graph_rebuilds;
    long long step_count;                        // steps taken by the batch
    // device-side loop of a chunk launch (set by the host before each launch)
    int loop_left;         // body iterations still to run
    int timeout;           // the loop hit loop_limit before loop_left reached 0
    long long loop_iters;  // iterations run by this launch
    long long loop_limit;  // upper bound on loop_iters
};

__device__ __forceinline__ bool sys_rebuild(const SysState* st, int s) { return st[s].rebuild != 0; }

// ---- integration -----------------------------------------------------------
static __global__ void __launch_bounds__(kThreads)
b_kick_drift_kernel(const int* __restrict__ blk_sys, const int* __restrict__ blk_first, const SysDev* __restrict__ sys,
                    SysState* st, int Ntot, double4* __restrict__ pos, Soa s, const double* __restrict__ bd) {
    int sidx = blk_sys[blockIdx.x];
    const SysDev& S = sys[sidx];
    if (!st[sidx].active) return;
    int i = blk_first[blockIdx.x] + threadIdx.x;
    bool own = i < S.atom_off + S.natoms;
    double m = 0.0;
    if (own) {
        double4 x = pos[i];
        double xs[3] = {x.x, x.y, x.z};
        double dt = S.pp.dt;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double v = kick(s.at(VX + k, i), s.at(FX + k, i), dt);
            double inc = __dmul_rn(v, dt);
            double xn = wrap(__dadd_rn(xs[k], inc), S.pp.L[k]);
            double dn = __dadd_rn(s.at(DX + k, i), inc);
            s.at(VX + k, i) = v;
            s.at(DX + k, i) = dn;
            xs[k] = xn;
            double e = dn - bd[(size_t)k * Ntot + i];
            m = fma(e, e, m);
        }
        pos[i] = make_double4(xs[0], xs[1], xs[2], 0.0);
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0 && m > 0.0)
        atomicMax(&st[sidx].max_disp2, (unsigned long long)__double_as_longlong(m));
}

// Per-system rebuild decision; opens the graph conditional if any system rebuilds.
static __global__ void b_decide_kernel(const SysDev* __restrict__ sys, SysState* st, int nsys, BatchFlags* fl,
                                       int ring_cap, cudaGraphConditionalHandle h, int use_handle) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < nsys; s += blockDim.x) {
        bool r = st[s].active &&
                 (sys[s].always || st[s].need_rebuild ||
                  __longlong_as_double((long long)st[s].max_disp2) > sys[s].thresh2);
        st[s].rebuild = r ? 1 : 0;
        if (r) atomicExch(&any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        fl->any_rebuild = any;
        fl->slot = (int)(fl->step_count % ring_cap);
        fl->step_count += 1;
        if (any) fl->graph_rebuilds += 1;
        if (use_handle) cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}

// End of one body iteration of a chunk launch: continue while iterations are
// left.  The iteration count is bounded independently of loop_left: a launch
// never runs more than loop_limit iterations, and one that would is stopped
// with the timeout flag set (the host then returns LJ_ERR_TIMEOUT).
static __global__ void b_loop_kernel(BatchFlags* fl, cudaGraphConditionalHandle h) {
    int left = --fl->loop_left;
    long long it = ++fl->loop_iters;
    bool go = left > 0;
    if (go && it >= fl->loop_limit) {
        fl->timeout = 1;
        go = false;
    }
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// ---- rebuild chain (systems with st[s].rebuild only) -------------------------
static __global__ void __launch_bounds__(kThreads)
b_bin_kernel(const int* __restrict__ sys_of, const SysDev* __restrict__ sys, const SysState* st, int Ntot,
             const double4* __restrict__ pos, int* __restrict__ cell_of, int* __restrict__ rank,
             int* __restrict__ count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Ntot) return;
    int s = sys_of[i];
    if (!sys_rebuild(st, s)) return;
    const Grid& g = sys[s].grid;
    double4 x = pos[i];
    int c = sys[s].cell_off + g.flat(cell_coord(x.x, g.ratio[0], g.n[0]), cell_coord(x.y, g.ratio[1], g.n[1]),
                                     cell_coord(x.z, g.ratio[2], g.n[2]));
    cell_of[i] = c;
    rank[i] = atomicAdd(&count[c], 1);
}

// One block per system: exclusive scan of its cells' counts, offset by its first slot.
static __global__ void __launch_bounds__(1024)
b_scan_kernel(const SysDev* __restrict__ sys, const SysState* st, int* __restrict__ count, int* __restrict__ start) {
    int s = blockIdx.x;
    if (!sys_rebuild(st, s)) return;
    __shared__ int tot;
    int base = sys[s].atom_off;
    int c0 = sys[s].cell_off, nc = sys[s].ncell;
    for (int t0 = 0; t0 < nc; t0 += 4 * 1024) {
        int idx = t0 + threadIdx.x * 4;
        int c[4], sum = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            c[q] = idx + q < nc ? count[c0 + idx + q] : 0;
            sum += c[q];
        }
        int ex = block_exclusive_scan<1024>(sum, &tot) + base;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (idx + q < nc) {
                start[c0 + idx + q] = ex;
                count[c0 + idx + q] = 0;
            }
            ex += c[q];
        }
        base += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) start[c0 + nc] = sys[s].atom_off + sys[s].natoms;
}

static __global__ void __launch_bounds__(kThreads)
b_scatter_kernel(const int* __restrict__ sys_of, const SysState* st, int Ntot, const int* __restrict__ cell_of,
                 const int* __restrict__ rank, const int* __restrict__ start, int* __restrict__ order) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Ntot || !sys_rebuild(st, sys_of[i])) return;
    order[start[cell_of[i]] + rank[i]] = i;
}

static __global__ void __launch_bounds__(32 * kSortWarps)
b_cell_sort_kernel(const int* __restrict__ cell_sys, const SysState* st, int ncell, const int* __restrict__ start,
                   int* __restrict__ order) {
    int lane = threadIdx.x & 31;
    int c = blockIdx.x * kSortWarps + (threadIdx.x >> 5);
    if (c >= ncell || !sys_rebuild(st, cell_sys[c])) return;
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

static __global__ void __launch_bounds__(kThreads)
b_gather_kernel(const int* __restrict__ sys_of, const SysState* st, int Ntot, const int* __restrict__ order,
                const double4* __restrict__ pos, double4* __restrict__ pos_out, Soa s, Soa s_out,
                const int* __restrict__ ids, int* __restrict__ ids_out, double* __restrict__ bd) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Ntot || !sys_rebuild(st, sys_of[k])) return;
    int o = order[k];
    pos_out[k] = pos[o];
#pragma unroll
    for (int f = 0; f < SOA_FIELDS; ++f) s_out.at(f, k) = s.at(f, o);
    ids_out[k] = ids[o];
#pragma unroll
    for (int q = 0; q < 3; ++q) bd[(size_t)q * Ntot + k] = s.at(DX + q, o);
}

static __global__ void __launch_bounds__(kThreads)
b_copy_back_kernel(const int* __restrict__ sys_of, const SysState* st, int Ntot, const double4* __restrict__ pos_in,
                   double4* __restrict__ pos, Soa s_in, Soa s, const int* __restrict__ ids_in, int* __restrict__ ids,
                   float4* __restrict__ posf) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Ntot || !sys_rebuild(st, sys_of[k])) return;
    double4 x = pos_in[k];
    pos[k] = x;
    posf[k] = make_float4((float)x.x, (float)x.y, (float)x.z, 0.f);
#pragma unroll
    for (int f = 0; f < SOA_FIELDS; ++f) s.at(f, k) = s_in.at(f, k);
    ids[k] = ids_in[k];
}

// Warp-per-cell list build: the per-cell body of build_list_warp_kernel, on
// the grid and slot ranges of the cell's own system (entries identical to a
// single-system build of that system).  W cells (warps) per block, the list
// tile a batch tunes; 24 resident warps leave it up to 80 registers, where it
// does not spill (the per-system indexing costs the registers the
// single-system kernel fits into 64).
template <int W>
static __global__ void __launch_bounds__(32 * W, 24 / W)
b_build_list_kernel(const int* __restrict__ cell_sys, const SysDev* __restrict__ sys, SysState* st, int ncell_tot,
                    int Ntot, const float4* __restrict__ posf, const int* __restrict__ start, int cap,
                    uint4* __restrict__ nbr4, int* __restrict__ cnt, BatchFlags* fl) {
    __shared__ BuildSmem bs[W];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int c = blockIdx.x * W + warp;
    if (c >= ncell_tot) return;
    int sidx = cell_sys[c];
    if (!sys_rebuild(st, sidx)) return;
    const SysDev& S = sys[sidx];
    const Grid& g = S.grid;
    int lc = c - S.cell_off;
    int wmax = build_cell_lists(lc / (g.n[1] * g.n[2]), (lc / g.n[2]) % g.n[1], lc % g.n[2], g, start + S.cell_off,
                                posf, S.Lf, S.cut2, cap, nbr4, cnt, Ntot, bs[warp], lane);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) wmax = max(wmax, __shfl_down_sync(0xffffffffu, wmax, off));
    if (lane == 0 && wmax > cap) atomicExch(&fl->overflow, 1);
    if (lc == 0 && lane == 0) atomicAdd((unsigned long long*)&st[sidx].builds, 1ull);
}

// ---- pair force: per block one system, same loop as force_fp64_kernel ---------
template <int BS>
static __global__ void __launch_bounds__(BS, 512 / BS)
b_force_kernel(const int* __restrict__ blk_sys, const int* __restrict__ blk_first, const SysDev* __restrict__ sys,
               const SysState* st, int Ntot, const double4* __restrict__ pos, Soa s, const uint4* __restrict__ nbr4,
               const int* __restrict__ cnt, double* __restrict__ partials) {
    int sidx = blk_sys[blockIdx.x];
    if (!st[sidx].active) return;
    const SysDev& S = sys[sidx];
    const PairParams pp = S.pp;
    int i = blk_first[blockIdx.x] + threadIdx.x;
    double acc[4] = {0, 0, 0, 0};
    if (i < S.atom_off + S.natoms) {
        const double4 xi = pos[i];
        bool near = !(xi.x >= pp.near_lo && xi.x < pp.near_hi[0] && xi.y >= pp.near_lo &&
                      xi.y < pp.near_hi[1] && xi.z >= pp.near_lo && xi.z < pp.near_hi[2]);
        LjSums a;
        int ng = (cnt[i] + 3) >> 2;
        uint4 cur = ng > 0 ? __ldcs(&nbr4[i]) : make_uint4(0, 0, 0, 0);
        for (int g = 0; g < ng; ++g) {
            uint4 nxt = g + 1 < ng ? __ldcs(&nbr4[(size_t)(g + 1) * Ntot + i]) : cur;
            unsigned e[4] = {cur.x, cur.y, cur.z, cur.w};
            double4 q[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) q[u] = ld_pos(pos + entry_slot(e[u]));
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                double dx, dy, dz;
                separation<false>(xi, q[u], e[u], near, pp, dx, dy, dz);
                lj_accumulate(pp, dx, dy, dz, a);
            }
            cur = nxt;
        }
        s.at(FX, i) = a.fx;
        s.at(FY, i) = a.fy;
        s.at(FZ, i) = a.fz;
        lj_energy(pp, a, acc[1], acc[2]);
        double f3[3] = {a.fx, a.fy, a.fz};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double v = kick(s.at(VX + k, i), f3[k], pp.dt);
            s.at(VX + k, i) = v;
            acc[0] = fma(v, v, acc[0]);
            double d = s.at(DX + k, i);
            acc[3] = fma(d, d, acc[3]);
        }
    }
    block_sum<4, BS>(acc);
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; ++q) partials[(size_t)blockIdx.x * 4 + q] = acc[q];
}

// One block per system: the single-system finalize over that system's blocks
// (after a step the pair kernel's blocks, after a measurement the kThreads ones).
static __global__ void __launch_bounds__(1024)
b_finalize_kernel(const SysDev* __restrict__ sys, SysState* st, int nsys, const double* __restrict__ partials,
                  double* __restrict__ ring, int ring_cap, int mode, BatchFlags* fl) {
    int sidx = blockIdx.x;
    const SysDev& S = sys[sidx];
    SysState& T = st[sidx];
    if (mode == 0 && !T.active) return;
    // thread 0 loads the state it updates before the reduction, so that those
    // loads overlap the partials' (only this block changes them while it runs)
    double t0 = 0, pe0 = 0, vir0 = 0;
    long long steps0 = 0;
    int slot = 0;
    if (threadIdx.x == 0) {
        t0 = T.t;
        pe0 = T.pe;
        vir0 = T.vir;
        steps0 = T.steps;
        slot = fl->slot;
    }
    double acc[4] = {0, 0, 0, 0};
    int off = mode == 2 ? S.blk_off : S.fblk_off, nb = mode == 2 ? S.nblk : S.nfblk;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] += partials[(size_t)(off + b) * 4 + q];
    block_sum<4, 1024>(acc);
    if (threadIdx.x == 0) {
        double pe = pe0, vir = vir0, t = t0;
        if (mode != 2) {
            pe = 0.5 * acc[1];
            vir = 0.5 * acc[2];
            T.pe = pe;
            T.vir = vir;
        }
        double* out = ring + 7 * ((size_t)(mode == 0 ? slot : ring_cap) * nsys + sidx);
        if (mode == 0) {
            t = t0 + S.pp.dt;
            T.t = t;
            T.steps = steps0 + 1;
        }
        double ke = 0.5 * acc[0];
        if (mode != 1) {
            out[0] = t;
            out[1] = ke;
            out[2] = pe;
            out[3] = pe + ke;
            out[4] = vir;
            out[5] = (2. / 3.) * ke / (double)S.natoms;
            out[6] = acc[3] / (double)S.natoms;
        }
        if (!isfinite(ke) || !isfinite(pe) || !isfinite(vir)) atomicExch(&fl->nonfinite, 1);
        if (mode == 0) {
            T.max_disp2 = 0ull;
            T.need_rebuild = 0;
            T.rebuild = 0;
        }
    }
}

// Measurement partial sums without a step (for set_temperature / measure).
static __global__ void __launch_bounds__(kThreads)
b_measure_kernel(const int* __restrict__ blk_sys, const int* __restrict__ blk_first, const SysDev* __restrict__ sys,
                 Soa s, double* __restrict__ partials) {
    int sidx = blk_sys[blockIdx.x];
    const SysDev& S = sys[sidx];
    int i = blk_first[blockIdx.x] + threadIdx.x;
    double acc[4] = {0, 0, 0, 0};
    if (i < S.atom_off + S.natoms) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double v = s.at(VX + k, i), d = s.at(DX + k, i);
            acc[0] = fma(v, v, acc[0]);
            acc[3] = fma(d, d, acc[3]);
        }
    }
    block_sum<4, kThreads>(acc);
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; ++q) partials[(size_t)blockIdx.x * 4 + q] = acc[q];
}

static __global__ void __launch_bounds__(kThreads)
b_scale_kernel(int first, int n, Soa s, double factor) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int k = 0; k < 3; ++k) s.at(VX + k, first + i) = __dmul_rn(s.at(VX + k, first + i), factor);
}

static __global__ void b_unpack_kernel(int first, int n, const double* __restrict__ in, int stride, int field,
                                       double4* __restrict__ pos, Soa s, int* __restrict__ ids) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* p = in + (size_t)i * stride;
    int k = first + i;
    if (field < 0) {
        pos[k] = make_double4(p[0], p[1], p[2], 0.0);
        ids[k] = i;
    } else {
        for (int q = 0; q < 3; ++q) s.at(field + q, k) = p[q];
    }
}

static __global__ void b_pack_kernel(int first, int n, double* __restrict__ out, int stride, int field,
                                     const double4* __restrict__ pos, Soa s, const int* __restrict__ ids) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int slot = first + k;
    double* p = out + (size_t)ids[slot] * stride;
    double v[3];
    if (field < 0) {
        double4 x = pos[slot];
        v[0] = x.x; v[1] = x.y; v[2] = x.z;
    } else {
        for (int q = 0; q < 3; ++q) v[q] = s.at(field + q, slot);
    }
    for (int q = 0; q < 3; ++q) p[q] = v[q];
    if (stride == 4) p[3] = 0.0;
}

int hiword_b(double x) {
    long long b;
    std::memcpy(&b, &x, 8);
    return (int)(b >> 32);
}

}  // namespace

struct lj_batch {
    int nsys = 0, Ntot = 0, ncell = 0, nblk = 0, cap = 0, device = 0;
    cudaStream_t stream = nullptr, side = nullptr;
    std::vector<SysDev> hsys;
    SysDev* sys = nullptr;
    SysState* st = nullptr;
    BatchFlags* fl = nullptr;
    int *blk_sys = nullptr, *blk_first = nullptr, *sys_of = nullptr, *cell_sys = nullptr;
    int force_block = kThreads, nfblk = 0;
    int list_tile = kBuildWarps;  // list cells (warps) per block of the list build
    int *fblk_sys = nullptr, *fblk_first = nullptr;  // pair-kernel block tables (room for 64-atom blocks)
    double4 *pos = nullptr, *pos_tmp = nullptr;
    float4* posf = nullptr;
    double *soa = nullptr, *soa_tmp = nullptr, *bd = nullptr, *partials = nullptr, *ring = nullptr;
    double* host_ring = nullptr;
    int ring_cap = 256;
    int *ids = nullptr, *ids_tmp = nullptr, *cell_of = nullptr, *rank = nullptr, *order = nullptr;
    int *count = nullptr, *start = nullptr, *cnt = nullptr;
    uint4* nbr = nullptr;
    double* dstats = nullptr;  // window statistics: nsys x 6 results, then nsys densities
    int* natoms = nullptr;     // atoms per system
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    bool graph_tried = false;
    int loop_limit_override = 0;  // > 0: iteration bound of a chunk launch (testing the timeout path)
    long long chunk_launches = 0;
    long long host_steps = 0;
    long long launches = 0;
    char err[512] = {0};
};

namespace {

#define BK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            std::snprintf(b->err, sizeof b->err, "%s: %s", #call, cudaGetErrorString(e_));        \
            return LJ_ERR_CUDA;                                                                   \
        }                                                                                         \
    } while (0)
#define BKL()                                                                                      \
    do {                                                                                           \
        ++b->launches;                                                                             \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess) {                                                                   \
            std::snprintf(b->err, sizeof b->err, "launch: %s", cudaGetErrorString(e_));            \
            return LJ_ERR_CUDA;                                                                    \
        }                                                                                          \
    } while (0)

int nb(int n, int t = kThreads) { return (n + t - 1) / t; }

int launch_rebuild_b(lj_batch* b) {
    Soa s{b->soa, b->Ntot}, st{b->soa_tmp, b->Ntot};
    b_bin_kernel<<<nb(b->Ntot), kThreads, 0, b->stream>>>(b->sys_of, b->sys, b->st, b->Ntot, b->pos, b->cell_of,
                                                          b->rank, b->count);
    BKL();
    b_scan_kernel<<<b->nsys, 1024, 0, b->stream>>>(b->sys, b->st, b->count, b->start);
    BKL();
    b_scatter_kernel<<<nb(b->Ntot), kThreads, 0, b->stream>>>(b->sys_of, b->st, b->Ntot, b->cell_of, b->rank,
                                                              b->start, b->order);
    BKL();
    b_cell_sort_kernel<<<nb(b->ncell, kSortWarps), 32 * kSortWarps, 0, b->stream>>>(b->cell_sys, b->st, b->ncell,
                                                                                   b->start, b->order);
    BKL();
    b_gather_kernel<<<nb(b->Ntot), kThreads, 0, b->stream>>>(b->sys_of, b->st, b->Ntot, b->order, b->pos,
                                                             b->pos_tmp, s, st, b->ids, b->ids_tmp, b->bd);
    BKL();
    b_copy_back_kernel<<<nb(b->Ntot), kThreads, 0, b->stream>>>(b->sys_of, b->st, b->Ntot, b->pos_tmp, b->pos, st, s,
                                                                b->ids_tmp, b->ids, b->posf);
    BKL();
#define LJ_BBUILD(W)                                                                                 \
    b_build_list_kernel<W><<<nb(b->ncell, W), 32 * W, 0, b->stream>>>(b->cell_sys, b->sys, b->st, b->ncell, \
                                                                      b->Ntot, b->posf, b->start, b->cap,   \
                                                                      b->nbr, b->cnt, b->fl)
    if (b->list_tile == 2) LJ_BBUILD(2);
    else if (b->list_tile == 8) LJ_BBUILD(8);
    else LJ_BBUILD(4);
#undef LJ_BBUILD
    BKL();
    return LJ_OK;
}

int launch_step_b(lj_batch* b, cudaGraphConditionalHandle* h) {
    Soa s{b->soa, b->Ntot};
    b_kick_drift_kernel<<<b->nblk, kThreads, 0, b->stream>>>(b->blk_sys, b->blk_first, b->sys, b->st, b->Ntot, b->pos,
                                                             s, b->bd);
    BKL();
    b_decide_kernel<<<1, 256, 0, b->stream>>>(b->sys, b->st, b->nsys, b->fl, b->ring_cap,
                                              h ? *h : cudaGraphConditionalHandle{}, h ? 1 : 0);
    BKL();
    return LJ_OK;
}

int launch_force_b(lj_batch* b) {
    Soa s{b->soa, b->Ntot};
#define LJ_BFORCE(BS)                                                                                          \
    b_force_kernel<BS><<<b->nfblk, BS, 0, b->stream>>>(b->fblk_sys, b->fblk_first, b->sys, b->st, b->Ntot, b->pos, s, \
                                                      b->nbr, b->cnt, b->partials)
    if (b->force_block == 64) LJ_BFORCE(64);
    else if (b->force_block == 256) LJ_BFORCE(256);
    else LJ_BFORCE(128);
#undef LJ_BFORCE
    BKL();
    b_finalize_kernel<<<b->nsys, 1024, 0, b->stream>>>(b->sys, b->st, b->nsys, b->partials, b->ring, b->ring_cap, 0,
                                                       b->fl);
    BKL();
    return LJ_OK;
}

// One step launched kernel by kernel (the rebuild chain always runs; its kernels skip
// the systems that do not rebuild).
int direct_step_b(lj_batch* b) {
    int rc = launch_step_b(b, nullptr);
    if (!rc) rc = launch_rebuild_b(b);
    if (!rc) rc = launch_force_b(b);
    return rc;
}

constexpr int kBatchGraphSteps = 8;

// Capture kBatchGraphSteps steps onto b->stream, which is capturing into some
// graph: per step kick_drift -> decide -> IF(rebuild chain, captured on
// b->side) -> force -> finalize.
int capture_steps_b(lj_batch* b) {
    cudaStream_t main = b->stream;
    int rc = LJ_OK;
    for (int k = 0; k < kBatchGraphSteps && rc == LJ_OK; ++k) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        cudaGraphConditionalHandle h;
        if (cudaStreamGetCaptureInfo(main, &cs, nullptr, &g, &deps, &ndeps) != cudaSuccess ||
            cudaGraphConditionalHandleCreate(&h, g, 0, 0) != cudaSuccess) {
            rc = LJ_ERR_CUDA;
            break;
        }
        if ((rc = launch_step_b(b, &h))) break;
        if (cudaStreamGetCaptureInfo(main, &cs, nullptr, &g, &deps, &ndeps) != cudaSuccess) {
            rc = LJ_ERR_CUDA;
            break;
        }
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        if (cudaGraphAddNode(&cnode, g, deps, ndeps, &cp) != cudaSuccess ||
            cudaStreamUpdateCaptureDependencies(main, &cnode, 1, cudaStreamSetCaptureDependencies) != cudaSuccess ||
            cudaStreamBeginCaptureToGraph(b->side, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            rc = LJ_ERR_CUDA;
            break;
        }
        b->stream = b->side;
        rc = launch_rebuild_b(b);
        b->stream = main;
        cudaGraph_t body = nullptr;
        if (cudaStreamEndCapture(b->side, &body) != cudaSuccess && rc == LJ_OK) rc = LJ_ERR_CUDA;
        if (rc) break;
        rc = launch_force_b(b);
    }
    b->stream = main;
    return rc;
}

// The chunk graph: one WHILE conditional node whose body is kBatchGraphSteps
// steps followed by b_loop_kernel, so that one launch runs a whole chunk of
// loop_left * kBatchGraphSteps steps with no host involvement (the loop
// handle restarts at 1 on every launch: the body runs at least once).
int build_graph_b(lj_batch* b) {
    long long l0 = b->launches;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = LJ_OK;
    cudaGraphConditionalHandle hw;
    cudaGraphNodeParams wp = {};
    cudaGraphNode_t wn;
    if (cudaGraphCreate(&graph, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&hw, graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
        rc = LJ_ERR_CUDA;
    } else {
        wp.type = cudaGraphNodeTypeConditional;
        wp.conditional.handle = hw;
        wp.conditional.type = cudaGraphCondTypeWhile;
        wp.conditional.size = 1;
        if (cudaGraphAddNode(&wn, graph, nullptr, 0, &wp) != cudaSuccess ||
            cudaStreamBeginCaptureToGraph(b->stream, wp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            rc = LJ_ERR_CUDA;
        } else {
            rc = capture_steps_b(b);
            if (rc == LJ_OK) {
                b_loop_kernel<<<1, 1, 0, b->stream>>>(b->fl, hw);
                if (cudaGetLastError() != cudaSuccess) rc = LJ_ERR_CUDA;
            }
            cudaGraph_t body = nullptr;
            if (cudaStreamEndCapture(b->stream, &body) != cudaSuccess && rc == LJ_OK) rc = LJ_ERR_CUDA;
        }
    }
    b->launches = l0;  // captured launches are not executions
    if (rc == LJ_OK && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        b->graph = exec;
        b->graph_steps = kBatchGraphSteps;
    } else {
        b->graph = nullptr;
        b->graph_steps = 0;
        rc = LJ_ERR_CUDA;
        cudaGetLastError();
    }
    if (graph) cudaGraphDestroy(graph);
    return rc;
}

// Enqueue nsteps steps: one chunk-graph launch for the whole multiples of
// kBatchGraphSteps (its loop count and bound set on the device first), single
// launches for the rest.
int enqueue_b(lj_batch* b, int nsteps) {
    if (!b->graph_tried) {
        b->graph_tried = true;
        build_graph_b(b);
    }
    int s = 0;
    if (b->graph_steps > 0 && nsteps >= b->graph_steps) {
        int iters = nsteps / b->graph_steps;
        struct {
            int loop_left, timeout;
            long long loop_iters, loop_limit;
        } ctl = {iters, 0, 0, b->loop_limit_override > 0 ? b->loop_limit_override : iters};
        static_assert(sizeof ctl == sizeof(BatchFlags) - offsetof(BatchFlags, loop_left), "loop fields");
        BK(cudaMemcpyAsync(&b->fl->loop_left, &ctl, sizeof ctl, cudaMemcpyHostToDevice, b->stream));
        BK(cudaGraphLaunch(b->graph, b->stream));
        ++b->chunk_launches;
        s = iters * b->graph_steps;
    }
    for (; s < nsteps; ++s) {
        int rc = direct_step_b(b);
        if (rc) return rc;
    }
    b->host_steps += nsteps;
    return LJ_OK;
}

int read_flags_b(lj_batch* b) {
    BatchFlags h;
    BK(cudaMemcpyAsync(&h, b->fl, sizeof h, cudaMemcpyDeviceToHost, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    if (h.overflow) {
        std::snprintf(b->err, sizeof b->err, "neighbour list capacity exceeded");
        return LJ_ERR_CAPACITY;
    }
    if (h.nonfinite) {
        std::snprintf(b->err, sizeof b->err, "non-finite energy or virial");
        return LJ_ERR_NONFINITE;
    }
    if (h.timeout) {
        // the launch took fewer steps than were enqueued: follow the device's
        // step count (the ring slots) and clear the flag for the next call
        b->host_steps = h.step_count;
        BK(cudaMemsetAsync(&b->fl->timeout, 0, sizeof(int), b->stream));
        BK(cudaStreamSynchronize(b->stream));
        std::snprintf(b->err, sizeof b->err, "a chunk launch stopped at its iteration bound (%lld iterations)",
                      h.loop_iters);
        return LJ_ERR_TIMEOUT;
    }
    return LJ_OK;
}

void free_b(lj_batch* b) {
    void* ptrs[] = {b->sys, b->st, b->fl, b->blk_sys, b->blk_first, b->fblk_sys, b->fblk_first, b->sys_of, b->cell_sys, b->pos, b->pos_tmp,
                    b->posf, b->soa, b->soa_tmp, b->bd, b->partials, b->ring, b->ids, b->ids_tmp, b->cell_of,
                    b->rank, b->order, b->count, b->start, b->cnt, b->nbr, b->dstats, b->natoms};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (b->host_ring) cudaFreeHost(b->host_ring);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->stream) cudaStreamDestroy(b->stream);
}

// Pair-kernel block tables for blocks of bs atoms (each block inside one
// system, as the single-system pair kernel of that block size partitions it),
// uploaded with the system table; the chunk graph is rebuilt on next use.
int set_force_blocks(lj_batch* b, int bs) {
    std::vector<int> fs, ff;
    int off = 0;
    for (SysDev& S : b->hsys) {
        S.fblk_off = off;
        S.nfblk = (S.natoms + bs - 1) / bs;
        for (int j = 0; j < S.nfblk; ++j) {
            fs.push_back((int)(&S - b->hsys.data()));
            ff.push_back(S.atom_off + j * bs);
        }
        off += S.nfblk;
    }
    BK(cudaMemcpy(b->fblk_sys, fs.data(), sizeof(int) * fs.size(), cudaMemcpyHostToDevice));
    BK(cudaMemcpy(b->fblk_first, ff.data(), sizeof(int) * ff.size(), cudaMemcpyHostToDevice));
    BK(cudaMemcpy(b->sys, b->hsys.data(), sizeof(SysDev) * b->nsys, cudaMemcpyHostToDevice));
    b->force_block = bs;
    b->nfblk = off;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = 0;
    b->graph_tried = false;
    return LJ_OK;
}

}  // namespace

extern "C" {

int lj_batch_create(const lj_batch_system* systems, int nsys, double cutoff, int device, lj_batch** out) {
    if (!systems || nsys < 1 || !out || !(cutoff * cutoff > std::cbrt(2.0))) return LJ_ERR_ARG;
    *out = nullptr;
    lj_batch* b = new (std::nothrow) lj_batch();
    if (!b) return LJ_ERR_ARG;
    b->nsys = nsys;
    b->device = device;
    double rc = cutoff;
    long long Ntot = 0, ncell = 0, nblk = 0;
    double rho_max = 0, cutmax = 0;
    b->hsys.resize((size_t)nsys);
    for (int s = 0; s < nsys; ++s) {
        const lj_batch_system& q = systems[s];
        SysDev& S = b->hsys[(size_t)s];
        std::memset(&S, 0, sizeof S);
        if (q.particle_count < 1) { delete b; return LJ_ERR_ARG; }
        double Lmin = std::min(q.box[0], std::min(q.box[1], q.box[2]));
        if (!(Lmin >= 3 * rc)) { delete b; return LJ_ERR_ARG; }  // needs >= 3 cells of edge rc per axis
        double skin = list_skin(q.skin, Lmin, rc);
        S.atom_off = (int)Ntot;
        S.natoms = q.particle_count;
        PairParams& pp = S.pp;
        pp.rc = rc;
        pp.rc2 = rc * rc;
        pp.inv_rc2 = 1.0 / pp.rc2;
        double rcm6 = 1 / (pp.rc2 * pp.rc2 * pp.rc2);
        pp.alpha = -4.0 * rcm6 * (rcm6 - 1.0);
        pp.beta = 12.0 * rcm6 * (2.0 * rcm6 - 1.0);
        pp.dt = q.time_delta;
        double near = rc * (1.0 + 1e-9);
        pp.near_lo = near;
        double Lmax = 0;
        for (int k = 0; k < 3; ++k) {
            pp.L[k] = q.box[k];
            pp.halfL[k] = 0.5 * q.box[k];
            pp.halfL_hi[k] = hiword_b(0.5 * q.box[k]);
            pp.near_hi[k] = q.box[k] - near;
            S.grid.n[k] = std::max(1, (int)std::floor(q.box[k] / (rc + skin)));
            S.grid.ratio[k] = (double)S.grid.n[k] / q.box[k];
            Lmax = std::max(Lmax, q.box[k]);
        }
        double h = 0.5 * skin;
        S.thresh2 = h * h * 0.999;
        S.always = skin == 0.0 ? 1 : 0;
        double cut = rc + skin + 8.0 * Lmax * std::ldexp(1.0, -24) + 1e-6;
        S.cut2 = (float)(cut * cut);
        S.Lf = make_float3((float)q.box[0], (float)q.box[1], (float)q.box[2]);
        S.cell_off = (int)ncell;
        S.ncell = S.grid.ncell();
        S.blk_off = (int)nblk;
        S.nblk = (q.particle_count + kThreads - 1) / kThreads;
        Ntot += q.particle_count;
        ncell += S.ncell;
        nblk += S.nblk;
        rho_max = std::max(rho_max, q.particle_count / (q.box[0] * q.box[1] * q.box[2]));
        cutmax = std::max(cutmax, rc + skin);
    }
    if (Ntot >= kMaxAtoms) { delete b; return LJ_ERR_ARG; }
    b->Ntot = (int)Ntot;
    b->ncell = (int)ncell;
    b->nblk = (int)nblk;
    double expect = 4.0 / 3.0 * M_PI * cutmax * cutmax * cutmax * std::max(rho_max, 1.2);
    b->cap = ((int)std::ceil(1.5 * expect + 32) + 3) & ~3;
    // device set-up; on an error everything allocated so far is released
    auto init = [&]() -> int {
        BK(cudaSetDevice(device));
        BK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        BK(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking));
        int N = b->Ntot;
        std::vector<int> blk_sys((size_t)nblk), blk_first((size_t)nblk), sys_of((size_t)N), cell_sys((size_t)ncell);
        for (int s = 0; s < nsys; ++s) {
            const SysDev& S = b->hsys[(size_t)s];
            for (int j = 0; j < S.nblk; ++j) {
                blk_sys[(size_t)(S.blk_off + j)] = s;
                blk_first[(size_t)(S.blk_off + j)] = S.atom_off + j * kThreads;
            }
            for (int i = 0; i < S.natoms; ++i) sys_of[(size_t)(S.atom_off + i)] = s;
            for (int c = 0; c < S.ncell; ++c) cell_sys[(size_t)(S.cell_off + c)] = s;
        }
        BK(cudaMalloc(&b->sys, sizeof(SysDev) * nsys));
        BK(cudaMalloc(&b->st, sizeof(SysState) * nsys));
        BK(cudaMalloc(&b->fl, sizeof(BatchFlags)));
        BK(cudaMalloc(&b->blk_sys, sizeof(int) * nblk));
        BK(cudaMalloc(&b->blk_first, sizeof(int) * nblk));
        BK(cudaMalloc(&b->sys_of, sizeof(int) * N));
        BK(cudaMalloc(&b->cell_sys, sizeof(int) * ncell));
        BK(cudaMalloc(&b->pos, sizeof(double4) * (N + 1)));
        BK(cudaMalloc(&b->pos_tmp, sizeof(double4) * N));
        BK(cudaMalloc(&b->posf, sizeof(float4) * (N + 1)));
        BK(cudaMalloc(&b->soa, sizeof(double) * SOA_FIELDS * N));
        BK(cudaMalloc(&b->soa_tmp, sizeof(double) * SOA_FIELDS * N));
        BK(cudaMalloc(&b->bd, sizeof(double) * 3 * N));
        long long nfblk64 = 0;
        for (const SysDev& S : b->hsys) nfblk64 += (S.natoms + 63) / 64;
        BK(cudaMalloc(&b->fblk_sys, sizeof(int) * nfblk64));
        BK(cudaMalloc(&b->fblk_first, sizeof(int) * nfblk64));
        BK(cudaMalloc(&b->partials, sizeof(double) * 4 * std::max<long long>(nblk, nfblk64)));
        BK(cudaMalloc(&b->ring, sizeof(double) * 7 * (size_t)(b->ring_cap + 1) * nsys));
        BK(cudaMallocHost(&b->host_ring, sizeof(double) * 7 * (size_t)(b->ring_cap + 1) * nsys));
        BK(cudaMalloc(&b->ids, sizeof(int) * N));
        BK(cudaMalloc(&b->ids_tmp, sizeof(int) * N));
        BK(cudaMalloc(&b->cell_of, sizeof(int) * N));
        BK(cudaMalloc(&b->rank, sizeof(int) * N));
        BK(cudaMalloc(&b->order, sizeof(int) * N));
        BK(cudaMalloc(&b->count, sizeof(int) * ncell));
        BK(cudaMalloc(&b->start, sizeof(int) * (ncell + 1)));
        BK(cudaMalloc(&b->cnt, sizeof(int) * N));
        BK(cudaMalloc(&b->nbr, sizeof(uint4) * (size_t)(b->cap / 4) * N));
        BK(cudaMalloc(&b->dstats, sizeof(double) * 7 * nsys));
        BK(cudaMalloc(&b->natoms, sizeof(int) * nsys));
        {
            std::vector<int> na((size_t)nsys);
            for (int s = 0; s < nsys; ++s) na[(size_t)s] = b->hsys[(size_t)s].natoms;
            BK(cudaMemcpy(b->natoms, na.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice));
        }
        BK(cudaMemcpy(b->sys, b->hsys.data(), sizeof(SysDev) * nsys, cudaMemcpyHostToDevice));
        std::vector<SysState> st0((size_t)nsys);
        for (auto& q : st0) {
            std::memset(&q, 0, sizeof q);
            q.active = 1;
            q.need_rebuild = 1;
        }
        BK(cudaMemcpy(b->st, st0.data(), sizeof(SysState) * nsys, cudaMemcpyHostToDevice));
        BK(cudaMemset(b->fl, 0, sizeof(BatchFlags)));
        BK(cudaMemcpy(b->blk_sys, blk_sys.data(), sizeof(int) * nblk, cudaMemcpyHostToDevice));
        BK(cudaMemcpy(b->blk_first, blk_first.data(), sizeof(int) * nblk, cudaMemcpyHostToDevice));
        BK(cudaMemcpy(b->sys_of, sys_of.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
        BK(cudaMemcpy(b->cell_sys, cell_sys.data(), sizeof(int) * ncell, cudaMemcpyHostToDevice));
        BK(cudaMemset(b->pos, 0, sizeof(double4) * N));
        BK(cudaMemset(b->soa, 0, sizeof(double) * SOA_FIELDS * N));
        BK(cudaMemset(b->bd, 0, sizeof(double) * 3 * N));
        BK(cudaMemset(b->count, 0, sizeof(int) * ncell));
        BK(cudaMemset(b->cnt, 0, sizeof(int) * N));
        const double4 ghost = make_double4(1e18, 1e18, 1e18, 0.0);
        const float4 ghostf = make_float4(1e18f, 1e18f, 1e18f, 0.f);
        BK(cudaMemcpy(b->pos + N, &ghost, sizeof ghost, cudaMemcpyHostToDevice));
        BK(cudaMemcpy(b->posf + N, &ghostf, sizeof ghostf, cudaMemcpyHostToDevice));
        std::vector<int> ident((size_t)N);
        for (int s = 0; s < nsys; ++s)
            for (int i = 0; i < b->hsys[(size_t)s].natoms; ++i) ident[(size_t)(b->hsys[(size_t)s].atom_off + i)] = i;
        BK(cudaMemcpy(b->ids, ident.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
        int sentinel = N;
        BK(cudaMemcpy(b->start + ncell, &sentinel, sizeof(int), cudaMemcpyHostToDevice));
        return set_force_blocks(b, kThreads);
    };
    if (int rc = init()) {
        cudaSetDevice(device);
        if (b->stream) cudaStreamSynchronize(b->stream);
        free_b(b);
        delete b;
        return rc;
    }
    *out = b;
    return LJ_OK;
}

int lj_batch_destroy(lj_batch* b) {
    if (!b) return LJ_ERR_ARG;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_b(b);
    delete b;
    return LJ_OK;
}

const char* lj_batch_last_error(const lj_batch* b) { return b ? b->err : "null batch"; }

int lj_batch_upload_system(lj_batch* b, int sys, const double* x, const double* v, int stride) {
    if (!b || sys < 0 || sys >= b->nsys || !x || (stride != 3 && stride != 4)) return LJ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    const SysDev& S = b->hsys[(size_t)sys];
    int n = S.natoms;
    double* stage = reinterpret_cast<double*>(b->pos_tmp) + 4 * (size_t)S.atom_off;  // this system's room
    Soa s{b->soa, b->Ntot};
    const double* src[2] = {x, v};
    int field[2] = {-1, VX};
    for (int q = 0; q < 2; ++q) {
        if (!src[q]) {
            BK(cudaMemsetAsync(b->soa + (size_t)VX * b->Ntot + S.atom_off, 0, sizeof(double) * n, b->stream));
            BK(cudaMemsetAsync(b->soa + (size_t)VY * b->Ntot + S.atom_off, 0, sizeof(double) * n, b->stream));
            BK(cudaMemsetAsync(b->soa + (size_t)VZ * b->Ntot + S.atom_off, 0, sizeof(double) * n, b->stream));
            continue;
        }
        BK(cudaMemcpyAsync(stage, src[q], sizeof(double) * stride * n, cudaMemcpyHostToDevice, b->stream));
        b_unpack_kernel<<<nb(n), kThreads, 0, b->stream>>>(S.atom_off, n, stage, stride, field[q], b->pos, s, b->ids);
        BKL();
    }
    for (int f : {DX, DY, DZ, FX, FY, FZ})
        BK(cudaMemsetAsync(b->soa + (size_t)f * b->Ntot + S.atom_off, 0, sizeof(double) * n, b->stream));
    SysState q;
    std::memset(&q, 0, sizeof q);
    q.active = 1;
    q.need_rebuild = 1;
    BK(cudaMemcpyAsync(b->st + sys, &q, sizeof q, cudaMemcpyHostToDevice, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    return LJ_OK;
}

int lj_batch_download_system(lj_batch* b, int sys, double* x, double* v, double* F, int stride) {
    if (!b || sys < 0 || sys >= b->nsys || (stride != 3 && stride != 4)) return LJ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    const SysDev& S = b->hsys[(size_t)sys];
    int n = S.natoms;
    double* stage = reinterpret_cast<double*>(b->pos_tmp) + 4 * (size_t)S.atom_off;
    Soa s{b->soa, b->Ntot};
    double* dst[3] = {x, v, F};
    int field[3] = {-1, VX, FX};
    for (int q = 0; q < 3; ++q) {
        if (!dst[q]) continue;
        b_pack_kernel<<<nb(n), kThreads, 0, b->stream>>>(S.atom_off, n, stage, stride, field[q], b->pos, s, b->ids);
        BKL();
        BK(cudaMemcpyAsync(dst[q], stage, sizeof(double) * stride * n, cudaMemcpyDeviceToHost, b->stream));
    }
    BK(cudaStreamSynchronize(b->stream));
    return LJ_OK;
}

int lj_batch_set_active(lj_batch* b, int sys, int active) {
    if (!b || sys < 0 || sys >= b->nsys) return LJ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    int a = active ? 1 : 0;
    BK(cudaMemcpyAsync(&b->st[sys].active, &a, sizeof(int), cudaMemcpyHostToDevice, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    return LJ_OK;
}

// nsteps steps of every active system; out (may be NULL) receives nsteps x nsys
// records (step-major; inactive systems' records are left as they were).
int lj_batch_step(lj_batch* b, int nsteps, lj_thermo* out) {
    if (!b || nsteps < 0) return LJ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    int done = 0;
    size_t per = 7 * (size_t)b->nsys;
    while (done < nsteps) {
        int chunk = std::min(nsteps - done, b->ring_cap);
        long long first = b->host_steps;
        int rc = enqueue_b(b, chunk);
        if (rc) return rc;
        if (out) {
            int s0 = (int)(first % b->ring_cap);
            int n1 = std::min(chunk, b->ring_cap - s0);
            BK(cudaMemcpyAsync(b->host_ring, b->ring + per * s0, sizeof(double) * per * n1, cudaMemcpyDeviceToHost,
                               b->stream));
            if (n1 < chunk)
                BK(cudaMemcpyAsync(b->host_ring + per * n1, b->ring, sizeof(double) * per * (chunk - n1),
                                   cudaMemcpyDeviceToHost, b->stream));
        }
        if ((rc = read_flags_b(b))) return rc;
        if (out) std::memcpy(out + (size_t)done * b->nsys, b->host_ring, sizeof(double) * per * chunk);
        done += chunk;
    }
    return LJ_OK;
}

// Instantaneous measurement of every system: out receives nsys records.
int lj_batch_measure(lj_batch* b, lj_thermo* out) {
    if (!b || !out) return LJ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    Soa s{b->soa, b->Ntot};
    b_measure_kernel<<<b->nblk, kThreads, 0, b->stream>>>(b->blk_sys, b->blk_first, b->sys, s, b->partials);
    BKL();
    b_finalize_kernel<<<b->nsys, 1024, 0, b->stream>>>(b->sys, b->st, b->nsys, b->partials, b->ring, b->ring_cap, 2,
                                                       b->fl);
    BKL();
    size_t per = 7 * (size_t)b->nsys;
    BK(cudaMemcpyAsync(b->host_ring, b->ring + per * b->ring_cap, sizeof(double) * per, cudaMemcpyDeviceToHost,
                       b->stream));
    BK(cudaStreamSynchronize(b->stream));
    std::memcpy(out, b->host_ring, sizeof(double) * per);
    return LJ_OK;
}

// physics::set_temperature for one system.
int lj_batch_set_temperature(lj_batch* b, int sys, double target, double* measured) {
    if (!b || sys < 0 || sys >= b->nsys || !(target >= 0)) return LJ_ERR_ARG;
    std::vector<lj_thermo> m((size_t)b->nsys);
    int rc = lj_batch_measure(b, m.data());
    if (rc) return rc;
    double T = m[(size_t)sys].temperature;
    if (!(T > 0)) return LJ_ERR_ARG;
    if (measured) *measured = T;
    const SysDev& S = b->hsys[(size_t)sys];
    Soa s{b->soa, b->Ntot};
    b_scale_kernel<<<nb(S.natoms), kThreads, 0, b->stream>>>(S.atom_off, S.natoms, s, std::sqrt(target / T));
    BKL();
    BK(cudaStreamSynchronize(b->stream));
    return LJ_OK;
}

int lj_batch_set_force_block(lj_batch* b, int force_block) {
    if (!b || (force_block != 64 && force_block != 128 && force_block != 256)) return LJ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    BK(cudaStreamSynchronize(b->stream));
    return set_force_blocks(b, force_block);
}

int lj_batch_set_list_tile(lj_batch* b, int cells) {
    if (!b || (cells != 2 && cells != 4 && cells != 8)) return LJ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    BK(cudaStreamSynchronize(b->stream));
    b->list_tile = cells;
    if (b->graph) cudaGraphExecDestroy(b->graph);  // the chunk graph holds the old launch shape
    b->graph = nullptr;
    b->graph_steps = 0;
    b->graph_tried = false;
    return LJ_OK;
}

int lj_batch_set_iteration_limit(lj_batch* b, int limit) {
    if (!b || limit < 0) return LJ_ERR_ARG;
    b->loop_limit_override = limit;
    return LJ_OK;
}

int lj_batch_window_stats(lj_batch* b, int sample_size, const double* density, lj_observation* out) {
    if (!b || !density || !out || sample_size < 2 || sample_size > b->ring_cap || sample_size > b->host_steps)
        return LJ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    double* dens = b->dstats + 6 * (size_t)b->nsys;
    BK(cudaMemcpyAsync(dens, density, sizeof(double) * b->nsys, cudaMemcpyHostToDevice, b->stream));
    window_stats_kernel<<<b->nsys, kStatsThreads, 0, b->stream>>>(b->ring, b->ring_cap, b->nsys, b->host_steps - 1,
                                                                 sample_size, b->natoms, dens, b->dstats);
    BKL();
    static_assert(sizeof(lj_observation) == 6 * sizeof(double), "lj_observation is 6 doubles");
    BK(cudaMemcpyAsync(out, b->dstats, sizeof(double) * 6 * b->nsys, cudaMemcpyDeviceToHost, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    return LJ_OK;
}

// Batch autotuner: every candidate (Verlet skin of all systems x pair-kernel
// block size x list cells per list-build block) runs in a fresh batch from the
// caller's state -- 16 steps to build the chunk graph and the first lists,
// then `steps` timed steps -- and the fastest is returned.
int lj_batch_autotune(const lj_batch_system* systems, int nsys, double cutoff, int device, const double* x,
                      const double* v, int stride, int steps, lj_batch_tuning* best) {
    if (!systems || nsys < 1 || !x || !best || steps < 8 || (stride != 3 && stride != 4)) return LJ_ERR_ARG;
    const double skins[] = {0.2, 0.3, 0.4, 0.5};
    const int blocks[] = {64, 128, 256};
    const int tiles[] = {2, 4, 8};
    std::vector<lj_batch_system> table(systems, systems + nsys);
    lj_batch_tuning win{-1.0, 0, 0, 1e300};
    for (double sk : skins) {
        for (lj_batch_system& q : table) q.skin = sk;
        for (int cand = 0; cand < 9; ++cand) {
            int bs = blocks[cand / 3], tile = tiles[cand % 3];
            lj_batch* b = nullptr;
            int rc = lj_batch_create(table.data(), nsys, cutoff, device, &b);
            if (rc) return rc;
            rc = lj_batch_set_force_block(b, bs);
            if (!rc) rc = lj_batch_set_list_tile(b, tile);
            size_t off = 0;
            for (int s = 0; s < nsys && !rc; ++s) {
                rc = lj_batch_upload_system(b, s, x + off, v ? v + off : nullptr, stride);
                off += (size_t)stride * systems[s].particle_count;
            }
            if (!rc) rc = lj_batch_step(b, 16, nullptr);
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            float ms = 0.f;
            if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) rc = LJ_ERR_CUDA;
            if (!rc) {
                cudaEventRecord(e0, b->stream);
                rc = lj_batch_step(b, steps, nullptr);
                cudaEventRecord(e1, b->stream);
            }
            if (!rc && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
                rc = LJ_ERR_CUDA;
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            lj_batch_destroy(b);
            if (rc) return rc;
            if (ms / steps < win.ms_per_step) win = lj_batch_tuning{sk, bs, tile, (double)ms / steps};
        }
    }
    *best = win;
    return LJ_OK;
}

int lj_batch_info(const lj_batch* b, int* total_atoms, long long* builds_per_system, long long* kernel_launches) {
    if (!b) return LJ_ERR_ARG;
    if (total_atoms) *total_atoms = b->Ntot;
    if (builds_per_system) {
        std::vector<SysState> st((size_t)b->nsys);
        if (cudaMemcpy(st.data(), b->st, sizeof(SysState) * b->nsys, cudaMemcpyDeviceToHost) != cudaSuccess)
            return LJ_ERR_CUDA;
        for (int s = 0; s < b->nsys; ++s) builds_per_system[s] = st[(size_t)s].builds;
    }
    if (kernel_launches) *kernel_launches = b->launches;
    return LJ_OK;
}

}  // extern "C"
