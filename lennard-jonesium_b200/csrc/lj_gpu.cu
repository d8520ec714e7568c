// lj_gpu.cu -- host side of the C ABI declared in include/lj_gpu.h.
//
// One context = one system on one device, driven on the context's own stream.
// A velocity-Verlet step (integrator.cpp:62-88) is the launch sequence
//   kick_drift -> [rebuild chain] -> force (+ second kick + partial sums) -> finalize
// where the rebuild chain (cell binning by counting sort, neighbour list) is
// launched every step but returns at once unless the device-side skin
// criterion (max displacement since the last build > skin / 2) or the host
// asked for a rebuild.  Per-step records land in a device ring and are copied
// to the host once per lj_gpu_step call.

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lj_gpu.h"
#include "lj_kernels.cuh"
#include "lj_mixed.cuh"

using namespace ljb;

struct Trajectory;  // the trajectory stream (below)

// One instantiated step graph.
struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    int steps = 0;          // steps per launch
    int kernels = 0;        // kernel nodes outside the rebuild bodies
    long long launches = 0;
};

struct lj_ctx {
    lj_params p{};
    int N = 0;
    PairParams pp{};
    double skin = 0.0;
    bool small_box = false;
    bool rebuild_always = false;
    Grid list_grid{};
    Grid ref_grid{};
    int cap = 0;
    int nblocks = 0;      // blocks of kThreads atoms (integration, measurement)
    int force_block = 128;
    int fblocks = 0;      // blocks of the pair kernel
    cudaStream_t stream = nullptr;

    // device buffers
    double4* pos = nullptr;
    double4* pos_tmp = nullptr;
    double* soa = nullptr;
    double* soa_tmp = nullptr;
    double* bd = nullptr;
    int* ids = nullptr;
    int* ids_tmp = nullptr;
    int* cell_of = nullptr;
    int* rank = nullptr;
    int* order = nullptr;
    int* count = nullptr;
    int* start = nullptr;
    int* tile_sums = nullptr;
    uint4* nbr = nullptr;        // neighbour list, groups of 4 entries
    float4* posf = nullptr;      // FP32 copy of the sorted positions (list builds)
    int* cnt = nullptr;
    double* partials = nullptr;
    Scalars* sc = nullptr;
    double* ring = nullptr;     // ring_cap records of 7 doubles
    double* dscratch = nullptr; // small device scratch (set_temperature factor, L)
    double* dL = nullptr;
    double* dstats = nullptr;   // window statistics: 6 results, density, atom count
    int ring_cap = 0;
    double* host_ring = nullptr;  // pinned

    // second position buffers: a step graph's fused pair kernels write the next
    // step's positions here while this step's are still being read
    double4* pos_b = nullptr;
    float4* posl_b = nullptr;
    // mixed-precision buffers
    float4* posl = nullptr;
    double* bx = nullptr;  // x at build (unwrapped reference for local coordinates)

    // debug (reference grid) buffers, allocated on first use
    int* dbg_count = nullptr;
    int* dbg_start = nullptr;
    int* dbg_members = nullptr;
    int* dbg_cell_of = nullptr;
    int* dbg_tiles = nullptr;
    // RDF cell-list scratch and device accumulator, sized on first use
    RdfScratch rdf{};
    Trajectory* traj = nullptr;  // open trajectory stream, if any

    long long launches = 0;       // kernels launched directly (gated-off ones included)
    long long host_steps = 0;     // mirror of the device step counter
    // step graphs: kick_drift -> decide -> IF(rebuild chain) -> force -> finalize, unrolled;
    // a long one for runs of steps and a short one for the remainder
    cudaStream_t side = nullptr;  // captures the conditional body
    StepGraph graphs[2];
    bool graph_tried = false;
    int rebuild_kernels = 0;      // kernels in one rebuild chain
    // the rebuild chain as a graph of its own, for the per-phase timing pass
    cudaGraphExec_t rebuild_exec = nullptr;
    bool rebuild_graph_tried = false;
    int rebuild_graph_kernels = 0;
    char err[512] = {0};
};

namespace {

const char* kStatus[] = {"ok", "invalid argument", "CUDA error", "non-finite energy or virial",
                         "device loop reached its bound", "neighbour list capacity exceeded"};

int set_err(lj_ctx* c, int code, const char* msg) {
    if (c) std::snprintf(c->err, sizeof c->err, "%s", msg);
    return code;
}

#define CK(call)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            if (ctx) std::snprintf(ctx->err, sizeof ctx->err, "%s: %s (%s:%d)", #call, \
                                   cudaGetErrorString(e_), __FILE__, __LINE__);        \
            return LJ_ERR_CUDA;                                                        \
        }                                                                              \
    } while (0)

#define CKL()                                                                           \
    do {                                                                                \
        ++ctx->launches;                                                                \
        cudaError_t e_ = cudaGetLastError();                                            \
        if (e_ != cudaSuccess) {                                                        \
            std::snprintf(ctx->err, sizeof ctx->err, "launch: %s (%s:%d)",              \
                          cudaGetErrorString(e_), __FILE__, __LINE__);                  \
            return LJ_ERR_CUDA;                                                         \
        }                                                                               \
    } while (0)

int blocks_for(int n, int t = kThreads) { return (n + t - 1) / t; }

Grid make_grid(const double L[3], double cell_min) {
    Grid g;
    for (int k = 0; k < 3; ++k) {
        g.n[k] = std::max(1, (int)std::floor(L[k] / cell_min));
        g.ratio[k] = (double)g.n[k] / L[k];
    }
    return g;
}

int hiword(double x) {
    long long b;
    std::memcpy(&b, &x, 8);
    return (int)(b >> 32);
}

Gate gate_of(lj_ctx* c) {
    Gate g;
    g.sc = c->sc;
    double h = 0.5 * c->skin;
    g.thresh2 = h * h * 0.999;
    g.always = c->rebuild_always ? 1 : 0;
    return g;
}

Soa soa_of(double* p, int N) { return Soa{p, N}; }

}  // namespace

// Verlet skin for a box: the requested skin (default 0.3), shrunk so the list
// grid keeps >= 3 cells of edge >= rc + skin per axis (the minimum-image form);
// 0 (a rebuild every step) when that leaves less than 0.05.
double list_skin(double requested, double Lmin, double rc) {
    double skin = requested < 0 ? 0.3 : requested;
    double fit = Lmin / 3.0 - rc - 1e-9 * Lmin;
    if (skin > fit) skin = fit;
    return skin >= 0.05 ? skin : 0.0;
}

namespace {

// Counting sort of atoms into grid g (histogram, scan, scatter); rank/cell_of per slot.
template <bool GATED>
int launch_binning(lj_ctx* ctx, const Grid& g, int* count, int* start, int* tiles, Gate gate) {
    int nc = g.ncell();
    int ntiles = (nc + kScanTile - 1) / kScanTile;
    bin_count_kernel<GATED><<<blocks_for(ctx->N), kThreads, 0, ctx->stream>>>(
        ctx->N, ctx->pos, g, ctx->cell_of, ctx->rank, count, gate);
    CKL();
    scan_reduce_kernel<GATED><<<ntiles, 1024, 0, ctx->stream>>>(count, nc, tiles, gate);
    CKL();
    scan_tiles_kernel<GATED><<<1, 1024, 0, ctx->stream>>>(tiles, ntiles, gate);
    CKL();
    scan_apply_kernel<GATED><<<ntiles, 1024, 0, ctx->stream>>>(count, nc, tiles, start, gate);
    CKL();
    return LJ_OK;
}

// Rebuild chain: bin into the list grid, sort, gather, list.  Every kernel
// returns at once when the gate is closed.
int launch_rebuild(lj_ctx* ctx) {
    Gate gate = gate_of(ctx);
    int N = ctx->N;
    int rc = launch_binning<true>(ctx, ctx->list_grid, ctx->count, ctx->start, ctx->tile_sums, gate);
    if (rc) return rc;
    scatter_kernel<true><<<blocks_for(N), kThreads, 0, ctx->stream>>>(N, ctx->cell_of, ctx->rank,
                                                                        ctx->start, ctx->order, gate);
    CKL();
    cell_sort_kernel<true><<<blocks_for(ctx->list_grid.ncell(), kSortWarps), 32 * kSortWarps, 0, ctx->stream>>>(
        ctx->list_grid.ncell(), ctx->start, ctx->order, gate);
    CKL();
    gather_kernel<<<blocks_for(N), kThreads, 0, ctx->stream>>>(
        N, ctx->order, ctx->pos, ctx->pos_tmp, soa_of(ctx->soa, N), soa_of(ctx->soa_tmp, N), ctx->ids,
        ctx->ids_tmp, ctx->bd, gate);
    CKL();
    copy_back_kernel<<<blocks_for(N), kThreads, 0, ctx->stream>>>(
        N, ctx->pos_tmp, ctx->pos, soa_of(ctx->soa_tmp, N), soa_of(ctx->soa, N), ctx->ids_tmp, ctx->ids,
        ctx->posf, gate);
    CKL();
    // FP32 candidate radius, widened past FP32 rounding of box coordinates so the
    // list is a superset of the FP64 pair set
    double Lmax = std::max(ctx->pp.L[0], std::max(ctx->pp.L[1], ctx->pp.L[2]));
    double cut = ctx->pp.rc + ctx->skin + 8.0 * Lmax * std::ldexp(1.0, -24) + 1e-6;
    float cut2 = (float)(cut * cut);
    float3 Lf = make_float3((float)ctx->pp.L[0], (float)ctx->pp.L[1], (float)ctx->pp.L[2]);
    if (ctx->small_box)
        build_list_kernel<true><<<blocks_for(N), kThreads, 0, ctx->stream>>>(
            N, ctx->pos, ctx->posf, ctx->list_grid, ctx->start, Lf, cut2, ctx->cap, ctx->nbr, ctx->cnt, ctx->sc, gate);
    else
        build_list_warp_kernel<<<blocks_for(ctx->list_grid.ncell(), kBuildWarps), 32 * kBuildWarps, 0, ctx->stream>>>(
            N, ctx->pos, ctx->posf, ctx->list_grid, ctx->start, Lf, cut2, ctx->cap, ctx->nbr, ctx->cnt, ctx->sc, gate);
    CKL();
    if (ctx->p.precision == LJ_PRECISION_MIXED) {
        mixed_build_local_kernel<<<blocks_for(N), kThreads, 0, ctx->stream>>>(
            N, ctx->pos, soa_of(ctx->soa, N), ctx->list_grid, ctx->bx, ctx->posl, gate);
        CKL();
    }
    return LJ_OK;
}

template <int BS>
int launch_force_bs(lj_ctx* ctx, bool kick, const Fuse& fz) {
    int N = ctx->N;
    Soa s = soa_of(ctx->soa, N);
    dim3 gr(ctx->fblocks), bl(BS);
    int kind = ctx->p.force_kind;
    if (ctx->p.precision == LJ_PRECISION_MIXED && kind == LJ_FORCE_LJ && !ctx->small_box) {
        MixedParams mp = mixed_params(ctx->pp, ctx->list_grid);
#define LJ_MIXED_LAUNCH(KK, PP)                                                                          \
    force_mixed_kernel<KK, BS, PP><<<gr, bl, 0, ctx->stream>>>(N, ctx->posl, s, ctx->nbr, ctx->cnt, ctx->pp, mp, \
                                                               ctx->partials, fz)
        if (ctx->p.mixed_per_pair) {
            if (kick) LJ_MIXED_LAUNCH(true, true); else LJ_MIXED_LAUNCH(false, true);
        } else {
            if (kick) LJ_MIXED_LAUNCH(true, false); else LJ_MIXED_LAUNCH(false, false);
        }
#undef LJ_MIXED_LAUNCH
        CKL();
        return LJ_OK;
    }
#define LJ_FORCE_LAUNCH(K, S, KK)                                                                       \
    force_fp64_kernel<K, S, KK, BS><<<gr, bl, 0, ctx->stream>>>(N, ctx->pos, s, ctx->nbr, ctx->cnt, \
                                                                ctx->pp, ctx->partials, fz)
    bool sm = ctx->small_box;
    if (kind == LJ_FORCE_LJ) {
        if (sm) { if (kick) LJ_FORCE_LAUNCH(KIND_LJ, true, true); else LJ_FORCE_LAUNCH(KIND_LJ, true, false); }
        else { if (kick) LJ_FORCE_LAUNCH(KIND_LJ, false, true); else LJ_FORCE_LAUNCH(KIND_LJ, false, false); }
    } else {
        if (sm) { if (kick) LJ_FORCE_LAUNCH(KIND_CONST, true, true); else LJ_FORCE_LAUNCH(KIND_CONST, true, false); }
        else { if (kick) LJ_FORCE_LAUNCH(KIND_CONST, false, true); else LJ_FORCE_LAUNCH(KIND_CONST, false, false); }
    }
#undef LJ_FORCE_LAUNCH
    CKL();
    return LJ_OK;
}

// Whether a pair kernel can carry the next step's kick and drift (every
// configuration with a force calculation).
bool can_fuse(const lj_ctx* ctx) { return ctx->p.force_kind != LJ_FORCE_NONE; }

// Pair kernel at the context's block size (64, 128 or 256 atoms per block).
// With pos_next / posl_next it also runs the next step's first half kick and
// drift, writing the new positions there.
int launch_force(lj_ctx* ctx, bool kick, double4* pos_next = nullptr, float4* posl_next = nullptr) {
    Fuse fz{};
    if (kick && pos_next) {
        fz.pos_next = pos_next;
        fz.posl_next = posl_next;
        fz.pos = ctx->pos;
        fz.bd = ctx->bd;
        fz.bx = ctx->bx;
        fz.sc = ctx->sc;
        fz.track = !ctx->rebuild_always;
        fz.local = ctx->p.precision == LJ_PRECISION_MIXED && ctx->p.force_kind == LJ_FORCE_LJ && !ctx->small_box;
        fz.periodic = ctx->p.periodic;
    }
    switch (ctx->force_block) {
        case 64: return launch_force_bs<64>(ctx, kick, fz);
        case 256: return launch_force_bs<256>(ctx, kick, fz);
        default: return launch_force_bs<128>(ctx, kick, fz);
    }
}

// Number of partial-sum blocks the last step's measurement pass wrote.
int partial_blocks(const lj_ctx* ctx, bool forces) {
    return forces ? ctx->fblocks : ctx->nblocks;
}

int launch_kick_drift(lj_ctx* ctx, double4* pos_out = nullptr, float4* posl_out = nullptr) {
    int N = ctx->N;
    bool track = !ctx->rebuild_always && ctx->p.force_kind != LJ_FORCE_NONE;
    bool local = ctx->p.precision == LJ_PRECISION_MIXED && ctx->p.force_kind == LJ_FORCE_LJ && !ctx->small_box;
    Soa s = soa_of(ctx->soa, N);
    dim3 gr(ctx->nblocks), bl(kThreads);
#define LJ_KD(P, T, Lc) \
    kick_drift_kernel<P, T, Lc><<<gr, bl, 0, ctx->stream>>>(N, ctx->pos, pos_out ? pos_out : ctx->pos, s, ctx->bd, \
                                                            ctx->bx, posl_out ? posl_out : ctx->posl, ctx->pp, ctx->sc)
    if (!ctx->p.periodic) LJ_KD(false, false, false);
    else if (local) { if (track) LJ_KD(true, true, true); else LJ_KD(true, false, true); }
    else { if (track) LJ_KD(true, true, false); else LJ_KD(true, false, false); }
#undef LJ_KD
    CKL();
    return LJ_OK;
}

// One velocity-Verlet step; its record goes to ring slot (step index mod ring_cap).
int launch_step(lj_ctx* ctx) {
    int rc = launch_kick_drift(ctx);
    if (rc) return rc;
    bool forces = ctx->p.force_kind != LJ_FORCE_NONE;
    if (forces) {
        rc = launch_rebuild(ctx);
        if (rc) return rc;
        rc = launch_force(ctx, true);
        if (rc) return rc;
    } else {
        kick_measure_kernel<<<ctx->nblocks, kThreads, 0, ctx->stream>>>(ctx->N, soa_of(ctx->soa, ctx->N),
                                                                         ctx->pp.dt, 1, ctx->partials);
        CKL();
    }
    finalize_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->partials, partial_blocks(ctx, forces), ctx->N, ctx->pp.dt, 0,
                                                 forces ? 1 : 0, ctx->sc, ctx->ring, ctx->ring_cap, NextStep{});
    CKL();
    return LJ_OK;
}

// Capture `nsteps` steps into one executable graph.  Each step is
//   kick_drift -> [decide] -> IF(rebuild chain) -> force(+kick) -> finalize
// where the conditional is set on the device from the rebuild gate, so the
// rebuild kernels are not even launched on the steps that do not need them.
// The gate reads the displacement of the step's own positions: with fused
// steps the previous step's pair kernel computed it and that step's finalize
// sets the conditional; otherwise (and on the first step) a one-thread
// `decide` kernel after kick_drift does.
// With an even step count the pair kernels of all but the last step also run
// the next step's kick and drift (Fuse), alternating between the two position
// buffers: kick_drift only opens the graph (writing the second buffer) and the
// last, unfused step leaves the state in the first buffer again.
// Returns LJ_OK with `out` filled, or an error (the caller then keeps
// launching the steps one kernel at a time).
int build_step_graph(lj_ctx* ctx, int nsteps, StepGraph& out) {
    cudaStream_t main = ctx->stream;
    long long launches0 = ctx->launches;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return set_err(ctx, LJ_ERR_CUDA, cudaGetErrorString(e));
    int rc = LJ_OK;
    int kernels = 0;
    bool forces = ctx->p.force_kind != LJ_FORCE_NONE;
    bool fuse = forces && can_fuse(ctx) && nsteps % 2 == 0;
    double4* const posA = ctx->pos;
    float4* const poslA = ctx->posl;
    auto other = [&](double4*& x, float4*& xl) {
        x = ctx->pos == posA ? ctx->pos_b : posA;
        xl = ctx->posl == poslA ? ctx->posl_b : poslA;
    };
    auto new_handle = [&](cudaGraphConditionalHandle& h) -> bool {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        return (e = cudaStreamGetCaptureInfo(main, &cs, nullptr, &g, nullptr, nullptr)) == cudaSuccess &&
               (e = cudaGraphConditionalHandleCreate(&h, g, 0, 0)) == cudaSuccess;
    };
    cudaGraphConditionalHandle h = 0;  // this step's rebuild conditional
    for (int st = 0; st < nsteps && rc == LJ_OK; ++st) {
        if (!fuse) {
            rc = launch_kick_drift(ctx);
            ++kernels;
        } else if (st == 0) {
            rc = launch_kick_drift(ctx, ctx->pos_b, ctx->posl_b);
            ++kernels;
            ctx->pos = ctx->pos_b;
            ctx->posl = ctx->posl_b;
        }
        if (rc) break;
        if (forces) {
            if (st == 0 || !fuse) {
                if (!new_handle(h)) {
                    rc = LJ_ERR_CUDA;
                    break;
                }
                decide_rebuild_kernel<<<1, 1, 0, main>>>(gate_of(ctx), h, ctx->sc);
                ++kernels;
                if ((e = cudaGetLastError()) != cudaSuccess) {
                    rc = LJ_ERR_CUDA;
                    break;
                }
            }
            cudaStreamCaptureStatus cs;
            cudaGraph_t g = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t ndeps = 0;
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeIf;
            cp.conditional.size = 1;
            cudaGraphNode_t cnode;
            if ((e = cudaStreamGetCaptureInfo(main, &cs, nullptr, &g, &deps, &ndeps)) != cudaSuccess ||
                (e = cudaGraphAddNode(&cnode, g, deps, ndeps, &cp)) != cudaSuccess ||
                (e = cudaStreamUpdateCaptureDependencies(main, &cnode, 1, cudaStreamSetCaptureDependencies)) !=
                    cudaSuccess) {
                rc = LJ_ERR_CUDA;
                break;
            }
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            if ((e = cudaStreamBeginCaptureToGraph(ctx->side, body, nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
                rc = LJ_ERR_CUDA;
                break;
            }
            long long l0 = ctx->launches;
            ctx->stream = ctx->side;
            rc = launch_rebuild(ctx);
            ctx->stream = main;
            ctx->rebuild_kernels = (int)(ctx->launches - l0);
            cudaGraph_t body_out = nullptr;
            cudaError_t e2 = cudaStreamEndCapture(ctx->side, &body_out);
            if (rc == LJ_OK && e2 != cudaSuccess) {
                e = e2;
                rc = LJ_ERR_CUDA;
            }
            if (rc) break;
            if (fuse && st + 1 < nsteps) {
                double4* nx = nullptr;
                float4* nxl = nullptr;
                other(nx, nxl);
                rc = launch_force(ctx, true, nx, nxl);
            } else {
                rc = launch_force(ctx, true);
            }
            ++kernels;
        } else {
            kick_measure_kernel<<<ctx->nblocks, kThreads, 0, main>>>(ctx->N, soa_of(ctx->soa, ctx->N), ctx->pp.dt, 1,
                                                                     ctx->partials);
            ++kernels;
            if (cudaGetLastError() != cudaSuccess) rc = LJ_ERR_CUDA;
        }
        if (rc) break;
        NextStep next{};
        if (forces && fuse && st + 1 < nsteps) {
            if (!new_handle(h)) {  // the next step's conditional, set by this finalize
                rc = LJ_ERR_CUDA;
                break;
            }
            next = NextStep{gate_of(ctx), h, 1};
        }
        finalize_kernel<<<1, 1024, 0, main>>>(ctx->partials, partial_blocks(ctx, forces), ctx->N, ctx->pp.dt, 0,
                                              forces ? 1 : 0, ctx->sc, ctx->ring, ctx->ring_cap, next);
        ++kernels;
        if (cudaGetLastError() != cudaSuccess) rc = LJ_ERR_CUDA;
        if (fuse && st + 1 < nsteps) {
            double4* nx = nullptr;
            float4* nxl = nullptr;
            other(nx, nxl);
            ctx->pos = nx;
            ctx->posl = nxl;
        }
    }
    if (fuse && rc == LJ_OK && ctx->pos != posA) rc = set_err(ctx, LJ_ERR_CUDA, "step graph: buffer parity");
    ctx->pos = posA;
    ctx->posl = poslA;
    ctx->stream = main;
    cudaError_t ee = cudaStreamEndCapture(main, &graph);
    ctx->launches = launches0;  // captured launches are not executions
    if (rc == LJ_OK && ee != cudaSuccess) {
        e = ee;
        rc = LJ_ERR_CUDA;
    }
    if (rc == LJ_OK) {
        e = cudaGraphInstantiate(&out.exec, graph, 0);
        if (e != cudaSuccess) rc = LJ_ERR_CUDA;
    }
    if (graph) cudaGraphDestroy(graph);
    if (rc) {
        out.exec = nullptr;
        std::snprintf(ctx->err, sizeof ctx->err, "step graph unavailable: %s", cudaGetErrorString(e));
        cudaGetLastError();  // clear the sticky-free error state of the failed capture
    } else {
        out.steps = nsteps;
        out.kernels = kernels;
    }
    return rc;
}

// Steps per launch of the two step graphs: the long one amortises the
// graph-opening kick_drift over more steps.
constexpr int kGraphSteps[2] = {32, 8};

// Enqueue nsteps steps: whole step graphs where available, single launches for the rest.
int enqueue_run(lj_ctx* ctx, int nsteps) {
    if (!ctx->graph_tried) {
        ctx->graph_tried = true;
        for (int q = 0; q < 2; ++q)
            if (build_step_graph(ctx, kGraphSteps[q], ctx->graphs[q]) != LJ_OK) break;
    }
    int s = 0;
    for (StepGraph& g : ctx->graphs) {
        if (!g.exec) break;
        for (; s + g.steps <= nsteps; s += g.steps) {
            CK(cudaGraphLaunch(g.exec, ctx->stream));
            ++g.launches;
        }
    }
    for (; s < nsteps; ++s) {
        int rc = launch_step(ctx);
        if (rc) return rc;
    }
    ctx->host_steps += nsteps;
    return LJ_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Trajectory stream: every `every` steps the state (x, v, F in atom-id order)
// is packed on the device, copied with one cudaMemcpyAsync into one of two
// pinned host buffers, and a writer thread formats it in the snapshot format
// of output/sinks.cpp:162-204 while the GPU runs on.  The enqueueing thread
// waits only when both buffers are still being written out.
// ---------------------------------------------------------------------------
static __global__ void __launch_bounds__(kThreads)
frame_pack_kernel(int N, const double4* __restrict__ pos, Soa s, const int* __restrict__ ids,
                  double* __restrict__ out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    double* o = out + 9 * (size_t)ids[k];
    double4 x = pos[k];
    o[0] = x.x;
    o[1] = x.y;
    o[2] = x.z;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        o[3 + q] = s.at(VX + q, k);
        o[6 + q] = s.at(FX + q, k);
    }
}

namespace ljb {
// Snapshot rows of n atoms (x, y, z, vx, vy, vz, fx, fy, fz each) at time_step (lj_sim.cpp).
int write_snapshot_rows(long long time_step, const double* xvf, int n, FILE* f);
}  // namespace ljb

struct Trajectory {
    FILE* f = nullptr;
    int every = 1;
    int N = 0;
    int device = 0;
    double* dstage = nullptr;      // N x 9 doubles on the device
    double* host[2] = {nullptr, nullptr};  // pinned frames
    cudaEvent_t ev[2] = {nullptr, nullptr};
    long long step_of[2] = {0, 0};
    bool busy[2] = {false, false};  // queued for, or being written by, the writer
    int next = 0;
    long long frames = 0;
    int error = 0;  // a write failed
    std::mutex m;
    std::condition_variable cv;
    std::deque<int> q;
    bool stop = false;
    std::thread th;

    void run() {
        cudaSetDevice(device);
        for (;;) {
            int b;
            {
                std::unique_lock<std::mutex> g(m);
                cv.wait(g, [this] { return stop || !q.empty(); });
                if (q.empty()) return;
                b = q.front();
                q.pop_front();
            }
            int err = cudaEventSynchronize(ev[b]) != cudaSuccess ||
                      write_snapshot_rows(step_of[b], host[b], N, f) != 0;
            {
                std::lock_guard<std::mutex> g(m);
                busy[b] = false;
                if (err) error = 1;
            }
            cv.notify_all();
        }
    }
    // wait until every queued frame is written
    void drain() {
        std::unique_lock<std::mutex> g(m);
        cv.wait(g, [this] { return q.empty() && !busy[0] && !busy[1]; });
    }
};

namespace {

void traj_close(Trajectory* t) {
    if (!t) return;
    if (t->th.joinable()) {
        t->drain();
        {
            std::lock_guard<std::mutex> g(t->m);
            t->stop = true;
        }
        t->cv.notify_all();
        t->th.join();
    }
    if (t->f) std::fclose(t->f);
    for (int b = 0; b < 2; ++b) {
        if (t->host[b]) cudaFreeHost(t->host[b]);
        if (t->ev[b]) cudaEventDestroy(t->ev[b]);
    }
    if (t->dstage) cudaFree(t->dstage);
    delete t;
}

// Enqueue the frame of the current state (step count ctx->host_steps).
int traj_frame(lj_ctx* ctx) {
    Trajectory* t = ctx->traj;
    int b = t->next;
    {
        std::unique_lock<std::mutex> g(t->m);
        t->cv.wait(g, [&] { return !t->busy[b]; });
    }
    frame_pack_kernel<<<ctx->nblocks, kThreads, 0, ctx->stream>>>(ctx->N, ctx->pos, soa_of(ctx->soa, ctx->N),
                                                                   ctx->ids, t->dstage);
    CKL();
    CK(cudaMemcpyAsync(t->host[b], t->dstage, sizeof(double) * 9 * (size_t)ctx->N, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaEventRecord(t->ev[b], ctx->stream));
    {
        std::lock_guard<std::mutex> g(t->m);
        t->busy[b] = true;
        t->step_of[b] = ctx->host_steps;
        t->q.push_back(b);
    }
    t->cv.notify_all();
    t->next = b ^ 1;
    ++t->frames;
    return LJ_OK;
}

// Enqueue nsteps steps, stopping at every step count that is a multiple of the
// trajectory interval to enqueue its frame.
int enqueue_steps(lj_ctx* ctx, int nsteps) {
    if (!ctx->traj) return enqueue_run(ctx, nsteps);
    int done = 0;
    while (done < nsteps) {
        long long every = ctx->traj->every;
        int n = (int)std::min<long long>(nsteps - done, every - ctx->host_steps % every);
        int rc = enqueue_run(ctx, n);
        if (rc) return rc;
        done += n;
        if (ctx->host_steps % every == 0 && (rc = traj_frame(ctx))) return rc;
    }
    return LJ_OK;
}

// The rebuild chain launched as one graph (the chain the step graphs run
// behind their conditional node), so that in the per-phase pass its kernels
// start back to back as inside a step graph instead of one host launch
// apiece; direct launches if the capture is not available.
int launch_rebuild_graph(lj_ctx* ctx) {
    if (!ctx->rebuild_graph_tried) {
        ctx->rebuild_graph_tried = true;
        long long l0 = ctx->launches;
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            int rc = launch_rebuild(ctx);
            cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
            if (rc != LJ_OK || e != cudaSuccess || cudaGraphInstantiate(&ctx->rebuild_exec, g, 0) != cudaSuccess)
                ctx->rebuild_exec = nullptr;
            if (g) cudaGraphDestroy(g);
        }
        ctx->rebuild_graph_kernels = (int)(ctx->launches - l0);
        ctx->launches = l0;   // captured launches are not executions
        cudaGetLastError();   // a failed capture leaves no error behind
    }
    if (!ctx->rebuild_exec) return launch_rebuild(ctx);
    CK(cudaGraphLaunch(ctx->rebuild_exec, ctx->stream));
    ctx->launches += ctx->rebuild_graph_kernels;
    return LJ_OK;
}

int read_flags(lj_ctx* ctx) {
    Scalars h;
    CK(cudaMemcpyAsync(&h, ctx->sc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h.overflow) return set_err(ctx, LJ_ERR_CAPACITY, "neighbour list capacity exceeded");
    if (h.nonfinite) return set_err(ctx, LJ_ERR_NONFINITE, "non-finite energy or virial");
    return LJ_OK;
}

void free_all(lj_ctx* c) {
    void* ptrs[] = {c->posf, c->pos, c->pos_tmp, c->soa, c->soa_tmp, c->bd, c->ids, c->ids_tmp, c->cell_of,
                    c->rank, c->order, c->count, c->start, c->tile_sums, c->nbr, c->cnt, c->partials,
                    c->sc, c->ring, c->dscratch, c->dstats, c->posl, c->bx, c->pos_b, c->posl_b, c->dbg_count,
                    c->dbg_start,
                    c->dbg_members, c->dbg_cell_of, c->dbg_tiles};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    rdf_release(c->rdf);
    traj_close(c->traj);
    c->traj = nullptr;
    if (c->host_ring) cudaFreeHost(c->host_ring);
    for (StepGraph& g : c->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (c->rebuild_exec) cudaGraphExecDestroy(c->rebuild_exec);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
}

// Everything of lj_gpu_create past the host-side argument checks; on an error
// the caller releases what was allocated.
int init_ctx(lj_ctx* ctx, const lj_params& p) {
    ctx->p = p;
    int N = ctx->N = p.particle_count;
    CK(cudaSetDevice(p.device));
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));

    // pair constants (lennard_jones_force.cpp:33-74)
    PairParams& pp = ctx->pp;
    double rc = p.cutoff_distance;
    pp.rc = rc;
    pp.rc2 = rc * rc;
    pp.inv_rc2 = 1.0 / pp.rc2;
    double rcm6 = 1 / (pp.rc2 * pp.rc2 * pp.rc2);
    pp.alpha = -4.0 * rcm6 * (rcm6 - 1.0);
    pp.beta = 12.0 * rcm6 * (2.0 * rcm6 - 1.0);
    pp.strength = p.force_strength;
    pp.dt = p.time_delta;
    double near = rc * (1.0 + 1e-9);
    pp.near_lo = near;
    for (int k = 0; k < 3; ++k) {
        pp.L[k] = p.box[k];
        pp.halfL[k] = 0.5 * p.box[k];
        pp.halfL_hi[k] = hiword(0.5 * p.box[k]);
        pp.near_hi[k] = p.box[k] - near;
    }

    // neighbour-list grid: cells of at least rc + skin, and >= 3 per axis for
    // the minimum-image form; otherwise zero skin and a rebuild every step.
    double Lmin = std::min(p.box[0], std::min(p.box[1], p.box[2]));
    double skin = p.force_kind == LJ_FORCE_NONE ? 0.0 : list_skin(p.skin, Lmin, rc);
    ctx->skin = skin;
    ctx->ref_grid = make_grid(p.box, rc);
    ctx->list_grid = make_grid(p.box, rc + skin);
    ctx->small_box = std::min(ctx->list_grid.n[0], std::min(ctx->list_grid.n[1], ctx->list_grid.n[2])) < 3;
    ctx->rebuild_always = skin == 0.0;
    if (ctx->list_grid.ncell() > kScanTile * kMaxScanTiles || ctx->ref_grid.ncell() > kScanTile * kMaxScanTiles) {
        return LJ_ERR_ARG;
    }

    double V = p.box[0] * p.box[1] * p.box[2];
    double rho = N / V;
    double cut = rc + skin;
    double expect = 4.0 / 3.0 * M_PI * cut * cut * cut * std::max(rho, 1.2);
    int cap = p.neighbor_capacity > 0 ? p.neighbor_capacity : (int)std::ceil(1.5 * expect + 32);
    cap = std::min(cap, std::max(N - 1, 1) * 27);
    cap = (std::max(cap, 1) + 3) & ~3;  // whole groups of 4 entries
    ctx->cap = cap;
    ctx->nblocks = blocks_for(N);
    if (p.force_block != 0 && p.force_block != 64 && p.force_block != 128 && p.force_block != 256) {
        return LJ_ERR_ARG;
    }
    ctx->force_block = p.force_block ? p.force_block : 128;
    ctx->fblocks = blocks_for(N, ctx->force_block);
    int ncl = ctx->list_grid.ncell();
    // slot N is a ghost far outside the box: it pads the last neighbour group
    CK(cudaMalloc(&ctx->pos, sizeof(double4) * (N + 1)));
    CK(cudaMalloc(&ctx->pos_b, sizeof(double4) * (N + 1)));
    CK(cudaMalloc(&ctx->posf, sizeof(float4) * (N + 1)));
    CK(cudaMalloc(&ctx->pos_tmp, sizeof(double4) * N));
    CK(cudaMalloc(&ctx->soa, sizeof(double) * SOA_FIELDS * N));
    CK(cudaMalloc(&ctx->soa_tmp, sizeof(double) * SOA_FIELDS * N));
    CK(cudaMalloc(&ctx->bd, sizeof(double) * 3 * N));
    CK(cudaMalloc(&ctx->ids, sizeof(int) * N));
    CK(cudaMalloc(&ctx->ids_tmp, sizeof(int) * N));
    CK(cudaMalloc(&ctx->cell_of, sizeof(int) * N));
    CK(cudaMalloc(&ctx->rank, sizeof(int) * N));
    CK(cudaMalloc(&ctx->order, sizeof(int) * N));
    CK(cudaMalloc(&ctx->count, sizeof(int) * ncl));
    CK(cudaMalloc(&ctx->start, sizeof(int) * (ncl + 1)));
    CK(cudaMalloc(&ctx->tile_sums, sizeof(int) * kMaxScanTiles));
    CK(cudaMalloc(&ctx->nbr, sizeof(uint4) * (size_t)(cap / 4) * N));
    CK(cudaMalloc(&ctx->cnt, sizeof(int) * N));
    CK(cudaMalloc(&ctx->partials, sizeof(double) * 4 * std::max(ctx->nblocks, ctx->fblocks)));
    CK(cudaMalloc(&ctx->sc, sizeof(Scalars)));
    ctx->ring_cap = 1024;
    CK(cudaMalloc(&ctx->ring, sizeof(double) * 7 * (ctx->ring_cap + 1)));
    CK(cudaMalloc(&ctx->dscratch, sizeof(double) * 8));
    CK(cudaMalloc(&ctx->dstats, sizeof(double) * 8));
    ctx->dL = ctx->dscratch + 4;
    CK(cudaMallocHost(&ctx->host_ring, sizeof(double) * 7 * ctx->ring_cap));
    if (p.precision == LJ_PRECISION_MIXED) {
        CK(cudaMalloc(&ctx->posl, sizeof(float4) * (N + 1)));
        CK(cudaMalloc(&ctx->posl_b, sizeof(float4) * (N + 1)));
        CK(cudaMalloc(&ctx->bx, sizeof(double) * 3 * N));
        CK(cudaMemsetAsync(ctx->posl, 0, sizeof(float4) * N, ctx->stream));
        float4 gl = make_float4(1e18f, 1e18f, 1e18f, 0.f);
        CK(cudaMemcpyAsync(ctx->posl + N, &gl, sizeof gl, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->posl_b + N, &gl, sizeof gl, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemsetAsync(ctx->bx, 0, sizeof(double) * 3 * N, ctx->stream));
    }
    CK(cudaMemsetAsync(ctx->pos, 0, sizeof(double4) * N, ctx->stream));
    CK(cudaMemsetAsync(ctx->posf, 0, sizeof(float4) * N, ctx->stream));
    static const double4 ghost = make_double4(1e18, 1e18, 1e18, 0.0);
    static const float4 ghostf = make_float4(1e18f, 1e18f, 1e18f, 0.f);
    CK(cudaMemcpyAsync(ctx->pos + N, &ghost, sizeof ghost, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->pos_b + N, &ghost, sizeof ghost, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->posf + N, &ghostf, sizeof ghostf, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(ctx->soa, 0, sizeof(double) * SOA_FIELDS * N, ctx->stream));
    CK(cudaMemsetAsync(ctx->bd, 0, sizeof(double) * 3 * N, ctx->stream));
    CK(cudaMemsetAsync(ctx->count, 0, sizeof(int) * ncl, ctx->stream));
    CK(cudaMemsetAsync(ctx->cnt, 0, sizeof(int) * N, ctx->stream));
    CK(cudaMemsetAsync(ctx->sc, 0, sizeof(Scalars), ctx->stream));
    CK(cudaMemcpyAsync(ctx->dL, p.box, sizeof(double) * 3, cudaMemcpyHostToDevice, ctx->stream));
    // identity permutation
    std::vector<int> ident(N);
    for (int i = 0; i < N; ++i) ident[i] = i;
    CK(cudaMemcpyAsync(ctx->ids, ident.data(), sizeof(int) * N, cudaMemcpyHostToDevice, ctx->stream));
    int one = 1;
    CK(cudaMemcpyAsync(&ctx->sc->need_rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return LJ_OK;
}

// Argument checks, grid and scratch of one RDF sample (allocates only when
// the scratch must grow: the first sample, or a larger nbins).
int rdf_prepare(lj_ctx* ctx, int nbins, double rmax, Grid& g) {
    if (nbins < 1 || !(rmax > 0)) return set_err(ctx, LJ_ERR_ARG, "bad rdf arguments");
    if ((size_t)nbins * sizeof(unsigned) > 200 * 1024)
        return set_err(ctx, LJ_ERR_ARG, "rdf: too many bins for the shared-memory histogram");
    for (int k = 0; k < 3; ++k)
        if (rmax > 0.5 * ctx->pp.L[k]) return set_err(ctx, LJ_ERR_ARG, "rmax exceeds half the box");
    CK(cudaSetDevice(ctx->p.device));
    g = rdf_grid(ctx->pp.L, rmax, (long long)kScanTile * kMaxScanTiles);
    if (rdf_reserve(ctx->rdf, ctx->N, rdf_uses_cells(g) ? g.ncell() : 1, nbins) || rdf_set_smem(nbins))
        return set_err(ctx, LJ_ERR_CUDA, "rdf: scratch allocation failed");
    return LJ_OK;
}

}  // namespace

extern "C" {

void lj_gpu_default_params(lj_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->particle_count = 0;
    p->box[0] = p->box[1] = p->box[2] = 1.0;
    p->cutoff_distance = 2.5;
    p->time_delta = 0.005;
    p->precision = LJ_PRECISION_FP64;
    p->force_kind = LJ_FORCE_LJ;
    p->force_strength = 0.0;
    p->periodic = 1;
    p->device = 0;
    p->skin = -1.0;
    p->neighbor_capacity = 0;
}

const char* lj_gpu_status_string(int s) {
    return (s >= 0 && s <= 5) ? kStatus[s] : "unknown status";
}

const char* lj_gpu_last_error(const lj_ctx* ctx) { return ctx ? ctx->err : "null context"; }

int lj_gpu_create(const lj_params* params, lj_ctx** out) {
    lj_ctx* ctx = nullptr;
    if (!params || !out) return LJ_ERR_ARG;
    *out = nullptr;
    const lj_params& p = *params;
    if (p.particle_count < 1 || p.particle_count >= kMaxAtoms) return LJ_ERR_ARG;
    if (!(p.cutoff_distance > 0) || !(p.time_delta >= 0)) return LJ_ERR_ARG;
    for (int k = 0; k < 3; ++k) {
        if (!(p.box[k] > 0) || !std::isfinite(p.box[k])) return LJ_ERR_ARG;
        // particle_pair_filter.cpp:61-64 -- only a pair filter needs box >= rc
        if (p.force_kind != LJ_FORCE_NONE && !(p.box[k] >= p.cutoff_distance)) return LJ_ERR_ARG;
    }
    if (p.force_kind < LJ_FORCE_NONE || p.force_kind > LJ_FORCE_CONSTANT) return LJ_ERR_ARG;
    if (p.precision != LJ_PRECISION_FP64 && p.precision != LJ_PRECISION_MIXED) return LJ_ERR_ARG;
    if (!p.periodic && p.force_kind != LJ_FORCE_NONE) return LJ_ERR_ARG;
    if (p.mixed_per_pair != 0 && p.mixed_per_pair != 1) return LJ_ERR_ARG;
    if (p.force_block != 0 && p.force_block != 64 && p.force_block != 128 && p.force_block != 256) return LJ_ERR_ARG;
    // lennard_jones_force.cpp:45 -- the cutoff must lie beyond the potential minimum
    if (p.force_kind == LJ_FORCE_LJ && !(p.cutoff_distance * p.cutoff_distance > std::cbrt(2.0)))
        return LJ_ERR_ARG;

    ctx = new (std::nothrow) lj_ctx();
    if (!ctx) return LJ_ERR_ARG;
    int rc = init_ctx(ctx, p);
    if (rc) {
        cudaSetDevice(p.device);
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        free_all(ctx);
        delete ctx;
        return rc;
    }
    *out = ctx;
    return LJ_OK;
}

int lj_gpu_destroy(lj_ctx* ctx) {
    if (!ctx) return LJ_ERR_ARG;
    cudaSetDevice(ctx->p.device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_all(ctx);
    delete ctx;
    return LJ_OK;
}

int lj_gpu_upload_state(lj_ctx* ctx, const double* x, const double* v, const double* disp,
                        const double* F, int stride, double time, double pe, double virial) {
    if (!ctx || !x || (stride != 3 && stride != 4)) return set_err(ctx, LJ_ERR_ARG, "bad upload arguments");
    CK(cudaSetDevice(ctx->p.device));
    int N = ctx->N;
    size_t bytes = sizeof(double) * (size_t)stride * N;
    double* stage = reinterpret_cast<double*>(ctx->pos_tmp);  // 4N doubles of room
    Soa s = soa_of(ctx->soa, N);
    const double* src[4] = {x, v, disp, F};
    int field[4] = {-1, VX, DX, FX};
    for (int q = 0; q < 4; ++q) {
        if (!src[q]) {
            CK(cudaMemsetAsync(ctx->soa + (size_t)field[q] * N, 0, sizeof(double) * 3 * N, ctx->stream));
            continue;
        }
        CK(cudaMemcpyAsync(stage, src[q], bytes, cudaMemcpyHostToDevice, ctx->stream));
        unpack_kernel<<<blocks_for(N), kThreads, 0, ctx->stream>>>(N, stage, stride, field[q], ctx->pos, s,
                                                                    ctx->ids);
        CKL();
    }
    Scalars h{};
    h.t = time;
    h.pe = pe;
    h.vir = virial;
    h.need_rebuild = 1;
    Scalars old;
    CK(cudaMemcpyAsync(&old, ctx->sc, sizeof old, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    h.builds = old.builds;
    h.steps = old.steps;
    CK(cudaMemcpyAsync(ctx->sc, &h, sizeof h, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return LJ_OK;
}

int lj_gpu_download_state(lj_ctx* ctx, double* x, double* v, double* disp, double* F, int stride,
                          double* time, double* pe, double* virial) {
    if (!ctx || (stride != 3 && stride != 4)) return set_err(ctx, LJ_ERR_ARG, "bad download arguments");
    CK(cudaSetDevice(ctx->p.device));
    int N = ctx->N;
    size_t bytes = sizeof(double) * (size_t)stride * N;
    double* stage = reinterpret_cast<double*>(ctx->pos_tmp);
    Soa s = soa_of(ctx->soa, N);
    double* dst[4] = {x, v, disp, F};
    int field[4] = {-1, VX, DX, FX};
    for (int q = 0; q < 4; ++q) {
        if (!dst[q]) continue;
        pack_kernel<<<blocks_for(N), kThreads, 0, ctx->stream>>>(N, stage, stride, field[q], ctx->pos, s,
                                                                  ctx->ids);
        CKL();
        CK(cudaMemcpyAsync(dst[q], stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    }
    Scalars h;
    CK(cudaMemcpyAsync(&h, ctx->sc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (time) *time = h.t;
    if (pe) *pe = h.pe;
    if (virial) *virial = h.vir;
    return LJ_OK;
}

int lj_gpu_compute_forces(lj_ctx* ctx, double* pe, double* virial) {
    if (!ctx) return LJ_ERR_ARG;
    CK(cudaSetDevice(ctx->p.device));
    if (ctx->p.force_kind == LJ_FORCE_NONE) {
        // no force calculation configured: clear_dynamics only
        CK(cudaMemsetAsync(ctx->soa + (size_t)FX * ctx->N, 0, sizeof(double) * 3 * ctx->N, ctx->stream));
        double z[3] = {0, 0, 0};
        CK(cudaMemcpyAsync(&ctx->sc->pe, z, sizeof(double) * 2, cudaMemcpyHostToDevice, ctx->stream));
    } else {
        int one = 1;
        CK(cudaMemcpyAsync(&ctx->sc->need_rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        int rc = launch_rebuild(ctx);
        if (rc) return rc;
        rc = launch_force(ctx, false);
        if (rc) return rc;
        finalize_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->partials, partial_blocks(ctx, true), ctx->N, ctx->pp.dt, 1, 1,
                                                     ctx->sc, ctx->ring, ctx->ring_cap, NextStep{});
        CKL();
    }
    int rc = read_flags(ctx);
    if (rc) return rc;
    Scalars h;
    CK(cudaMemcpyAsync(&h, ctx->sc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (pe) *pe = h.pe;
    if (virial) *virial = h.vir;
    return LJ_OK;
}

int lj_gpu_step(lj_ctx* ctx, int nsteps, lj_thermo* out) {
    if (!ctx || nsteps < 0) return set_err(ctx, LJ_ERR_ARG, "bad step arguments");
    CK(cudaSetDevice(ctx->p.device));
    int done = 0;
    while (done < nsteps) {
        int chunk = std::min(nsteps - done, ctx->ring_cap);
        long long first = ctx->host_steps;
        int rc = enqueue_steps(ctx, chunk);
        if (rc) return rc;
        if (out) {
            // records of steps first .. first+chunk-1 sit at ring slots (step mod ring_cap)
            int s0 = (int)(first % ctx->ring_cap);
            int n1 = std::min(chunk, ctx->ring_cap - s0);
            CK(cudaMemcpyAsync(ctx->host_ring, ctx->ring + 7 * (size_t)s0, sizeof(double) * 7 * n1,
                               cudaMemcpyDeviceToHost, ctx->stream));
            if (n1 < chunk)
                CK(cudaMemcpyAsync(ctx->host_ring + 7 * (size_t)n1, ctx->ring, sizeof(double) * 7 * (chunk - n1),
                                   cudaMemcpyDeviceToHost, ctx->stream));
        }
        rc = read_flags(ctx);  // synchronises
        if (rc) return rc;
        if (out) std::memcpy(out + done, ctx->host_ring, sizeof(double) * 7 * chunk);
        done += chunk;
    }
    return LJ_OK;
}

int lj_gpu_measure(lj_ctx* ctx, lj_thermo* out) {
    if (!ctx || !out) return set_err(ctx, LJ_ERR_ARG, "bad measure arguments");
    CK(cudaSetDevice(ctx->p.device));
    kick_measure_kernel<<<ctx->nblocks, kThreads, 0, ctx->stream>>>(ctx->N, soa_of(ctx->soa, ctx->N), 0.0, 0,
                                                                     ctx->partials);
    CKL();
    finalize_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->partials, ctx->nblocks, ctx->N, ctx->pp.dt, 2, 0,
                                                 ctx->sc, ctx->ring, ctx->ring_cap, NextStep{});
    CKL();
    CK(cudaMemcpyAsync(ctx->host_ring, ctx->ring + 7 * (size_t)ctx->ring_cap, sizeof(double) * 7,
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::memcpy(out, ctx->host_ring, sizeof(double) * 7);
    return LJ_OK;
}

int lj_gpu_scale_velocities(lj_ctx* ctx, double factor) {
    if (!ctx || !std::isfinite(factor)) return set_err(ctx, LJ_ERR_ARG, "bad scale factor");
    CK(cudaSetDevice(ctx->p.device));
    scale_kernel<<<ctx->nblocks, kThreads, 0, ctx->stream>>>(ctx->N, soa_of(ctx->soa, ctx->N), factor);
    CKL();
    CK(cudaStreamSynchronize(ctx->stream));
    return LJ_OK;
}

int lj_gpu_set_temperature(lj_ctx* ctx, double target, double* measured) {
    if (!ctx || !(target >= 0)) return set_err(ctx, LJ_ERR_ARG, "bad target temperature");
    lj_thermo m;
    int rc = lj_gpu_measure(ctx, &m);
    if (rc) return rc;
    if (!(m.temperature > 0)) return set_err(ctx, LJ_ERR_ARG, "cannot scale a zero-temperature state");
    if (measured) *measured = m.temperature;
    return lj_gpu_scale_velocities(ctx, std::sqrt(target / m.temperature));
}

int lj_gpu_debug_cells(lj_ctx* ctx, int* shape, int* cell_of, int* offsets, int* members) {
    if (!ctx) return LJ_ERR_ARG;
    CK(cudaSetDevice(ctx->p.device));
    const Grid& g = ctx->ref_grid;
    if (shape)
        for (int k = 0; k < 3; ++k) shape[k] = g.n[k];
    if (!cell_of && !offsets && !members) return LJ_OK;
    int nc = g.ncell(), N = ctx->N;
    if (!ctx->dbg_count) {
        CK(cudaMalloc(&ctx->dbg_count, sizeof(int) * nc));
        CK(cudaMalloc(&ctx->dbg_start, sizeof(int) * (nc + 1)));
        CK(cudaMalloc(&ctx->dbg_members, sizeof(int) * N));
        CK(cudaMalloc(&ctx->dbg_cell_of, sizeof(int) * N));
        CK(cudaMalloc(&ctx->dbg_tiles, sizeof(int) * kMaxScanTiles));
        CK(cudaMemsetAsync(ctx->dbg_count, 0, sizeof(int) * nc, ctx->stream));
    }
    Gate open{};
    open.sc = ctx->sc;
    open.always = 1;
    int rc = launch_binning<false>(ctx, g, ctx->dbg_count, ctx->dbg_start, ctx->dbg_tiles, open);
    if (rc) return rc;
    debug_members_kernel<<<blocks_for(N), kThreads, 0, ctx->stream>>>(N, ctx->cell_of, ctx->rank, ctx->dbg_start,
                                                                       ctx->ids, ctx->dbg_members, ctx->dbg_cell_of);
    CKL();
    sort_members_kernel<<<blocks_for(nc), kThreads, 0, ctx->stream>>>(nc, ctx->dbg_start, ctx->dbg_members);
    CKL();
    if (cell_of) CK(cudaMemcpyAsync(cell_of, ctx->dbg_cell_of, sizeof(int) * N, cudaMemcpyDeviceToHost, ctx->stream));
    if (offsets) CK(cudaMemcpyAsync(offsets, ctx->dbg_start, sizeof(int) * (nc + 1), cudaMemcpyDeviceToHost, ctx->stream));
    if (members) CK(cudaMemcpyAsync(members, ctx->dbg_members, sizeof(int) * N, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // the shared cell_of/rank scratch now holds the reference grid: force a list rebuild
    int one = 1;
    CK(cudaMemcpy(&ctx->sc->need_rebuild, &one, sizeof(int), cudaMemcpyHostToDevice));
    return LJ_OK;
}

long long lj_gpu_debug_pairs(lj_ctx* ctx, long long cap, int* pi, int* pj, int* pimg, double* pr2) {
    if (!ctx || cap < 0 || (cap > 0 && (!pi || !pj || !pimg || !pr2))) return -LJ_ERR_ARG;
    if (ctx->p.force_kind == LJ_FORCE_NONE) return 0;
    if (cudaSetDevice(ctx->p.device) != cudaSuccess) return -LJ_ERR_CUDA;
    // make sure the list reflects the current positions
    int one = 1;
    if (cudaMemcpyAsync(&ctx->sc->need_rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        return -LJ_ERR_CUDA;
    int rc = launch_rebuild(ctx);
    if (rc) return -rc;
    int* di = nullptr; int* dj = nullptr; int* dm = nullptr; double* dr = nullptr;
    unsigned long long* counter = nullptr;
    long long c = cap > 0 ? cap : 1;
    cudaError_t e = cudaMalloc(&di, sizeof(int) * c);
    if (e == cudaSuccess) e = cudaMalloc(&dj, sizeof(int) * c);
    if (e == cudaSuccess) e = cudaMalloc(&dm, sizeof(int) * c);
    if (e == cudaSuccess) e = cudaMalloc(&dr, sizeof(double) * c);
    if (e == cudaSuccess) e = cudaMalloc(&counter, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), ctx->stream);
    unsigned long long total = 0;
    if (e == cudaSuccess) {
        if (ctx->small_box)
            debug_pairs_kernel<true><<<ctx->nblocks, kThreads, 0, ctx->stream>>>(
                ctx->N, ctx->pos, ctx->nbr, ctx->cnt, ctx->ids, ctx->pp, cap, di, dj, dm, dr, counter);
        else
            debug_pairs_kernel<false><<<ctx->nblocks, kThreads, 0, ctx->stream>>>(
                ctx->N, ctx->pos, ctx->nbr, ctx->cnt, ctx->ids, ctx->pp, cap, di, dj, dm, dr, counter);
        e = cudaGetLastError();
        ++ctx->launches;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, counter, sizeof total, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    long long n = std::min<long long>((long long)total, cap);
    if (e == cudaSuccess && n > 0) {
        e = cudaMemcpy(pi, di, sizeof(int) * n, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(pj, dj, sizeof(int) * n, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(pimg, dm, sizeof(int) * n, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(pr2, dr, sizeof(double) * n, cudaMemcpyDeviceToHost);
    }
    cudaFree(di); cudaFree(dj); cudaFree(dm); cudaFree(dr); cudaFree(counter);
    if (e != cudaSuccess) {
        std::snprintf(ctx->err, sizeof ctx->err, "debug_pairs: %s", cudaGetErrorString(e));
        return -LJ_ERR_CUDA;
    }
    int st = read_flags(ctx);
    if (st) return -st;
    return (long long)total;
}

int lj_gpu_get_stats(const lj_ctx* ctx_c, lj_stats* out) {
    lj_ctx* ctx = const_cast<lj_ctx*>(ctx_c);
    if (!ctx || !out) return LJ_ERR_ARG;
    CK(cudaSetDevice(ctx->p.device));
    Scalars h;
    CK(cudaMemcpyAsync(&h, ctx->sc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    out->steps = h.steps;
    out->list_builds = h.builds;
    out->neighbor_capacity = ctx->cap;
    for (int k = 0; k < 3; ++k) out->list_cells[k] = ctx->list_grid.n[k];
    out->max_neighbors = h.max_count;
    out->small_box = ctx->small_box ? 1 : 0;
    out->skin = ctx->skin;
    // direct launches + kernel nodes executed by step graphs (each launch's
    // kernels, and the rebuild chain each time a conditional opened)
    out->kernel_launches = ctx->launches + (long long)ctx->rebuild_kernels * h.graph_rebuilds;
    for (const StepGraph& g : ctx->graphs) out->kernel_launches += g.launches * g.kernels;
    return LJ_OK;
}

int lj_gpu_rdf(lj_ctx* ctx, int nbins, double rmax, unsigned long long* hist) {
    if (!ctx || !hist) return set_err(ctx, LJ_ERR_ARG, "bad rdf arguments");
    Grid g{};
    int rc = rdf_prepare(ctx, nbins, rmax, g);
    if (rc) return rc;
    // a single sample goes to the second half of the scratch histogram, so a
    // running accumulation is left alone
    unsigned long long* once = ctx->rdf.hist + ctx->rdf.bins;
    CK(cudaMemsetAsync(once, 0, sizeof(unsigned long long) * nbins, ctx->stream));
    if (rdf_enqueue(ctx->N, ctx->pos, ctx->pp, g, nbins, rmax, ctx->rdf, once, ctx->stream, &ctx->launches))
        return set_err(ctx, LJ_ERR_CUDA, "rdf: kernel launch failed");
    CK(cudaMemcpyAsync(hist, once, sizeof(unsigned long long) * nbins, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return LJ_OK;
}

int lj_gpu_rdf_accumulate(lj_ctx* ctx, int nbins, double rmax) {
    if (!ctx) return LJ_ERR_ARG;
    RdfScratch& r = ctx->rdf;
    if (r.samples > 0 && (nbins != r.acc_bins || rmax != r.acc_rmax))
        return set_err(ctx, LJ_ERR_ARG, "rdf_accumulate: nbins and rmax differ from the running accumulation");
    Grid g{};
    int rc = rdf_prepare(ctx, nbins, rmax, g);
    if (rc) return rc;
    if (r.samples == 0) {
        CK(cudaMemsetAsync(r.hist, 0, sizeof(unsigned long long) * nbins, ctx->stream));
        r.acc_bins = nbins;
        r.acc_rmax = rmax;
    }
    if (rdf_enqueue(ctx->N, ctx->pos, ctx->pp, g, nbins, rmax, r, r.hist, ctx->stream, &ctx->launches))
        return set_err(ctx, LJ_ERR_CUDA, "rdf: kernel launch failed");
    ++r.samples;
    return LJ_OK;
}

int lj_gpu_rdf_read(lj_ctx* ctx, unsigned long long* hist, long long* samples) {
    if (!ctx) return LJ_ERR_ARG;
    CK(cudaSetDevice(ctx->p.device));
    const RdfScratch& r = ctx->rdf;
    if (samples) *samples = r.samples;
    if (hist && r.samples > 0) {
        CK(cudaMemcpyAsync(hist, r.hist, sizeof(unsigned long long) * r.acc_bins, cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return LJ_OK;
}

int lj_gpu_rdf_reset(lj_ctx* ctx) {
    if (!ctx) return LJ_ERR_ARG;
    ctx->rdf.samples = 0;
    ctx->rdf.acc_bins = 0;
    ctx->rdf.acc_rmax = 0.0;
    return LJ_OK;
}

}  // extern "C"

extern "C" {

void* lj_gpu_stream(lj_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int lj_gpu_step_async(lj_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 0) return set_err(ctx, LJ_ERR_ARG, "bad step arguments");
    CK(cudaSetDevice(ctx->p.device));
    return enqueue_steps(ctx, nsteps);
}

int lj_gpu_synchronize(lj_ctx* ctx) {
    if (!ctx) return LJ_ERR_ARG;
    CK(cudaSetDevice(ctx->p.device));
    return read_flags(ctx);
}

int lj_gpu_step_timed(lj_ctx* ctx, int nsteps, lj_phase_times* out) {
    if (!ctx || nsteps < 0 || !out) return set_err(ctx, LJ_ERR_ARG, "bad step arguments");
    CK(cudaSetDevice(ctx->p.device));
    std::memset(out, 0, sizeof *out);
    // ev[1] after kick/drift, ev[5] once the host has read the rebuild
    // criterion: the host round trip between them belongs to no phase
    cudaEvent_t ev[6];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    Scalars before;
    CK(cudaMemcpy(&before, ctx->sc, sizeof before, cudaMemcpyDeviceToHost));
    bool forces = ctx->p.force_kind != LJ_FORCE_NONE;
    const Gate gate = gate_of(ctx);
    for (int s = 0; s < nsteps; ++s) {
        int rc;
        CK(cudaEventRecord(ev[0], ctx->stream));
        if ((rc = launch_kick_drift(ctx))) return rc;
        CK(cudaEventRecord(ev[1], ctx->stream));
        if (forces) {
            // launch the rebuild chain only on the steps whose gate is open, as
            // the step graphs' conditional node does (the host reads the
            // criterion kick_drift just computed)
            Scalars h;
            CK(cudaMemcpyAsync(&h, ctx->sc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            double d2;
            std::memcpy(&d2, &h.max_disp2, sizeof d2);
            bool open = gate.always || h.need_rebuild || d2 > gate.thresh2;
            CK(cudaEventRecord(ev[5], ctx->stream));
            if (open && (rc = launch_rebuild_graph(ctx))) return rc;
        } else {
            CK(cudaEventRecord(ev[5], ctx->stream));
        }
        CK(cudaEventRecord(ev[2], ctx->stream));
        if (forces) {
            if ((rc = launch_force(ctx, true))) return rc;
        } else {
            kick_measure_kernel<<<ctx->nblocks, kThreads, 0, ctx->stream>>>(ctx->N, soa_of(ctx->soa, ctx->N),
                                                                             ctx->pp.dt, 1, ctx->partials);
            CKL();
        }
        CK(cudaEventRecord(ev[3], ctx->stream));
        finalize_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->partials, partial_blocks(ctx, forces), ctx->N, ctx->pp.dt,
                                                     0, forces ? 1 : 0, ctx->sc, ctx->ring, ctx->ring_cap, NextStep{});
        CKL();
        CK(cudaEventRecord(ev[4], ctx->stream));
        CK(cudaEventSynchronize(ev[4]));
        float ms[4];
        for (int q = 0; q < 4; ++q) CK(cudaEventElapsedTime(&ms[q], ev[q == 1 ? 5 : q], ev[q + 1]));
        out->kick_drift_ms += ms[0];
        out->rebuild_ms += ms[1];
        out->force_ms += ms[2];
        out->finalize_ms += ms[3];
    }
    for (auto& e : ev) cudaEventDestroy(e);
    Scalars after;
    CK(cudaMemcpy(&after, ctx->sc, sizeof after, cudaMemcpyDeviceToHost));
    out->steps = nsteps;
    out->rebuilds = after.builds - before.builds;
    ctx->host_steps += nsteps;
    return read_flags(ctx);
}

}  // extern "C"

extern "C" {

int lj_gpu_window_stats(lj_ctx* ctx, int sample_size, double density, lj_observation* out) {
    if (!ctx || !out || sample_size < 2 || sample_size > ctx->ring_cap || sample_size > ctx->host_steps)
        return set_err(ctx, LJ_ERR_ARG, "window_stats: need 2 <= sample_size <= min(1024, steps taken)");
    CK(cudaSetDevice(ctx->p.device));
    double in[2];
    int n = ctx->N;
    in[0] = density;
    std::memcpy(&in[1], &n, sizeof n);
    CK(cudaMemcpyAsync(ctx->dstats + 6, in, sizeof in, cudaMemcpyHostToDevice, ctx->stream));
    window_stats_kernel<<<1, kStatsThreads, 0, ctx->stream>>>(ctx->ring, ctx->ring_cap, 1, ctx->host_steps - 1,
                                                             sample_size, reinterpret_cast<int*>(ctx->dstats + 7),
                                                             ctx->dstats + 6, ctx->dstats);
    CKL();
    double o[6];
    CK(cudaMemcpyAsync(o, ctx->dstats, sizeof o, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *out = lj_observation{o[0], o[1], o[2], o[3], o[4], o[5]};
    return LJ_OK;
}

int lj_gpu_trajectory_open(lj_ctx* ctx, const char* path, int every) {
    if (!ctx || !path || every < 1) return set_err(ctx, LJ_ERR_ARG, "bad trajectory arguments");
    if (ctx->traj) return set_err(ctx, LJ_ERR_ARG, "a trajectory is already open");
    CK(cudaSetDevice(ctx->p.device));
    Trajectory* t = new (std::nothrow) Trajectory();
    if (!t) return set_err(ctx, LJ_ERR_ARG, "out of host memory");
    t->every = every;
    t->N = ctx->N;
    t->device = ctx->p.device;
    size_t bytes = sizeof(double) * 9 * (size_t)ctx->N;
    t->f = std::fopen(path, "w");
    int rc = LJ_OK;
    if (!t->f) {
        rc = set_err(ctx, LJ_ERR_ARG, "cannot open the trajectory file");
    } else if (cudaMalloc(&t->dstage, bytes) != cudaSuccess || cudaMallocHost(&t->host[0], bytes) != cudaSuccess ||
               cudaMallocHost(&t->host[1], bytes) != cudaSuccess ||
               cudaEventCreateWithFlags(&t->ev[0], cudaEventDisableTiming) != cudaSuccess ||
               cudaEventCreateWithFlags(&t->ev[1], cudaEventDisableTiming) != cudaSuccess) {
        rc = set_err(ctx, LJ_ERR_CUDA, "trajectory buffers: allocation failed");
    } else {
        // the two header rows of output/sinks.cpp:162-183
        std::fputs("TimeStep,ParticleID,Position,Position,Position,Velocity,Velocity,Velocity,Force,Force,Force\n"
                   "TimeStep,ParticleID,X,Y,Z,X,Y,Z,X,Y,Z\n",
                   t->f);
        t->th = std::thread([t] { t->run(); });
    }
    if (rc) {
        traj_close(t);
        return rc;
    }
    ctx->traj = t;
    return LJ_OK;
}

int lj_gpu_trajectory_close(lj_ctx* ctx, long long* frames) {
    if (!ctx) return LJ_ERR_ARG;
    Trajectory* t = ctx->traj;
    if (!t) return set_err(ctx, LJ_ERR_ARG, "no trajectory is open");
    CK(cudaSetDevice(ctx->p.device));
    t->drain();
    int err = t->error;
    if (frames) *frames = t->frames;
    ctx->traj = nullptr;
    traj_close(t);
    return err ? set_err(ctx, LJ_ERR_ARG, "trajectory: a frame could not be written") : LJ_OK;
}

// Project autotuner: for the caller's system (base params + state), time
// `steps` velocity-Verlet steps for every candidate and return the fastest
// parameters.  Candidates: the Verlet skin, which sets the list-cell edge
// rc + skin and, against it, the rebuild frequency; and per skin the pair
// kernel's block size (atoms per block: 64, 128, 256).
// Each candidate runs in its own context from the same initial state after a
// warm-up long enough to build the step graph and the first neighbour list.
int lj_gpu_autotune(const lj_params* base, const double* x, const double* v, int stride, int steps,
                    lj_params* best, double* best_ms_per_step) {
    if (!base || !x || !best || steps < 1 || (stride != 3 && stride != 4)) return LJ_ERR_ARG;
    const double skins[] = {0.15, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7};
    const int blocks[] = {64, 128, 256};
    double best_ms = 1e300;
    lj_params winner = *base;
    double Lmin = std::min(base->box[0], std::min(base->box[1], base->box[2]));
    double last_skin = -1.0;
    for (double sk : skins) {
        double eff = list_skin(sk, Lmin, base->cutoff_distance);
        if (eff == last_skin) continue;  // the box clips this skin to one already tried
        last_skin = eff;
        for (int bs : blocks) {
            lj_params p = *base;
            p.skin = sk;
            p.force_block = bs;
            lj_ctx* ctx = nullptr;
            int rc = lj_gpu_create(&p, &ctx);
            if (rc) return rc;
            float ms = 0;
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            rc = lj_gpu_upload_state(ctx, x, v, nullptr, nullptr, stride, 0.0, 0.0, 0.0);
            if (!rc) rc = lj_gpu_step_async(ctx, 16);
            if (!rc) rc = lj_gpu_synchronize(ctx);
            if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) rc = LJ_ERR_CUDA;
            if (!rc) {
                cudaEventRecord(e0, ctx->stream);
                rc = lj_gpu_step_async(ctx, steps);
                cudaEventRecord(e1, ctx->stream);
            }
            if (!rc) rc = lj_gpu_synchronize(ctx);
            if (!rc && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) rc = LJ_ERR_CUDA;
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            lj_gpu_destroy(ctx);
            if (rc) return rc;
            if (ms / steps < best_ms) {
                best_ms = ms / steps;
                winner = p;
            }
        }
    }
    *best = winner;
    if (best_ms_per_step) *best_ms_per_step = best_ms;
    return LJ_OK;
}

}  // extern "C"
