// lj_adjoint.cu -- differentiable NVE: a hand-written discrete adjoint of
// velocity Verlet with the LJ force Hessian-vector product.
//
// Potential with energy and length scales (the reference fixes eps = sigma = 1,
// physics/lennard_jones_force.cpp:107-121): with u = r / sigma and the cutoff
// u_c = rc / sigma held fixed,
//     V(r) = eps * [4 u^-6 (u^-6 - 1) + alpha + beta (u^2 / u_c^2 - 1)]
//     W(r) = -r V'(r) = eps * [24 u^-6 (2 u^-6 - 1) - 2 beta u^2 / u_c^2]
//     F_i  = sum_j f(q_ij) r_ij,   f = W / q,   q = r^2
// with alpha, beta the reference's spline constants for u_c (:68-73).
//
// Forward (the reference's step, integrator.cpp:62-88, starting from
// F_0 = F(x_0)): h = v_n + dt/2 F(x_n); x_{n+1} = x_n + dt h (wrapped);
// v_{n+1} = h + dt/2 F(x_{n+1}).  Outputs: the time averages over states 1..M
// of the total potential energy PE and of the virial pressure
// P = rho (T + W / (3N)) (physics/analyzers.cpp:73-75), T = (2/3) KE / N.
// Loss L = (1/M) sum_{n=1..M} l_n, l_n = w_pe PE_n + w_p P_n.
//
// Reverse sweep (exact gradient of the discrete trajectory), one Hessian-vector
// product per step:  for n = M .. 1, with adjoints ax, av and a pending c = 0,
//     av += dl/dv_n;   u = dt/2 av + c
//     ax += dl/dx_n + J(x_n) u;    a_theta += dl/dtheta|_n + (dF/dtheta)(x_n) . u
//     av = av + dt ax;             c = dt/2 av
// (l_n = the loss of state n) and finally ax += J(x_0) c and
// a_theta += (dF/dtheta)(x_0) . c.  Then dL/dx_0 = ax, dL/dv_0 = av.  J = dF/dx is
// the (negative) Hessian: (J u)_i = sum_j [f (u_i - u_j) + 2 f' (r_ij . (u_i - u_j)) r_ij],
// f' = df/dq.  States are recomputed per segment from checkpoints kept every
// k steps.  Pairs are found exactly (FP64, r^2 < rc^2) at every state, so the
// trajectory and the gradient follow the same pair set; atoms stay in id order.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lj_gpu.h"
#include "lj_kernels.cuh"

using namespace ljb;

namespace {

constexpr int kAdjCap = 192;  // list entries per atom (the exact pair set at any liquid density)

struct AdjParams {
    double L[3], halfL[3];
    double eps, sigma, rc2;  // rc2 = (u_c sigma)^2
    double alpha, beta;      // spline constants for u_c
    double inv_uc2s2;        // 1 / (u_c^2 sigma^2)
    double inv_sigma;
    double dt;
};

// Pair quantities at q = r^2: V, W = -r V', f = W / q, dW/dq, f' = df/dq and
// the sigma derivatives of V, W and f.
struct PairQ {
    double V, W, f, dWdq, fp, dVds, dWds, dfds;
};

__device__ __forceinline__ PairQ pair_q(const AdjParams& P, double q) {
    PairQ o;
    double iq = 1.0 / q;  // the only division
    double s2 = P.sigma * P.sigma * iq;
    double s6 = s2 * s2 * s2;  // (sigma^2 / q)^3
    double s12 = s6 * s6;
    double x = q * P.inv_uc2s2;
    o.V = P.eps * (4.0 * s6 * (s6 - 1.0) + P.alpha + P.beta * (x - 1.0));
    o.W = P.eps * (48.0 * s12 - 24.0 * s6 - 2.0 * P.beta * x);
    o.f = o.W * iq;
    o.dWdq = P.eps * ((-288.0 * s12 + 72.0 * s6) * iq - 2.0 * P.beta * P.inv_uc2s2);
    o.fp = (o.dWdq - o.f) * iq;
    o.dVds = o.W * P.inv_sigma;
    o.dWds = P.eps * (576.0 * s12 - 144.0 * s6 + 4.0 * P.beta * x) * P.inv_sigma;
    o.dfds = o.dWds * iq;
    return o;
}

__device__ __forceinline__ double mimg(double d, double L, double halfL) {
    return d > halfL ? d - L : (d < -halfL ? d + L : d);
}

// Cells of edge >= cutoff (>= 3 per axis): cell of each atom and its arrival rank.
static __global__ void ad_bin_kernel(int N, const double4* __restrict__ x, Grid g, int* __restrict__ cell_of,
                                     int* __restrict__ rank, int* __restrict__ count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double4 p = x[i];
    int c = g.flat(cell_coord(p.x, g.ratio[0], g.n[0]), cell_coord(p.y, g.ratio[1], g.n[1]),
                   cell_coord(p.z, g.ratio[2], g.n[2]));
    cell_of[i] = c;
    rank[i] = atomicAdd(&count[c], 1);
}

static __global__ void ad_members_kernel(int N, const int* __restrict__ cell_of, const int* __restrict__ rank,
                                         const int* __restrict__ start, int* __restrict__ members) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    members[start[cell_of[i]] + rank[i]] = i;
}

// Members of each cell into id order (insertion sort; a cell holds a few tens
// of atoms), so the pair order and with it every sum is reproducible.
static __global__ void ad_sort_cells_kernel(int ncell, const int* __restrict__ start, int* __restrict__ members) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    int b = start[c], e = start[c + 1];
    for (int k = b + 1; k < e; ++k) {
        int v = members[k], m = k - 1;
        while (m >= b && members[m] > v) {
            members[m + 1] = members[m];
            --m;
        }
        members[m + 1] = v;
    }
}

// Exact neighbour list over the 27-cell stencil (minimum image): every j with
// r_ij^2 < rc^2, in stencil-then-id order, stored [slot][atom].  One warp per
// atom: the lanes test 32 candidates of a cell at a time and the hits are
// compacted in candidate order (ballot + prefix count).
static __global__ void __launch_bounds__(kThreads)
ad_list_kernel(int N, const double4* __restrict__ x, Grid g, const int* __restrict__ cell_of,
               const int* __restrict__ start, const int* __restrict__ members, const AdjParams* __restrict__ Pp,
               int* __restrict__ nbr, int* __restrict__ cnt, int* __restrict__ overflow) {
    int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= N) return;  // uniform across the warp
    const AdjParams P = *Pp;
    double4 xi = x[i];
    int c = cell_of[i];
    int ca = c / (g.n[1] * g.n[2]), cb = (c / g.n[2]) % g.n[1], cc = c % g.n[2];
    int n = 0;
    for (int a = -1; a <= 1; ++a)
        for (int b = -1; b <= 1; ++b)
            for (int d = -1; d <= 1; ++d) {
                int cell = g.flat((ca + a + g.n[0]) % g.n[0], (cb + b + g.n[1]) % g.n[1], (cc + d + g.n[2]) % g.n[2]);
                int ke = start[cell + 1];
                for (int k0 = start[cell]; k0 < ke; k0 += 32) {
                    int k = k0 + lane, j = -1;
                    bool hit = false;
                    if (k < ke) {
                        j = members[k];
                        if (j != i) {
                            double4 xj = x[j];
                            double dx = mimg(xi.x - xj.x, P.L[0], P.halfL[0]);
                            double dy = mimg(xi.y - xj.y, P.L[1], P.halfL[1]);
                            double dz = mimg(xi.z - xj.z, P.L[2], P.halfL[2]);
                            hit = dx * dx + dy * dy + dz * dz < P.rc2;
                        }
                    }
                    unsigned m = __ballot_sync(0xffffffffu, hit);
                    if (hit) {
                        int slot = n + __popc(m & ((1u << lane) - 1u));
                        if (slot < kAdjCap) nbr[(size_t)slot * N + i] = j;
                    }
                    n += __popc(m);
                }
            }
    if (lane == 0) {
        cnt[i] = min(n, kAdjCap);
        if (n > kAdjCap) atomicExch(overflow, 1);
    }
}

template <int Q>
__device__ __forceinline__ void write_partials(double (&acc)[Q], double* __restrict__ partials) {
    block_sum<Q, kThreads>(acc);
    if (threadIdx.x == 0)
        for (int q = 0; q < Q; ++q) partials[(size_t)blockIdx.x * Q + q] = acc[q];
}

// Sum over the 32 lanes of a warp (fixed tree; valid in lane 0).
template <int Q>
__device__ __forceinline__ void warp_reduce(double (&v)[Q]) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int q = 0; q < Q; ++q) v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
}

// Forces at x, one warp per atom (lanes take every 32nd list entry); block
// partials {2 PE, 2 W} (each pair seen from both ends).
static __global__ void __launch_bounds__(kThreads)
ad_force_kernel(int N, const double4* __restrict__ x, const int* __restrict__ nbr, const int* __restrict__ cnt,
                const AdjParams* __restrict__ Pp, double* __restrict__ F, double* __restrict__ partials) {
    const AdjParams P = *Pp;
    int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    double acc[2] = {0, 0};
    if (i < N) {  // uniform across the warp
        double4 xi = x[i];
        double t[5] = {0, 0, 0, 0, 0};  // fx, fy, fz, PE, W
        for (int k = lane; k < cnt[i]; k += 32) {
            double4 xj = x[nbr[(size_t)k * N + i]];
            double dx = mimg(xi.x - xj.x, P.L[0], P.halfL[0]);
            double dy = mimg(xi.y - xj.y, P.L[1], P.halfL[1]);
            double dz = mimg(xi.z - xj.z, P.L[2], P.halfL[2]);
            PairQ o = pair_q(P, dx * dx + dy * dy + dz * dz);
            t[0] += o.f * dx;
            t[1] += o.f * dy;
            t[2] += o.f * dz;
            t[3] += o.V;
            t[4] += o.W;
        }
        warp_reduce<5>(t);
        if (lane == 0) {
            F[3 * (size_t)i] = t[0];
            F[3 * (size_t)i + 1] = t[1];
            F[3 * (size_t)i + 2] = t[2];
            acc[0] = t[3];
            acc[1] = t[4];
        }
    }
    write_partials<2>(acc, partials);
}

// v += dt/2 F, then (drift) x = wrap(x + dt v).
static __global__ void ad_kick_kernel(int N, double4* __restrict__ x, double* __restrict__ v,
                                      const double* __restrict__ F, const AdjParams* __restrict__ Pp, int drift) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const AdjParams P = *Pp;
    double4 xi = x[i];
    double p[3] = {xi.x, xi.y, xi.z};
    for (int k = 0; k < 3; ++k) {
        double vk = v[3 * (size_t)i + k] + 0.5 * F[3 * (size_t)i + k] * P.dt;
        v[3 * (size_t)i + k] = vk;
        if (drift) p[k] = wrap(p[k] + vk * P.dt, P.L[k]);
    }
    if (drift) x[i] = make_double4(p[0], p[1], p[2], 0.0);
}

// block partials {2 KE}
static __global__ void __launch_bounds__(kThreads)
ad_ke_kernel(int N, const double* __restrict__ v, double* __restrict__ partials) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[1] = {0};
    if (i < N)
        for (int k = 0; k < 3; ++k) acc[0] += v[3 * (size_t)i + k] * v[3 * (size_t)i + k];
    write_partials<1>(acc, partials);
}

// Loss weights of one state, set before each backward pass: wpe (PE), wpw (W)
// and gv (d loss / d v = gv v).
struct AdjWeights {
    double wpe, wpw, gv;
};

// av += gv * v (the step's loss gradient in v); u = dt/2 av + c
static __global__ void ad_pre_kernel(int n3, const double* __restrict__ v, const AdjWeights* __restrict__ Wp,
                                     double* __restrict__ av, const double* __restrict__ c, double* __restrict__ u,
                                     const AdjParams* __restrict__ Pp) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n3) return;
    double a = av[q] + Wp->gv * v[q];
    av[q] = a;
    u[q] = 0.5 * Pp->dt * a + c[q];
}

// At state x, with the pending vector u, one warp per atom:
//   ax_i += (J u)_i + wpe * (-F_i) + wpw * sum_j 2 (dW/dq) r_ij
// (J = dF/dx; wpe, wpw the step's weights of PE and W in the loss) and the
// block partials {dF/deps . u, dF/dsigma . u, 2 PE, 2 W, 2 dPE/dsigma, 2 dW/dsigma}.
static __global__ void __launch_bounds__(kThreads)
ad_hvp_kernel(int N, const double4* __restrict__ x, const int* __restrict__ nbr, const int* __restrict__ cnt,
              const AdjParams* __restrict__ Pp, const double* __restrict__ u, const AdjWeights* __restrict__ Wp,
              int use_weights, double* __restrict__ ax, double* __restrict__ partials) {
    const AdjParams P = *Pp;
    const double wpe = use_weights ? Wp->wpe : 0.0, wpw = use_weights ? Wp->wpw : 0.0;
    int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (i < N) {  // uniform across the warp
        double4 xi = x[i];
        double ui[3] = {u[3 * (size_t)i], u[3 * (size_t)i + 1], u[3 * (size_t)i + 2]};
        // ju[3], F[3], gw[3], sum dfds r.u_i, V, W, dV/dsigma, dW/dsigma
        double t[14] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = lane; k < cnt[i]; k += 32) {
            int j = nbr[(size_t)k * N + i];
            double4 xj = x[j];
            double r[3] = {mimg(xi.x - xj.x, P.L[0], P.halfL[0]), mimg(xi.y - xj.y, P.L[1], P.halfL[1]),
                           mimg(xi.z - xj.z, P.L[2], P.halfL[2])};
            PairQ o = pair_q(P, r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            double du[3] = {ui[0] - u[3 * (size_t)j], ui[1] - u[3 * (size_t)j + 1], ui[2] - u[3 * (size_t)j + 2]};
            double rdu = r[0] * du[0] + r[1] * du[1] + r[2] * du[2];
            double rui = r[0] * ui[0] + r[1] * ui[1] + r[2] * ui[2];
            for (int m = 0; m < 3; ++m) {
                t[m] += o.f * du[m] + 2.0 * o.fp * rdu * r[m];
                t[3 + m] += o.f * r[m];
                t[6 + m] += 2.0 * o.dWdq * r[m];
            }
            t[9] += o.dfds * rui;
            t[10] += o.V;
            t[11] += o.W;
            t[12] += o.dVds;
            t[13] += o.dWds;
        }
        warp_reduce<14>(t);
        if (lane == 0) {
            acc[0] = (t[3] * ui[0] + t[4] * ui[1] + t[5] * ui[2]) / P.eps;
            acc[1] = t[9];
            acc[2] = t[10];
            acc[3] = t[11];
            acc[4] = t[12];
            acc[5] = t[13];
            for (int m = 0; m < 3; ++m) ax[3 * (size_t)i + m] += t[m] - wpe * t[3 + m] + wpw * t[6 + m];
        }
    }
    write_partials<6>(acc, partials);
}

// av = av + dt ax; c = dt/2 av
static __global__ void ad_post_kernel(int n3, const double* __restrict__ ax, double* __restrict__ av,
                                      double* __restrict__ c, const AdjParams* __restrict__ Pp) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n3) return;
    const double dt = Pp->dt;
    double b = av[q] + dt * ax[q];
    av[q] = b;
    c[q] = 0.5 * dt * b;
}

}  // namespace

struct lj_adj_ctx {
    lj_adj_params p{};
    int N = 0, nblk = 0, nbw = 0, M = 0, k = 0, ncell_alloc = 0;  // blocks: thread / warp per atom
    int nmax[3] = {0, 0, 0};
    AdjParams P{};
    Grid g{};
    double rho = 0;
    cudaStream_t stream = nullptr;
    AdjParams* dP = nullptr;    // device copy of P, read by every kernel
    AdjWeights* dW = nullptr;   // loss weights of the current backward pass
    // captured forward and backward passes (rebuilt when the cell grid changes)
    cudaGraphExec_t gfwd = nullptr, gbwd = nullptr;
    bool graphs_tried = false;
    double4* x = nullptr;
    double *v = nullptr, *F = nullptr, *ax = nullptr, *av = nullptr, *c = nullptr, *u = nullptr;
    double* fwd_part = nullptr;  // per step n = 0..M: nbw x {2 PE, 2 W} then nblk x {2 KE}
    double* bwd_part = nullptr;  // per state n = 0..M: nbw x 6
    int *cell_of = nullptr, *rank = nullptr, *count = nullptr, *start = nullptr, *members = nullptr,
        *tiles = nullptr, *nbr = nullptr, *cnt = nullptr, *overflow = nullptr;
    double4* ckx = nullptr;  // checkpoints: x at steps 0, k, 2k, ...
    double* ckv = nullptr;   //              v at the same steps
    double4* segx = nullptr; // the k + 1 states of one segment
    double* segv = nullptr;
    std::vector<double> series;  // per state 1..M: PE, W, KE, P
    bool have_forward = false;
    char err[256] = {0};
};

namespace {

#define AK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            std::snprintf(a->err, sizeof a->err, "%s: %s", #call, cudaGetErrorString(e_)); \
            return LJ_ERR_CUDA;                                                            \
        }                                                                                  \
    } while (0)

int nb(int n) { return (n + kThreads - 1) / kThreads; }

size_t fwd_stride(const lj_adj_ctx* a) { return (size_t)a->nbw * 2 + a->nblk; }

void drop_graphs(lj_adj_ctx* a);

// Potential constants and the cell grid for epsilon, sigma (nothing changes on error).
int set_potential(lj_adj_ctx* a, double eps, double sigma) {
    double uc = a->p.cutoff_sigma, uc2 = uc * uc;
    if (!(eps > 0) || !(sigma > 0) || !std::isfinite(eps) || !std::isfinite(sigma)) return LJ_ERR_ARG;
    double rcm6 = 1.0 / (uc2 * uc2 * uc2);
    AdjParams P{};
    Grid g{};
    P.alpha = -4.0 * rcm6 * (rcm6 - 1.0);
    P.beta = 12.0 * rcm6 * (2.0 * rcm6 - 1.0);
    P.eps = eps;
    P.sigma = sigma;
    double rc = uc * sigma;
    P.rc2 = rc * rc;
    P.inv_uc2s2 = 1.0 / (uc2 * sigma * sigma);
    P.inv_sigma = 1.0 / sigma;
    P.dt = a->p.time_delta;
    for (int k = 0; k < 3; ++k) {
        P.L[k] = a->p.box[k];
        P.halfL[k] = 0.5 * a->p.box[k];
        double nd = std::floor(a->p.box[k] / rc);
        int n = nd > 1 << 20 ? 1 << 20 : (int)nd;
        if (a->nmax[k]) n = std::min(n, a->nmax[k]);  // fewer, larger cells stay exact
        if (n < 3) {
            std::snprintf(a->err, sizeof a->err, "box edge %g holds fewer than 3 cells of edge %g", a->p.box[k], rc);
            return LJ_ERR_ARG;  // the minimum-image stencil needs >= 3 cells per axis
        }
        g.n[k] = n;
        g.ratio[k] = (double)n / a->p.box[k];
    }
    bool grid_changed = g.n[0] != a->g.n[0] || g.n[1] != a->g.n[1] || g.n[2] != a->g.n[2];
    a->P = P;
    a->g = g;
    a->have_forward = false;
    if (grid_changed) drop_graphs(a);
    return LJ_OK;
}

// Exact pair list at the positions in a->x.
int build_list(lj_adj_ctx* a) {
    int N = a->N, nc = a->g.ncell();
    int ntiles = (nc + kScanTile - 1) / kScanTile;
    ad_bin_kernel<<<nb(N), kThreads, 0, a->stream>>>(N, a->x, a->g, a->cell_of, a->rank, a->count);
    Gate open{};
    open.always = 1;
    scan_reduce_kernel<false><<<ntiles, 1024, 0, a->stream>>>(a->count, nc, a->tiles, open);
    scan_tiles_kernel<false><<<1, 1024, 0, a->stream>>>(a->tiles, ntiles, open);
    scan_apply_kernel<false><<<ntiles, 1024, 0, a->stream>>>(a->count, nc, a->tiles, a->start, open);  // zeroes count
    ad_members_kernel<<<nb(N), kThreads, 0, a->stream>>>(N, a->cell_of, a->rank, a->start, a->members);
    ad_sort_cells_kernel<<<nb(nc), kThreads, 0, a->stream>>>(nc, a->start, a->members);
    ad_list_kernel<<<nb(32 * N), kThreads, 0, a->stream>>>(N, a->x, a->g, a->cell_of, a->start, a->members, a->dP,
                                                           a->nbr, a->cnt, a->overflow);
    AK(cudaGetLastError());
    return LJ_OK;
}

// Forces at a->x into a->F; energy partials into part.
int forces(lj_adj_ctx* a, double* part) {
    int rc = build_list(a);
    if (rc) return rc;
    ad_force_kernel<<<a->nbw, kThreads, 0, a->stream>>>(a->N, a->x, a->nbr, a->cnt, a->dP, a->F, part);
    AK(cudaGetLastError());
    return LJ_OK;
}

// One step from (x, v, F = F(x)); partials of the new state into part.
int step(lj_adj_ctx* a, double* part) {
    ad_kick_kernel<<<nb(a->N), kThreads, 0, a->stream>>>(a->N, a->x, a->v, a->F, a->dP, 1);
    int rc = forces(a, part);
    if (rc) return rc;
    ad_kick_kernel<<<nb(a->N), kThreads, 0, a->stream>>>(a->N, a->x, a->v, a->F, a->dP, 0);
    ad_ke_kernel<<<a->nblk, kThreads, 0, a->stream>>>(a->N, a->v, part + 2 * (size_t)a->nbw);
    AK(cudaGetLastError());
    return LJ_OK;
}

int check_overflow(lj_adj_ctx* a) {
    int ov = 0;
    AK(cudaMemcpyAsync(&ov, a->overflow, sizeof(int), cudaMemcpyDeviceToHost, a->stream));
    AK(cudaStreamSynchronize(a->stream));
    if (ov) {
        std::snprintf(a->err, sizeof a->err, "a neighbour list exceeded %d entries", kAdjCap);
        return LJ_ERR_CAPACITY;
    }
    return LJ_OK;
}

// The forward pass after x, v and the parameters are on the device: F_0, then
// M steps with a checkpoint every k steps.  Captured once as a graph.
int enqueue_forward(lj_adj_ctx* a) {
    int N = a->N, M = a->M, k = a->k, n3 = 3 * N;
    int rc = forces(a, a->fwd_part);  // F_0 = F(x_0), as the integrator's first force evaluation
    if (rc) return rc;
    for (int n = 0; n < M; ++n) {
        if (n % k == 0) {
            AK(cudaMemcpyAsync(a->ckx + (size_t)(n / k) * N, a->x, sizeof(double4) * N, cudaMemcpyDeviceToDevice,
                               a->stream));
            AK(cudaMemcpyAsync(a->ckv + (size_t)(n / k) * n3, a->v, sizeof(double) * n3, cudaMemcpyDeviceToDevice,
                               a->stream));
        }
        if ((rc = step(a, a->fwd_part + fwd_stride(a) * (n + 1)))) return rc;
    }
    return LJ_OK;
}

// The backward pass after the loss weights are on the device: per segment
// (last first) recompute its states from the checkpoint, then the reverse
// sweep over them.  Captured once as a graph.
int enqueue_backward(lj_adj_ctx* a) {
    int N = a->N, M = a->M, k = a->k, n3 = 3 * N;
    AK(cudaMemsetAsync(a->ax, 0, sizeof(double) * n3, a->stream));
    AK(cudaMemsetAsync(a->av, 0, sizeof(double) * n3, a->stream));
    AK(cudaMemsetAsync(a->c, 0, sizeof(double) * n3, a->stream));
    int rc;
    int nseg = (M + k - 1) / k;
    for (int sgi = nseg - 1; sgi >= 0; --sgi) {
        int n0 = sgi * k, n1 = std::min(M, n0 + k);  // this segment holds states n0 .. n1
        AK(cudaMemcpyAsync(a->x, a->ckx + (size_t)sgi * N, sizeof(double4) * N, cudaMemcpyDeviceToDevice, a->stream));
        AK(cudaMemcpyAsync(a->v, a->ckv + (size_t)sgi * n3, sizeof(double) * n3, cudaMemcpyDeviceToDevice, a->stream));
        AK(cudaMemcpyAsync(a->segv, a->v, sizeof(double) * n3, cudaMemcpyDeviceToDevice, a->stream));
        AK(cudaMemcpyAsync(a->segx, a->x, sizeof(double4) * N, cudaMemcpyDeviceToDevice, a->stream));
        if ((rc = forces(a, a->fwd_part))) return rc;  // recompute: same values as the forward pass
        for (int n = n0; n < n1; ++n) {
            if ((rc = step(a, a->fwd_part + fwd_stride(a) * (n + 1)))) return rc;
            int s = n + 1 - n0;
            AK(cudaMemcpyAsync(a->segx + (size_t)s * N, a->x, sizeof(double4) * N, cudaMemcpyDeviceToDevice,
                               a->stream));
            AK(cudaMemcpyAsync(a->segv + (size_t)s * n3, a->v, sizeof(double) * n3, cudaMemcpyDeviceToDevice,
                               a->stream));
        }
        // reverse over states n1 .. n0 + 1, and state 0 at the very end
        for (int n = n1; n > n0 || n == 0; --n) {
            int s = n - n0;
            AK(cudaMemcpyAsync(a->x, a->segx + (size_t)s * N, sizeof(double4) * N, cudaMemcpyDeviceToDevice,
                               a->stream));
            if ((rc = build_list(a))) return rc;
            double* part = a->bwd_part + 6 * (size_t)a->nbw * n;
            if (n == 0) {
                // x_0 carries no loss: ax += J(x_0) c, theta += dF/dtheta(x_0) . c
                ad_hvp_kernel<<<a->nbw, kThreads, 0, a->stream>>>(N, a->x, a->nbr, a->cnt, a->dP, a->c, a->dW, 0,
                                                                   a->ax, part);
                AK(cudaGetLastError());
                break;
            }
            ad_pre_kernel<<<nb(n3), kThreads, 0, a->stream>>>(n3, a->segv + (size_t)s * n3, a->dW, a->av, a->c, a->u,
                                                              a->dP);
            ad_hvp_kernel<<<a->nbw, kThreads, 0, a->stream>>>(N, a->x, a->nbr, a->cnt, a->dP, a->u, a->dW, 1, a->ax,
                                                               part);
            ad_post_kernel<<<nb(n3), kThreads, 0, a->stream>>>(n3, a->ax, a->av, a->c, a->dP);
            AK(cudaGetLastError());
        }
    }
    return LJ_OK;
}

void drop_graphs(lj_adj_ctx* a) {
    if (a->gfwd) cudaGraphExecDestroy(a->gfwd);
    if (a->gbwd) cudaGraphExecDestroy(a->gbwd);
    a->gfwd = a->gbwd = nullptr;
    a->graphs_tried = false;
}

// One pass captured from the stream into an executable graph; on failure
// *out stays null and the pass is launched kernel by kernel instead.
void capture(lj_adj_ctx* a, int (*pass)(lj_adj_ctx*), cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    int rc = pass(a);
    cudaError_t e = cudaStreamEndCapture(a->stream, &g);
    if (rc == LJ_OK && e == cudaSuccess && g && cudaGraphInstantiate(out, g, 0) != cudaSuccess) *out = nullptr;
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
}

// Capture both passes once per cell grid (a new sigma can change the grid,
// and with it the launch shapes of the binning).
int prepare_graphs(lj_adj_ctx* a) {
    if (a->graphs_tried) return LJ_OK;
    a->graphs_tried = true;
    capture(a, enqueue_forward, &a->gfwd);
    capture(a, enqueue_backward, &a->gbwd);
    return LJ_OK;
}

void free_a(lj_adj_ctx* a) {
    drop_graphs(a);
    void* ptrs[] = {a->x,     a->v,     a->F,     a->ax,    a->av,   a->c,    a->u,   a->fwd_part,
                    a->bwd_part, a->cell_of, a->rank, a->count, a->start, a->members, a->tiles, a->nbr,
                    a->cnt,   a->overflow, a->ckx, a->ckv,  a->segx,  a->segv, a->dP, a->dW};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (a->stream) cudaStreamDestroy(a->stream);
}

}  // namespace

extern "C" {

int lj_adj_create(const lj_adj_params* p, lj_adj_ctx** out) {
    if (!out) return LJ_ERR_ARG;
    *out = nullptr;
    if (!p || p->particle_count < 2 || p->particle_count > (1 << 25) || p->steps < 1 || p->checkpoint_every < 1 || !(p->time_delta > 0) ||
        !(p->cutoff_sigma * p->cutoff_sigma > std::cbrt(2.0)) || !std::isfinite(p->cutoff_sigma))
        return LJ_ERR_ARG;  // lennard_jones_force.cpp:45 asserts rc^2 > 2^(1/3)
    for (int k = 0; k < 3; ++k)
        if (!(p->box[k] > 0) || !std::isfinite(p->box[k])) return LJ_ERR_ARG;
    lj_adj_ctx* a = new (std::nothrow) lj_adj_ctx();
    if (!a) return LJ_ERR_ARG;
    a->p = *p;
    int rc = set_potential(a, p->epsilon, p->sigma);
    if (rc) {
        delete a;
        return rc;
    }
    for (int k = 0; k < 3; ++k) a->nmax[k] = a->g.n[k];
    int N = a->N = p->particle_count;
    a->M = p->steps;
    a->k = std::min(p->checkpoint_every, p->steps);
    a->nblk = nb(N);
    a->nbw = nb(32 * N);
    a->rho = N / (p->box[0] * p->box[1] * p->box[2]);
    int nc = a->ncell_alloc = a->g.ncell();
    if ((nc + kScanTile - 1) / kScanTile > kMaxScanTiles) {
        delete a;
        return LJ_ERR_ARG;
    }
    int nck = (a->M + a->k - 1) / a->k;
    *out = a;  // from here on, errors leave a context that lj_adj_destroy frees
    AK(cudaSetDevice(p->device));
    AK(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking));
    AK(cudaMalloc(&a->x, sizeof(double4) * N));
    for (double** q : {&a->v, &a->F, &a->ax, &a->av, &a->c, &a->u}) AK(cudaMalloc(q, sizeof(double) * 3 * N));
    AK(cudaMalloc(&a->fwd_part, sizeof(double) * fwd_stride(a) * (a->M + 1)));
    AK(cudaMalloc(&a->bwd_part, sizeof(double) * 6 * (size_t)a->nbw * (a->M + 1)));
    for (int** q : {&a->cell_of, &a->rank, &a->members, &a->cnt}) AK(cudaMalloc(q, sizeof(int) * N));
    AK(cudaMalloc(&a->count, sizeof(int) * nc));
    AK(cudaMemset(a->count, 0, sizeof(int) * nc));
    AK(cudaMalloc(&a->start, sizeof(int) * (nc + 1)));
    AK(cudaMalloc(&a->tiles, sizeof(int) * kMaxScanTiles));
    AK(cudaMalloc(&a->nbr, sizeof(int) * (size_t)kAdjCap * N));
    AK(cudaMalloc(&a->overflow, sizeof(int)));
    AK(cudaMalloc(&a->dP, sizeof(AdjParams)));
    AK(cudaMalloc(&a->dW, sizeof(AdjWeights)));
    AK(cudaMemset(a->overflow, 0, sizeof(int)));
    AK(cudaMalloc(&a->ckx, sizeof(double4) * (size_t)N * nck));
    AK(cudaMalloc(&a->ckv, sizeof(double) * 3 * (size_t)N * nck));
    AK(cudaMalloc(&a->segx, sizeof(double4) * (size_t)N * (a->k + 1)));
    AK(cudaMalloc(&a->segv, sizeof(double) * 3 * (size_t)N * (a->k + 1)));
    return LJ_OK;
}

int lj_adj_destroy(lj_adj_ctx* a) {
    if (!a) return LJ_ERR_ARG;
    cudaSetDevice(a->p.device);
    if (a->stream) cudaStreamSynchronize(a->stream);
    free_a(a);
    delete a;
    return LJ_OK;
}

const char* lj_adj_last_error(const lj_adj_ctx* a) { return a ? a->err : "null context"; }

int lj_adj_set_potential(lj_adj_ctx* a, double eps, double sigma) {
    if (!a) return LJ_ERR_ARG;
    return set_potential(a, eps, sigma);
}

int lj_adj_forward(lj_adj_ctx* a, const double* x0, const double* v0, int stride, double* out2, double* series) {
    if (!a || !x0 || !v0 || (stride != 3 && stride != 4) || !out2) return LJ_ERR_ARG;
    AK(cudaSetDevice(a->p.device));
    a->have_forward = false;
    int N = a->N, M = a->M, n3 = 3 * N;
    std::vector<double4> hx((size_t)N);
    std::vector<double> hv((size_t)n3);
    for (int i = 0; i < N; ++i) {
        const double* xi = x0 + (size_t)i * stride;
        hx[(size_t)i] = make_double4(xi[0], xi[1], xi[2], 0.0);
        for (int q = 0; q < 3; ++q) hv[3 * (size_t)i + q] = v0[(size_t)i * stride + q];
    }
    AK(cudaMemcpyAsync(a->x, hx.data(), sizeof(double4) * N, cudaMemcpyHostToDevice, a->stream));
    AK(cudaMemcpyAsync(a->v, hv.data(), sizeof(double) * n3, cudaMemcpyHostToDevice, a->stream));
    AK(cudaMemcpyAsync(a->dP, &a->P, sizeof(AdjParams), cudaMemcpyHostToDevice, a->stream));
    int rc = prepare_graphs(a);
    if (rc) return rc;
    if (a->gfwd) {
        AK(cudaGraphLaunch(a->gfwd, a->stream));
    } else if ((rc = enqueue_forward(a))) {
        return rc;
    }
    std::vector<double> h(fwd_stride(a) * (M + 1));
    AK(cudaMemcpyAsync(h.data(), a->fwd_part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, a->stream));
    if ((rc = check_overflow(a))) return rc;
    a->series.assign(4 * (size_t)M, 0.0);
    double pe_avg = 0, p_avg = 0;
    for (int n = 1; n <= M; ++n) {
        const double* part = h.data() + fwd_stride(a) * n;
        double pe = 0, w = 0, ke = 0;
        for (int b = 0; b < a->nbw; ++b) {  // blocks in order
            pe += part[2 * b];
            w += part[2 * b + 1];
        }
        for (int b = 0; b < a->nblk; ++b) ke += part[2 * (size_t)a->nbw + b];
        pe *= 0.5;
        w *= 0.5;
        ke *= 0.5;
        double T = (2.0 / 3.0) * ke / N;                  // KE = (3/2) N T
        double P = a->rho * (T + w / (3.0 * N));          // analyzers.cpp:73-75
        double* s = a->series.data() + 4 * (size_t)(n - 1);
        s[0] = pe;
        s[1] = w;
        s[2] = ke;
        s[3] = P;
        pe_avg += pe;
        p_avg += P;
    }
    pe_avg /= M;
    p_avg /= M;
    if (!std::isfinite(pe_avg) || !std::isfinite(p_avg)) return LJ_ERR_NONFINITE;
    out2[0] = pe_avg;
    out2[1] = p_avg;
    if (series) std::memcpy(series, a->series.data(), sizeof(double) * 4 * M);
    a->have_forward = true;
    return LJ_OK;
}

int lj_adj_backward(lj_adj_ctx* a, double w_pe, double w_p, double* dx0, double* dv0, int stride, double* deps,
                    double* dsigma) {
    if (!a || !a->have_forward || (stride != 3 && stride != 4) || !std::isfinite(w_pe) || !std::isfinite(w_p))
        return LJ_ERR_ARG;
    AK(cudaSetDevice(a->p.device));
    int N = a->N, M = a->M, n3 = 3 * N;
    // the loss of state n: (w_pe PE_n + w_p P_n) / M, P_n = rho (2 KE_n / 3N + W_n / 3N)
    AdjWeights wts;
    wts.wpe = w_pe / M;
    wts.wpw = w_p / M * a->rho / (3.0 * N);     // weight of W
    wts.gv = w_p / M * a->rho * 2.0 / (3.0 * N);  // d loss / d v = gv v
    const double wpe = wts.wpe, wpw = wts.wpw;
    AK(cudaMemcpyAsync(a->dW, &wts, sizeof wts, cudaMemcpyHostToDevice, a->stream));
    int rc;
    if (a->gbwd) {
        AK(cudaGraphLaunch(a->gbwd, a->stream));
    } else if ((rc = enqueue_backward(a))) {
        return rc;
    }
    std::vector<double> hax((size_t)n3), hav((size_t)n3), hp(6 * (size_t)a->nbw * (M + 1));
    AK(cudaMemcpyAsync(hax.data(), a->ax, sizeof(double) * n3, cudaMemcpyDeviceToHost, a->stream));
    AK(cudaMemcpyAsync(hav.data(), a->av, sizeof(double) * n3, cudaMemcpyDeviceToHost, a->stream));
    AK(cudaMemcpyAsync(hp.data(), a->bwd_part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, a->stream));
    if ((rc = check_overflow(a))) return rc;
    double aeps = 0, asig = 0;
    for (int n = 0; n <= M; ++n) {
        double pr[6] = {0, 0, 0, 0, 0, 0};
        const double* part = hp.data() + 6 * (size_t)a->nbw * n;
        for (int b = 0; b < a->nbw; ++b)
            for (int q = 0; q < 6; ++q) pr[q] += part[6 * (size_t)b + q];
        aeps += pr[0];
        asig += pr[1];
        if (n > 0) {  // explicit parameter dependence of the loss at state n
            double PE = 0.5 * pr[2], W = 0.5 * pr[3], dPEds = 0.5 * pr[4], dWds = 0.5 * pr[5];
            aeps += (wpe * PE + wpw * W) / a->P.eps;
            asig += wpe * dPEds + wpw * dWds;
        }
    }
    for (int i = 0; i < N; ++i)
        for (int q = 0; q < 3; ++q) {
            if (dx0) dx0[(size_t)i * stride + q] = hax[3 * (size_t)i + q];
            if (dv0) dv0[(size_t)i * stride + q] = hav[3 * (size_t)i + q];
        }
    if (deps) *deps = aeps;
    if (dsigma) *dsigma = asig;
    return LJ_OK;
}

}  // extern "C"
