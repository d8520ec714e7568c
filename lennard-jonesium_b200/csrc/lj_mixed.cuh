// lj_mixed.cuh -- mixed-precision pair kernel: FP32 pair arithmetic (r^2, the
// r^-6 terms, V, W and the force magnitude), FP64 per-atom force accumulation,
// FP64 integration and FP64 global sums.
//
// Positions for the pair kernel are FP32 *cell-local* coordinates: at each
// list build an atom's offset from the origin of its list cell, xl = x - c*a
// (a = L / n, the cell edge), is kept in FP64 (bx); every step
// xl = bx + (d - d_build) follows the unwrapped displacement, so a periodic
// wrap never moves it.  The neighbour entry carries the stencil offset delta of
// the neighbour's cell, and the separation is
//     s = (xl_i - xl_j) - delta * a
// which equals the reference's (x_i - x_j) - image * L (particle_pair_filter.cpp:180-183)
// in exact arithmetic while keeping every FP32 operand below a few sigma, so
// the FP32 rounding error of s is ~1e-7 absolute instead of ~1e-5 for box
// coordinates at L ~ 100.
//
// Pair forces are summed in FP32 over chunks of 8 consecutive neighbours and
// each chunk sum is added into the FP64 per-atom accumulator, which keeps the
// FP64 conversion traffic at one per chunk per component; PER_PAIR instead
// converts and adds every pair's terms in FP64 (no FP32 sum at all, the mixed
// step 15 % slower at 1M atoms).  The energy and virial come, as on the FP64
// path, from the power sums sum u^2, sum u, sum r^2 and the pair count
// (lj_energy), formed in FP64 from the FP32 chunk sums.  The loop structure
// (groups of 4 with the next group's indices in flight, branch-free cutoff) is
// that of the FP64 kernel; the FP32 reciprocal is the hardware approximation
// (rcp.approx, about 1 ulp), adequate for FP32 pair arithmetic.
#pragma once

#include "lj_kernels.cuh"

namespace ljb {

struct MixedParams {
    float rc2, inv_rc2, alpha, beta;
    float a[3];  // list-cell edge per axis
    // the spline's virial as a function of r^2: W = u(48u - 24) + wq r^2 with
    // u = r^-6 (lennard_jones_force.cpp:107-119), so the force magnitude over r
    // is f = W / r^2 = u(48u - 24) r^-2 + wq
    float wq;
};

inline MixedParams mixed_params(const PairParams& pp, const Grid& g) {
    MixedParams m;
    m.rc2 = (float)pp.rc2;
    m.inv_rc2 = (float)pp.inv_rc2;
    m.alpha = (float)pp.alpha;
    m.beta = (float)pp.beta;
    for (int k = 0; k < 3; ++k) m.a[k] = (float)(pp.L[k] / g.n[k]);
    m.wq = (float)(-2.0 * pp.beta * pp.inv_rc2);
    return m;
}

// After a list build: local coordinate of each slot relative to its list cell.
static __global__ void __launch_bounds__(kThreads)
mixed_build_local_kernel(int N, const double4* __restrict__ pos, Soa s, Grid g, double* __restrict__ bx,
                         float4* __restrict__ posl, Gate gate) {
    if (!gate.open()) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double4 x = pos[i];
    double xs[3] = {x.x, x.y, x.z};
    float l[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        int c = cell_coord(xs[k], g.ratio[k], g.n[k]);
        double o = (double)c * (1.0 / g.ratio[k]);
        double b = xs[k] - o;
        bx[(size_t)k * N + i] = b;
        l[k] = (float)b;
    }
    posl[i] = make_float4(l[0], l[1], l[2], 0.f);
}

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The 4 neighbour positions of one list group.
__device__ __forceinline__ void gather4(const float4* __restrict__ posl, const uint4 grp, float4 (&q)[4]) {
    q[0] = posl[entry_slot(grp.x)];
    q[1] = posl[entry_slot(grp.y)];
    q[2] = posl[entry_slot(grp.z)];
    q[3] = posl[entry_slot(grp.w)];
}

// Stencil offset of one axis from its 2-bit code c = i + 1 at bit position
// 2k: 2^23 + (c << 2k) is exact in FP32, so subtracting 2^23 + (1 << 2k)
// gives i * 4^k exactly (no shift needed to extract the field); the offset
// i * a is then that value times a / 4^k, an exact product.
__device__ __forceinline__ float code_bias(unsigned e, unsigned field_mask) {
    return __uint_as_float(0x4b000000u | (e & field_mask));
}

template <bool KICK, int BS = kThreads, bool PER_PAIR = false>
static __global__ void __launch_bounds__(BS, 768 / BS)
force_mixed_kernel(int N, const float4* __restrict__ posl, Soa s, const uint4* __restrict__ nbr4,
                   const int* __restrict__ cnt, PairParams pp, MixedParams mp,
                   double* __restrict__ partials, Fuse fu) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0, 0, 0, 0};
    double m = 0.0;
    const float2 na_xy = make_float2(-mp.a[0], -0.25f * mp.a[1]);
    const float az16 = 0.0625f * mp.a[2];
    const float2 unbias = make_float2(-8388609.0f, -8388612.0f);
    if (i < N) {
        const float4 xi = posl[i];
        const float2 xi_xy = make_float2(xi.x, xi.y);
        // FP64 per-atom accumulators: the force and the power sums of the
        // energy and virial (sum u^2, sum u, sum r^2, pair count; lj_energy)
        double fx = 0, fy = 0, fz = 0, su2 = 0, su = 0, sr2 = 0;
        int nh = 0;
        // list indices stream from HBM: two groups in flight ahead of the two
        // being evaluated (the neighbour positions, mostly L1/L2 hits, are
        // gathered per group)
        int ng = (cnt[i] + 3) >> 2;
        const uint4* lp = nbr4 + i;
        const uint4 z4 = make_uint4(0u, 0u, 0u, 0u);
        uint4 A = ng > 0 ? __ldcs(lp) : z4;
        uint4 B = ng > 1 ? __ldcs(lp + (size_t)N) : z4;
        const float2 mone = make_float2(-1.f, -1.f);
        // one group: 4 neighbours into the FP32 chunk sums, (x, y) of the force
        // and (sum u^2, sum u) as packed pairs
        auto group = [&](const uint4 grp, float2& cxy, float& cz, float2& cuu, float& cr2) {
            float4 Q[4];
            gather4(posl, grp, Q);
            const unsigned e[4] = {grp.x, grp.y, grp.z, grp.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                // s = (xl_i - xl_j) - offset * a, the offset product exact
                float2 t_xy = __fadd2_rn(make_float2(code_bias(e[u], 0x3u), code_bias(e[u], 0xcu)), unbias);
                float tz = code_bias(e[u], 0x30u) - 8388624.0f;
                float2 d_xy = __ffma2_rn(make_float2(Q[u].x, Q[u].y), mone, xi_xy);  // xi - q, one rounding
                d_xy = __ffma2_rn(t_xy, na_xy, d_xy);
                float dx = d_xy.x, dy = d_xy.y;
                float dz = fmaf(-tz, az16, xi.z - Q[u].z);
                float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                bool hit = r2 < mp.rc2;
                float ir2 = rcp_approx(r2);
                float ir6 = ir2 * ir2 * ir2;
                // f = W / r^2 = u(48u - 24) r^-2 + wq
                float f = hit ? fmaf(ir6 * fmaf(48.f, ir6, -24.f), ir2, mp.wq) : 0.f;
                float uh = hit ? ir6 : 0.f;
                float rh = hit ? r2 : 0.f;
                nh += hit ? 1 : 0;
                if (PER_PAIR) {
                    fx += (double)(f * dx);
                    fy += (double)(f * dy);
                    fz += (double)(f * dz);
                    su2 += (double)(uh * uh);
                    su += (double)uh;
                    sr2 += (double)rh;
                } else {
                    cxy = __ffma2_rn(make_float2(f, f), d_xy, cxy);
                    cz = fmaf(f, dz, cz);
                    cuu = __ffma2_rn(make_float2(uh, uh), make_float2(uh, 1.f), cuu);
                    cr2 += rh;
                }
            }
        };
        // chunks of 2 groups = 8 neighbours summed in FP32, then added in FP64
        for (int g = 0; g < ng; g += 2) {
            uint4 C = g + 2 < ng ? __ldcs(lp + (size_t)(g + 2) * N) : z4;
            uint4 D = g + 3 < ng ? __ldcs(lp + (size_t)(g + 3) * N) : z4;
            float2 cxy = make_float2(0.f, 0.f), cuu = make_float2(0.f, 0.f);
            float cz = 0.f, cr2 = 0.f;
            group(A, cxy, cz, cuu, cr2);
            if (g + 1 < ng) group(B, cxy, cz, cuu, cr2);
            if (!PER_PAIR) {
                fx += (double)cxy.x;
                fy += (double)cxy.y;
                fz += (double)cz;
                su2 += (double)cuu.x;
                su += (double)cuu.y;
                sr2 += (double)cr2;
            }
            A = C;
            B = D;
        }
        s.at(FX, i) = fx;
        s.at(FY, i) = fy;
        s.at(FZ, i) = fz;
        LjSums a;
        a.su2 = su2;
        a.su = su;
        a.sr2 = sr2;
        a.nh = nh;
        lj_energy(pp, a, acc[1], acc[2]);
        if (KICK) {
            const double f3[3] = {fx, fy, fz};
            const double4 x = fu.pos_next ? fu.pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
            m = step_epilogue(N, i, s, x, f3, pp, fu, acc);
        }
    }
    if (KICK) fused_track(fu, m);
    block_sum<4, BS>(acc);
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; ++q) partials[(size_t)blockIdx.x * 4 + q] = acc[q];
}

// Radial distribution histogram (lj_rdf.cu).
//
// Scratch of the cell-list histogram: sized on first use and kept, so that a
// sample costs no allocation and no synchronisation.  hist holds two
// histograms of `bins` counts: the running accumulator, then a single sample.
struct RdfScratch {
    int atoms = 0, cells = 0, bins = 0;  // capacities
    int* cell_of = nullptr;
    int* rank = nullptr;
    int* count = nullptr;
    int* start = nullptr;
    int* tiles = nullptr;
    double4* sorted = nullptr;
    unsigned long long* hist = nullptr;
    // the running accumulation (lj_gpu_rdf_accumulate)
    int acc_bins = 0;
    double acc_rmax = 0.0;
    long long samples = 0;
};

// Grid of cells of edge >= rmax with at most max_cells cells (coarser cells
// where the box holds more; the histogram does not depend on the cell size).
Grid rdf_grid(const double L[3], double rmax, long long max_cells);
// The cell-list kernels need >= 3 cells per axis; otherwise all pairs.
bool rdf_uses_cells(const Grid& g);
// Grow the scratch to N atoms, ncell cells and nbins bins (returns 2 on a CUDA error).
int rdf_reserve(RdfScratch& s, int N, int ncell, int nbins);
void rdf_release(RdfScratch& s);
// Allow a shared-memory histogram of nbins counts (above 48 KB).
int rdf_set_smem(int nbins);
// Enqueue one sample: ordered pairs counted into hist (device, nbins counts),
// which is added to, not cleared.  Returns 0, or 2 on a CUDA error.
int rdf_enqueue(int N, const double4* pos, const PairParams& pp, const Grid& g, int nbins, double rmax,
                const RdfScratch& s, unsigned long long* hist, cudaStream_t stream, long long* launches);

}  // namespace ljb
