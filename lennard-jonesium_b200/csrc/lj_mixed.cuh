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
// FP64 conversion traffic at one per chunk per component.  The loop structure
// (groups of 4 with the next group's indices in flight, branch-free cutoff) is
// that of the FP64 kernel; the FP32 reciprocal is the hardware approximation
// (rcp.approx, about 1 ulp), adequate for FP32 pair arithmetic.
#pragma once

#include "lj_kernels.cuh"

namespace ljb {

struct MixedParams {
    float rc2, inv_rc2, alpha, beta;
    float a[3];  // list-cell edge per axis
};

inline MixedParams mixed_params(const PairParams& pp, const Grid& g) {
    MixedParams m;
    m.rc2 = (float)pp.rc2;
    m.inv_rc2 = (float)pp.inv_rc2;
    m.alpha = (float)pp.alpha;
    m.beta = (float)pp.beta;
    for (int k = 0; k < 3; ++k) m.a[k] = (float)(pp.L[k] / g.n[k]);
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

template <bool KICK, int BS = kThreads>
static __global__ void __launch_bounds__(BS, 512 / BS)
force_mixed_kernel(int N, const float4* __restrict__ posl, Soa s, const uint4* __restrict__ nbr4,
                   const int* __restrict__ cnt, PairParams pp, MixedParams mp,
                   double* __restrict__ partials) {
    __shared__ float4 off[27];
    if (threadIdx.x < 27) {
        int c = threadIdx.x;
        off[c] = make_float4((float)(c / 9 - 1) * mp.a[0], (float)((c / 3) % 3 - 1) * mp.a[1],
                             (float)(c % 3 - 1) * mp.a[2], 0.f);
    }
    __syncthreads();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0, 0, 0, 0};
    if (i < N) {
        const float4 xi = posl[i];
        double fx = 0, fy = 0, fz = 0, pe = 0, w = 0;
        int ng = (cnt[i] + 3) >> 2;
        uint4 cur = ng > 0 ? __ldcs(&nbr4[i]) : make_uint4(0, 0, 0, 0);
        for (int g0 = 0; g0 < ng; g0 += 2) {
            // one chunk = 2 groups = 8 neighbours summed in FP32, then added in FP64
            float cx = 0.f, cy = 0.f, cz = 0.f, cv = 0.f, cw = 0.f;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                int g = g0 + h;
                if (g < ng) {
                    uint4 nxt = g + 1 < ng ? __ldcs(&nbr4[(size_t)(g + 1) * N + i]) : cur;
                    unsigned e[4] = {cur.x, cur.y, cur.z, cur.w};
                    float4 q[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) q[u] = posl[e[u] & kSlotMask];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        float4 o = off[e[u] >> kSlotBits];
                        float dx = (xi.x - q[u].x) - o.x;
                        float dy = (xi.y - q[u].y) - o.y;
                        float dz = (xi.z - q[u].z) - o.z;
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
                    cur = nxt;
                }
            }
            fx += (double)cx;
            fy += (double)cy;
            fz += (double)cz;
            pe += (double)cv;
            w += (double)cw;
        }
        s.at(FX, i) = fx;
        s.at(FY, i) = fy;
        s.at(FZ, i) = fz;
        acc[1] = pe;
        acc[2] = w;
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
    block_sum<4, BS>(acc);
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; ++q) partials[(size_t)blockIdx.x * 4 + q] = acc[q];
}

// Radial distribution histogram (lj_rdf.cu).
int rdf_launch(int N, const double4* pos, const PairParams& pp, int nbins, double rmax,
               unsigned long long* hist_host, cudaStream_t stream, char* err, size_t errlen,
               long long* launches);

}  // namespace ljb
