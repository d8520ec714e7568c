// lj_common.cuh -- device helpers shared by the engine's kernels.
//
// Arithmetic that must reproduce the reference bit-for-bit (integration,
// periodic wrap, cell index, separation, r^2 and the cutoff test) is written
// with explicit round-to-nearest intrinsics so that nvcc cannot contract it
// into FMAs; the CPU oracle (oracle/ljref.cpp) uses the same fixed order.
#pragma once

#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

namespace ljb {

constexpr int kThreads = 128;             // block size of per-atom kernels
// Neighbour entry: slot << 6 | offset code, the code holding i + 1 (0, 1, 2)
// for each axis' offset i in {-1, 0, 1} in 2 bits (x: bits 0-1, y: 2-3, z: 4-5)
// -- the stencil cell's offset from the home cell, or in small-box lists the
// lattice image.
constexpr unsigned kCodeBits = 6;
constexpr unsigned kGhostCode = 0x15;     // offset (0, 0, 0)
constexpr int kMaxAtoms = 1 << 26;        // 67M atoms per context
constexpr int kScanTile = 4096;           // cells per scan tile (1024 threads x 4)
constexpr int kMaxScanTiles = 1024;

struct Grid {
    int n[3];
    double ratio[3];  // n_k / L_k, computed first as in particle_pair_filter.cpp:144-147
    __host__ __device__ int ncell() const { return n[0] * n[1] * n[2]; }
    __host__ __device__ int flat(int a, int b, int c) const { return (a * n[1] + b) * n[2] + c; }
};

// Device-resident scalars of one system.
struct Scalars {
    double t, pe, vir;
    unsigned long long max_disp2;  // bits of a non-negative double: max |d - d_build|^2 this step
    unsigned long long max_disp2_next;  // the same for the next step, from a fused pair-kernel epilogue
    int need_rebuild;              // set by the host (upload, forced rebuild)
    int overflow;                  // a neighbour list overflowed
    int nonfinite;                 // a non-finite energy or virial was seen
    int max_count;                 // largest neighbour count at the last build
    long long builds;              // neighbour-list builds so far
    long long steps;
    long long graph_rebuilds;      // rebuild subgraphs executed by step graphs
};

// Physical constants of the pair kernel.
struct PairParams {
    double L[3];
    double halfL[3];
    int halfL_hi[3];   // high word of L/2: a cheap |d| > L/2 test on the integer pipe
    double rc, rc2, inv_rc2;
    double alpha, beta;  // LJ spline (lennard_jones_force.cpp:68-73)
    double strength;     // constant-force mock
    double near_lo, near_hi[3];  // an atom with all coords in [near_lo, near_hi) needs no image
    double dt;
};

// ---- reference-order arithmetic ------------------------------------------

// v += (1/2) F dt  (integrator.cpp:70 and :82)
__device__ __forceinline__ double kick(double v, double f, double dt) {
    return __dadd_rn(v, __dmul_rn(__dmul_rn(0.5, f), dt));
}

// x -= floor(x / L) * L  (boundary_condition.cpp:45-48)
__device__ __forceinline__ double wrap(double x, double L) {
    return __dsub_rn(x, __dmul_rn(floor(__ddiv_rn(x, L)), L));
}

// clamp(floor(x * (n / L)), 0, n - 1)  (particle_pair_filter.cpp:144-147; the
// clamp only touches positions the reference would index out of bounds)
__device__ __forceinline__ int cell_coord(double x, double ratio, int n) {
    int c = (int)floor(__dmul_rn(x, ratio));
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

// fma(s_z, s_z, fma(s_y, s_y, s_x * s_x))
__device__ __forceinline__ double norm2(double sx, double sy, double sz) {
    return __fma_rn(sz, sz, __fma_rn(sy, sy, __dmul_rn(sx, sx)));
}

__device__ __forceinline__ int image_code(int ix, int iy, int iz) {
    return 9 * (ix + 1) + 3 * (iy + 1) + (iz + 1);
}

__host__ __device__ __forceinline__ unsigned offset_code(int ix, int iy, int iz) {
    return (unsigned)(ix + 1) | ((unsigned)(iy + 1) << 2) | ((unsigned)(iz + 1) << 4);
}

__host__ __device__ __forceinline__ unsigned make_entry(unsigned slot, unsigned code) {
    return (slot << kCodeBits) | code;
}

__device__ __forceinline__ unsigned entry_slot(unsigned e) { return e >> kCodeBits; }

// offset of axis k (0, 1, 2) in {-1, 0, 1}
__device__ __forceinline__ int entry_axis(unsigned e, int k) { return (int)((e >> (2 * k)) & 3u) - 1; }

// ---- reductions ------------------------------------------------------------

template <int Q>
__device__ __forceinline__ void warp_sum(double (&v)[Q]) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int q = 0; q < Q; ++q) v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
}

// Deterministic block sum of Q doubles; result valid in thread 0.
template <int Q, int NT>
__device__ __forceinline__ void block_sum(double (&v)[Q]) {
    __shared__ double sm[NT / 32][Q];
    warp_sum<Q>(v);
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < Q; ++q) sm[warp][q] = v[q];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < Q; ++q) v[q] = lane < NT / 32 ? sm[lane][q] : 0.0;
        warp_sum<Q>(v);
    }
    __syncthreads();
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    return v;
}

// Exclusive scan of one int per thread across a block of NT threads.
template <int NT>
__device__ __forceinline__ int block_exclusive_scan(int x, int* total) {
    __shared__ int warp_tot[NT / 32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = x;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = lane < NT / 32 ? warp_tot[lane] : 0;
        int wi = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, wi, off);
            if (lane >= off) wi += y;
        }
        if (lane < NT / 32) warp_tot[lane] = wi - w;
        if (lane == NT / 32 - 1 && total) *total = wi;
    }
    __syncthreads();
    int res = incl - x + warp_tot[warp];
    __syncthreads();
    return res;
}

}  // namespace ljb
