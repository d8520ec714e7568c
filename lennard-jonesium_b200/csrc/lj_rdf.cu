// lj_rdf.cu -- radial distribution histogram (new: the reference has no RDF).
//
// Ordered pairs (i != j) at minimum-image distance r < rmax are counted in bin
// floor(sqrt(r^2) * (nbins / rmax)).  The separation, r^2 and the bin follow
// exactly the arithmetic of the CPU oracle (dd - image * L with image from
// dd > L/2, fma-ordered r^2, IEEE sqrt), so histograms agree bit-for-bit.
//
// Boxes with at least 3 cells of edge >= rmax per axis use a cell list over
// the 27-cell stencil (counting sort into an RDF grid, positions copied in that
// order); smaller boxes use all pairs.  Each block accumulates a shared-memory
// histogram and adds it to the global 64-bit histogram once.

#include <cstdio>

#include "lj_mixed.cuh"

namespace ljb {

namespace {

__device__ __forceinline__ double min_image(double dd, double L, double halfL) {
    double img = dd > halfL ? 1.0 : (dd < -halfL ? -1.0 : 0.0);
    return __dsub_rn(dd, __dmul_rn(img, L));
}

__device__ __forceinline__ void rdf_count(const double4& xi, const double4& xj, const PairParams& pp,
                                          double rmax2, double inv_dr, int nbins, unsigned* sh) {
    double sx = min_image(__dsub_rn(xi.x, xj.x), pp.L[0], pp.halfL[0]);
    double sy = min_image(__dsub_rn(xi.y, xj.y), pp.L[1], pp.halfL[1]);
    double sz = min_image(__dsub_rn(xi.z, xj.z), pp.L[2], pp.halfL[2]);
    double r2 = norm2(sx, sy, sz);
    if (r2 < rmax2) {
        int b = (int)__dmul_rn(__dsqrt_rn(r2), inv_dr);
        if (b < nbins) atomicAdd(&sh[b], 1u);
    }
}

__device__ __forceinline__ void flush(unsigned* sh, int nbins, unsigned long long* hist) {
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        if (sh[b]) atomicAdd(&hist[b], (unsigned long long)sh[b]);
}

__global__ void __launch_bounds__(kThreads)
rdf_all_pairs_kernel(int N, const double4* __restrict__ pos, PairParams pp, double rmax2, double inv_dr,
                     int nbins, unsigned long long* __restrict__ hist) {
    extern __shared__ unsigned sh[];
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) sh[b] = 0;
    __syncthreads();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) {
        double4 xi = pos[i];
        for (int j = 0; j < N; ++j)
            if (j != i) rdf_count(xi, pos[j], pp, rmax2, inv_dr, nbins, sh);
    }
    flush(sh, nbins, hist);
}

__global__ void __launch_bounds__(kThreads)
rdf_cells_kernel(int N, const double4* __restrict__ sorted, Grid g, const int* __restrict__ start,
                 PairParams pp, double rmax2, double inv_dr, int nbins, unsigned long long* __restrict__ hist) {
    extern __shared__ unsigned sh[];
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) sh[b] = 0;
    __syncthreads();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) {
        double4 xi = sorted[i];
        int ci[3] = {cell_coord(xi.x, g.ratio[0], g.n[0]), cell_coord(xi.y, g.ratio[1], g.n[1]),
                     cell_coord(xi.z, g.ratio[2], g.n[2])};
        for (int a = -1; a <= 1; ++a) {
            int na = (ci[0] + a + g.n[0]) % g.n[0];
            for (int b = -1; b <= 1; ++b) {
                int nb = (ci[1] + b + g.n[1]) % g.n[1];
                for (int c = -1; c <= 1; ++c) {
                    int nc = (ci[2] + c + g.n[2]) % g.n[2];
                    int cell = g.flat(na, nb, nc);
                    for (int j = start[cell]; j < start[cell + 1]; ++j)
                        if (j != i) rdf_count(xi, sorted[j], pp, rmax2, inv_dr, nbins, sh);
                }
            }
        }
    }
    flush(sh, nbins, hist);
}

__global__ void rdf_bin_kernel(int N, const double4* __restrict__ pos, Grid g, int* __restrict__ cell_of,
                               int* __restrict__ rank, int* __restrict__ count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double4 x = pos[i];
    int c = g.flat(cell_coord(x.x, g.ratio[0], g.n[0]), cell_coord(x.y, g.ratio[1], g.n[1]),
                   cell_coord(x.z, g.ratio[2], g.n[2]));
    cell_of[i] = c;
    rank[i] = atomicAdd(&count[c], 1);
}

__global__ void rdf_place_kernel(int N, const double4* __restrict__ pos, const int* __restrict__ cell_of,
                                 const int* __restrict__ rank, const int* __restrict__ start,
                                 double4* __restrict__ sorted) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    sorted[start[cell_of[i]] + rank[i]] = pos[i];
}

}  // namespace

int rdf_launch(int N, const double4* pos, const PairParams& pp, int nbins, double rmax,
               unsigned long long* hist_host, cudaStream_t stream, char* err, size_t errlen,
               long long* launches) {
    if ((size_t)nbins * sizeof(unsigned) > 200 * 1024) {
        std::snprintf(err, errlen, "rdf: too many bins for the shared-memory histogram");
        return 1;  // LJ_ERR_ARG
    }
    Grid g;
    int nmin = 1 << 30;
    for (int k = 0; k < 3; ++k) {
        g.n[k] = (int)floor(pp.L[k] / rmax);
        if (g.n[k] < 1) g.n[k] = 1;
        g.ratio[k] = (double)g.n[k] / pp.L[k];
        nmin = g.n[k] < nmin ? g.n[k] : nmin;
    }
    bool cells = nmin >= 3 && g.ncell() <= kScanTile * kMaxScanTiles;
    unsigned long long* dh = nullptr;
    int *cell_of = nullptr, *rank = nullptr, *count = nullptr, *start = nullptr, *tiles = nullptr;
    double4* sorted = nullptr;
    cudaError_t e = cudaMalloc(&dh, sizeof(unsigned long long) * nbins);
    size_t shm = sizeof(unsigned) * nbins;
    if (e == cudaSuccess) e = cudaMemsetAsync(dh, 0, sizeof(unsigned long long) * nbins, stream);
    if (e == cudaSuccess && shm > 48 * 1024) {
        e = cudaFuncSetAttribute(rdf_cells_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(rdf_all_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    }
    double rmax2 = rmax * rmax, inv_dr = (double)nbins / rmax;
    int blocks = (N + kThreads - 1) / kThreads;
    if (e == cudaSuccess && !cells) {
        rdf_all_pairs_kernel<<<blocks, kThreads, shm, stream>>>(N, pos, pp, rmax2, inv_dr, nbins, dh);
        e = cudaGetLastError();
        ++*launches;
    } else if (e == cudaSuccess) {
        int nc = g.ncell();
        int ntiles = (nc + kScanTile - 1) / kScanTile;
        e = cudaMalloc(&cell_of, sizeof(int) * N);
        if (e == cudaSuccess) e = cudaMalloc(&rank, sizeof(int) * N);
        if (e == cudaSuccess) e = cudaMalloc(&count, sizeof(int) * nc);
        if (e == cudaSuccess) e = cudaMalloc(&start, sizeof(int) * (nc + 1));
        if (e == cudaSuccess) e = cudaMalloc(&tiles, sizeof(int) * kMaxScanTiles);
        if (e == cudaSuccess) e = cudaMalloc(&sorted, sizeof(double4) * N);
        if (e == cudaSuccess) e = cudaMemsetAsync(count, 0, sizeof(int) * nc, stream);
        if (e == cudaSuccess) {
            Gate open{};
            open.always = 1;
            rdf_bin_kernel<<<blocks, kThreads, 0, stream>>>(N, pos, g, cell_of, rank, count);
            scan_reduce_kernel<false><<<ntiles, 1024, 0, stream>>>(count, nc, tiles, open);
            scan_tiles_kernel<false><<<1, 1024, 0, stream>>>(tiles, ntiles, open);
            scan_apply_kernel<false><<<ntiles, 1024, 0, stream>>>(count, nc, tiles, start, open);
            rdf_place_kernel<<<blocks, kThreads, 0, stream>>>(N, pos, cell_of, rank, start, sorted);
            rdf_cells_kernel<<<blocks, kThreads, shm, stream>>>(N, sorted, g, start, pp, rmax2, inv_dr, nbins, dh);
            e = cudaGetLastError();
            *launches += 6;
        }
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hist_host, dh, sizeof(unsigned long long) * nbins, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(dh);
    cudaFree(cell_of);
    cudaFree(rank);
    cudaFree(count);
    cudaFree(start);
    cudaFree(tiles);
    cudaFree(sorted);
    if (e != cudaSuccess) {
        std::snprintf(err, errlen, "rdf: %s", cudaGetErrorString(e));
        return 2;  // LJ_ERR_CUDA
    }
    return 0;
}

}  // namespace ljb
