// lj_rdf.cu -- radial distribution histogram (new: the reference has no RDF).
//
// Ordered pairs (i != j) at minimum-image distance r < rmax are counted in bin
// floor(sqrt(r^2) * (nbins / rmax)).  The separation, r^2 and the bin follow
// exactly the arithmetic of the CPU oracle (dd - image * L with image from
// dd > L/2, fma-ordered r^2, IEEE sqrt), so histograms agree bit-for-bit.
//
// Boxes with at least 3 cells of edge >= rmax per axis use a cell list over
// the half-shell stencil (counting sort into an RDF grid, positions copied in
// that order; each unordered pair evaluated once and counted twice); smaller
// boxes use all pairs.  Each block accumulates a shared-memory
// histogram and adds it to the global 64-bit histogram once.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>

#include "lj_mixed.cuh"

namespace ljb {

namespace {

__device__ __forceinline__ double min_image(double dd, double L, double halfL) {
    double img = dd > halfL ? 1.0 : (dd < -halfL ? -1.0 : 0.0);
    return __dsub_rn(dd, __dmul_rn(img, L));
}

template <unsigned INC>
__device__ __forceinline__ void rdf_count(const double4& xi, const double4& xj, const PairParams& pp,
                                          double rmax2, double inv_dr, int nbins, unsigned* sh) {
    double sx = min_image(__dsub_rn(xi.x, xj.x), pp.L[0], pp.halfL[0]);
    double sy = min_image(__dsub_rn(xi.y, xj.y), pp.L[1], pp.halfL[1]);
    double sz = min_image(__dsub_rn(xi.z, xj.z), pp.L[2], pp.halfL[2]);
    double r2 = norm2(sx, sy, sz);
    if (r2 < rmax2) {
        int b = (int)__dmul_rn(__dsqrt_rn(r2), inv_dr);
        if (b < nbins) atomicAdd(&sh[b], INC);
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
            if (j != i) rdf_count<1u>(xi, pos[j], pp, rmax2, inv_dr, nbins, sh);
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
        // half shell: the own cell's later atoms and the 13 stencil cells after
        // the own cell in (a, b, c) order; each unordered pair is met once and
        // counts for both ordered pairs (the separation of (j, i) is exactly the
        // negated one of (i, j), so both fall in the same bin)
        for (int j = i + 1; j < start[g.flat(ci[0], ci[1], ci[2]) + 1]; ++j)
            rdf_count<2u>(xi, sorted[j], pp, rmax2, inv_dr, nbins, sh);
        for (int s = 14; s < 27; ++s) {
            int a = s / 9 - 1, b = (s / 3) % 3 - 1, c = s % 3 - 1;
            int cell = g.flat((ci[0] + a + g.n[0]) % g.n[0], (ci[1] + b + g.n[1]) % g.n[1],
                              (ci[2] + c + g.n[2]) % g.n[2]);
            for (int j = start[cell]; j < start[cell + 1]; ++j)
                rdf_count<2u>(xi, sorted[j], pp, rmax2, inv_dr, nbins, sh);
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

Grid rdf_grid(const double L[3], double rmax, long long max_cells) {
    // floor(L / rmax) in double: a tiny rmax gives a huge count, not an int overflow
    double n[3];
    for (int k = 0; k < 3; ++k) n[k] = std::max(1.0, std::floor(L[k] / rmax));
    double prod = n[0] * n[1] * n[2];
    if (prod > (double)max_cells) {
        double f = std::cbrt((double)max_cells / prod);
        for (int k = 0; k < 3; ++k) n[k] = std::max(1.0, std::floor(n[k] * f));
        while (n[0] * n[1] * n[2] > (double)max_cells) {
            int k = n[0] >= n[1] ? (n[0] >= n[2] ? 0 : 2) : (n[1] >= n[2] ? 1 : 2);
            n[k] -= 1.0;
        }
    }
    Grid g;
    for (int k = 0; k < 3; ++k) {
        g.n[k] = (int)n[k];
        g.ratio[k] = (double)g.n[k] / L[k];
    }
    return g;
}

bool rdf_uses_cells(const Grid& g) { return g.n[0] >= 3 && g.n[1] >= 3 && g.n[2] >= 3; }

int rdf_enqueue(int N, const double4* pos, const PairParams& pp, const Grid& g, int nbins, double rmax,
                const RdfScratch& s, unsigned long long* hist, cudaStream_t stream, long long* launches) {
    double rmax2 = rmax * rmax, inv_dr = (double)nbins / rmax;
    size_t shm = sizeof(unsigned) * nbins;
    int blocks = (N + kThreads - 1) / kThreads;
    if (!rdf_uses_cells(g)) {
        rdf_all_pairs_kernel<<<blocks, kThreads, shm, stream>>>(N, pos, pp, rmax2, inv_dr, nbins, hist);
        ++*launches;
        return cudaGetLastError() == cudaSuccess ? 0 : 2;
    }
    int nc = g.ncell();
    int ntiles = (nc + kScanTile - 1) / kScanTile;
    if (cudaMemsetAsync(s.count, 0, sizeof(int) * nc, stream) != cudaSuccess) return 2;
    Gate open{};
    open.always = 1;
    rdf_bin_kernel<<<blocks, kThreads, 0, stream>>>(N, pos, g, s.cell_of, s.rank, s.count);
    scan_reduce_kernel<false><<<ntiles, 1024, 0, stream>>>(s.count, nc, s.tiles, open);
    scan_tiles_kernel<false><<<1, 1024, 0, stream>>>(s.tiles, ntiles, open);
    scan_apply_kernel<false><<<ntiles, 1024, 0, stream>>>(s.count, nc, s.tiles, s.start, open);
    rdf_place_kernel<<<blocks, kThreads, 0, stream>>>(N, pos, s.cell_of, s.rank, s.start, s.sorted);
    rdf_cells_kernel<<<blocks, kThreads, shm, stream>>>(N, s.sorted, g, s.start, pp, rmax2, inv_dr, nbins, hist);
    *launches += 6;
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int rdf_set_smem(int nbins) {
    size_t shm = sizeof(unsigned) * nbins;
    if (shm <= 48 * 1024) return 0;
    if (cudaFuncSetAttribute(rdf_cells_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm) != cudaSuccess ||
        cudaFuncSetAttribute(rdf_all_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm) !=
            cudaSuccess)
        return 2;
    return 0;
}

int rdf_reserve(RdfScratch& s, int N, int ncell, int nbins) {
    if (N > s.atoms) {
        cudaFree(s.cell_of);
        cudaFree(s.rank);
        cudaFree(s.sorted);
        s.cell_of = s.rank = nullptr;
        s.sorted = nullptr;
        s.atoms = 0;
        if (cudaMalloc(&s.cell_of, sizeof(int) * N) != cudaSuccess ||
            cudaMalloc(&s.rank, sizeof(int) * N) != cudaSuccess ||
            cudaMalloc(&s.sorted, sizeof(double4) * N) != cudaSuccess)
            return 2;
        s.atoms = N;
    }
    if (ncell > s.cells) {
        cudaFree(s.count);
        cudaFree(s.start);
        s.count = s.start = nullptr;
        s.cells = 0;
        if (cudaMalloc(&s.count, sizeof(int) * ncell) != cudaSuccess ||
            cudaMalloc(&s.start, sizeof(int) * (ncell + 1)) != cudaSuccess)
            return 2;
        s.cells = ncell;
    }
    if (!s.tiles && cudaMalloc(&s.tiles, sizeof(int) * kMaxScanTiles) != cudaSuccess) return 2;
    if (nbins > s.bins) {
        unsigned long long* h = nullptr;
        if (cudaMalloc(&h, sizeof(unsigned long long) * 2 * (size_t)nbins) != cudaSuccess) return 2;
        // a running accumulation moves to the new buffer (rare: a larger
        // single sample taken in the middle of an accumulation)
        // (the samples were enqueued on a non-blocking stream: wait for the device first)
        if (s.samples > 0 &&
            (cudaDeviceSynchronize() != cudaSuccess ||
             cudaMemcpy(h, s.hist, sizeof(unsigned long long) * s.acc_bins, cudaMemcpyDeviceToDevice) != cudaSuccess)) {
            cudaFree(h);
            return 2;
        }
        cudaFree(s.hist);
        s.hist = h;
        s.bins = nbins;
    }
    return 0;
}

void rdf_release(RdfScratch& s) {
    void* ptrs[] = {s.cell_of, s.rank, s.count, s.start, s.tiles, s.sorted, s.hist};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    s = RdfScratch{};
}

}  // namespace ljb

namespace ljb {

// ---------------------------------------------------------------------------
// Allocation-free RDF entry point.
//
// For callers that may not call cudaMalloc: an application whose GPU memory is
// owned by its own pool allocator (a deep-learning framework, for instance,
// whose caching allocator must see every allocation), or a per-step analysis
// hook in a time-critical loop, where cudaMalloc's latency and the implicit
// device-wide synchronisation that cudaMalloc/cudaFree can cause are not
// acceptable.  They pass device buffers they already own for the positions and
// the histogram; the cell-list scratch comes from the fixed device array below.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// library holds it (about 5.3 MB) until the process exits.  All calls on a
// device share it and it keeps the last call's contents; each call clears what
// must start at zero (the cell counts and the output histogram) on its stream.
// Calls whose work overlaps on the GPU (different streams, or several host
// threads) race on the shared array: serialise them.
// ---------------------------------------------------------------------------

namespace {

constexpr int kNoAllocMaxAtoms = 131072;
constexpr int kNoAllocMaxCells = 32768;
constexpr int kNoAllocMaxBins = 12288;  // 48 KB shared-memory histogram, no attribute change needed
constexpr size_t kOffSorted = 0;
constexpr size_t kOffCellOf = kOffSorted + sizeof(double4) * kNoAllocMaxAtoms;
constexpr size_t kOffRank = kOffCellOf + sizeof(int) * kNoAllocMaxAtoms;
constexpr size_t kOffCount = kOffRank + sizeof(int) * kNoAllocMaxAtoms;
constexpr size_t kOffStart = kOffCount + sizeof(int) * kNoAllocMaxCells;
constexpr size_t kOffTiles = kOffStart + sizeof(int) * (kNoAllocMaxCells + 256);
constexpr size_t kNoAllocBytes = kOffTiles + sizeof(int) * kMaxScanTiles;
static_assert(kOffCellOf % 256 == 0 && kOffRank % 256 == 0 && kOffCount % 256 == 0 &&
              kOffStart % 256 == 0 && kOffTiles % 256 == 0, "scratch sub-buffers must stay aligned");

__device__ __align__(256) unsigned char g_rdf_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::atomic<unsigned char*> g_scratch_addr[kMaxDevices];

// Device address of g_rdf_scratch on the current device, looked up on the
// first call on each device and cached for the life of the process.  A
// cudaDeviceReset (or anything else that destroys and recreates the device's
// primary context) reloads the module and may move the array: the cached
// address is then stale, so a process that resets a device must not call
// lj_gpu_rdf_noalloc on it afterwards.
int scratch_address(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 2;
    unsigned char* p = g_scratch_addr[dev].load();
    if (!p) {
        void* q = nullptr;
        if (cudaGetSymbolAddress(&q, g_rdf_scratch) != cudaSuccess || !q) return 2;
        p = static_cast<unsigned char*>(q);
        g_scratch_addr[dev].store(p);
    }
    *out = p;
    return 0;
}

}  // namespace

}  // namespace ljb

extern "C" int lj_gpu_rdf_noalloc(const double* pos, int N, const double* box, int nbins, double rmax,
                                  unsigned long long* hist, void* stream_handle) {
    using namespace ljb;
    if (!pos || !box || !hist || N < 1 || nbins < 1 || !(rmax > 0)) return 1;  // LJ_ERR_ARG
    if (N > kNoAllocMaxAtoms || nbins > kNoAllocMaxBins) return 1;
    // double4 position loads need 16-byte alignment, the 64-bit histogram atomics 8
    if ((reinterpret_cast<uintptr_t>(pos) & 15) != 0 || (reinterpret_cast<uintptr_t>(hist) & 7) != 0) return 1;
    PairParams pp{};
    for (int k = 0; k < 3; ++k) {
        if (!(box[k] > 0) || !std::isfinite(box[k]) || rmax > 0.5 * box[k]) return 1;
        pp.L[k] = box[k];
        pp.halfL[k] = 0.5 * box[k];
    }
    // cells of edge >= rmax, coarser where the box holds more than the array's
    // kNoAllocMaxCells of them (the histogram does not depend on the cell size)
    Grid g = rdf_grid(pp.L, rmax, kNoAllocMaxCells);
    unsigned char* base = nullptr;
    if (scratch_address(&base)) return 2;  // LJ_ERR_CUDA
    RdfScratch sc{};
    sc.sorted = reinterpret_cast<double4*>(base + kOffSorted);
    sc.cell_of = reinterpret_cast<int*>(base + kOffCellOf);
    sc.rank = reinterpret_cast<int*>(base + kOffRank);
    sc.count = reinterpret_cast<int*>(base + kOffCount);
    sc.start = reinterpret_cast<int*>(base + kOffStart);
    sc.tiles = reinterpret_cast<int*>(base + kOffTiles);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    if (cudaMemsetAsync(hist, 0, sizeof(unsigned long long) * nbins, stream) != cudaSuccess) return 2;
    long long launches = 0;
    return rdf_enqueue(N, reinterpret_cast<const double4*>(pos), pp, g, nbins, rmax, sc, hist, stream, &launches);
}
