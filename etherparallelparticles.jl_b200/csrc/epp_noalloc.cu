// epp_noalloc.cu -- cell-list build for callers that cannot allocate device memory.
//
// Some hosts of this library may not call cudaMalloc while they drive a simulation: a host
// application whose device memory comes from its own fixed pool, or a caller in the middle of a
// step where a device allocation would synchronise the device or is simply not permitted.  For
// them epp_cell_sort_noalloc runs the same bin -> count -> scan -> scatter -> rank-by-id pipeline
// as the context's search!, on device buffers the caller passes in, with every intermediate
// array in one statically sized device array declared below.  That array is part of the library:
// every GPU that loads libepp.so holds it until the process exits.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <mutex>

#include "epp_cells.cuh"

using namespace epp;

namespace {

constexpr int kNaMaxParticles = 1 << 20;   // largest n accepted
constexpr int kNaMaxCells = 1 << 20;       // largest domain (cells) accepted
constexpr int kNaTiles = (kNaMaxCells + 1 + kScanTile - 1) / kScanTile;

// Layout of the scratch (bytes, each part 256-aligned):
//   counts   int   [kNaMaxCells + 2]
//   scan     u64   [kNaTiles + 1]        look-back state of the scan
//   cs       int2  [kNaMaxParticles]     (cell, slot) per particle
//   perm     int2  [kNaMaxParticles]     (id, particle) in arrival order
//   start    int   [kNaMaxCells + 2]     offsets before they are copied out
//   occ      int   [kNaMaxCells + 1]     occupied cells (written by the scan, unused here)
//   meta     int   [64]
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kOffCounts = 0;
constexpr size_t kOffScan = kOffCounts + align256(sizeof(int) * (kNaMaxCells + 2));
constexpr size_t kOffCs = kOffScan + align256(sizeof(unsigned long long) * (kNaTiles + 1));
constexpr size_t kOffPerm = kOffCs + align256(sizeof(int2) * kNaMaxParticles);
constexpr size_t kOffStart = kOffPerm + align256(sizeof(int2) * kNaMaxParticles);
constexpr size_t kOffOcc = kOffStart + align256(sizeof(int) * (kNaMaxCells + 2));
constexpr size_t kOffMeta = kOffOcc + align256(sizeof(int) * (kNaMaxCells + 1));
constexpr size_t kScratchBytes = kOffMeta + align256(sizeof(int) * 64);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
// Device address of the scratch, per device, looked up on the first call on that device.  The
// look-up is guarded, so first calls from several host threads at once are safe (the calls
// themselves still share the scratch and must not overlap on the GPU).
std::atomic<unsigned char*> g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mu;

// Bin particle i (positions column-major: x at pos[i], y at pos[n + i], z at pos[2n + i]); outside
// the domain -> dead bin (n_cells), as NeighbourSearch.jl:41-43 kills it.
template <int D>
__global__ void k_na_bin(int n, DevDomain dom, const float* pos, int* count, int2* cs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 x = make_float4(pos[i], pos[(size_t)n + i], D == 3 ? pos[(size_t)2 * n + i] : 0.0f, 0.0f);
    int c = cell_of<D>(dom, x, 0);
    if (c < 0) c = dom.n_cells;
    const int slot = atomicAdd(&count[c], 1);
    cs[i] = make_int2(c, slot);
}

// Rank inside the cell by particle id; writes the 1-based id to its sorted position.
// A permutation entry or destination outside 0..n-1 is skipped and reported (EPP_STATUS_QUEUE).
__global__ void k_na_rank(int n, int n_cells, const int2* perm, const int2* cs, const int* start,
                          int* sorted_ids, unsigned* status) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int2 e = perm[p];
    const int src = e.y;
    if (src < 0 || src >= n) {
        atomicOr(status, EPP_STATUS_QUEUE);
        return;
    }
    const int c = cs[src].x;
    if (c >= n_cells) return;   // dead particles are not part of the cell list
    const int s = start[c], en = min(start[c + 1], n);
    int rank = 0;
    for (int q = max(s, 0); q < en; ++q) rank += perm[q].x < e.x;
    const int dst = s + rank;
    if (dst < 0 || dst >= n) {
        atomicOr(status, EPP_STATUS_QUEUE);
        return;
    }
    sorted_ids[dst] = e.x + 1;
}

// Scatter in arrival order: perm[start[c] + slot] = (particle id, particle id).
__global__ void k_na_scatter(int n, const int2* cs, const int* start, int2* perm, unsigned* status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 c = cs[i];
    const int dst = start[c.x] + c.y;
    if (dst < 0 || dst >= n) {
        atomicOr(status, EPP_STATUS_QUEUE);
        return;
    }
    perm[dst] = make_int2(i, i);
}

__global__ void k_na_counts(int n_cells, const int* start, int* counts, int* offsets) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n_cells && counts) counts[c] = start[c + 1] - start[c];
    if (c <= n_cells && offsets) offsets[c] = start[c];
}

}  // namespace

extern "C" {

int32_t epp_noalloc_limits(int32_t* max_particles, int32_t* max_cells, int64_t* scratch_bytes) {
    if (max_particles) *max_particles = kNaMaxParticles;
    if (max_cells) *max_cells = kNaMaxCells;
    if (scratch_bytes) *scratch_bytes = (int64_t)kScratchBytes;
    return EPP_OK;
}

int32_t epp_cell_sort_noalloc(const epp_domain* domain, int32_t n, const float* pos, int32_t* counts,
                              int32_t* offsets, int32_t* sorted_ids, int32_t* n_alive, void* stream) {
    if (!domain || n < 0 || (n > 0 && !pos) || !sorted_ids || !n_alive) return EPP_ERR_INVALID_ARGUMENT;
    if (n > kNaMaxParticles) return EPP_ERR_CAPACITY;
    DevDomain dom;
    std::memset(&dom, 0, sizeof dom);
    if (const int rc = plan_domain(*domain, 1, kNaMaxCells, dom)) return rc;   // the context's cell grid
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return EPP_ERR_CUDA;
    // set-up, once per device, with that device current: the scratch's device address
    unsigned char* base = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!base) {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        base = g_scratch_addr[dev].load(std::memory_order_acquire);
        if (!base) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return EPP_ERR_CUDA;
            base = static_cast<unsigned char*>(p);
            g_scratch_addr[dev].store(base, std::memory_order_release);
        }
    }
    int* count = reinterpret_cast<int*>(base + kOffCounts);
    unsigned long long* scan = reinterpret_cast<unsigned long long*>(base + kOffScan);
    int2* cs = reinterpret_cast<int2*>(base + kOffCs);
    int2* perm = reinterpret_cast<int2*>(base + kOffPerm);
    int* start = reinterpret_cast<int*>(base + kOffStart);
    int* occ = reinterpret_cast<int*>(base + kOffOcc);
    int* meta = reinterpret_cast<int*>(base + kOffMeta);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nc = dom.n_cells;
    const int tiles = (nc + 1 + kScanTile - 1) / kScanTile;
    // the scratch keeps the last call's contents: clear what must start at zero
    if (cudaMemsetAsync(count, 0, sizeof(int) * (nc + 2), s) != cudaSuccess ||
        cudaMemsetAsync(scan, 0, sizeof(unsigned long long) * (tiles + 1), s) != cudaSuccess ||
        cudaMemsetAsync(meta, 0, sizeof(int) * 64, s) != cudaSuccess)
        return EPP_ERR_CUDA;
    const int T = 128;
    const int gb = (n + T - 1) / T;
    if (n > 0) {
        if (domain->dim == 2) k_na_bin<2><<<gb, T, 0, s>>>(n, dom, pos, count, cs);
        else k_na_bin<3><<<gb, T, 0, s>>>(n, dom, pos, count, cs);
    }
    k_scan<<<tiles, kScanThreads, 0, s>>>(nc + 1, count, start, occ, meta, scan,
                                          reinterpret_cast<unsigned*>(meta + 1));
    unsigned* status = reinterpret_cast<unsigned*>(meta + 1);
    if (n > 0) {
        k_na_scatter<<<gb, T, 0, s>>>(n, cs, start, perm, status);
        k_na_rank<<<gb, T, 0, s>>>(n, nc, perm, cs, start, sorted_ids, status);
    }
    k_na_counts<<<(nc + 1 + T - 1) / T, T, 0, s>>>(nc, start, counts, offsets);
    if (cudaGetLastError() != cudaSuccess) return EPP_ERR_CUDA;
    unsigned st = 0;
    if (cudaMemcpyAsync(n_alive, start + nc, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&st, status, sizeof st, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return EPP_ERR_CUDA;
    return st ? EPP_ERR_DEVICE_STATUS : EPP_OK;
}

}  // extern "C"
