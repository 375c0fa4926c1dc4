// epp_cells.cuh -- cell-list build: bin + atomic count, single-pass exclusive scan, scatter,
// rank-by-id gather (a counting sort with a deterministic within-cell order).
//
// Replaces the reference's fixed-capacity buckets (NeighbourSearch.jl:12-47, clean! at
// NeighbourSystem.jl:43-54): the counts, offsets and membership of every cell equal the
// reference's bucket counts, their exclusive scan and the buckets sorted by particle id.
#pragma once
#include "epp_math.cuh"

namespace epp {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;   // 2048 cells per tile
constexpr long long kSpinLimit = 1ll << 22;            // bounded look-back wait

__device__ __forceinline__ void set_status(unsigned* status, unsigned bits) {
    if (bits) atomicOr(status, bits);
}

// Per-call search, pass 1 (insertParticlesIntoCells!, NeighbourSearch.jl:12-47):
//   immovable particles with a cell keep it; others are binned from their position;
//   particles outside the domain are killed (dead bin = n_cells).
// Block 0 also clears the look-back state of the scan that follows.
template <int D>
__global__ void k_bin_count(int n, DevDomain dom, State s, int* count, int2* cs, int max_cell,
                            unsigned* status, unsigned long long* scan_state, int n_scan_words) {
    if (blockIdx.x == 0)
        for (int t = threadIdx.x; t < n_scan_words; t += blockDim.x) scan_state[t] = 0ull;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = s.cell[i];
    unsigned st = 0;
    if (c != dom.n_cells) {
        int tm = s.tagm[i];
        if (movable_of(tm) || c < 0) {
            c = cell_of<D>(dom, s.xh[i], inst_of(tm));
            if (c < 0) {
                c = dom.n_cells;
                st |= EPP_STATUS_KILLED;
            }
            s.cell[i] = c;
        }
    }
    int slot = atomicAdd(&count[c], 1);
    if (max_cell > 0 && c < dom.n_cells && slot >= max_cell) st |= EPP_STATUS_CELL_OVERFLOW;
    cs[i] = make_int2(c, slot);
    set_status(status, st);
}

// Single-pass exclusive scan with decoupled look-back over m = n_cells + 1 counts (the last is
// the dead bin).  Writes start[0..m], the list of occupied cells occ[0..n_occ) in cell order
// (meta[0] = n_occ) and clears the counts for the next binning pass.  Tiles take a ticket in
// launch order so every predecessor is already running; the wait on a predecessor is bounded
// and reports EPP_STATUS_SPIN_TIMEOUT instead of hanging.
// scan_state layout: [0] ticket, [1 + t] status word of tile t:
//   (flag << 62) | (occupied cells << 31) | particles,  flag 1 = aggregate, 2 = inclusive prefix.
__device__ __forceinline__ unsigned long long pack_status(unsigned long long flag,
                                                          unsigned long long v) {
    // v = (occ << 32) | count  ->  status word
    return (flag << 62) | ((v >> 32) << 31) | (v & 0x7fffffffull);
}
__device__ __forceinline__ unsigned long long unpack_status(unsigned long long w) {
    return (((w >> 31) & 0x7fffffffull) << 32) | (w & 0x7fffffffull);
}

static __global__ void __launch_bounds__(kScanThreads) k_scan(int m, int* count, int* start, int* occ,
                                                       int* meta, unsigned long long* scan_state,
                                                       unsigned* status) {
    __shared__ int s_tile;
    __shared__ unsigned long long s_warp[kScanThreads / 32];
    __shared__ unsigned long long s_prefix;
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(&scan_state[0], 1ull);
    __syncthreads();
    const int tile = s_tile;
    const int base = tile * kScanTile + threadIdx.x * kScanItems;
    const bool full = base + kScanItems <= m;   // the thread's 8 cells are all in range (aligned)
    int v[kScanItems];
    if (full) {   // two 16-byte loads, then zero the counts for the next step
        const int4 a = reinterpret_cast<const int4*>(count + base)[0];
        const int4 b = reinterpret_cast<const int4*>(count + base)[1];
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
        reinterpret_cast<int4*>(count + base)[0] = make_int4(0, 0, 0, 0);
        reinterpret_cast<int4*>(count + base)[1] = make_int4(0, 0, 0, 0);
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            v[k] = base + k < m ? count[base + k] : 0;
            if (base + k < m) count[base + k] = 0;
        }
    }
    unsigned long long tsum = 0;   // (occupied << 32) | particles
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int idx = base + k;
        tsum += (unsigned long long)v[k] + ((idx < m - 1 && v[k] > 0) ? (1ull << 32) : 0ull);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long incl = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = lane < kScanThreads / 32 ? s_warp[lane] : 0ull;
        unsigned long long wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = wi - w;   // exclusive warp offsets
        const unsigned long long total = __shfl_sync(0xffffffffu, wi, kScanThreads / 32 - 1);   // block total
        unsigned long long prefix = 0;
        if (tile == 0) {
            if (lane == 0) atomicExch(&scan_state[1], pack_status(2, total));
        } else {
            if (lane == 0) atomicExch(&scan_state[1 + tile], pack_status(1, total));
            // decoupled look-back, 32 predecessors per round: lane l reads tile p - l; the round
            // ends at the nearest tile with its inclusive prefix published (flag 2), summing the
            // aggregates (flag 1) of the tiles in between; waits (bounded) while any of those has
            // published nothing yet
            volatile unsigned long long* st = scan_state + 1;
            int p = tile - 1;
            long long spins = 0;
            for (;;) {
                const int q = p - lane;
                const unsigned long long w2 = q >= 0 ? st[q] : (2ull << 62);   // before tile 0: inclusive 0
                const unsigned flag = (unsigned)(w2 >> 62);
                const unsigned incl_mask = __ballot_sync(0xffffffffu, flag == 2);
                const unsigned zero_mask = __ballot_sync(0xffffffffu, flag == 0);
                const unsigned need = incl_mask ? ((incl_mask & (0u - incl_mask)) << 1) - 1u : 0xffffffffu;
                if (zero_mask & need) {
                    if (++spins > kSpinLimit) {
                        if (lane == 0) atomicOr(status, EPP_STATUS_SPIN_TIMEOUT);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                unsigned long long x = ((need >> lane) & 1u) ? unpack_status(w2) : 0ull;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                prefix += x;
                if (incl_mask) break;
                p -= 32;
            }
            if (lane == 0) {
                __threadfence();
                atomicExch(&scan_state[1 + tile], pack_status(2, prefix + total));
            }
        }
        if (lane == 0) s_prefix = prefix;
    }
    __syncthreads();
    unsigned long long run = s_prefix + s_warp[warp] + incl - tsum;
    int out[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int idx = base + k;
        out[k] = (int)(run & 0xffffffffull);
        const int oc = (int)(run >> 32);
        if (idx < m - 1 && v[k] > 0) occ[oc] = idx;
        run += (unsigned long long)v[k] + ((idx < m - 1 && v[k] > 0) ? (1ull << 32) : 0ull);
        if (idx == m - 1) {
            start[m] = (int)(run & 0xffffffffull);
            meta[0] = (int)(run >> 32);
        }
    }
    if (full) {
        reinterpret_cast<int4*>(start + base)[0] = make_int4(out[0], out[1], out[2], out[3]);
        reinterpret_cast<int4*>(start + base)[1] = make_int4(out[4], out[5], out[6], out[7]);
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k)
            if (base + k < m) start[base + k] = out[k];
    }
}

// Scatter in arrival order: perm[start[c] + slot] = (id, source index).  A destination outside
// [0, n) can only come from a failed scan; it is reported, never written.
static __global__ void k_scatter(int n, const int2* cs, const int* start, const int* id, int2* perm,
                          unsigned* status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int2 c = cs[i];
    int dst = start[c.x] + c.y;
    if (dst < 0 || dst >= n) {
        atomicOr(status, EPP_STATUS_QUEUE);
        return;
    }
    perm[dst] = make_int2(id[i], i);
}

// Rank within the cell by particle id and hand (src, dst, cell) to the mover.  The dead bin
// keeps arrival order (dead particles never interact).
template <class Mover>
__global__ void k_rank_gather(int n, int n_cells, const int2* perm, const int2* cs,
                              const int* start, Mover mv, unsigned* status) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int2 e = perm[p];
    int src = e.y;
    if (src < 0 || src >= n) {
        atomicOr(status, EPP_STATUS_QUEUE);
        return;
    }
    int c = cs[src].x;
    int s = start[c];
    int rank;
    if (c == n_cells) {
        rank = p - s;
    } else {
        int en = min(start[c + 1], n);
        rank = 0;
        for (int q = max(s, 0); q < en; ++q) rank += perm[q].x < e.x;
    }
    const int dst = s + rank;
    if (dst < 0 || dst >= n) {
        atomicOr(status, EPP_STATUS_QUEUE);
        return;
    }
    mv(src, dst, c);
}

// Mover of the per-call search: every state array follows the particle.
struct MoverAll {
    State a, b;
    __device__ __forceinline__ void operator()(int src, int dst, int c) const {
        b.xh[dst] = a.xh[src];
        b.vm[dst] = a.vm[src];
        b.dv[dst] = a.dv[src];
        b.comp[dst] = a.comp[src];
        b.rho[dst] = a.rho[src];
        b.drho[dst] = a.drho[src];
        b.vol[dst] = a.vol[src];
        b.p[dst] = a.p[src];
        b.tagm[dst] = a.tagm[src];
        b.id[dst] = a.id[src];
        b.cell[dst] = c;
    }
};

}  // namespace epp
