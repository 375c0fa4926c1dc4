// epp_tile.cuh -- the default pair passes: warp tiles over a shared candidate list.
//
// A warp takes 32 consecutive particles in cell order.  When their cells lie in one cell row
// (x from xa to xb at fixed y, z) the union of their 3^D stencils is, for each of the 3^(D-1)
// stencil rows (y+dy, z+dz), the cells xa-1 .. xb+1 -- contiguous in cell order, so 3 (2D) or
// 9 (3D) contiguous particle ranges shared by the whole warp.  A warp that crosses a row end
// (about 2% of them) uses each lane's own stencil instead; both passes make the same choice.
//
// Phase A (search pass): the candidates are staged 32 at a time in shared memory with one
// coalesced 16-byte load per lane; every lane then tests all 32 staged candidates against its own
// particle with broadcast shared-memory reads -- all lanes in lockstep, no divergence -- using
// the reference's IEEE criterion, and packs the results into one 32-bit word per chunk: the
// particle's neighbour mask over the first CAP candidates of the warp's enumeration.  Phase B:
// each lane walks the set bits of its own mask in one flattened loop (candidate order), checks
// the active-pair matrix and adds the pair term; candidates past CAP (very dense cells) follow
// in a per-lane tail loop, in order.  The search pass stores each particle's accepted
// neighbours (sorted indices, in summation order) as a list; the next momentum pass sees the
// same positions and cells, so it walks that list (k_list) instead of searching again.
//
// Summation order per particle = stencil rows (z, y offset), then cell order, then id order
// inside a cell: deterministic, a rounding-level reordering of the reference's list order.
#pragma once
#include "epp_cellpair.cuh"

namespace epp {

// (2 harmonic(h_i, h_j))^2 with IEEE operations; kept out of line (rare: h_j != cached h_j).
__device__ __noinline__ float pair_r2(float hi, float hj) {
    const float h2 = harmonic2_exact(hi, hj);
    return __fmul_rn(h2, h2);
}

template <int D>
struct TileConf {
    static constexpr int NR = D == 2 ? 3 : 9;    // stencil rows of one cell row
    static constexpr int NRMAX = NR;             // ranges of a tile (one cell row) or one particle
    static constexpr int NW = D == 2 ? 8 : 32;   // mask words per particle (32 candidates each)
    static constexpr int CAP = 32 * NW;          // candidates covered by the mask
};

struct TileMask {
    unsigned* words;   // [NW * cap]: word w of particle i at w * cap + i
    int cap;
    int* list;         // [LCAP * cap]: k-th neighbour (sorted index) of particle i at k * cap + i
};

template <int D>
struct ListConf {
    static constexpr int LCAP = D == 2 ? 64 : 160;   // neighbours kept per particle
};

// Candidate ranges (contiguous particle index ranges) of a warp tile or of one particle.
template <int D>
struct TileRanges {
    int lo[TileConf<D>::NRMAX], len[TileConf<D>::NRMAX];
    int n, total;

    __device__ __forceinline__ void add(const PairArgs& A, int row, int xa, int xb) {
        // cells xa..xb (clamped) of linear cell row `row`
        const int n0 = A.dom.n[0];
        xa = max(xa, 0);
        xb = min(xb, n0 - 1);
        int l = 0, h = 0;
        if (xa <= xb) {
            l = max(A.start[row * n0 + xa], 0);
            h = min(A.start[row * n0 + xb + 1], A.n_max);
            h = max(h, l);
        }
        lo[n] = l;
        len[n] = h - l;
        total += h - l;
        ++n;
    }
    // The stencil of the cells [xa, xb] of cell row (y, z): rows (y+dy, z+dz), x in [xa-1, xb+1].
    __device__ __forceinline__ void stencil(const PairArgs& A, int y, int z, int xa, int xb) {
        const int n1 = A.dom.n[1];
#pragma unroll
        for (int dz = (D == 3 ? -1 : 0); dz <= (D == 3 ? 1 : 0); ++dz) {
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
                const int yy = y + dy, zz = z + dz;
                const bool in = yy >= 0 && yy < n1 && (D == 2 || (zz >= 0 && zz < A.dom.n[2]));
                if (in) add(A, yy + n1 * zz, xa - 1, xb + 1);
                else add(A, 0, 1, 0);   // empty range keeps the row slots aligned
            }
        }
    }
    // candidate index k (0 <= k < total) -> particle index
    __device__ __forceinline__ int at(int k) const {
        int j = 0;
#pragma unroll
        for (int r = 0; r < TileConf<D>::NRMAX; ++r) {
            if (r < n && k >= 0 && k < len[r]) j = lo[r] + k;
            k -= r < n ? len[r] : 0;
        }
        return j;
    }
};

// UH: every particle has the same h (checked at upload), so both criteria reduce to
// dr^2 <= R^2 with one constant (gap^2, or (2 harmonic(h, h))^2 -- the same IEEE value).
template <int D, bool BUILD, class Act, bool EPI, bool UH>
__global__ void __launch_bounds__(128, D == 2 ? 8 : 6) k_tile(PairArgs A, TileMask M, Act act, unsigned long long* pairs,
                                                 unsigned long long* scan_state, int n_scan_words) {
    static_assert(BUILD, "the reuse pass is k_list");
    constexpr int NW = TileConf<D>::NW;
    constexpr int CAP = TileConf<D>::CAP;
    __shared__ float4 s_x[4][32];
    if (EPI && blockIdx.x == 0)
        for (int t = threadIdx.x; t < n_scan_words; t += blockDim.x) scan_state[t] = 0ull;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int w0 = i - lane;
    int cnt = 0;
    if (w0 < n_alive) {   // warp-uniform
        const bool on = i < n_alive;
        const int c_first = A.s.cell[w0];
        const int c_last = A.s.cell[min(w0 + 31, n_alive - 1)];
        EPP_CHECK(c_first >= 0 && c_first < A.dom.n_cells && c_last >= c_first && c_last < A.dom.n_cells, 11, c_last);
        const int n0 = A.dom.n[0];
        const int r0 = c_first / n0, r1 = c_last / n0;
        // tile mode: the warp's cells lie in one cell row (all but the ~2% of warps that cross
        // a row end); otherwise every lane uses its own stencil (same choice in every pass)
        const bool tiled = r1 == r0;
        TileRanges<D> R;
        if (tiled) {
            R.n = 0;
            R.total = 0;
            R.stencil(A, r0 % A.dom.n[1], r0 / A.dom.n[1], c_first - r0 * n0, c_last - r0 * n0);
        } else {
            const int c = A.s.cell[min(i, n_alive - 1)];
            const int ry = (c / n0) % A.dom.n[1], rz = (c / n0) / A.dom.n[1];
            R.n = 0;
            R.total = 0;
            R.stencil(A, ry, rz, c % n0, c % n0);
        }
        const float4 xi = on ? A.s.xh[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const int ti = on ? tag_of(A.s.tagm[i]) : 0;
        const bool valid = on && ti >= 1 && ti <= A.n_tags;
        if (on && !valid) atomicOr(A.status, EPP_STATUS_BAD_TAG);
        const bool want = valid && act.wants(ti);
        const TargetConst tc = target_const<D>(on ? xi.w : 1.0f);
        unsigned st = 0;
        float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        unsigned local_words[NW];   // this pass's mask (dynamic index: local memory, L1)
        float hc_h = xi.w;                      // criterion cache: last h_j and its exact R^2
        float hc_r2 = A.crit == EPP_CRITERION_DEFAULT ? A.dom.gap_square : tc.h2sq;
        // ---- phase A: lockstep filter over staged chunks (search pass only) ----
        if (BUILD && !tiled) {
            // per-lane stencil (warps that cross a cell-row end): mask bits of the first CAP candidates
            unsigned cur = 0u;
            int k = 0;
            for (int r = 0; r < R.n && k < CAP; ++r) {
                for (int j = R.lo[r]; j < R.lo[r] + R.len[r] && k < CAP; ++j, ++k) {
                    EPP_CHECK(j >= 0 && j < A.n_max, 14, j);
                    bool ok = false;
                    if (want) {
                        const float4 xj = A.s.xh[j];
                        const float dx = __fsub_rn(xi.x, xj.x);
                        const float dy = __fsub_rn(xi.y, xj.y);
                        float dr2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                        if (D == 3) {
                            const float dz = __fsub_rn(xi.z, xj.z);
                            dr2 = __fadd_rn(dr2, __fmul_rn(dz, dz));
                        }
                        if (A.crit == EPP_CRITERION_DEFAULT) {
                            ok = dr2 <= A.dom.gap_square;
                        } else if (xj.w == xi.w) {
                            ok = dr2 <= tc.h2sq;
                        } else {
                            const float h2 = harmonic2_exact(xi.w, xj.w);
                            ok = dr2 <= __fmul_rn(h2, h2);
                        }
                    }
                    cur |= (unsigned)ok << (k & 31);
                    if ((k & 31) == 31) {
                        local_words[k >> 5] = cur;
                        if (M.words && on) M.words[(size_t)(k >> 5) * M.cap + i] = cur;
                        cur = 0u;
                    }
                }
            }
            if (k & 31) {
                local_words[k >> 5] = cur;
                if (M.words && on) M.words[(size_t)(k >> 5) * M.cap + i] = cur;
            }
        }
        if (BUILD && tiled) {
            // mask words of the first CAP candidates (the rest: tail loop below)
            const int nchunk = min((R.total + 31) >> 5, NW);
            for (int ch = 0; ch < nchunk; ++ch) {
                const int k = (ch << 5) + lane;
                const int jj = k < R.total ? R.at(k) : 0;
                EPP_CHECK(jj >= 0 && jj < A.n_max, 12, jj);
                // padding past the last candidate is far away with h = 0: it fails every test
                s_x[wib][lane] = k < R.total ? A.s.xh[jj] : make_float4(1e30f, 1e30f, 1e30f, 0.0f);
                __syncwarp();
                unsigned word = 0u;
                if (UH) {
                    const float R2 = A.crit == EPP_CRITERION_DEFAULT ? A.dom.gap_square : tc.h2sq;
#pragma unroll 16
                    for (int b = 0; b < 32; ++b) {
                        const float4 xj = s_x[wib][b];
                        const float dx = __fsub_rn(xi.x, xj.x);
                        const float dy = __fsub_rn(xi.y, xj.y);
                        float dr2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                        if (D == 3) {
                            const float dz = __fsub_rn(xi.z, xj.z);
                            dr2 = __fadd_rn(dr2, __fmul_rn(dz, dz));
                        }
                        word |= (unsigned)(dr2 <= R2) << b;
                    }
                } else {
                    // a handful of distinct h values: cache the exact bound of the last h_j seen
#pragma unroll 8
                    for (int b = 0; b < 32; ++b) {
                        const float4 xj = s_x[wib][b];
                        const float dx = __fsub_rn(xi.x, xj.x);
                        const float dy = __fsub_rn(xi.y, xj.y);
                        float dr2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                        if (D == 3) {
                            const float dz = __fsub_rn(xi.z, xj.z);
                            dr2 = __fadd_rn(dr2, __fmul_rn(dz, dz));
                        }
                        if (xj.w != hc_h) {
                            hc_h = xj.w;
                            hc_r2 = A.crit == EPP_CRITERION_DEFAULT ? A.dom.gap_square : pair_r2(xi.w, xj.w);
                        }
                        word |= (unsigned)(dr2 <= hc_r2) << b;
                    }
                }
                if (!want) word = 0u;
                EPP_CHECK(!(M.words && on) || i < M.cap, 15, i);
                local_words[ch] = word;
                if (M.words && on) M.words[(size_t)ch * M.cap + i] = word;
                __syncwarp();
            }
        }
        // ---- phase B: the lane's own neighbours, in candidate order.  All loads of a neighbour
        //      are issued together (tag, position, state) and the next mask word is fetched one
        //      word ahead, so each pair costs one memory round trip. ----
        if (want) {
            const int nwords = min((R.total + 31) >> 5, NW);
            const unsigned amask = A.adj[ti - 1];
            const typename Act::Self me = act.self(i);
            HPairCache pc{-1.0f, 0.0f, 0.0f, 0.0f};
            float4 part = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            int w = 0;
            unsigned bits = 0u, ahead = 0u;
            if (nwords > 0) bits = local_words[0];
            if (nwords > 1) ahead = local_words[1];
            int r = 0, roff = 0;   // range cursor: k increases monotonically
            for (;;) {
                while (!bits && ++w < nwords) {
                    bits = ahead;
                    if (w + 1 < nwords) ahead = local_words[w + 1];
                }
                if (!bits) break;
                const int b = __ffs(bits) - 1;
                bits &= bits - 1u;
                const int k = (w << 5) + b;
                while (r < R.n - 1 && k >= roff + R.len[r]) {
                    roff += R.len[r];
                    ++r;
                }
                const int j = R.lo[r] + (k - roff);
                EPP_CHECK(j >= 0 && j < A.n_max, 13, j);
                const int tj = tag_of(A.s.tagm[j]);
                const float4 xj = A.s.xh[j];
                const typename Act::Nb nb = act.fetch(j, ti, tj);
                if (j == i) continue;
                if (tj < 1 || tj > A.n_tags) {
                    st |= EPP_STATUS_BAD_TAG;
                    continue;
                }
                if (!((amask >> (tj - 1)) & 1u)) continue;
                if (M.list && cnt < ListConf<D>::LCAP) M.list[(size_t)cnt * M.cap + i] = j;
                const float4 c = act.term(me, nb, ti, tj, xj, geometry<D>(xi, xj), tc, pc);
                part.x += c.x;
                part.y += c.y;
                part.z += c.z;
                ++cnt;
            }
            sum = part;
            // candidates past the mask's capacity (very dense cells): filtered inline, in
            // candidate order, after the mask's pairs -- the order of the stored list too
            if (R.total > CAP) {
                int k0 = 0;
                for (int r = 0; r < R.n; ++r) {
                    for (int j = R.lo[r] + max(CAP - k0, 0); j < R.lo[r] + R.len[r]; ++j) {
                        EPP_CHECK(j >= 0 && j < A.n_max, 17, j);
                        const float4 xj = A.s.xh[j];
                        if (!accept<D>(A, i, xi, amask, tc.h2sq, j, xj, st)) continue;
                        const int tj = tag_of(A.s.tagm[j]);
                        if (M.list && cnt < ListConf<D>::LCAP) M.list[(size_t)cnt * M.cap + i] = j;
                        const float4 c = act.term(me, act.fetch(j, ti, tj), ti, tj, xj, geometry<D>(xi, xj), tc, pc);
                        sum.x += c.x;
                        sum.y += c.y;
                        sum.z += c.z;
                        ++cnt;
                    }
                    k0 += R.len[r];
                }
            }
        }
        if (st) atomicOr(A.status, st);
        if (on) {
            if (want) act.end(i, ti, sum, cnt);
            else act.end_idle(i, ti);
        }
    } else if (EPI && i < A.n_max) {
        act.end_idle(i, tag_of(A.s.tagm[i]));
    }
    if (EPI && w0 < n_alive && i >= n_alive && i < A.n_max) act.end_idle(i, tag_of(A.s.tagm[i]));
    count_pairs(pairs, cnt);
}

// Neighbours of particle i from its own stencil, filtered inline (used when the list of the last
// search overflowed); same order as the search pass.
template <int D, class Act>
__device__ __noinline__ float4 neighbours_by_stencil(const PairArgs& A, int i, float4 xi, int ti,
                                                     const TargetConst& tc, const Act& act, int* count) {
    const int c = A.s.cell[i];
    const int n0 = A.dom.n[0];
    TileRanges<D> R;
    R.n = 0;
    R.total = 0;
    R.stencil(A, (c / n0) % A.dom.n[1], (c / n0) / A.dom.n[1], c % n0, c % n0);
    const unsigned amask = A.adj[ti - 1];
    unsigned st = 0;
    const typename Act::Self me = act.self(i);
    HPairCache pc{-1.0f, 0.0f, 0.0f, 0.0f};
    float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    int cnt = 0;
    for (int r = 0; r < R.n; ++r)
        for (int j = R.lo[r]; j < R.lo[r] + R.len[r]; ++j) {
            const float4 xj = A.s.xh[j];
            if (!accept<D>(A, i, xi, amask, tc.h2sq, j, xj, st)) continue;
            const int tj = tag_of(A.s.tagm[j]);
            const float4 t = act.term(me, act.fetch(j, ti, tj), ti, tj, xj, geometry<D>(xi, xj), tc, pc);
            sum.x += t.x;
            sum.y += t.y;
            sum.z += t.z;
            ++cnt;
        }
    if (st) atomicOr(A.status, st);
    *count = cnt;
    return sum;
}

// Momentum over the neighbour list written by the last search pass (same positions, cells and
// criterion): one thread per particle, a coalesced list read per neighbour, the next index
// fetched one ahead.  EPI: fused step (integrate + bin for every particle, dead bin included;
// block 0 clears the scan state).
template <int D, class Act, bool EPI>
__global__ void __launch_bounds__(128, D == 2 ? 8 : 4) k_list(PairArgs A, TileMask M, const int* ncount, Act act,
                                                             unsigned long long* scan_state, int n_scan_words) {
    if (EPI && blockIdx.x == 0)
        for (int t = threadIdx.x; t < n_scan_words; t += blockDim.x) scan_state[t] = 0ull;
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_alive) {
        const float4 xi = A.s.xh[i];
        const int ti = tag_of(A.s.tagm[i]);
        if (ti < 1 || ti > A.n_tags || !act.wants(ti)) {
            act.end_idle(i, ti);
        } else {
            const TargetConst tc = target_const<D>(xi.w);
            const int cnt = ncount[i];
            float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            int got = cnt;
            if (cnt <= ListConf<D>::LCAP) {
                const typename Act::Self me = act.self(i);
                HPairCache pc{-1.0f, 0.0f, 0.0f, 0.0f};
                int j = cnt > 0 ? M.list[i] : 0;
                for (int k = 0; k < cnt; ++k) {
                    EPP_CHECK(j >= 0 && j < A.n_max, 16, j);
                    const int jn = k + 1 < cnt ? M.list[(size_t)(k + 1) * M.cap + i] : 0;
                    const int tj = tag_of(A.s.tagm[j]);
                    const float4 xj = A.s.xh[j];
                    const float4 t = act.term(me, act.fetch(j, ti, tj), ti, tj, xj, geometry<D>(xi, xj), tc, pc);
                    sum.x += t.x;
                    sum.y += t.y;
                    sum.z += t.z;
                    j = jn;
                }
            } else {
                sum = neighbours_by_stencil<D>(A, i, xi, ti, tc, act, &got);
            }
            act.end(i, ti, sum, got);
        }
    } else if (EPI && i < A.n_max) {
        act.end_idle(i, tag_of(A.s.tagm[i]));
    }
}

}  // namespace epp
