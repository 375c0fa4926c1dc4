// epp_mask.cuh -- the 2D pair passes over stencil-row masks.
//
// In 2D a particle's 3x3 cell stencil is three stencil rows (dy = -1, 0, +1); in each row its
// candidates are the contiguous cell-order range of cells cx-1 .. cx+1 (a "window" of about 27
// particles at h = 1.5 dx).  The search pass records, per particle and stencil row, one 32-bit
// word whose bit k says whether candidate k of that window passed the reference's criterion and
// the active-pair matrix: 12 bytes per particle in place of a neighbour list of about 25 entries.
// Every pair pass walks the set bits in ascending order -- stencil rows, then cell order, then id
// order inside a cell, the order of the neighbour lists -- so the sums are the same.
//
// A warp takes 32 consecutive particles in cell order.  When their cells lie in one cell row, the
// union of their windows in stencil row r is one contiguous range (cells xa-1 .. xb+1); the warp
// stages it in shared memory (one union row of up to 64 candidates at a time, two coalesced loads
// per lane) and every lane reads its own window from there.  The search pass tests only its own
// window (27 candidates, not the ~190 of the warp's union) and folds the continuity sum of the
// search action into the same walk over the accepted bits, so no separate continuity pass reads
// the neighbours again.  Warps that cross a cell-row end, and union rows longer than 64, read the
// candidates from global memory instead; a particle whose window holds more than 32 candidates
// (dense neighbourhoods) is marked and takes its neighbours from its stencil in every pass.
#pragma once
#include "epp_tile.cuh"

namespace epp {

constexpr int kRowSlots = 64;                    // union candidates of one stencil row staged at once
constexpr unsigned kMaskOverflow = 0xffffffffu;  // own-row word of a particle read from its stencil:
                                                 // its own bit is never set otherwise

struct RowWin {
    int lo, hi;   // candidate range [lo, hi) in cell order
};

// Linear cell row of stencil row r (0, 1, 2 for dy = -1, 0, +1) of the cell row `rid` (y + n1 k;
// k is the instance of a batch), or -1 when y + dy is outside the grid.
__device__ __forceinline__ int stencil_row(const PairArgs& A, int rid, int r) {
    const int y = rid % A.dom.n[1];
    const int yy = y + r - 1;
    return (yy >= 0 && yy < A.dom.n[1]) ? rid + r - 1 : -1;
}

// Candidates of cells xa .. xb (clamped to the grid) of linear cell row `row` (-1: none).
__device__ __forceinline__ RowWin row_range(const PairArgs& A, int row, int xa, int xb) {
    RowWin w{0, 0};
    if (row < 0) return w;
    const int n0 = A.dom.n[0];
    xa = max(xa, 0);
    xb = min(xb, n0 - 1);
    if (xa > xb) return w;
    const int l = max(A.start[row * n0 + xa], 0);
    const int h = min(A.start[row * n0 + xb + 1], A.n_max);
    w.lo = l;
    w.hi = max(h, l);
    return w;
}

// One staged union row of a warp.
template <class Act>
struct RowStage {
    float4 x[kRowSlots];                 // (x, y, z, h)
    int e[kRowSlots];                    // list entry: index | (tag - 1) << 28
    typename Act::Nb nb[kRowSlots];      // what the pair term reads of a neighbour
};

// Stages union row [u.lo, u.hi) (at most kRowSlots candidates; the rest are padding far away) and
// returns, for this lane, the union slots whose tag its row of the active-pair matrix allows.  A tag
// outside 1..n_tags sets EPP_STATUS_BAD_TAG in `st`.  Warp-collective.
template <class Act, bool FETCH>
__device__ __forceinline__ unsigned long long stage_row(const PairArgs& A, const Act& act, RowStage<Act>& S,
                                                        RowWin u, unsigned amask, int lane, unsigned& st,
                                                        bool& one_h, float& h0) {
    unsigned long long allowed = 0ull;
    one_h = true;
    h0 = 0.0f;
    __syncwarp();
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int k = half * 32 + lane;
        const int j = u.lo + k;
        const bool real = j < u.hi;
        const float4 xj = real ? A.s.xh[j] : make_float4(1e30f, 1e30f, 1e30f, 0.0f);
        const int tj = real ? tag_of(A.s.tagm[j]) : 0;
        S.x[k] = xj;
        S.e[k] = list_entry(j, tj >= 1 ? tj : 1);
        if (FETCH && real) S.nb[k] = act.fetch(j, 0, tj);
        if (__ballot_sync(0xffffffffu, real && (tj < 1 || tj > A.n_tags))) st |= EPP_STATUS_BAD_TAG;
        for (int t = 1; t <= A.n_tags; ++t) {
            const unsigned b = __ballot_sync(0xffffffffu, real && tj == t);
            if ((amask >> (t - 1)) & 1u) allowed |= (unsigned long long)b << (half * 32);
        }
        const float hf = __shfl_sync(0xffffffffu, xj.w, 0);
        if (half == 0) h0 = hf;
        one_h = __all_sync(0xffffffffu, !real || xj.w == h0) && one_h;
    }
    __syncwarp();
    return allowed;
}

// The acceptance word of one lane's window of `len` (<= 32) staged candidates starting at union
// slot `off`: bit k set when candidate k is within the criterion's radius, by the reference's IEEE
// arithmetic.  `r2u` is the exact bound when every candidate has the same h (h0); otherwise the
// bound is looked up per candidate.
__device__ __forceinline__ unsigned window_bits(const float4* sx, int off, int len, float4 xi, bool uniform,
                                                float r2u, float h2sq, bool dflt, float gap_square) {
    unsigned word = 0u;
    if (uniform) {
        // dr2 <= R2 as integers: non-negative floats order like their bit patterns, so
        // bits(dr2) - bits(R2) - 1 is negative exactly for the accepted candidates
        const int nR2 = -__float_as_int(r2u) - 1;
        for (int k = len - 1; k >= 0; --k) {
            const float4 xj = sx[off + k];
            const float dx = __fsub_rn(xi.x, xj.x);
            const float dy = __fsub_rn(xi.y, xj.y);
            const float d = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
            word = (word << 1) | ((unsigned)(__float_as_int(d) + nR2) >> 31);
        }
        return word;
    }
    float hc = xi.w, rc = dflt ? gap_square : h2sq;
    for (int k = len - 1; k >= 0; --k) {
        const float4 xj = sx[off + k];
        const float dx = __fsub_rn(xi.x, xj.x);
        const float dy = __fsub_rn(xi.y, xj.y);
        const float d = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
        if (xj.w != hc) {
            hc = xj.w;
            rc = dflt ? gap_square : (hc == xi.w ? h2sq : pair_r2(xi.w, hc));
        }
        word = (word << 1) | (d <= rc ? 1u : 0u);
    }
    return word;
}

// The search pass over stencil-row masks (2D): for each particle its three row words, nCount,
// and the search action of `Act` over the accepted neighbours (CPCont: continuity + density
// preview; CPCount: the count only), summed in list order.
template <class Act>
__global__ void __launch_bounds__(128) k_mask_build(const __grid_constant__ PairArgs A, unsigned* mask, int cap,
                                                    const __grid_constant__ Act act, unsigned long long* pairs) {
    __shared__ RowStage<Act> stage[4];
    const int lane = threadIdx.x & 31;
    RowStage<Act>& S = stage[threadIdx.x >> 5];
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int w0 = i - lane;
    int cnt = 0;
    if (w0 < n_alive) {   // warp-uniform
        const bool on = i < n_alive;
        const int n0 = A.dom.n[0];
        const int c_first = A.s.cell[w0];
        const int c_last = A.s.cell[min(w0 + 31, n_alive - 1)];
        EPP_CHECK(c_first >= 0 && c_last >= c_first && c_last < A.dom.n_cells, 31, c_last);
        const int rid0 = c_first / n0;
        const bool tiled = rid0 == c_last / n0;
        const int c = A.s.cell[min(i, n_alive - 1)];
        const int rid = c / n0, cx = c - rid * n0;
        const float4 xi = on ? A.s.xh[i] : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        const int ti = on ? tag_of(A.s.tagm[i]) : 0;
        const bool valid = on && ti >= 1 && ti <= A.n_tags;
        unsigned st = (on && !valid) ? EPP_STATUS_BAD_TAG : 0u;
        const unsigned amask = valid ? A.adj[ti - 1] : 0u;
        const TargetConst tc = target_const<2>(on ? xi.w : 1.0f);
        const bool dflt = A.crit == EPP_CRITERION_DEFAULT;
        typename Act::Self me{};
        if (valid) me = act.self(i);
        RowWin win[3];
        bool over = false;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            win[r] = row_range(A, stencil_row(A, rid, r), cx - 1, cx + 1);
            over |= win[r].hi - win[r].lo > 32;
        }
        const bool walk = valid && !over;
        unsigned words[3] = {0u, 0u, 0u};
        float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            RowWin u{0, 0};
            if (tiled) u = row_range(A, stencil_row(A, rid0, r), c_first - rid0 * n0 - 1, c_last - rid0 * n0 + 1);
            const bool staged = tiled && u.hi - u.lo <= kRowSlots;   // warp-uniform
            bool one_h = false;
            float h0 = 0.0f;
            unsigned long long allowed = 0ull;
            if (staged) allowed = stage_row<Act, Act::NC != 0>(A, act, S, u, amask, lane, st, one_h, h0);
            if (walk) {
                const int len = win[r].hi - win[r].lo;
                unsigned word;
                int off = 0;
                if (staged) {
                    off = win[r].lo - u.lo;
                    const bool uniform = one_h && (dflt || h0 == xi.w);
                    word = window_bits(S.x, off, len, xi, uniform, dflt ? A.dom.gap_square : tc.h2sq, tc.h2sq,
                                       dflt, A.dom.gap_square);
                    word &= (unsigned)(allowed >> off);
                } else {
                    word = 0u;
                    for (int k = len - 1; k >= 0; --k) {
                        const int j = win[r].lo + k;
                        word = (word << 1) | (accept<2>(A, i, xi, amask, tc.h2sq, j, A.s.xh[j], st) ? 1u : 0u);
                    }
                }
                if (len < 32) word &= (1u << len) - 1u;
                if (r == 1) word &= ~(1u << (i - win[1].lo));   // not its own neighbour
                words[r] = word;
                // the search action over this row's neighbours, in candidate order
                unsigned wk = word;
                while (wk) {
                    const int k = __ffs(wk) - 1;
                    wk &= wk - 1u;
                    ++cnt;
                    if (Act::NC == 0) continue;
                    float4 xj;
                    int tj;
                    typename Act::Nb nb;
                    if (staged) {
                        xj = S.x[off + k];
                        tj = entry_tag(S.e[off + k]);
                        nb = S.nb[off + k];
                    } else {
                        const int j = win[r].lo + k;
                        xj = A.s.xh[j];
                        tj = tag_of(A.s.tagm[j]);
                        nb = act.fetch(j, ti, tj);
                    }
                    const float4 t = act.term(me, nb, ti, tj, xj, geometry<2>(xi, xj), tc);
                    sum.x += t.x;
                    sum.y += t.y;
                    sum.z += t.z;
                }
            }
        }
        if (on) {
            if (!valid) {
                act.end_idle(i, ti);
            } else if (over) {   // dense neighbourhood: its neighbours come from its stencil
                words[0] = words[2] = 0u;
                words[1] = kMaskOverflow;
                sum = neighbours_by_stencil<2>(A, i, xi, ti, tc, act);
                cnt = (int)sum.w;
                sum.w = 0.0f;
                act.end(i, ti, sum, cnt);
            } else {
                act.end(i, ti, sum, cnt);
            }
            mask[i] = words[0];
            mask[(size_t)cap + i] = words[1];
            mask[(size_t)2 * cap + i] = words[2];
        }
        if (st) atomicOr(A.status, st);
    }
    count_pairs(pairs, cnt);
}

// A pair action over the masks of the last search (same order, positions and criterion), one
// thread per particle.  STAGE: the warp stages each union row (positions, tags and the action's
// neighbour records) in shared memory; otherwise neighbours are read from global memory (actions
// whose neighbour reads may overlap the pass's own writes).  EPI: fused momentum step (integrate
// + bin for every particle, dead bin included; block 0 clears the scan state).
template <class Act, bool EPI, bool STAGE>
__global__ void __launch_bounds__(128) k_mask_walk(const __grid_constant__ PairArgs A, const unsigned* mask, int cap,
                                                   const __grid_constant__ Act act, unsigned long long* scan_state,
                                                   int n_scan_words) {
    __shared__ RowStage<Act> stage[STAGE ? 4 : 1];
    if (EPI && blockIdx.x == 0)
        for (int t = threadIdx.x; t < n_scan_words; t += blockDim.x) scan_state[t] = 0ull;
    const int lane = threadIdx.x & 31;
    RowStage<Act>& S = stage[STAGE ? (threadIdx.x >> 5) : 0];
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int w0 = i - lane;
    if (w0 < n_alive) {   // warp-uniform
        const bool on = i < n_alive;
        const int n0 = A.dom.n[0];
        const int c_first = A.s.cell[w0];
        const int c_last = A.s.cell[min(w0 + 31, n_alive - 1)];
        EPP_CHECK(c_first >= 0 && c_last >= c_first && c_last < A.dom.n_cells, 32, c_last);
        const int rid0 = c_first / n0;
        const bool tiled = rid0 == c_last / n0;
        const int c = A.s.cell[min(i, n_alive - 1)];
        const int rid = c / n0, cx = c - rid * n0;
        const float4 xi = on ? A.s.xh[i] : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        const int ti = on ? tag_of(A.s.tagm[i]) : 0;
        const bool valid = on && ti >= 1 && ti <= A.n_tags && act.wants(ti);
        unsigned words[3] = {0u, 0u, 0u};
        if (on) {
            words[0] = mask[i];
            words[1] = mask[(size_t)cap + i];
            words[2] = mask[(size_t)2 * cap + i];
        }
        const bool over = words[1] == kMaskOverflow;
        const bool walk = valid && !over;
        const TargetConst tc = target_const<2>(on ? xi.w : 1.0f);
        typename Act::Self me{};
        if (walk) me = act.self(i);
        float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        int cnt = 0;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const RowWin win = row_range(A, stencil_row(A, rid, r), cx - 1, cx + 1);
            RowWin u{0, 0};
            bool staged = false;
            if (STAGE && tiled) {
                u = row_range(A, stencil_row(A, rid0, r), c_first - rid0 * n0 - 1, c_last - rid0 * n0 + 1);
                staged = u.hi - u.lo <= kRowSlots;
            }
            if (staged) {
                unsigned st = 0u;
                bool one_h;
                float h0;
                stage_row<Act, true>(A, act, S, u, 0u, lane, st, one_h, h0);
            }
            if (!walk) continue;
            const int off = win.lo - u.lo;
            unsigned wk = words[r];
            while (wk) {
                const int k = __ffs(wk) - 1;
                wk &= wk - 1u;
                ++cnt;
                float4 xj;
                int tj;
                typename Act::Nb nb;
                if (staged) {
                    xj = S.x[off + k];
                    tj = entry_tag(S.e[off + k]);
                    nb = S.nb[off + k];
                } else {
                    const int j = win.lo + k;
                    EPP_CHECK(j < A.n_max, 33, j);
                    xj = __ldg(&A.s.xh[j]);
                    tj = tag_of(A.s.tagm[j]);
                    nb = act.fetch(j, ti, tj);
                }
                const float4 t = act.term(me, nb, ti, tj, xj, geometry<2>(xi, xj), tc);
                sum.x += t.x;
                sum.y += t.y;
                sum.z += t.z;
            }
        }
        if (on) {
            if (!valid) {
                act.end_idle(i, ti);
            } else {
                if (over) {
                    sum = neighbours_by_stencil<2>(A, i, xi, ti, tc, act);
                    cnt = (int)sum.w;
                    sum.w = 0.0f;
                }
                act.end(i, ti, sum, cnt);
            }
        } else if (EPI && i < A.n_max) {
            act.end_idle(i, tag_of(A.s.tagm[i]));
        }
    } else if (EPI && i < A.n_max) {
        act.end_idle(i, tag_of(A.s.tagm[i]));
    }
}

}  // namespace epp
