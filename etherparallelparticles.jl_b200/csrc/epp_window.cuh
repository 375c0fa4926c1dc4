// epp_window.cuh -- the 2D search pass over per-particle stencil-row windows, with the search
// action folded in.
//
// A particle's 3x3 cell stencil is three stencil rows (dy = -1, 0, +1); in each row its
// candidates are one contiguous cell-order range, cells cx-1 .. cx+1 (its "window", about 27
// particles at h = 1.5 dx).  The list search pass (k_build) tests, in lockstep, every candidate of
// the warp's union of stencils against every lane -- about 190 per particle; here each lane tests
// only its own window, 81 candidates.
//
// A warp takes 32 consecutive particles in cell order.  When their cells lie in one cell row, the
// union of their windows in a stencil row is one contiguous range; the warp stages the three union
// rows (up to 64 candidates each) in shared memory in one round -- position and h, the list entry
// (index and tag) in the unused z lane, and the search action's neighbour record -- and every lane
// reads its own window from there.  The lane builds one acceptance word per stencil row with the
// reference's IEEE criterion (and the active-pair matrix, applied from per-row tag bitmaps), then
// walks the set bits of the three words in list order, in one loop: it appends the neighbour to
// its list (the lists the momentum, filter and extrapolation passes read; same layout and order as
// k_build's: stencil rows, then cell order, then id order inside a cell) and adds the search
// action's term -- the continuity rate -- from the staged record, so no separate continuity pass
// walks the neighbours again.  Windows beyond 32 candidates (dense neighbourhoods) go row by row
// in 32-candidate chunks.  A warp that crosses a cell-row end takes one such round per cell
// row of its particles; union rows longer than 64 are read from global memory instead.
#pragma once
#include "epp_tile.cuh"

namespace epp {

struct RowWin {
    int lo, hi;   // candidate range [lo, hi) in cell order
};

// Linear cell row of stencil row r (0, 1, 2 for dy = -1, 0, +1) of the cell row `rid` = y + n1 k
// (k is the instance of a batch; the caller passes y = rid mod n1), or -1 when y + dy is outside
// the grid.
__device__ __forceinline__ int stencil_row2(const PairArgs& A, int rid, int y, int r) {
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

template <class Act>
struct Stage2 {
    float4 x[3 * 64];                 // (x, y, list entry as bits, h)
    typename Act::Nb nb[3 * 64];
};

// Stages union rows u[0..2] (each at most 64 candidates) and records, per row, the union slots
// whose tag this lane's row of the active-pair matrix allows and whether every candidate of the
// row has one h (one_h, h0).  A tag outside 1..n_tags sets EPP_STATUS_BAD_TAG.  Warp-collective.
template <class Act, bool FETCH>
__device__ __forceinline__ void stage_rows2(const PairArgs& A, const Act& act, Stage2<Act>& S, const RowWin (&u)[3],
                                            unsigned amask, int lane, unsigned& st, unsigned long long (&allowed)[3],
                                            bool (&one_h)[3], float (&h0)[3]) {
    __syncwarp();
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        allowed[r] = 0ull;
        one_h[r] = true;
        h0[r] = 0.0f;
#pragma unroll
        for (int part = 0; part < 2; ++part) {
            if (u[r].lo + part * 32 >= u[r].hi) break;   // warp-uniform: nothing left in this row
            const int k = part * 32 + lane;
            const int j = u[r].lo + k;
            const bool real = j < u[r].hi;
            const float4 xj = real ? A.s.xh[j] : make_float4(1e30f, 1e30f, 0.0f, 0.0f);
            const int tj = real ? tag_of(A.s.tagm[j]) : 0;
            S.x[64 * r + k] = make_float4(xj.x, xj.y, __int_as_float(list_entry(j, tj >= 1 ? tj : 1)), xj.w);
            if (FETCH && real) S.nb[64 * r + k] = act.fetch(j, 0, tj);
            if (__ballot_sync(0xffffffffu, real && (tj < 1 || tj > A.n_tags))) st |= EPP_STATUS_BAD_TAG;
            for (int t = 1; t <= A.n_tags; ++t) {
                const unsigned b = __ballot_sync(0xffffffffu, real && tj == t);
                if ((amask >> (t - 1)) & 1u) allowed[r] |= (unsigned long long)b << (part * 32);
            }
            const float hf = __shfl_sync(0xffffffffu, xj.w, 0);
            if (part == 0) h0[r] = hf;
            one_h[r] = __all_sync(0xffffffffu, !real || xj.w == h0[r]) && one_h[r];
        }
    }
    __syncwarp();
}

// Acceptance bits of staged candidates [k0, k1) (k1 - k0 <= 32) of a lane's window starting at
// slot `off`: bit k - k0 set when candidate k is within the criterion's radius, by the reference's
// IEEE arithmetic.  `uniform`: every candidate has the lane's h (or the default criterion), so one
// exact bound `r2u` serves; otherwise the bound is looked up per candidate.
__device__ __forceinline__ unsigned window_bits(const float4* sx, int off, int k0, int k1, float4 xi, bool uniform,
                                                float r2u, float h2sq, bool dflt, float gap_square) {
    // (dx, dy) and (dx^2, dy^2) on the packed f32x2 pipe (each half rounds like __fsub_rn /
    // __fmul_rn), the sum scalar
    const f32x2 XY = f2_pack(xi.x, xi.y);
    unsigned word = 0u;
    if (uniform) {
        // dr2 <= R2 as integers: non-negative floats order like their bit patterns, so
        // bits(dr2) - bits(R2) - 1 is negative exactly for the accepted candidates
        const int nR2 = -__float_as_int(r2u) - 1;
        for (int k = k1 - 1; k >= k0; --k) {
            const f32x2 d = f2_sub(XY, *reinterpret_cast<const f32x2*>(&sx[off + k]));
            float dx2, dy2;
            f2_unpack(f2_mul(d, d), dx2, dy2);
            word = (word << 1) | ((unsigned)(__float_as_int(__fadd_rn(dx2, dy2)) + nR2) >> 31);
        }
        return word;
    }
    float hc = xi.w, rc = dflt ? gap_square : h2sq;
    for (int k = k1 - 1; k >= k0; --k) {
        const float hj = sx[off + k].w;
        const f32x2 d = f2_sub(XY, *reinterpret_cast<const f32x2*>(&sx[off + k]));
        float dx2, dy2;
        f2_unpack(f2_mul(d, d), dx2, dy2);
        if (hj != hc) {
            hc = hj;
            rc = dflt ? gap_square : (hc == xi.w ? h2sq : pair_r2(xi.w, hc));
        }
        word = (word << 1) | (__fadd_rn(dx2, dy2) <= rc ? 1u : 0u);
    }
    return word;
}

// What the general per-lane search hands back to the search pass.
struct WinOut {
    int cnt;
    float sx, sy;
    unsigned st;
};

// The per-lane search of the 2D search pass in its general form: windows of any length, row by
// row 32 candidates at a time, from the staged union rows u[] or, when `staged` is false, from
// global memory.  Only dense neighbourhoods (a window beyond 32 candidates) and union rows beyond
// the staging area come here.  Inlined: as an out-of-line call it cost the kernel registers (the
// values live across the call) and 13% of its time.
// uniform_rows: bit r set when every candidate of staged row r has the lane's h (or the default
// criterion), so one exact bound serves the row.
template <class Act>
__device__ __forceinline__ WinOut win_lane_general(const PairArgs& A, const TileMask& M, const Act& act,
                                                const Stage2<Act>& S, bool staged, RowWin u0, RowWin u1, RowWin u2,
                                                unsigned long long al0, unsigned long long al1, unsigned long long al2,
                                                unsigned uniform_rows, int i, int ti, float4 xi, unsigned amask,
                                                int rid, int cx) {
    const TargetConst tc = target_const<2>(xi.w);
    const bool dflt = A.crit == EPP_CRITERION_DEFAULT;
    typename Act::Self me = act.self(i);
    ListWriter<2> L = list_writer<2>(M, i);
    WinOut o{0, 0.0f, 0.0f, 0u};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const RowWin win = row_range(A, stencil_row2(A, rid, rid % A.dom.n[1], r), cx - 1, cx + 1);
        const RowWin u = r == 0 ? u0 : (r == 1 ? u1 : u2);
        const unsigned long long allowed = r == 0 ? al0 : (r == 1 ? al1 : al2);
        const int len = win.hi - win.lo;
        const int woff = win.lo - u.lo;
        const bool uniform = staged && ((uniform_rows >> r) & 1u);
        for (int k0 = 0; k0 < len; k0 += 32) {
            const int k1 = min(len, k0 + 32);
            unsigned word;
            if (staged) {
                word = window_bits(S.x, 64 * r + woff, k0, k1, xi, uniform, dflt ? A.dom.gap_square : tc.h2sq,
                                   tc.h2sq, dflt, A.dom.gap_square);
                word &= (unsigned)(allowed >> (woff + k0));
            } else {
                word = 0u;
                for (int k = k1 - 1; k >= k0; --k) {
                    const int j = win.lo + k;
                    word = (word << 1) | (accept<2>(A, i, xi, amask, tc.h2sq, j, A.s.xh[j], o.st) ? 1u : 0u);
                }
            }
            if (k1 - k0 < 32) word &= (1u << (k1 - k0)) - 1u;
            if (r == 1) {   // not its own neighbour
                const int ks = i - win.lo - k0;
                if (ks >= 0 && ks < 32) word &= ~(1u << ks);
            }
            while (word) {   // append and run the search action, in list order
                const int k = k0 + __ffs(word) - 1;
                word &= word - 1u;
                float4 xj;
                int e, tj;
                typename Act::Nb nb;
                if (staged) {
                    const float4 xs = S.x[64 * r + woff + k];
                    e = __float_as_int(xs.z);
                    xj = make_float4(xs.x, xs.y, 0.0f, xs.w);
                    tj = entry_tag(e);
                    if (Act::NC != 0) nb = S.nb[64 * r + woff + k];
                } else {
                    const int j = win.lo + k;
                    xj = A.s.xh[j];
                    tj = tag_of(A.s.tagm[j]);
                    e = list_entry(j, tj);
                    if (Act::NC != 0) nb = act.fetch(j, ti, tj);
                }
                L.put(o.cnt++, e);
                if (Act::NC != 0) {
                    const float4 t = act.term(me, nb, ti, tj, xj, geometry<2>(xi, xj), tc);
                    o.sx = __fadd_rn(o.sx, t.x);
                    o.sy = __fadd_rn(o.sy, t.y);
                }
            }
        }
    }
    L.flush(o.cnt);
    return o;
}

// The 2D search pass: neighbour lists and nCount, and the search action of `Act` over the accepted
// neighbours in list order (CPCont: continuity + density preview; CPCount: the count only).  A
// particle with more neighbours than a list keeps has only those stored (the pair passes read its
// stencil); its search action still covers all of them.
template <class Act>
__global__ void __launch_bounds__(128, 7) k_win_build(const __grid_constant__ PairArgs A, const __grid_constant__ TileMask M,
                                                   const __grid_constant__ Act act, unsigned long long* pairs) {
    __shared__ Stage2<Act> stage[4];
    const int lane = threadIdx.x & 31;
    Stage2<Act>& S = stage[threadIdx.x >> 5];
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int w0 = i - lane;
    int cnt = 0;
    if (w0 < n_alive) {   // warp-uniform
        const bool on = i < n_alive;
        const int n0 = A.dom.n[0];
        const int c = A.s.cell[min(i, n_alive - 1)];
        EPP_CHECK(!__any_sync(0xffffffffu, c < 0 || c >= A.dom.n_cells), 34, c);
        const int rid = c / n0, cx = c - rid * n0;
        const int y = rid % A.dom.n[1];
        const float4 xi = on ? A.s.xh[i] : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        const int ti = on ? tag_of(A.s.tagm[i]) : 0;
        const bool valid = on && ti >= 1 && ti <= A.n_tags;
        unsigned st = (on && !valid) ? EPP_STATUS_BAD_TAG : 0u;
        const unsigned amask = valid ? A.adj[ti - 1] : 0u;
        float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        // One round per cell row among the warp's particles (cell order keeps each row's lanes
        // contiguous): a warp inside one cell row -- all but about 2% -- takes one round; a warp
        // that crosses a row end stages the union rows of each part in turn instead of reading
        // candidates from global memory one dependent load at a time.
        unsigned pending = __ballot_sync(0xffffffffu, on);
        while (pending) {   // warp-uniform
            const int lead = __ffs(pending) - 1;
            const int rid_g = __shfl_sync(0xffffffffu, rid, lead);
            const int y_g = __shfl_sync(0xffffffffu, y, lead);
            const bool mine = ((pending >> lane) & 1u) && rid == rid_g;
            const unsigned members = __ballot_sync(0xffffffffu, mine);
            const int xa = __shfl_sync(0xffffffffu, cx, lead) - 1;
            const int xb = __shfl_sync(0xffffffffu, cx, 31 - __clz(members)) + 1;
            pending &= ~members;
            RowWin u[3];
            bool staged = true;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                u[r] = row_range(A, stencil_row2(A, rid_g, y_g, r), xa, xb);
                staged = staged && u[r].hi - u[r].lo <= 64;   // warp-uniform
            }
            unsigned long long allowed[3] = {0ull, 0ull, 0ull};
            bool one_h[3] = {false, false, false};
            float h0[3] = {0.0f, 0.0f, 0.0f};
            if (staged) stage_rows2<Act, Act::NC != 0>(A, act, S, u, amask, lane, st, allowed, one_h, h0);
            if (!(mine && valid)) continue;
            const bool dflt = A.crit == EPP_CRITERION_DEFAULT;
            RowWin win[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) win[r] = row_range(A, stencil_row2(A, rid, y, r), cx - 1, cx + 1);
            unsigned uniform_rows = 0u;
#pragma unroll
            for (int r = 0; r < 3; ++r)
                if (one_h[r] && (dflt || h0[r] == xi.w)) uniform_rows |= 1u << r;
            if (!staged || win[0].hi - win[0].lo > 32 || win[1].hi - win[1].lo > 32 || win[2].hi - win[2].lo > 32) {
                const WinOut o = win_lane_general<Act>(A, M, act, S, staged, u[0], u[1], u[2], allowed[0], allowed[1],
                                                       allowed[2], uniform_rows, i, ti, xi, amask, rid, cx);
                cnt = o.cnt;
                sum.x = o.sx;
                sum.y = o.sy;
                st |= o.st;
                continue;
            }
            // every window in one word: the three words first, then one walk over all of them, so
            // a warp iterates as often as its busiest lane's neighbour count (not the sum over rows
            // of each row's busiest lane)
            const TargetConst tc = target_const<2>(xi.w);
            unsigned w[3];
            int off[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int len = win[r].hi - win[r].lo;
                const int woff = win[r].lo - u[r].lo;   // the window's first slot in its staged row
                off[r] = 64 * r + woff;
                unsigned word = 0u;
                if (len > 0) {
                    word = window_bits(S.x, off[r], 0, len, xi, (uniform_rows >> r) & 1u,
                                       dflt ? A.dom.gap_square : tc.h2sq, tc.h2sq, dflt, A.dom.gap_square);
                    word &= (unsigned)(allowed[r] >> woff);
                    if (len < 32) word &= (1u << len) - 1u;
                }
                if (r == 1) word &= ~(1u << (i - win[1].lo));   // not its own neighbour
                w[r] = word;
            }
            typename Act::Self me = act.self(i);
            ListWriter<2> L = list_writer<2>(M, i);
            unsigned a = w[0], b = w[1], c2 = w[2];
            while (a | b | c2) {   // append and run the search action, in list order
                const int r = a ? 0 : (b ? 1 : 2);
                const unsigned cur = a ? a : (b ? b : c2);
                const int slot = (r == 0 ? off[0] : (r == 1 ? off[1] : off[2])) + __ffs(cur) - 1;
                const unsigned rest = cur & (cur - 1u);
                if (r == 0) a = rest;
                else if (r == 1) b = rest;
                else c2 = rest;
                const float4 xs = S.x[slot];
                const int e = __float_as_int(xs.z);
                L.put(cnt++, e);
                if (Act::NC != 0) {
                    const int tj = entry_tag(e);
                    const float4 xj = make_float4(xs.x, xs.y, 0.0f, xs.w);
                    const float4 t = act.term(me, S.nb[slot], ti, tj, xj, geometry<2>(xi, xj), tc);
                    sum.x = __fadd_rn(sum.x, t.x);
                    sum.y = __fadd_rn(sum.y, t.y);
                }
            }
            L.flush(cnt);
        }
        if (on) {
            if (!valid) act.end_idle(i, ti);
            else act.end(i, ti, sum, cnt);
        }
        if (st) atomicOr(A.status, st);
    }
    count_pairs(pairs, cnt);
}

}  // namespace epp
