// epp_mask.cuh -- pair passes over stencil-row masks.
//
// A particle's 3^D cell stencil is 3^(D-1) stencil rows (dy, and dz in 3D, from -1 to +1); in each
// row its candidates are the contiguous cell-order range of cells cx-1 .. cx+1 (a "window": about
// 27 particles in 2D at h = 1.5 dx, about 53 in 3D at h = 1.3 dx).  The search pass records, per
// particle and stencil row, W 32-bit words (W = 1 in 2D, 2 in 3D) whose bit k says whether
// candidate k of that window passed the reference's criterion and the active-pair matrix: 12 bytes
// per particle in 2D and 72 in 3D, in place of neighbour lists of about 25 and 62 entries.  Every
// pair pass walks the set bits in ascending order -- stencil rows (dz, then dy), then cell order,
// then id order inside a cell, the order of the neighbour lists -- so the sums add the same terms
// in the same order (equal to FP32 rounding: the compiler may fuse a multiply and an add
// differently in these kernels and in the list passes).
//
// A warp takes 32 consecutive particles in cell order.  When their cells lie in one cell row, the
// union of their windows in stencil row r is one contiguous range (cells xa-1 .. xb+1); the warp
// stages it in shared memory (one union row at a time, up to 64 candidates in 2D and 128 in 3D,
// with coalesced loads) and every lane reads its own window from there.  The search pass tests
// only its own window (in 2D 27 candidates, not the ~190 of the warp's union) and folds the search
// action (continuity and the density preview) into the same walk over the accepted bits, so no
// separate continuity pass reads the neighbours again.  Warps that cross a cell-row end, and union
// rows longer than the staging area, read the candidates from global memory instead; a particle
// whose window holds more than 32 W candidates (dense neighbourhoods) is marked and takes its
// neighbours from its stencil in every pass.
#pragma once
#include "epp_tile.cuh"

namespace epp {

template <int D>
struct MaskConf {
    static constexpr int ROWS = D == 2 ? 3 : 9;      // stencil rows
    static constexpr int W = D == 2 ? 1 : 2;         // 32-bit words per row window
    static constexpr int SLOTS = D == 2 ? 64 : 128;  // union candidates of a row staged at once
    static constexpr int WORDS = ROWS * W;           // words per particle
    static constexpr int OWN = ROWS / 2;             // the particle's own stencil row
};
constexpr unsigned kMaskOverflow = 0xffffffffu;  // every word of the own row: the particle's
                                                 // neighbours come from its stencil (its own bit is
                                                 // never set otherwise)

struct RowWin {
    int lo, hi;   // candidate range [lo, hi) in cell order
};

// Linear cell row of stencil row r of the cell row `rid` (y + n1 z; z is the instance of a 2D
// batch), or -1 when it lies outside the grid.  Rows go dz-major then dy, as the list passes'.
template <int D>
__device__ __forceinline__ int stencil_row(const PairArgs& A, int rid, int r) {
    const int n1 = A.dom.n[1];
    const int y = rid % n1, z = rid / n1;
    const int yy = y + (D == 2 ? r : r % 3) - 1;
    const int zz = D == 2 ? z : z + r / 3 - 1;
    if (yy < 0 || yy >= n1) return -1;
    if (D == 3 && (zz < 0 || zz >= A.dom.n[2])) return -1;
    return yy + n1 * zz;
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
template <int D, class Act>
struct RowStage {
    float4 x[MaskConf<D>::SLOTS];                 // (x, y, z, h)
    int e[MaskConf<D>::SLOTS];                    // list entry: index | (tag - 1) << 28
    typename Act::Nb nb[MaskConf<D>::SLOTS];      // what the pair term reads of a neighbour
};

// Bits [off, off + 32) of a bitmap of 64 NW bits held in 64-bit words.
template <int NW>
__device__ __forceinline__ unsigned bits_at(const unsigned long long (&m)[NW], int off) {
    const int q = off >> 6, s = off & 63;
    unsigned long long lo = 0ull, hi = 0ull;
#pragma unroll
    for (int t = 0; t < NW; ++t) {   // selects, not a dynamic index: m stays in registers
        if (t == q) lo = m[t];
        if (t == q + 1) hi = m[t];
    }
    unsigned long long v = lo >> s;
    if (s) v |= hi << (64 - s);
    return (unsigned)v;
}

// Stages union row [u.lo, u.hi) (at most SLOTS candidates) and records, for this lane, the union
// slots whose tag its row of the active-pair matrix allows.  A tag outside 1..n_tags sets
// EPP_STATUS_BAD_TAG in `st`.  Warp-collective.
template <int D, class Act, bool FETCH>
__device__ __forceinline__ void stage_row(const PairArgs& A, const Act& act, RowStage<D, Act>& S, RowWin u,
                                          unsigned amask, int lane, unsigned& st, bool& one_h, float& h0,
                                          unsigned long long (&allowed)[MaskConf<D>::SLOTS / 64]) {
    constexpr int NW = MaskConf<D>::SLOTS / 64;
#pragma unroll
    for (int q = 0; q < NW; ++q) allowed[q] = 0ull;
    one_h = true;
    h0 = 0.0f;
    __syncwarp();
#pragma unroll
    for (int part = 0; part < MaskConf<D>::SLOTS / 32; ++part) {
        const int k = part * 32 + lane;
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
            if ((amask >> (t - 1)) & 1u) allowed[part >> 1] |= (unsigned long long)b << ((part & 1) * 32);
        }
        const float hf = __shfl_sync(0xffffffffu, xj.w, 0);
        if (part == 0) h0 = hf;
        one_h = __all_sync(0xffffffffu, !real || xj.w == h0) && one_h;
        if (u.lo + (part + 1) * 32 >= u.hi) break;   // warp-uniform: the slots beyond are never read
    }
    __syncwarp();
}

// The acceptance bits of candidates [k0, k1) (k1 - k0 <= 32) of one lane's window starting at
// union slot `off`: bit k - k0 set when candidate k is within the criterion's radius, by the
// reference's IEEE arithmetic.  `uniform`: every candidate has the lane's h (or the default
// criterion), so one exact bound `r2u` serves; otherwise the bound is looked up per candidate.
template <int D>
__device__ __forceinline__ unsigned window_bits(const float4* sx, int off, int k0, int k1, float4 xi, bool uniform,
                                                float r2u, float h2sq, bool dflt, float gap_square) {
    unsigned word = 0u;
    if (uniform) {
        // dr2 <= R2 as integers: non-negative floats order like their bit patterns, so
        // bits(dr2) - bits(R2) - 1 is negative exactly for the accepted candidates
        const int nR2 = -__float_as_int(r2u) - 1;
        for (int k = k1 - 1; k >= k0; --k) {
            const float4 xj = sx[off + k];
            const float dx = __fsub_rn(xi.x, xj.x);
            const float dy = __fsub_rn(xi.y, xj.y);
            float d = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
            if (D == 3) {
                const float dz = __fsub_rn(xi.z, xj.z);
                d = __fadd_rn(d, __fmul_rn(dz, dz));
            }
            word = (word << 1) | ((unsigned)(__float_as_int(d) + nR2) >> 31);
        }
        return word;
    }
    float hc = xi.w, rc = dflt ? gap_square : h2sq;
    for (int k = k1 - 1; k >= k0; --k) {
        const float4 xj = sx[off + k];
        const float dx = __fsub_rn(xi.x, xj.x);
        const float dy = __fsub_rn(xi.y, xj.y);
        float d = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
        if (D == 3) {
            const float dz = __fsub_rn(xi.z, xj.z);
            d = __fadd_rn(d, __fmul_rn(dz, dz));
        }
        if (xj.w != hc) {
            hc = xj.w;
            rc = dflt ? gap_square : (hc == xi.w ? h2sq : pair_r2(xi.w, hc));
        }
        word = (word << 1) | (d <= rc ? 1u : 0u);
    }
    return word;
}

// The search pass over stencil-row masks: for each particle its row words, nCount, and the search
// action of `Act` over the accepted neighbours (CPCont: continuity + density preview; CPCount: the
// count only), summed in list order.
template <int D, class Act>
__global__ void __launch_bounds__(128) k_mask_build(const __grid_constant__ PairArgs A, unsigned* mask, int cap,
                                                    const __grid_constant__ Act act, unsigned long long* pairs) {
    using MC = MaskConf<D>;
    __shared__ RowStage<D, Act> stage[4];
    const int lane = threadIdx.x & 31;
    RowStage<D, Act>& S = stage[threadIdx.x >> 5];
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
        const TargetConst tc = target_const<D>(on ? xi.w : 1.0f);
        const bool dflt = A.crit == EPP_CRITERION_DEFAULT;
        typename Act::Self me{};
        if (valid) me = act.self(i);
        bool over = false;
        for (int r = 0; r < MC::ROWS; ++r) {
            const RowWin w = row_range(A, stencil_row<D>(A, rid, r), cx - 1, cx + 1);
            over |= w.hi - w.lo > 32 * MC::W;
        }
        const bool walk = valid && !over;
        float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (int r = 0; r < MC::ROWS; ++r) {
            const RowWin win = row_range(A, stencil_row<D>(A, rid, r), cx - 1, cx + 1);
            RowWin u{0, 0};
            if (tiled) u = row_range(A, stencil_row<D>(A, rid0, r), c_first - rid0 * n0 - 1, c_last - rid0 * n0 + 1);
            const bool staged = tiled && u.hi - u.lo <= MC::SLOTS;   // warp-uniform
            bool one_h = false;
            float h0 = 0.0f;
            unsigned long long allowed[MC::SLOTS / 64];
            if (staged) stage_row<D, Act, Act::NC != 0>(A, act, S, u, amask, lane, st, one_h, h0, allowed);
            unsigned words[MC::W];
#pragma unroll
            for (int q = 0; q < MC::W; ++q) words[q] = 0u;
            if (walk) {
                const int len = win.hi - win.lo;
                const int off = win.lo - u.lo;
#pragma unroll
                for (int q = 0; q < MC::W; ++q) {
                    const int k0 = 32 * q, k1 = min(len, 32 * (q + 1));
                    if (k0 >= k1) continue;
                    unsigned word;
                    if (staged) {
                        const bool uniform = one_h && (dflt || h0 == xi.w);
                        word = window_bits<D>(S.x, off, k0, k1, xi, uniform, dflt ? A.dom.gap_square : tc.h2sq,
                                              tc.h2sq, dflt, A.dom.gap_square);
                        word &= bits_at<MC::SLOTS / 64>(allowed, off + k0);
                    } else {
                        word = 0u;
                        for (int k = k1 - 1; k >= k0; --k) {
                            const int j = win.lo + k;
                            word = (word << 1) | (accept<D>(A, i, xi, amask, tc.h2sq, j, A.s.xh[j], st) ? 1u : 0u);
                        }
                    }
                    if (k1 - k0 < 32) word &= (1u << (k1 - k0)) - 1u;
                    if (r == MC::OWN) {   // not its own neighbour
                        const int ks = i - win.lo - k0;
                        if (ks >= 0 && ks < 32) word &= ~(1u << ks);
                    }
                    words[q] = word;
                    // the search action over this word's neighbours, in candidate order
                    unsigned wk = word;
                    while (wk) {
                        const int k = k0 + __ffs(wk) - 1;
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
                            const int j = win.lo + k;
                            xj = A.s.xh[j];
                            tj = tag_of(A.s.tagm[j]);
                            nb = act.fetch(j, ti, tj);
                        }
                        const float4 t = act.term(me, nb, ti, tj, xj, geometry<D>(xi, xj), tc);
                        sum.x += t.x;
                        sum.y += t.y;
                        sum.z += t.z;
                    }
                }
            }
            if (on) {
#pragma unroll
                for (int q = 0; q < MC::W; ++q) {
                    const unsigned v = !valid ? 0u : over ? (r == MC::OWN ? kMaskOverflow : 0u) : words[q];
                    mask[(size_t)(r * MC::W + q) * cap + i] = v;
                }
            }
        }
        if (on) {
            if (!valid) {
                act.end_idle(i, ti);
            } else if (over) {   // dense neighbourhood: its neighbours come from its stencil
                sum = neighbours_by_stencil<D>(A, i, xi, ti, tc, act);
                cnt = (int)sum.w;
                sum.w = 0.0f;
                act.end(i, ti, sum, cnt);
            } else {
                act.end(i, ti, sum, cnt);
            }
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
template <int D, class Act, bool EPI, bool STAGE>
__global__ void __launch_bounds__(128) k_mask_walk(const __grid_constant__ PairArgs A, const unsigned* mask, int cap,
                                                   const __grid_constant__ Act act, unsigned long long* scan_state,
                                                   int n_scan_words) {
    using MC = MaskConf<D>;
    __shared__ RowStage<D, Act> stage[STAGE ? 4 : 1];
    if (EPI && blockIdx.x == 0)
        for (int t = threadIdx.x; t < n_scan_words; t += blockDim.x) scan_state[t] = 0ull;
    const int lane = threadIdx.x & 31;
    RowStage<D, Act>& S = stage[STAGE ? (threadIdx.x >> 5) : 0];
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
        bool over = on;
#pragma unroll
        for (int q = 0; q < MC::W; ++q)
            over = over && mask[(size_t)(MC::OWN * MC::W + q) * cap + min(i, n_alive - 1)] == kMaskOverflow;
        const bool walk = valid && !over;
        const TargetConst tc = target_const<D>(on ? xi.w : 1.0f);
        typename Act::Self me{};
        if (walk) me = act.self(i);
        float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        int cnt = 0;
        for (int r = 0; r < MC::ROWS; ++r) {
            RowWin u{0, 0};
            bool staged = false;
            if (STAGE && tiled) {
                u = row_range(A, stencil_row<D>(A, rid0, r), c_first - rid0 * n0 - 1, c_last - rid0 * n0 + 1);
                staged = u.hi - u.lo <= MC::SLOTS;
            }
            unsigned words[MC::W];
#pragma unroll
            for (int q = 0; q < MC::W; ++q) words[q] = walk ? mask[(size_t)(r * MC::W + q) * cap + i] : 0u;
            if (staged) {
                unsigned st = 0u;
                bool one_h;
                float h0;
                unsigned long long allowed[MC::SLOTS / 64];
                stage_row<D, Act, true>(A, act, S, u, 0u, lane, st, one_h, h0, allowed);
            }
            if (!walk) continue;
            const RowWin win = row_range(A, stencil_row<D>(A, rid, r), cx - 1, cx + 1);
            const int off = win.lo - u.lo;
#pragma unroll
            for (int q = 0; q < MC::W; ++q) {
                unsigned wk = words[q];
                while (wk) {
                    const int k = 32 * q + __ffs(wk) - 1;
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
                    const float4 t = act.term(me, nb, ti, tj, xj, geometry<D>(xi, xj), tc);
                    sum.x += t.x;
                    sum.y += t.y;
                    sum.z += t.z;
                }
            }
        }
        if (on) {
            if (!valid) {
                act.end_idle(i, ti);
            } else {
                if (over) {
                    sum = neighbours_by_stencil<D>(A, i, xi, ti, tc, act);
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

// ---------------------------------------------------------------------------------------------
// 2D: all three union rows staged at once and one walk over the three row words.  The per-row
// form above iterates, per stencil row, as often as the lane with the most neighbours in that
// row; summed over the rows that is ~10% more iterations than the busiest lane's total, and each
// row pays its own staging round.  Here the warp stages the three rows (up to 64 candidates each)
// in one round and walks the bits of row 0, then 1, then 2 as one sequence.  Records are slim:
// the list entry (index and tag) rides in the unused z lane of the position record.

template <class Act>
struct Stage2 {
    float4 x[3 * 64];                 // (x, y, list entry as bits, h)
    typename Act::Nb nb[3 * 64];
};

// Stages union rows u[0..2] (each at most 64 candidates).  TAGS: also the union slots whose tag this
// lane's row of the active-pair matrix allows (per row) and whether every candidate of a row has one
// h (one_h, h0).  Warp-collective.
template <class Act, bool FETCH, bool TAGS>
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
            if (TAGS) {
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
    }
    __syncwarp();
}

// The next set bit of the concatenated row words (a, b, c), lowest row first: its bit index k and
// row r; the bit is cleared.  Branch-free, so lanes at different rows stay converged.
__device__ __forceinline__ void next_bit3(unsigned& a, unsigned& b, unsigned& c, int& k, int& r) {
    const unsigned cur = a ? a : (b ? b : c);
    r = a ? 0 : (b ? 1 : 2);
    k = __ffs(cur) - 1;
    const unsigned nxt = cur & (cur - 1u);
    a = r == 0 ? nxt : a;
    b = r == 1 ? nxt : b;
    c = r == 2 ? nxt : c;
}

template <class Act>
__global__ void __launch_bounds__(128) k_mask2_build(const __grid_constant__ PairArgs A, unsigned* mask, int cap,
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
        const int c_first = A.s.cell[w0];
        const int c_last = A.s.cell[min(w0 + 31, n_alive - 1)];
        EPP_CHECK(c_first >= 0 && c_last >= c_first && c_last < A.dom.n_cells, 34, c_last);
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
        RowWin win[3], u[3];
        bool over = false, staged = tiled;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            win[r] = row_range(A, stencil_row<2>(A, rid, r), cx - 1, cx + 1);
            over |= win[r].hi - win[r].lo > 32;
            u[r] = RowWin{0, 0};
            if (tiled) {
                u[r] = row_range(A, stencil_row<2>(A, rid0, r), c_first - rid0 * n0 - 1, c_last - rid0 * n0 + 1);
                staged = staged && u[r].hi - u[r].lo <= 64;   // warp-uniform
            }
        }
        const bool walk = valid && !over;
        unsigned long long allowed[3];
        bool one_h[3];
        float h0[3];
        if (staged) stage_rows2<Act, Act::NC != 0, true>(A, act, S, u, amask, lane, st, allowed, one_h, h0);
        unsigned w[3] = {0u, 0u, 0u};
        int off[3];
        if (walk) {
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int len = win[r].hi - win[r].lo;
                off[r] = staged ? 64 * r + win[r].lo - u[r].lo : win[r].lo;
                unsigned word;
                if (staged) {
                    const bool uniform = one_h[r] && (dflt || h0[r] == xi.w);
                    word = window_bits<2>(S.x, off[r], 0, len, xi, uniform, dflt ? A.dom.gap_square : tc.h2sq, tc.h2sq,
                                          dflt, A.dom.gap_square);
                    word &= (unsigned)(allowed[r] >> (win[r].lo - u[r].lo));
                } else {
                    word = 0u;
                    for (int k = len - 1; k >= 0; --k) {
                        const int j = win[r].lo + k;
                        word = (word << 1) | (accept<2>(A, i, xi, amask, tc.h2sq, j, A.s.xh[j], st) ? 1u : 0u);
                    }
                }
                if (len < 32) word &= (1u << len) - 1u;
                if (r == 1) word &= ~(1u << (i - win[1].lo));   // not its own neighbour
                w[r] = word;
            }
            cnt = __popc(w[0]) + __popc(w[1]) + __popc(w[2]);
        }
        float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (walk && Act::NC != 0) {
            typename Act::Self me = act.self(i);
            unsigned a = w[0], b = w[1], cc = w[2];
            while (a | b | cc) {   // the search action over the neighbours, in list order
                int k, r;
                next_bit3(a, b, cc, k, r);
                const int base = r == 0 ? off[0] : (r == 1 ? off[1] : off[2]);
                float4 xj;
                int tj;
                typename Act::Nb nb;
                if (staged) {
                    const float4 xs = S.x[base + k];
                    xj = make_float4(xs.x, xs.y, 0.0f, xs.w);
                    tj = entry_tag(__float_as_int(xs.z));
                    nb = S.nb[base + k];
                } else {
                    const int j = base + k;
                    xj = A.s.xh[j];
                    tj = tag_of(A.s.tagm[j]);
                    nb = act.fetch(j, ti, tj);
                }
                const float4 t = act.term(me, nb, ti, tj, xj, geometry<2>(xi, xj), tc);
                sum.x += t.x;
                sum.y += t.y;
            }
        }
        if (on) {
            if (!valid) {
                act.end_idle(i, ti);
                w[0] = w[1] = w[2] = 0u;
            } else if (over) {   // dense neighbourhood: its neighbours come from its stencil
                w[0] = w[2] = 0u;
                w[1] = kMaskOverflow;
                sum = neighbours_by_stencil<2>(A, i, xi, ti, tc, act);
                cnt = (int)sum.w;
                sum.w = 0.0f;
                act.end(i, ti, sum, cnt);
            } else {
                act.end(i, ti, sum, cnt);
            }
            mask[i] = w[0];
            mask[(size_t)cap + i] = w[1];
            mask[(size_t)2 * cap + i] = w[2];
        }
        if (st) atomicOr(A.status, st);
    }
    count_pairs(pairs, cnt);
}

template <class Act, bool EPI, bool STAGE>
__global__ void __launch_bounds__(128) k_mask2_walk(const __grid_constant__ PairArgs A, const unsigned* mask, int cap,
                                                    const __grid_constant__ Act act, unsigned long long* scan_state,
                                                    int n_scan_words) {
    __shared__ Stage2<Act> stage[STAGE ? 4 : 1];
    if (EPI && blockIdx.x == 0)
        for (int t = threadIdx.x; t < n_scan_words; t += blockDim.x) scan_state[t] = 0ull;
    const int lane = threadIdx.x & 31;
    Stage2<Act>& S = stage[STAGE ? (threadIdx.x >> 5) : 0];
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int w0 = i - lane;
    if (w0 < n_alive) {   // warp-uniform
        const bool on = i < n_alive;
        const int n0 = A.dom.n[0];
        const int c_first = A.s.cell[w0];
        const int c_last = A.s.cell[min(w0 + 31, n_alive - 1)];
        EPP_CHECK(c_first >= 0 && c_last >= c_first && c_last < A.dom.n_cells, 35, c_last);
        const int rid0 = c_first / n0;
        const bool tiled = rid0 == c_last / n0;
        const int c = A.s.cell[min(i, n_alive - 1)];
        const int rid = c / n0, cx = c - rid * n0;
        const float4 xi = on ? A.s.xh[i] : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        const int ti = on ? tag_of(A.s.tagm[i]) : 0;
        const bool valid = on && ti >= 1 && ti <= A.n_tags && act.wants(ti);
        unsigned w[3] = {0u, 0u, 0u};
        if (on) {
            w[0] = mask[i];
            w[1] = mask[(size_t)cap + i];
            w[2] = mask[(size_t)2 * cap + i];
        }
        const bool over = w[1] == kMaskOverflow;
        const bool walk = valid && !over;
        RowWin u[3];
        int off[3];
        bool staged = STAGE && tiled;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const RowWin win = row_range(A, stencil_row<2>(A, rid, r), cx - 1, cx + 1);
            u[r] = RowWin{0, 0};
            if (STAGE && tiled) {
                u[r] = row_range(A, stencil_row<2>(A, rid0, r), c_first - rid0 * n0 - 1, c_last - rid0 * n0 + 1);
                staged = staged && u[r].hi - u[r].lo <= 64;
            }
            off[r] = win.lo;
        }
        if (staged) {
            unsigned st = 0u;
            unsigned long long allowed[3];
            bool one_h[3];
            float h0[3];
            stage_rows2<Act, true, false>(A, act, S, u, 0u, lane, st, allowed, one_h, h0);
#pragma unroll
            for (int r = 0; r < 3; ++r) off[r] = 64 * r + off[r] - u[r].lo;
        }
        const TargetConst tc = target_const<2>(on ? xi.w : 1.0f);
        float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        int cnt = 0;
        if (walk) {
            typename Act::Self me = act.self(i);
            unsigned a = w[0], b = w[1], cc = w[2];
            cnt = __popc(a) + __popc(b) + __popc(cc);
            while (a | b | cc) {
                int k, r;
                next_bit3(a, b, cc, k, r);
                const int base = r == 0 ? off[0] : (r == 1 ? off[1] : off[2]);
                float4 xj;
                int tj;
                typename Act::Nb nb;
                if (staged) {
                    const float4 xs = S.x[base + k];
                    xj = make_float4(xs.x, xs.y, 0.0f, xs.w);
                    tj = entry_tag(__float_as_int(xs.z));
                    nb = S.nb[base + k];
                } else {
                    const int j = base + k;
                    EPP_CHECK(j < A.n_max, 36, j);
                    xj = __ldg(&A.s.xh[j]);
                    tj = tag_of(A.s.tagm[j]);
                    nb = act.fetch(j, ti, tj);
                }
                const float4 t = act.term(me, nb, ti, tj, xj, geometry<2>(xi, xj), tc);
                sum.x += t.x;
                sum.y += t.y;
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
