// epp_pass.cuh -- the default pair passes: one thread per particle, filter once per step.
//
// A particle's candidates are the particles of its 3^D stencil, enumerated row by row (the 3
// cells x-1..x+1 of a stencil row are contiguous in cell-sorted order).  The search pass filters
// every candidate with the reference's IEEE criterion and active-pair matrix and records the
// accepted ones as bits of a per-particle mask over that enumeration; it then walks the set bits
// only, so the pair arithmetic runs with every lane busy instead of the ~1/3 of lanes that have a
// neighbour at any one candidate.  The next momentum pass sees the same positions, cells and
// criterion, so it reuses the mask and skips the filter entirely.  Candidates past the mask's
// capacity (very dense cells) are filtered and evaluated inline, in the same order.
//
// Summation order per particle = candidate order (row-major over the stencil, id order inside a
// cell): deterministic, and a rounding-level reordering of the reference's list order.
#pragma once
#include "epp_cellpair.cuh"

namespace epp {

template <int D>
struct MaskConf {
    static constexpr int NW = D == 2 ? 4 : 16;   // 32-bit words per particle
    static constexpr int CAP = 32 * NW;          // candidates covered by the mask
};

struct MaskArgs {
    unsigned* words;   // [NW * cap], word q of particle i at q * cap + i
    int cap;
};

// Row bounds of the stencil of cell c, iterated in order.
template <int D>
struct RowIter {
    int x0, x1, y0, y1, z0, z1, n0, n1;
    int yy, zz;
    __device__ __forceinline__ void init(const PairArgs& A, int c) {
        n0 = A.dom.n[0];
        n1 = A.dom.n[1];
        const int cx = c % n0, cy = (c / n0) % n1, cz = c / (n0 * n1);   // 2D: instance layer
        x0 = max(cx - 1, 0);
        x1 = min(cx + 1, n0 - 1);
        y0 = max(cy - 1, 0);
        y1 = min(cy + 1, n1 - 1);
        z0 = D == 3 ? max(cz - 1, 0) : cz;
        z1 = D == 3 ? min(cz + 1, A.dom.n[2] - 1) : cz;
        yy = y0;
        zz = z0;
    }
    // bounds of the current row; false when all rows are done
    __device__ __forceinline__ bool bounds(const PairArgs& A, int& lo, int& hi) const {
        if (zz > z1) return false;
        const int base = n0 * (yy + n1 * zz);
        lo = max(A.start[base + x0], 0);
        hi = min(A.start[base + x1 + 1], A.n_max);
        hi = max(hi, lo);
        return true;
    }
    __device__ __forceinline__ void next() {
        if (++yy > y1) {
            yy = y0;
            ++zz;
        }
    }
};

template <int NW>
__device__ __forceinline__ void mask_put(unsigned (&mw)[NW], int q, unsigned v) {
#pragma unroll
    for (int w = 0; w < NW; ++w)
        if (w == q) mw[w] = v;
}

// Candidate filter: the reference's criterion (IEEE, exact) and the active-pair matrix.
template <int D>
__device__ __forceinline__ bool accept(const PairArgs& A, int i, float4 xi, unsigned amask, float h2sq,
                                       int j, float4 xj, unsigned& st) {
    if (j == i) return false;
    const float dx = __fsub_rn(xi.x, xj.x);
    const float dy = __fsub_rn(xi.y, xj.y);
    float dr2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
    if (D == 3) {
        const float dz = __fsub_rn(xi.z, xj.z);
        dr2 = __fadd_rn(dr2, __fmul_rn(dz, dz));
    }
    bool ok;
    if (A.crit == EPP_CRITERION_DEFAULT) {
        ok = dr2 <= A.dom.gap_square;
    } else if (xj.w == xi.w) {
        ok = dr2 <= h2sq;
    } else {
        const float h2 = harmonic2_exact(xi.w, xj.w);
        ok = dr2 <= __fmul_rn(h2, h2);
    }
    if (!ok) return false;
    const int tj = tag_of(A.s.tagm[j]);
    if (tj < 1 || tj > A.n_tags) {
        st |= EPP_STATUS_BAD_TAG;
        return false;
    }
    return (amask >> (tj - 1)) & 1u;
}

template <int D>
__device__ __forceinline__ PairGeo geometry(float4 xi, float4 xj) {
    PairGeo g;
    g.dx = __fsub_rn(xi.x, xj.x);
    g.dy = __fsub_rn(xi.y, xj.y);
    g.dz = D == 3 ? __fsub_rn(xi.z, xj.z) : 0.0f;
    g.dr2 = __fadd_rn(__fmul_rn(g.dx, g.dx), __fmul_rn(g.dy, g.dy));
    if (D == 3) g.dr2 = __fadd_rn(g.dr2, __fmul_rn(g.dz, g.dz));
    return g;
}

// One pass over the neighbours of particle i.  BUILD: filter the candidates, store the mask
// (when M.words) and evaluate the accepted pairs.  !BUILD: read the mask written by the last
// search at these positions and evaluate its pairs.  Returns the number of neighbours.
template <int D, bool BUILD, class Act>
__device__ __forceinline__ int neighbours(const PairArgs& A, const MaskArgs& M, int i, float4 xi, int ti,
                                          const TargetConst& tc, const Act& act, float4& sum) {
    constexpr int NW = MaskConf<D>::NW;
    constexpr int CAP = MaskConf<D>::CAP;
    const unsigned amask = A.adj[ti - 1];
    unsigned st = 0;
    unsigned mw[NW];
    int count = 0;
    RowIter<D> rows;
    rows.init(A, A.s.cell[i]);
    if (BUILD) {
        // phase A: filter into mask bits; candidates past CAP are evaluated inline
        unsigned cur = 0;
        int k = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) mw[w] = 0u;
        RowIter<D> it = rows;
        int lo, hi;
        while (it.bounds(A, lo, hi)) {
            for (int j = lo; j < hi; ++j, ++k) {
                const float4 xj = A.s.xh[j];
                const bool ok = accept<D>(A, i, xi, amask, tc.h2sq, j, xj, st);
                if (k < CAP) {
                    cur |= (unsigned)ok << (k & 31);
                    if ((k & 31) == 31) {
                        mask_put<NW>(mw, k >> 5, cur);
                        cur = 0u;
                    }
                } else if (ok) {
                    const float4 c = act.contrib(i, j, ti, tag_of(A.s.tagm[j]), xi, xj, geometry<D>(xi, xj), tc);
                    sum.x += c.x;
                    sum.y += c.y;
                    sum.z += c.z;
                    ++count;
                }
            }
            it.next();
        }
        if (k < CAP && (k & 31)) mask_put<NW>(mw, k >> 5, cur);
        if (M.words) {
#pragma unroll
            for (int w = 0; w < NW; ++w) M.words[(size_t)w * M.cap + i] = mw[w];
        }
    } else {
#pragma unroll
        for (int w = 0; w < NW; ++w) mw[w] = M.words[(size_t)w * M.cap + i];
    }
    // phase B: the accepted pairs in candidate order
    float4 part = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    {
        int lo = 0, hi = 0, off = 0;
        bool more = rows.bounds(A, lo, hi);
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            unsigned bits = mw[w];
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1u;
                const int k = 32 * w + b;
                while (more && k >= off + (hi - lo)) {
                    off += hi - lo;
                    rows.next();
                    more = rows.bounds(A, lo, hi);
                }
                if (!more) break;
                const int j = lo + (k - off);
                const float4 xj = A.s.xh[j];
                const float4 c = act.contrib(i, j, ti, tag_of(A.s.tagm[j]), xi, xj, geometry<D>(xi, xj), tc);
                part.x += c.x;
                part.y += c.y;
                part.z += c.z;
                ++count;
            }
        }
    }
    // the mask's pairs precede the inline ones in candidate order
    sum.x = part.x + sum.x;
    sum.y = part.y + sum.y;
    sum.z = part.z + sum.z;
    if (!BUILD) {
        // candidates past CAP: filter inline (same order as the search that built the mask)
        RowIter<D> it;
        it.init(A, A.s.cell[i]);
        int k = 0, lo, hi;
        while (it.bounds(A, lo, hi)) {
            if (k + (hi - lo) > CAP) {
                for (int j = max(lo, lo + (CAP - k)); j < hi; ++j) {
                    const float4 xj = A.s.xh[j];
                    if (accept<D>(A, i, xi, amask, tc.h2sq, j, xj, st)) {
                        const float4 c =
                            act.contrib(i, j, ti, tag_of(A.s.tagm[j]), xi, xj, geometry<D>(xi, xj), tc);
                        sum.x += c.x;
                        sum.y += c.y;
                        sum.z += c.z;
                        ++count;
                    }
                }
            }
            k += hi - lo;
            it.next();
        }
    }
    if (st) atomicOr(A.status, st);
    return count;
}

// A pair pass, one thread per particle.  EPI: fused momentum (integrate + bin for every particle,
// the dead bin included; block 0 clears the scan state of the step's sort).
template <int D, bool BUILD, class Act, bool EPI>
__global__ void __launch_bounds__(128, 4) k_pass(PairArgs A, MaskArgs M, Act act, unsigned long long* pairs,
                                                 unsigned long long* scan_state, int n_scan_words) {
    if (EPI && blockIdx.x == 0)
        for (int t = threadIdx.x; t < n_scan_words; t += blockDim.x) scan_state[t] = 0ull;
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int cnt = 0;
    if (i < n_alive) {
        const float4 xi = A.s.xh[i];
        const int ti = tag_of(A.s.tagm[i]);
        if (ti < 1 || ti > A.n_tags) {
            atomicOr(A.status, EPP_STATUS_BAD_TAG);
            act.end_idle(i, ti);
        } else if (!act.wants(ti)) {
            act.end_idle(i, ti);
        } else {
            const TargetConst tc = target_const<D>(xi.w);
            float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            cnt = neighbours<D, BUILD>(A, M, i, xi, ti, tc, act, sum);
            act.end(i, ti, sum, cnt);
        }
    } else if (EPI && i < A.n_max) {
        act.end_idle(i, tag_of(A.s.tagm[i]));
    }
    count_pairs(pairs, cnt);
}

}  // namespace epp
