// epp_tile.cuh -- the default pair passes: warp tiles over a shared candidate list.
//
// A warp takes 32 consecutive particles in cell order.  When their cells lie in one cell row
// (x from xa to xb at fixed y, z) the union of their 3^D stencils is, for each of the 3^(D-1)
// stencil rows (y+dy, z+dz), the cells xa-1 .. xb+1 -- contiguous in cell order, so 3 (2D) or
// 9 (3D) contiguous particle ranges shared by the whole warp.  A warp that crosses a row end
// (about 2% of them) uses each lane's own stencil instead; both passes make the same choice.
//
// The search pass (k_build) stages each chunk of 32 candidates in shared memory with one
// coalesced load per lane; every lane then tests all 32 staged candidates against its own
// particle with broadcast shared-memory reads -- all lanes in lockstep -- using the reference's
// IEEE criterion and the active-pair matrix, and appends its accepted neighbours (sorted index
// and tag, candidate order) to its list.  The pair passes (k_list: continuity, momentum, the
// count actions) then walk each particle's list, one thread per particle, so every lane runs
// its own neighbour count without waiting for the others' candidates.
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

// Pairs of FP32 values in one 64-bit register: Blackwell's f32x2 arithmetic performs two IEEE
// round-to-nearest operations per instruction.  Packed sub and mul match __fsub_rn / __fmul_rn
// bit for bit (checked on B200 over 8M random pairs); a packed add fed directly by a packed
// multiply was measured to round like a fused multiply-add, so sums stay scalar __fadd_rn.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float a, float b) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_unpack(f32x2 v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

template <int D>
struct TileConf {
    static constexpr int NRMAX = D == 2 ? 3 : 9;   // stencil rows: ranges of a tile or of one particle
};

// A neighbour-list entry carries the neighbour's sorted index in its low 28 bits and its tag - 1
// in the top 4 (tags are 1..EPP_MAX_TAGS = 16), so the list passes get the tag with the index
// instead of gathering it.  Contexts hold at most 2^28 particles.
constexpr int kEntryBits = 28;
__device__ __forceinline__ int list_entry(int j, int tag) { return j | ((tag - 1) << kEntryBits); }
__device__ __forceinline__ int entry_index(int e) { return e & ((1 << kEntryBits) - 1); }
__device__ __forceinline__ int entry_tag(int e) { return (int)((unsigned)e >> kEntryBits) + 1; }

struct TileMask {
    int cap;
    int* list;   // [cap * LCAP]: row i holds the neighbours (sorted indices) of particle i in order
};

template <int D>
struct ListConf {
    static constexpr int LCAP = D == 2 ? 64 : 160;   // neighbours kept per particle (multiple of 4)
    // 3D: row-major, a particle's entries contiguous (written and read 16 bytes at a time);
    // 2D: column-major, entry k of particle i at k * cap + i (a warp's reads coalesce).
    static constexpr bool ROW = D == 3;
};

// Appends a lane's neighbours to its list; entries past LCAP are counted but not stored.
// Row-major lists take one int4 store per four neighbours.
template <int D>
struct ListWriter {
    int* base;   // row of the particle (row-major) or its column origin (column-major)
    int cap;
    int b0, b1, b2;
    __device__ __forceinline__ void put(int cnt, int j) {
        if (cnt >= ListConf<D>::LCAP) return;
        if (!ListConf<D>::ROW) {   // column-major: base advances one column per entry
            *base = j;
            base += cap;
            return;
        }
        // row-major: the last three entries wait in b0..b2 (oldest first); every fourth entry
        // stores the group and the row pointer moves on
        if ((cnt & 3) == 3) {
            *reinterpret_cast<int4*>(base) = make_int4(b0, b1, b2, j);
            base += 4;
        }
        b0 = b1;
        b1 = b2;
        b2 = j;
    }
    // the last partial group of a row (its unused slots are never read)
    __device__ __forceinline__ void flush(int cnt) {
        if (!ListConf<D>::ROW || cnt >= ListConf<D>::LCAP) return;
        const int r = cnt & 3;   // entries waiting: the newest r of b0..b2
        if (r == 1) *reinterpret_cast<int4*>(base) = make_int4(b2, 0, 0, 0);
        else if (r == 2) *reinterpret_cast<int4*>(base) = make_int4(b1, b2, 0, 0);
        else if (r == 3) *reinterpret_cast<int4*>(base) = make_int4(b0, b1, b2, 0);
    }
};

template <int D>
__device__ __forceinline__ ListWriter<D> list_writer(const TileMask& M, int i) {
    return ListWriter<D>{ListConf<D>::ROW ? M.list + (size_t)i * ListConf<D>::LCAP : M.list + i, M.cap, 0, 0, 0};
}

// Reads a particle's list in order, the next entries already in flight: 2D (column-major) one
// entry at a time through next(), with streaming loads (each entry is read once: evicted first,
// so the neighbour records the pass gathers keep the L1; momentum -1.7%); 3D (row-major) rows are
// read four entries at a time by k_list from the two groups start() loads, as ordinary loads (a
// row's next group shares its line: streaming loads there cost the 3D list passes 5-9%).
template <int D>
struct ListReader {
    const int* base;
    int cap, cnt;
    int4 q, qn;
    __device__ __forceinline__ void start(const TileMask& M, int i, int n) {
        cap = M.cap;
        cnt = n;
        if (ListConf<D>::ROW) {
            base = M.list + (size_t)i * ListConf<D>::LCAP;
            const int4* row = reinterpret_cast<const int4*>(base);
            q = n > 0 ? row[0] : make_int4(0, 0, 0, 0);
            qn = n > 4 ? row[1] : make_int4(0, 0, 0, 0);
        } else {
            base = M.list + i;
            q.x = n > 0 ? __ldcs(base) : 0;
        }
    }
    // entry k of a column-major list (called with k = 0, 1, 2, ... < cnt)
    __device__ __forceinline__ int next(int k) {
        const int j = q.x;
        if (k + 1 < cnt) {   // the next entry one column on
            base += cap;
            q.x = __ldcs(base);
        }
        return j;
    }
};

// Candidate ranges (contiguous particle index ranges) of a warp tile or of one particle.
template <int D>
struct TileRanges {
    int lo[TileConf<D>::NRMAX], len[TileConf<D>::NRMAX], cum[TileConf<D>::NRMAX];   // cum: first candidate index
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
        cum[n] = total;
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
    // candidate index k (0 <= k < total) -> particle index: the last range starting at or before k
    // holds it (empty ranges share their successor's start, which comes after them)
    __device__ __forceinline__ int at(int k) const {
        int b = lo[0];
#pragma unroll
        for (int r = 1; r < TileConf<D>::NRMAX; ++r)
            if (r < n && k >= cum[r]) b = lo[r] - cum[r];
        return k + b;
    }
};

// Neighbour list of one lane from its own stencil (warps that cross a cell-row end): candidates
// in order, each filtered with the reference's criterion and the active-pair matrix.
template <int D>
__device__ __forceinline__ int lane_stencil_list(const PairArgs& A, ListWriter<D>& L, const TileRanges<D>& R,
                                                 int i, float4 xi, int ti, float h2sq, unsigned& st) {
    const unsigned amask = A.adj[ti - 1];
    int cnt = 0;
    for (int r = 0; r < R.n; ++r) {
        for (int j = R.lo[r]; j < R.lo[r] + R.len[r]; ++j) {
            EPP_CHECK(j >= 0 && j < A.n_max, 14, j);
            if (!accept<D>(A, i, xi, amask, h2sq, j, A.s.xh[j], st)) continue;
            L.put(cnt++, list_entry(j, tag_of(A.s.tagm[j])));
        }
    }
    return cnt;
}

// The search pass: neighbour lists and nCount.  Each chunk of 32 candidates of the warp's union
// is staged in shared memory (position and index, one coalesced load per lane; the next chunk's
// loads are issued before the current chunk is tested); every lane tests all 32 against its own
// particle in lockstep with the reference's IEEE criterion.  A chunk whose candidates share one
// h (all of them away from material interfaces) is tested against one exact bound per lane;
// other chunks look the bound up per candidate.  One ballot per tag gives the chunk's candidates
// of each tag, so a lane keeps only the pairs its row of the active-pair matrix allows, then
// appends them to its list in candidate order.
template <int D>
__global__ void __launch_bounds__(128, D == 2 ? 8 : 6)
    k_build(const __grid_constant__ PairArgs A, const __grid_constant__ TileMask M, int* ncount,
            unsigned long long* pairs) {
    __shared__ __align__(16) float s_p[4][4][32];   // staged x, y, z, h of a chunk (per warp)
    __shared__ int s_j[4][32];
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
        // a row end); otherwise every lane uses its own stencil
        const bool tiled = r1 == r0;
        TileRanges<D> R;
        R.n = 0;
        R.total = 0;
        if (tiled) {
            R.stencil(A, r0 % A.dom.n[1], r0 / A.dom.n[1], c_first - r0 * n0, c_last - r0 * n0);
        } else {
            const int c = A.s.cell[min(i, n_alive - 1)];
            R.stencil(A, (c / n0) % A.dom.n[1], (c / n0) / A.dom.n[1], c % n0, c % n0);
        }
        const float4 xi = on ? A.s.xh[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const int ti = on ? tag_of(A.s.tagm[i]) : 0;
        const bool valid = on && ti >= 1 && ti <= A.n_tags;
        unsigned st = 0;
        if (on && !valid) st |= EPP_STATUS_BAD_TAG;
        const TargetConst tc = target_const<D>(on ? xi.w : 1.0f);
        const unsigned amask = valid ? A.adj[ti - 1] : 0u;
        ListWriter<D> L = list_writer<D>(M, min(i, n_alive - 1));
        if (!tiled) {
            if (valid) cnt = lane_stencil_list<D>(A, L, R, i, xi, ti, tc.h2sq, st);
        } else {
            const bool dflt = A.crit == EPP_CRITERION_DEFAULT;
            float hc_h = xi.w;   // exact bound of the last h_j seen
            float hc_r2 = dflt ? A.dom.gap_square : tc.h2sq;
            const int nchunk = (R.total + 31) >> 5;
            // this lane's own particle in the union: the middle stencil row holds it
            constexpr int RMID = D == 3 ? 4 : 1;
            const int k_self = on ? R.cum[RMID] + (i - R.lo[RMID]) : -1;
            // chunk 0 in flight
            bool real = lane < R.total;
            int jn = real ? R.at(lane) : 0;
            float4 xn = real ? A.s.xh[jn] : make_float4(1e30f, 1e30f, 1e30f, 0.0f);
            int tn = real ? tag_of(A.s.tagm[jn]) : 0;
            for (int ch = 0; ch < nchunk; ++ch) {
                EPP_CHECK(jn >= 0 && jn < A.n_max, 12, jn);
                // padding past the last candidate is far away: it fails every test
                s_p[wib][0][lane] = xn.x;
                s_p[wib][1][lane] = xn.y;
                s_p[wib][2][lane] = xn.z;
                s_p[wib][3][lane] = xn.w;
                s_j[wib][lane] = list_entry(jn, tn);   // appended as is (a real, allowed tag)
                const int tj = tn;
                const bool real_c = real;
                if (__ballot_sync(0xffffffffu, real_c && (tj < 1 || tj > A.n_tags))) st |= EPP_STATUS_BAD_TAG;
                // candidates whose tag this lane's row of the active-pair matrix accepts
                unsigned allowed = 0u;
                for (int t = 1; t <= A.n_tags; ++t) {
                    const unsigned of_t = __ballot_sync(0xffffffffu, real_c && tj == t);
                    if ((amask >> (t - 1)) & 1u) allowed |= of_t;
                }
                // one h for every real candidate of the chunk?
                const float h0 = __shfl_sync(0xffffffffu, xn.w, 0);
                const bool one_h = __all_sync(0xffffffffu, !real_c || xn.w == h0);
                __syncwarp();
                // next chunk's loads, in flight while this one is tested
                if (ch + 1 < nchunk) {
                    const int k = ((ch + 1) << 5) + lane;
                    real = k < R.total;
                    jn = real ? R.at(k) : 0;
                    xn = real ? A.s.xh[jn] : make_float4(1e30f, 1e30f, 1e30f, 0.0f);
                    tn = real ? tag_of(A.s.tagm[jn]) : 0;
                }
                unsigned word = 0u;
                if (one_h) {
                    if (h0 != hc_h) {
                        hc_h = h0;
                        hc_r2 = dflt ? A.dom.gap_square : h0 == xi.w ? tc.h2sq : pair_r2(xi.w, h0);
                    }
                    // dr2 <= R2 as integers: non-negative floats order like their bit patterns, so
                    // bits(dr2) - bits(R2) - 1 is negative exactly for the accepted candidates, and
                    // a funnel shift moves that sign bit into the chunk's word (candidate 0 ends in
                    // the top bit, where the append loop below starts)
                    const int nR2 = -__float_as_int(hc_r2) - 1;
                    // two candidates per packed sub / mul; dr2 = (dx dx + dy dy) + dz dz, IEEE
                    const f32x2 XI = f2_pack(xi.x, xi.x), YI = f2_pack(xi.y, xi.y), ZI = f2_pack(xi.z, xi.z);
                    const f32x2* px = reinterpret_cast<const f32x2*>(s_p[wib][0]);
                    const f32x2* py = reinterpret_cast<const f32x2*>(s_p[wib][1]);
                    const f32x2* pz = reinterpret_cast<const f32x2*>(s_p[wib][2]);
#pragma unroll
                    for (int b = 0; b < 16; ++b) {
                        const f32x2 dx = f2_sub(XI, px[b]);
                        const f32x2 dy = f2_sub(YI, py[b]);
                        float x0, x1, y0, y1;
                        f2_unpack(f2_mul(dx, dx), x0, x1);
                        f2_unpack(f2_mul(dy, dy), y0, y1);
                        float d0 = __fadd_rn(x0, y0), d1 = __fadd_rn(x1, y1);
                        if (D == 3) {
                            const f32x2 dz = f2_sub(ZI, pz[b]);
                            float z0, z1;
                            f2_unpack(f2_mul(dz, dz), z0, z1);
                            d0 = __fadd_rn(d0, z0);
                            d1 = __fadd_rn(d1, z1);
                        }
                        word = __funnelshift_l((unsigned)(__float_as_int(d0) + nR2), word, 1);
                        word = __funnelshift_l((unsigned)(__float_as_int(d1) + nR2), word, 1);
                    }
                } else {
#pragma unroll 8
                    for (int b = 0; b < 32; ++b) {
                        const float4 xj = make_float4(s_p[wib][0][b], s_p[wib][1][b], s_p[wib][2][b], s_p[wib][3][b]);
                        const float dx = __fsub_rn(xi.x, xj.x);
                        const float dy = __fsub_rn(xi.y, xj.y);
                        float dr2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                        if (D == 3) {
                            const float dz = __fsub_rn(xi.z, xj.z);
                            dr2 = __fadd_rn(dr2, __fmul_rn(dz, dz));
                        }
                        if (xj.w != hc_h) {
                            hc_h = xj.w;
                            hc_r2 = dflt ? A.dom.gap_square : xj.w == xi.w ? tc.h2sq : pair_r2(xi.w, xj.w);
                        }
                        word |= (unsigned)(dr2 <= hc_r2) << (31 - b);
                    }
                }
                // candidate b at bit 31 - b: walked from the top with count-leading-zeros
                word &= __brev(allowed);
                if ((k_self >> 5) == ch) word &= ~(0x80000000u >> (k_self & 31));   // not its own neighbour
                // this lane's neighbours among the chunk, in candidate order
                while (word) {
                    const int b = __clz(word);
                    word ^= 0x80000000u >> b;
                    L.put(cnt++, s_j[wib][b]);
                }
                __syncwarp();
            }
        }
        L.flush(cnt);
        if (st) atomicOr(A.status, st);
        if (on) ncount[i] = cnt;
    }
    count_pairs(pairs, cnt);
}

// Neighbours of particle i from its own stencil, filtered inline (used when the list of the last
// search overflowed); same order as the search pass.  Returns the sum with the count in w.
template <int D, class Act>
__device__ __noinline__ float4 neighbours_by_stencil(const PairArgs& A, int i, float4 xi, int ti,
                                                     const TargetConst& tc, const Act& act) {
    const int c = A.s.cell[i];
    const int n0 = A.dom.n[0];
    TileRanges<D> R;
    R.n = 0;
    R.total = 0;
    R.stencil(A, (c / n0) % A.dom.n[1], (c / n0) / A.dom.n[1], c % n0, c % n0);
    const unsigned amask = A.adj[ti - 1];
    unsigned st = 0;
    const typename Act::Self me = act.self(i);
    float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    int cnt = 0;
    for (int r = 0; r < R.n; ++r)
        for (int j = R.lo[r]; j < R.lo[r] + R.len[r]; ++j) {
            const float4 xj = A.s.xh[j];
            if (!accept<D>(A, i, xi, amask, tc.h2sq, j, xj, st)) continue;
            const int tj = tag_of(A.s.tagm[j]);
            const float4 t = act.term(me, act.fetch(j, ti, tj), ti, tj, xj, geometry<D>(xi, xj), tc);
            sum.x += t.x;
            sum.y += t.y;
            sum.z += t.z;
            ++cnt;
        }
    if (st) atomicOr(A.status, st);
    sum.w = (float)cnt;
    return sum;
}

// A pair action over the neighbour lists written by the last search pass (same positions,
// cells and criterion): one thread per particle walking its own list, the next entries already
// in flight.  EPI: fused momentum step (integrate + bin for every
// particle, dead bin included; block 0 clears the scan state).
template <int D, class Act, bool EPI>
__global__ void __launch_bounds__(128, D == 2 ? 9 : 4)   // 2D: 9 blocks (56 registers) beat 8, 10 and 12
    k_list(const __grid_constant__ PairArgs A, const __grid_constant__ TileMask M, const int* ncount,
           const __grid_constant__ Act act, unsigned long long* scan_state, int n_scan_words) {
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
                ListReader<D> lr;
                lr.start(M, i, cnt);
                if (D == 2) {   // 2D: a second neighbour record in flight costs more than it hides
                    for (int k = 0; k < cnt; ++k) {
                        const int e = lr.next(k);
                        const int j = entry_index(e);
                        EPP_CHECK(j < A.n_max, 16, j);
                        const int tj = entry_tag(e);
                        const float4 xj = __ldg(&A.s.xh[j]);
                        const float4 t =
                            act.term(me, act.fetch(j, ti, tj), ti, tj, xj, geometry<D>(xi, xj), tc);
                        sum.x += t.x;
                        sum.y += t.y;
                        sum.z += t.z;
                    }
                    act.end(i, ti, sum, got);
                    return;
                }
                // 3D: software pipeline, neighbour k + 1's loads in flight while k's term runs
                // the row is read four entries (16 bytes) at a time, two groups ahead; inside a
                // group the entry is picked at compile time
                const int4* row = reinterpret_cast<const int4*>(lr.base);
                int4 q = lr.q, qn = lr.qn;
                int en = cnt > 0 ? q.x : list_entry(0, 1);
                int jn = entry_index(en);
                EPP_CHECK(jn < A.n_max, 16, jn);
                float4 xn = cnt > 0 ? __ldg(&A.s.xh[jn]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                typename Act::Nb nn = act.fetch(jn, ti, entry_tag(en));
                for (int k0 = 0; k0 < cnt; k0 += 4) {
                    const int4 q2 = k0 + 8 < cnt ? row[(k0 >> 2) + 2] : make_int4(0, 0, 0, 0);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int k = k0 + u;
                        if (k >= cnt) break;
                        const int tj = entry_tag(en);
                        const float4 xj = xn;
                        const typename Act::Nb nb = nn;
                        if (k + 1 < cnt) {
                            en = u == 0 ? q.y : u == 1 ? q.z : u == 2 ? q.w : qn.x;
                            jn = entry_index(en);
                            EPP_CHECK(jn < A.n_max, 16, jn);
                            xn = __ldg(&A.s.xh[jn]);
                            nn = act.fetch(jn, ti, entry_tag(en));
                        }
                        const float4 t = act.term(me, nb, ti, tj, xj, geometry<D>(xi, xj), tc);
                        sum.x += t.x;
                        sum.y += t.y;
                        sum.z += t.z;
                    }
                    q = qn;
                    qn = q2;
                }
            } else {
                sum = neighbours_by_stencil<D>(A, i, xi, ti, tc, act);
                got = (int)sum.w;
                sum.w = 0.0f;
            }
            act.end(i, ti, sum, got);
        }
    } else if (EPI && i < A.n_max) {
        act.end_idle(i, tag_of(A.s.tagm[i]));
    }
}

}  // namespace epp
