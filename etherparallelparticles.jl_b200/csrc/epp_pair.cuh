// epp_pair.cuh -- the neighbour traversal shared by every pair pass, and its actions.
//
// Traversal = device_findNeighbourParticlesFromCells! (NeighbourSearch.jl:166-227) without the
// stored list: for each alive particle I (one thread, cell-sorted order) the 3^D neighbour
// cells are visited in the reference's table order (NeighbourSystemBase.jl:28-48: x offset
// outer, y inner; z innermost in 3D) and each cell's particles in id order, so neighbours are
// met in the same order as the reference's list.  The criterion is evaluated with IEEE
// operations (no contraction) so the neighbour sets are bit-exact.
#pragma once
#include "epp_cells.cuh"
#include "epp_kernels.cuh"

namespace epp {

struct PairArgs {
    DevDomain dom;
    State s;
    const int* start;        // cell offsets (start[n_cells] = number of alive particles)
    unsigned adj[kMaxTags];  // bit tj-1 of adj[ti-1]: pair (ti, tj) active
    int n_tags;
    int crit;                // EPP_CRITERION_*
    int n_max;               // particles held (bounds every index read from start[])
    unsigned* status;
};

// Visits the neighbours of alive particle i (cell-sorted index) and calls act.pair for each
// one that passes the criterion and the active-pair matrix.
template <int D, class Act>
__device__ __forceinline__ void traverse(const PairArgs& A, int i, float4 xi, int ti,
                                         const Act& act, typename Act::Acc& acc) {
    const unsigned amask = A.adj[ti - 1];
    const int c = A.s.cell[i];
    int cc[3];
    cc[0] = c % A.dom.n[0];
    cc[1] = (c / A.dom.n[0]) % A.dom.n[1];
    cc[2] = c / (A.dom.n[0] * A.dom.n[1]);   // 2D: the instance layer (no coupling across it)
    const float h2ii = harmonic2_exact(xi.w, xi.w);
    unsigned st = 0;
    for (int di = -1; di <= 1; ++di) {
        const int ii = cc[0] + di;
        if (ii < 0 || ii >= A.dom.n[0]) continue;
        for (int dj = -1; dj <= 1; ++dj) {
            const int jj = cc[1] + dj;
            if (jj < 0 || jj >= A.dom.n[1]) continue;
            for (int dk = (D == 3 ? -1 : 0); dk <= (D == 3 ? 1 : 0); ++dk) {
                const int kk = cc[2] + dk;
                if (D == 3 && (kk < 0 || kk >= A.dom.n[2])) continue;
                const int nc = ii + A.dom.n[0] * (jj + A.dom.n[1] * kk);
                const int je = min(A.start[nc + 1], A.n_max);
                for (int j = max(A.start[nc], 0); j < je; ++j) {
                    if (j == i) continue;
                    const float4 xj = A.s.xh[j];
                    const float dx = __fsub_rn(xi.x, xj.x);
                    const float dy = __fsub_rn(xi.y, xj.y);
                    const float dz = D == 3 ? __fsub_rn(xi.z, xj.z) : 0.0f;
                    float dr2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                    if (D == 3) dr2 = __fadd_rn(dr2, __fmul_rn(dz, dz));
                    bool ok;
                    if (A.crit == EPP_CRITERION_DEFAULT) {
                        ok = dr2 <= A.dom.gap_square;
                    } else {
                        const float h2 = xj.w == xi.w ? h2ii : harmonic2_exact(xi.w, xj.w);
                        ok = dr2 <= __fmul_rn(h2, h2);
                    }
                    if (!ok) continue;
                    const int tj = tag_of(A.s.tagm[j]);
                    if (tj < 1 || tj > A.n_tags) {
                        st |= EPP_STATUS_BAD_TAG;
                        continue;
                    }
                    if (!((amask >> (tj - 1)) & 1u)) continue;
                    act.pair(i, j, ti, tj, xi, xj, dx, dy, dz, dr2, acc);
                }
            }
        }
    }
    if (st) atomicOr(A.status, st);
}

// Adds the per-thread neighbour counts of a block's warps to *counter (all lanes take part).
__device__ __forceinline__ void count_pairs(unsigned long long* counter, int cnt) {
    unsigned long long c = (unsigned long long)cnt;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && counter && c) atomicAdd(counter, c);
}

template <int D, class Act>
__global__ void __launch_bounds__(128) k_pair(PairArgs A, Act act, unsigned long long* pairs) {
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int cnt = 0;
    if (i < n_alive) {
        const float4 xi = A.s.xh[i];
        const int ti = tag_of(A.s.tagm[i]);
        typename Act::Acc acc;
        act.begin(i, ti, xi, acc);
        const bool bad_i = ti < 1 || ti > A.n_tags;
        if (bad_i) atomicOr(A.status, EPP_STATUS_BAD_TAG);
        if (!bad_i && act.wants(ti)) traverse<D>(A, i, xi, ti, act, acc);
        act.end(i, ti, acc);
        cnt = act.count(acc);
    }
    count_pairs(pairs, cnt);
}

// Per-particle cached kernel geometry for h_j == h_i (the common case): bit-identical to the
// per-pair IEEE evaluation.
struct HCache {
    float h, hinv, hh;   // h_i, invharmonic(h_i, h_i), 1 / hinv
    __device__ __forceinline__ void init(float hi) {
        h = hi;
        hinv = invharmonic_exact(hi, hi);
        hh = __fdiv_rn(1.0f, hinv);
    }
    __device__ __forceinline__ float pair_hinv(float hj) const {
        return hj == h ? hinv : invharmonic_exact(h, hj);
    }
};

// ------------------------------------------------------------------------------------------
// search! action (exact reference order; used when the list is emitted): neighbour count, list (nIndex, nRVec, nR, nW, nDW, nHInv), and the
// dam-break continuity of main.jl:74-90 (iValueGradient! SPH/Library/Kernel.jl:114-128,
// iClassicContinuity! / iBalancedContinuity! Continuity.jl:23-47).
// FUSED: drho starts from 0 (sContinuity! zeroed it) and the density preview (rho + drho dt,
// eos) that the next momentum pass reads is written to rpn.
template <int D, bool EMIT, bool CONT, bool FUSED>
struct ActSearch {
    State s;
    NeighbourList L;
    DevPhys P;
    int* ncount;
    unsigned* status;

    struct Acc {
        int cnt;
        float drho, rho_i;
        float4 vi;
        HCache hc;
    };
    __device__ __forceinline__ bool wants(int) const { return true; }
    __device__ __forceinline__ void begin(int i, int ti, float4 xi, Acc& a) const {
        a.cnt = 0;
        if (CONT) {
            a.drho = FUSED ? 0.0f : s.drho[i];
            a.rho_i = s.rho[i];
            a.vi = s.vm[i];
            a.hc.init(xi.w);
        }
    }
    __device__ __forceinline__ void pair(int i, int j, int ti, int tj, float4 xi, float4 xj,
                                         float dx, float dy, float dz, float dr2, Acc& a) const {
        const int k = a.cnt;
        float r = 0.0f;
        if (EMIT || CONT) r = sqrtf(dr2);
        if (EMIT) {
            if (k < L.max_nb) {
                L.idx[(size_t)k * L.cap + i] = j;
                L.rvec[((size_t)D * k + 0) * L.cap + i] = dx;
                L.rvec[((size_t)D * k + 1) * L.cap + i] = dy;
                if (D == 3) L.rvec[((size_t)D * k + 2) * L.cap + i] = dz;
                L.r[(size_t)k * L.cap + i] = r;
            } else {
                atomicOr(status, EPP_STATUS_NEIGHBOUR_OVERFLOW);
            }
        }
        if (CONT) {
            const bool ff = ti == P.fluid && tj == P.fluid;
            const bool fw = ti == P.fluid && tj == P.wall;
            const bool wf = ti == P.wall && tj == P.fluid;
            if (ff || fw || wf) {
                const float hinv = a.hc.pair_hinv(xj.w);
                const float dw = kern_gradient<D>(P.kernel, r, hinv);
                if (EMIT && k < L.max_nb) {
                    L.hinv[(size_t)k * L.cap + i] = hinv;
                    L.w[(size_t)k * L.cap + i] = kern_value<D>(P.kernel, r, hinv);
                    L.dw[(size_t)k * L.cap + i] = dw;
                }
                const float4 vj = s.vm[j];
                float vdx = dx * (a.vi.x - vj.x);
                vdx += dy * (a.vi.y - vj.y);
                if (D == 3) vdx += dz * (a.vi.z - vj.z);
                if (ff) a.drho += fdiv(vj.w * vdx * dw, r);
                else a.drho += fdiv(a.rho_i * s.vol[j] * vdx * dw, r);
            }
        }
        a.cnt = k + 1;
    }
    __device__ __forceinline__ void end(int i, int ti, Acc& a) const {
        ncount[i] = a.cnt;
        if (CONT) {
            s.drho[i] = a.drho;
            // density preview of sContinuity! (Continuity.jl:10-21) + eos, exact FP32 order
            if (ti == P.fluid || ti == P.wall) {
                const int inst = inst_of(s.tagm[i]);
                const float rho = __fadd_rn(a.rho_i, __fmul_rn(a.drho, P.dt_of(inst)));
                s.rp4[i] = make_rp4(rho, eos(P, inst, rho));
            } else {
                s.rp4[i] = make_rp4(a.rho_i, s.p[i]);
            }
        }
    }
    __device__ __forceinline__ int count(const Acc& a) const { return a.cnt; }
};

// Outputs of the fused momentum pass (integrate + bin epilogue).
struct FusedOut {
    float4* xh;          // new (x, h)   in the current (old) order
    float4* vm;          // new (v, m)
    float4* comp;        // new Kahan compensation
    int2* cs;            // (cell, slot) for the counting sort
    int* count;          // per-cell counters (zero on entry)
    float4* accel;       // optional dv/dt output (momentum + gravity), may be null
    unsigned long long* scan_state;   // cleared by block 0 for the scan that follows
    int n_scan_words;
    int n;               // all particles (alive first, dead bin last)
};

}  // namespace epp
