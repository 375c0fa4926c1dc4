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
    cc[2] = D == 3 ? c / (A.dom.n[0] * A.dom.n[1]) : 0;
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
// search! action: neighbour count, optional list (nIndex, nRVec, nR, nW, nDW, nHInv), and the
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
                const float dw = wc2_gradient<D>(r, hinv);
                if (EMIT && k < L.max_nb) {
                    L.hinv[(size_t)k * L.cap + i] = hinv;
                    L.w[(size_t)k * L.cap + i] = wc2_value<D>(r, hinv);
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
            float2 rp;
            if (ti == P.fluid || ti == P.wall) {
                rp.x = __fadd_rn(a.rho_i, __fmul_rn(a.drho, P.dt));
                rp.y = eos(P, rp.x);
            } else {
                rp.x = a.rho_i;
                rp.y = s.p[i];
            }
            s.rpn[i] = rp;
        }
    }
    __device__ __forceinline__ int count(const Acc& a) const { return a.cnt; }
};

// ------------------------------------------------------------------------------------------
// interaction! action: dam-break momentum of main.jl:107-118 with the benchmark's artificial
// viscosity: fluid-fluid iClassicPressure! (Pressure.jl:24-41), fluid-wall iBalancedPressure!
// (:43-60), each followed by sArtificialViscosity! (Viscosity.jl:28-52).  Walls receive nothing.
// FUSED: rho and p come from the density preview (rpn) of the previous search, du starts at 0
// (sAccelerate! zeroed it) and the epilogue integrates (sGravity!, sAccelerate!, sMove!,
// Motion.jl:17-51) and bins the new position.
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

template <int D, bool FUSED>
struct ActMomentum {
    State s;
    DevPhys P;
    DevDomain dom;
    FusedOut F;
    unsigned* status;

    struct Acc {
        float du[3];
        float rho_i, p_i, pr_i;
        float4 vi;
        HCache hc;
    };
    __device__ __forceinline__ bool wants(int ti) const { return ti == P.fluid; }
    __device__ __forceinline__ void begin(int i, int ti, float4 xi, Acc& a) const {
        if (FUSED) {
            a.du[0] = a.du[1] = a.du[2] = 0.0f;
            const float2 rp = s.rpn[i];
            a.rho_i = rp.x;
            a.p_i = rp.y;
        } else {
            const float4 d = s.dv[i];
            a.du[0] = d.x; a.du[1] = d.y; a.du[2] = d.z;
            a.rho_i = s.rho[i];
            a.p_i = s.p[i];
        }
        if (ti == P.fluid) {
            a.pr_i = fdiv(a.p_i, a.rho_i * a.rho_i);
            a.vi = s.vm[i];
            a.hc.init(xi.w);
        }
    }
    __device__ __forceinline__ void pair(int i, int j, int ti, int tj, float4 xi, float4 xj,
                                         float dx, float dy, float dz, float dr2, Acc& a) const {
        const bool ff = tj == P.fluid;
        const bool fw = tj == P.wall;
        if (!(ff || fw)) return;
        const float r = sqrtf(dr2);
        const float hinv = a.hc.pair_hinv(xj.w);
        const float dw = wc2_gradient<D>(r, hinv);
        const float4 vj = s.vm[j];
        float rho_j, p_j;
        if (FUSED) {
            const float2 rp = s.rpn[j];
            rho_j = rp.x;
            p_j = rp.y;
        } else {
            rho_j = s.rho[j];
            p_j = s.p[j];
        }
        float p_rho_2 = ff ? a.pr_i + fdiv(p_j, rho_j * rho_j) : fdiv(a.p_i + p_j, a.rho_i * rho_j);
        p_rho_2 *= fdiv(-vj.w * dw, r);
        a.du[0] += p_rho_2 * dx;
        a.du[1] += p_rho_2 * dy;
        if (D == 3) a.du[2] += p_rho_2 * dz;
        float vdx = dx * (a.vi.x - vj.x);
        vdx += dy * (a.vi.y - vj.y);
        if (D == 3) vdx += dz * (a.vi.z - vj.z);
        if (vdx < 0.0f) {
            const float rhob = 0.5f * (a.rho_i + rho_j);
            const float hh = xj.w == a.hc.h ? a.hc.hh : fdiv(1.0f, hinv);
            const float az = r * r + 0.01f * hh * hh;
            const float phi = fdiv(vdx, hinv * az);
            float force = fdiv((-P.alpha * P.c0 + P.beta * phi) * phi, rhob);
            if (P.visc == EPP_VISCOSITY_REFERENCE) force *= fdiv(-vj.w, a.rho_i * rho_j * r) * dw;
            else force *= fdiv(-vj.w, r) * dw;
            a.du[0] += force * dx;
            a.du[1] += force * dy;
            if (D == 3) a.du[2] += force * dz;
        }
    }
    __device__ __forceinline__ void end(int i, int ti, Acc& a) const {
        if (!FUSED) {
            if (ti == P.fluid) s.dv[i] = make_float4(a.du[0], a.du[1], a.du[2], 0.0f);
            return;
        }
        integrate_and_bin(i, ti, &a);
    }
    __device__ __forceinline__ int count(const Acc&) const { return 0; }
    // Fused epilogue; also used (acc == nullptr) for particles outside the pair loop.
    __device__ __forceinline__ void integrate_and_bin(int i, int ti, const Acc* a) const {
        float4 x = s.xh[i];
        float4 v = s.vm[i];
        float4 cp = s.comp[i];
        const int tm = s.tagm[i];
        int c = s.cell[i];
        const bool alive = c != dom.n_cells;
        if (alive && ti == P.fluid && a) {
            float du[3] = {a->du[0], a->du[1], a->du[2]};
            float vv[3] = {v.x, v.y, v.z}, xx[3] = {x.x, x.y, x.z}, cc[3] = {cp.x, cp.y, cp.z};
#pragma unroll
            for (int k = 0; k < D; ++k) {
                du[k] = __fadd_rn(du[k], P.g[k]);                      // sGravity!
                vv[k] = __fadd_rn(vv[k], __fmul_rn(du[k], P.dt));      // sAccelerate!
            }
#pragma unroll
            for (int k = 0; k < D; ++k) {                              // sMove!
                if (P.kahan) {
                    const float y = __fsub_rn(__fmul_rn(vv[k], P.dt), cc[k]);
                    const float t = __fadd_rn(xx[k], y);
                    cc[k] = __fsub_rn(__fsub_rn(t, xx[k]), y);
                    xx[k] = t;
                } else {
                    xx[k] = __fadd_rn(xx[k], __fmul_rn(vv[k], P.dt));
                }
            }
            x.x = xx[0]; x.y = xx[1]; x.z = xx[2];
            v.x = vv[0]; v.y = vv[1]; v.z = vv[2];
            cp.x = cc[0]; cp.y = cc[1]; cp.z = cc[2];
            if (F.accel) F.accel[i] = make_float4(du[0], du[1], du[2], 0.0f);
            if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z)))
                atomicOr(status, EPP_STATUS_NONFINITE);
        }
        F.xh[i] = x;
        F.vm[i] = v;
        F.comp[i] = cp;
        // bin the new position (insertParticlesIntoCells!, NeighbourSearch.jl:26-45)
        if (alive && (movable_of(tm) || c < 0)) {
            c = cell_of<D>(dom, x);
            if (c < 0) {
                c = dom.n_cells;
                atomicOr(status, EPP_STATUS_KILLED);
            }
        }
        const int slot = atomicAdd(&F.count[c], 1);
        F.cs[i] = make_int2(c, slot);
    }
};

// Fused momentum pass: the pair kernel for alive particles, the epilogue alone for the dead
// bin; block 0 clears the scan's look-back state.
template <int D>
__global__ void __launch_bounds__(128) k_momentum_fused(PairArgs A, ActMomentum<D, true> act) {
    if (blockIdx.x == 0)
        for (int t = threadIdx.x; t < act.F.n_scan_words; t += blockDim.x) act.F.scan_state[t] = 0ull;
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= act.F.n) return;
    if (i >= n_alive) {
        act.integrate_and_bin(i, tag_of(A.s.tagm[i]), nullptr);
        return;
    }
    const float4 xi = A.s.xh[i];
    const int ti = tag_of(A.s.tagm[i]);
    typename ActMomentum<D, true>::Acc acc;
    act.begin(i, ti, xi, acc);
    const bool bad_i = ti < 1 || ti > A.n_tags;
    if (bad_i) atomicOr(A.status, EPP_STATUS_BAD_TAG);
    if (!bad_i && act.wants(ti)) traverse<D>(A, i, xi, ti, act, acc);
    act.integrate_and_bin(i, ti, (!bad_i && ti == act.P.fluid) ? &acc : nullptr);
}

// interaction! test action (ActionTest.jl:71-75): dVelocity += 1 per listed neighbour.
template <int D>
struct ActCount {
    State s;
    struct Acc {
        float n;
    };
    __device__ __forceinline__ bool wants(int) const { return true; }
    __device__ __forceinline__ void begin(int, int, float4, Acc& a) const { a.n = 0.0f; }
    __device__ __forceinline__ void pair(int, int, int, int, float4, float4, float, float, float,
                                         float, Acc& a) const {
        a.n += 1.0f;
    }
    __device__ __forceinline__ void end(int i, int, Acc& a) const {
        float4 d = s.dv[i];
        // one += per neighbour and component, as the reference loop adds 1.0 each time
        d.x += a.n;
        d.y += a.n;
        if (D == 3) d.z += a.n;
        s.dv[i] = d;
    }
    __device__ __forceinline__ int count(const Acc&) const { return 0; }
};

}  // namespace epp
