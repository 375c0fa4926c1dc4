// epp_cellpair.cuh -- cell-centric pair passes: one warp per occupied cell.
//
// All particles of a cell share the same 3^D stencil, whose cells form 3 (2D) or 9 (3D) rows
// that are contiguous in cell-sorted order.  A warp stages those candidates in shared memory
// with coalesced 16-byte loads, filters every (target, candidate) pair of the cell with the
// reference's IEEE criterion (so the neighbour sets stay bit-exact), and compacts the accepted
// pairs into a per-warp queue.  The pair arithmetic then runs on full warps, 32 pairs at a time,
// and each window is folded into the targets' accumulators by a segmented shuffle scan over runs
// of the same target -- a fixed order, so results are deterministic.  This replaces the
// thread-per-particle loop in which only about a third of the lanes had a neighbour at any time.
#pragma once
#include <type_traits>

#include "epp_pair_g.cuh"

namespace epp {

constexpr int kCPWarps = 4;       // warps per block
constexpr int kCPQueue = 64;      // queue ring (entries)

template <int D>
struct CPConf {
    static constexpr int C = D == 2 ? 192 : 512;   // staged candidates per chunk
    static constexpr int T = 64;                    // targets per batch
};

struct CellArgs {
    PairArgs A;
    const int* occ;      // occupied cells (cell order)
    const int* meta;     // meta[0] = number of occupied cells
};

struct TargetConst {   // per target: h, invharmonic(h,h), dW/r factor, 1/hinv, (2 harmonic(h,h))^2
    float h, hinv, kdw, hh;
    float h2sq;
};

// Kernel constants of a pair with h_j != h_i: the IEEE division of invharmonic, out of line.
// Equal h (every pair of a uniform-h case) takes the target's cached constants instead.
template <int D>
__device__ __noinline__ float4 hpair_consts(float hi, float hj) {
    const float hinv = invharmonic_exact(hi, hj);
    return make_float4(hinv, wc2_kdw<D>(hinv), __fdividef(1.0f, hinv), 0.0f);
}

template <int D>
__device__ __forceinline__ void pair_consts(const TargetConst& tc, float hj, float& hinv, float& kdw, float& hh) {
    if (hj == tc.h) {
        hinv = tc.hinv;
        kdw = tc.kdw;
        hh = tc.hh;
        return;
    }
    const float4 c = hpair_consts<D>(tc.h, hj);
    hinv = c.x;
    kdw = c.y;
    hh = c.z;
}

// (dW/dr) / r of a pair: the cached Wendland C2 closed form, or (GEN) the selected kernel's; 0
// outside the support.
template <int D, bool GEN>
__device__ __forceinline__ float pair_dwr(int kernel, float q, float hinv, float kdw) {
    if (!GEN || kernel == EPP_KERNEL_WENDLAND_C2) {
        if (!(q < 2.0f)) return 0.0f;   // W = dW = 0 at q >= 2 (WendlandC2.jl:23,44)
        const float u = __fsub_rn(2.0f, q);
        return __fmul_rn(kdw, __fmul_rn(__fmul_rn(u, u), u));
    }
    return kern_dwr<D>(kernel, q, hinv);
}

template <int D>
struct CPShared {
    float4 cx[CPConf<D>::C];     // staged candidate (x, h)
    int cj[CPConf<D>::C];        // staged candidate index
    int ct[CPConf<D>::C];        // staged candidate tag
    int queue[kCPQueue];         // (t << 16) | k
    float4 acc[CPConf<D>::T];    // per-target sums
    int cnt[CPConf<D>::T];       // per-target accepted pairs
    TargetConst tc[CPConf<D>::T];
};

template <int D>
__device__ __forceinline__ TargetConst target_const(float h) {
    TargetConst c;
    c.h = h;
    c.hinv = invharmonic_exact(h, h);
    c.kdw = wc2_kdw<D>(c.hinv);
    c.hh = __fdiv_rn(1.0f, c.hinv);
    const float h2 = harmonic2_exact(h, h);
    c.h2sq = __fmul_rn(h2, h2);
    return c;
}

// Geometry of a pair for the contribution functions.
struct PairGeo {
    float dx, dy, dz, dr2;
};

// ---------------------------------------------------------------------------------------------
// Continuity (search! action of main.jl:74-90) as a per-pair contribution.  GEN: any kernel of
// EPP_KERNEL_*; otherwise Wendland C2 from its cached closed form (the benchmark physics).
template <int D, bool FUSED, bool GEN = false>
struct CPCont {
    State s;
    DevPhys P;
    int* ncount;
    static constexpr int NC = 1;
    __device__ __forceinline__ bool wants(int) const { return true; }
    struct Self {
        float4 v;
        float rho;
    };
    // what the term reads of a neighbour: (vx, vy, vz, m) and V_j; in 2D V_j rides in the unused z
    // lane, so a record is 16 bytes (staged rows of the mask passes stay small)
    struct Nb3 {
        float4 v;
        float vol;
    };
    struct Nb2 {
        float4 v;   // (vx, vy, V, m)
    };
    using Nb = typename std::conditional<D == 2, Nb2, Nb3>::type;
    __device__ __forceinline__ static float vol_of(const Nb2& n) { return n.v.z; }
    __device__ __forceinline__ static float vol_of(const Nb3& n) { return n.vol; }
    __device__ __forceinline__ Self self(int i) const { return Self{s.vm[i], s.rho[i]}; }
    // Neighbour records go through the read-only path: no pass writes what it gathers.
    // V_j enters only the balanced (fluid-wall, wall-fluid) term: in 3D fluid-fluid pairs skip its
    // load (5% off the pass); in 2D, without the 3D software pipeline, the branch costs more than
    // the 4-byte gather saves
    __device__ __forceinline__ Nb fetch(int j, int ti, int tj) const {
        if constexpr (D == 2) {
            float4 v = __ldg(&s.vm[j]);
            v.z = __ldg(&s.vol[j]);
            return Nb{v};
        } else {
            return Nb{__ldg(&s.vm[j]), ti == P.fluid && tj == P.fluid ? 0.0f : __ldg(&s.vol[j])};
        }
    }
    __device__ __forceinline__ float4 term(const Self& me, const Nb& nb, int ti, int tj, float4 xj,
                                           const PairGeo& g, const TargetConst& tc) const {
        float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const bool ff = ti == P.fluid && tj == P.fluid;
        const bool fw = ti == P.fluid && tj == P.wall;
        const bool wf = ti == P.wall && tj == P.fluid;
        if (!(ff || fw || wf)) return out;
        // every operation rounded on its own (no contraction into fused multiply-adds), so the term
        // is the same bit for bit wherever a pass evaluates it
        const float r = sqrtf(g.dr2);
        float hinv, kdw, hh;
        pair_consts<D>(tc, xj.w, hinv, kdw, hh);
        const float dwr = pair_dwr<D, GEN>(P.kernel, __fmul_rn(r, hinv), hinv, kdw);
        if (dwr == 0.0f) return out;
        float vdx = __fmul_rn(g.dx, __fsub_rn(me.v.x, nb.v.x));
        vdx = __fadd_rn(vdx, __fmul_rn(g.dy, __fsub_rn(me.v.y, nb.v.y)));
        if (D == 3) vdx = __fadd_rn(vdx, __fmul_rn(g.dz, __fsub_rn(me.v.z, nb.v.z)));
        if (ff) out.x = __fmul_rn(__fmul_rn(nb.v.w, vdx), dwr);                              // iClassicContinuity!
        else out.x = __fmul_rn(__fmul_rn(__fmul_rn(me.rho, vol_of(nb)), vdx), dwr);         // iBalancedContinuity!
        return out;
    }
    __device__ __forceinline__ float4 contrib(int i, int j, int ti, int tj, float4 xi, float4 xj,
                                              const PairGeo& g, const TargetConst& tc) const {
        return term(self(i), fetch(j, ti, tj), ti, tj, xj, g, tc);
    }
    __device__ __forceinline__ void end(int i, int ti, float4 sum, int cnt) const {
        ncount[i] = cnt;
        const float rho_i = s.rho[i];
        const float drho = FUSED ? sum.x : s.drho[i] + sum.x;
        s.drho[i] = drho;
        if (ti == P.fluid || ti == P.wall) {
            const int inst = inst_of(s.tagm[i]);
            const float rho = __fadd_rn(rho_i, __fmul_rn(drho, P.dt_of(inst)));
            s.rp4[i] = make_rp4(rho, eos(P, inst, rho));
        } else {
            s.rp4[i] = make_rp4(rho_i, s.p[i]);
        }
    }
    __device__ __forceinline__ void end_idle(int i, int ti) const { end(i, ti, make_float4(0, 0, 0, 0), 0); }
};

// Count only (search! without an action).
template <int D>
struct CPCount {
    int* ncount;
    static constexpr int NC = 0;
    struct Self {};
    struct Nb {};
    __device__ __forceinline__ Self self(int) const { return Self{}; }
    __device__ __forceinline__ Nb fetch(int, int, int) const { return Nb{}; }
    __device__ __forceinline__ float4 term(const Self&, const Nb&, int, int, float4, const PairGeo&,
                                           const TargetConst&) const {
        return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    __device__ __forceinline__ bool wants(int) const { return true; }
    __device__ __forceinline__ float4 contrib(int, int, int, int, float4, float4, const PairGeo&,
                                              const TargetConst&) const {
        return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    __device__ __forceinline__ void end(int i, int, float4, int cnt) const { ncount[i] = cnt; }
    __device__ __forceinline__ void end_idle(int i, int) const { ncount[i] = 0; }
};

// interaction! test action: dVelocity += 1 per neighbour (ActionTest.jl:71-75).
template <int D>
struct CPCountDv {
    State s;
    static constexpr int NC = 0;
    struct Self {};
    struct Nb {};
    __device__ __forceinline__ Self self(int) const { return Self{}; }
    __device__ __forceinline__ Nb fetch(int, int, int) const { return Nb{}; }
    __device__ __forceinline__ float4 term(const Self&, const Nb&, int, int, float4, const PairGeo&,
                                           const TargetConst&) const {
        return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    __device__ __forceinline__ bool wants(int) const { return true; }
    __device__ __forceinline__ float4 contrib(int, int, int, int, float4, float4, const PairGeo&,
                                              const TargetConst&) const {
        return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    __device__ __forceinline__ void end(int i, int, float4, int cnt) const {
        float4 d = s.dv[i];
        d.x += (float)cnt;
        d.y += (float)cnt;
        if (D == 3) d.z += (float)cnt;
        s.dv[i] = d;
    }
    __device__ __forceinline__ void end_idle(int, int) const {}
};

// p_rho_2 of a pair from the two (rho, p, p/rho^2, 1/rho) records: iClassicPressure!,
// iBalancedPressure!, iDensityWeightedPressure! (Pressure.jl:24-83).
__device__ __forceinline__ float pressure_term(int form, float4 rpi, float4 rpj) {
    if (form == EPP_PRESSURE_CLASSIC) return rpi.z + rpj.z;
    if (form == EPP_PRESSURE_BALANCED) return (rpi.y + rpj.y) * rpi.w * rpj.w;
    return __fdiv_rn(2.0f * (rpi.y * rpi.x + rpj.y * rpj.x) * rpi.w * rpj.w, rpi.x + rpj.x);
}

// Momentum (interaction! of main.jl:107-118) as a per-pair contribution; FUSED adds the
// integrate + bin epilogue of the fused step.  GEN: any kernel and EPP_VISCOSITY_CLASSIC; otherwise
// Wendland C2 with artificial viscosity (the benchmark physics).
template <int D, bool FUSED, bool GEN = false>
struct CPMom {
    ActMomG<D, FUSED> m;   // state, physics, fused outputs, integrate_and_bin
    static constexpr int NC = 3;
    __device__ __forceinline__ bool wants(int ti) const { return ti == m.P.fluid; }
    struct Self {
        float4 v, rp;
        float c0;
        float gap;   // GEN with the tensile correction only
    };
    struct NbG {
        float4 v, rp;
        float gap;
    };
    struct NbP {   // the benchmark physics reads no gap
        float4 v, rp;
    };
    using Nb = typename std::conditional<GEN, NbG, NbP>::type;
    __device__ __forceinline__ float gap_of(int i) const {
        return GEN && m.P.tensile ? m.P.gap[m.s.id[i]] : 0.0f;
    }
    __device__ __forceinline__ Self self(int i) const {
        return Self{m.s.vm[i], m.s.rp4[i], m.P.c0_of(inst_of(m.s.tagm[i])), gap_of(i)};
    }
    __device__ __forceinline__ Nb fetch(int j, int, int) const {
        if constexpr (GEN) return Nb{__ldg(&m.s.vm[j]), __ldg(&m.s.rp4[j]), gap_of(j)};
        else return Nb{__ldg(&m.s.vm[j]), __ldg(&m.s.rp4[j])};
    }
    __device__ __forceinline__ float4 term(const Self& me, const Nb& nb, int ti, int tj, float4 xj,
                                           const PairGeo& g, const TargetConst& tc) const {
        float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const DevPhys& P = m.P;
        const bool ff = tj == P.fluid;
        const bool fw = tj == P.wall;
        if (!(ff || fw)) return out;
        const float r = sqrtf(g.dr2);
        float hinv, kdw, hh;
        pair_consts<D>(tc, xj.w, hinv, kdw, hh);
        const float dwr = pair_dwr<D, GEN>(P.kernel, r * hinv, hinv, kdw);
        if (dwr == 0.0f) return out;
        const float4 rpi = me.rp, rpj = nb.rp, vi = me.v, vj = nb.v;
        float p_rho_2;
        if constexpr (!GEN) {   // the dam break's pair: classic fluid-fluid, balanced fluid-wall
            p_rho_2 = ff ? rpi.z + rpj.z : (rpi.y + rpj.y) * rpi.w * rpj.w;
        } else {
            p_rho_2 = pressure_term(ff ? P.pff : P.pfw, rpi, rpj);
            if (P.tensile) {   // iPressureCorrection (Pressure.jl:10-22)
                const float w = kern_value<D>(P.kernel, r, hinv);
                const float w_gap = kern_value<D>(P.kernel, 0.5f * (me.gap + nb.gap), hinv);
                p_rho_2 += fabsf(p_rho_2) * __fdiv_rn(0.01f * w, w_gap);
            }
        }
        const float fp = p_rho_2 * (-vj.w * dwr);
        out.x = fp * g.dx;
        out.y = fp * g.dy;
        if (D == 3) out.z = fp * g.dz;
        if (GEN && P.visc == EPP_VISCOSITY_CLASSIC) {
            // iClassicViscosity! (Viscosity.jl:10-26): 2 mu m_j r dW / (rho_i rho_j (r^2 + 0.01 h^2))
            // times (u_i - u_j); r dW = r^2 (dW / r)
            const float az = g.dr2 + 0.01f * hh * hh;
            const float force = __fdividef(2.0f * P.mu * vj.w * g.dr2 * dwr * rpi.w * rpj.w, az);
            out.x += force * (vi.x - vj.x);
            out.y += force * (vi.y - vj.y);
            if (D == 3) out.z += force * (vi.z - vj.z);
            return out;
        }
        float vdx = g.dx * (vi.x - vj.x);
        vdx += g.dy * (vi.y - vj.y);
        if (D == 3) vdx += g.dz * (vi.z - vj.z);
        if (vdx < 0.0f) {
            const float rhob = 0.5f * (rpi.x + rpj.x);
            const float az = g.dr2 + 0.01f * hh * hh;
            const float phi = __fdividef(vdx, hinv * az);
            float force = __fdividef((-P.alpha * me.c0 + P.beta * phi) * phi, rhob);
            if (P.visc == EPP_VISCOSITY_REFERENCE) force *= (-vj.w * rpi.w * rpj.w) * dwr;
            else force *= -vj.w * dwr;
            out.x += force * g.dx;
            out.y += force * g.dy;
            if (D == 3) out.z += force * g.dz;
        }
        return out;
    }
    __device__ __forceinline__ float4 contrib(int i, int j, int ti, int tj, float4 xi, float4 xj,
                                              const PairGeo& g, const TargetConst& tc) const {
        return term(self(i), fetch(j, ti, tj), ti, tj, xj, g, tc);
    }
    __device__ __forceinline__ void end(int i, int ti, float4 sum, int) const {
        typename ActMomG<D, FUSED>::Acc a;
        a.du[0] = sum.x;
        a.du[1] = sum.y;
        a.du[2] = sum.z;
        m.end(i, ti, a);
    }
    __device__ __forceinline__ void end_idle(int i, int ti) const {
        if (FUSED) m.integrate_and_bin(i, ti, nullptr);
    }
};

// Kernel filter (iFilter of main.jl:128-134: iKernelFilter!, Filter.jl:10-23) over fluid-fluid
// pairs: the sums wv += W V_j and wv_rho += W m_j, added to the per-particle filter sums.
template <int D>
struct CPFilter {
    State s;
    DevPhys P;
    float* wv;
    float* wvr;
    static constexpr int NC = 2;
    __device__ __forceinline__ bool wants(int ti) const { return ti == P.fluid; }
    struct Self {};
    struct Nb {
        float vol, m;
    };
    __device__ __forceinline__ Self self(int) const { return Self{}; }
    __device__ __forceinline__ Nb fetch(int j, int, int) const { return Nb{s.vol[j], s.vm[j].w}; }
    __device__ __forceinline__ float4 term(const Self&, const Nb& nb, int, int tj, float4 xj, const PairGeo& g,
                                           const TargetConst& tc) const {
        float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (tj != P.fluid) return out;
        float hinv, kdw, hh;
        pair_consts<D>(tc, xj.w, hinv, kdw, hh);
        const float w = kern_value<D>(P.kernel, sqrtf(g.dr2), hinv);
        out.x = w * nb.vol;
        out.y = w * nb.m;
        return out;
    }
    __device__ __forceinline__ float4 contrib(int i, int j, int ti, int tj, float4, float4 xj, const PairGeo& g,
                                              const TargetConst& tc) const {
        return term(self(i), fetch(j, ti, tj), ti, tj, xj, g, tc);
    }
    __device__ __forceinline__ void end(int i, int, float4 sum, int) const {
        wv[i] += sum.x;
        wvr[i] += sum.y;
    }
    __device__ __forceinline__ void end_idle(int, int) const {}
};

// Wall pressure extrapolation over wall-fluid pairs (iExtrapolatePressure!, Pressure.jl:85-131):
// wv += W V_j and wv_p += W V_j (max(p_j, p0) + max(rho_j g.r_ij, p0)).  FUSED: inside epp_step,
// right after the density preview, so rho_j and p_j are the preview's (rp4) with V_j = m_j / rho_j,
// and each wall particle's thread finishes its own sums (sExtrapolatePressure!,
// Pressure.jl:133-150) into its preview record; only fluid records are read and only wall
// records are written, so the pass has no read-after-write hazard.  Otherwise the sums are added
// to wv / wvp for EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF.
template <int D, bool FUSED>
struct CPExtrap {
    State s;
    DevPhys P;
    float* wv;
    float* wvp;
    static constexpr int NC = 2;
    __device__ __forceinline__ bool wants(int ti) const { return ti == P.wall; }
    struct Self {};
    struct Nb {
        float rho, p, vol;
    };
    __device__ __forceinline__ Self self(int) const { return Self{}; }
    __device__ __forceinline__ Nb fetch(int j, int, int) const {
        if (FUSED) {
            const float4 rp = s.rp4[j];
            return Nb{rp.x, rp.y, __fdiv_rn(s.vm[j].w, rp.x)};
        }
        return Nb{s.rho[j], s.p[j], s.vol[j]};
    }
    __device__ __forceinline__ float4 term(const Self&, const Nb& nb, int, int tj, float4 xj, const PairGeo& g,
                                           const TargetConst& tc) const {
        float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (tj != P.fluid) return out;
        float hinv, kdw, hh;
        pair_consts<D>(tc, xj.w, hinv, kdw, hh);
        const float w = kern_value<D>(P.kernel, sqrtf(g.dr2), hinv);
        float g_dot_x = g.dx * P.g[0];
        g_dot_x += g.dy * P.g[1];
        if (D == 3) g_dot_x += g.dz * P.g[2];
        const float w_v = w * nb.vol;
        out.x = w_v;
        out.y = w_v * (fmaxf(nb.p, P.p0) + fmaxf(nb.rho * g_dot_x, P.p0));
        return out;
    }
    __device__ __forceinline__ float4 contrib(int i, int j, int ti, int tj, float4, float4 xj, const PairGeo& g,
                                              const TargetConst& tc) const {
        return term(self(i), fetch(j, ti, tj), ti, tj, xj, g, tc);
    }
    __device__ __forceinline__ void end(int i, int, float4 sum, int) const {
        if (FUSED) {
            const float p = sum.x > 0.0f ? __fdiv_rn(sum.y, sum.x) : P.p0;
            s.rp4[i] = make_rp4(s.rp4[i].x, p);
        } else {
            wv[i] += sum.x;
            wvp[i] += sum.y;
        }
    }
    __device__ __forceinline__ void end_idle(int, int) const {}
};

// Segmented inclusive scan over runs of equal key (keys are non-decreasing across lanes).
__device__ __forceinline__ float seg_scan(float v, int key, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float up = __shfl_up_sync(0xffffffffu, v, o);
        const int kup = __shfl_up_sync(0xffffffffu, key, o);
        if (lane >= o && kup == key) v += up;
    }
    return v;
}

template <int D, class Act>
__device__ __forceinline__ void cp_window(const CellArgs& CA, const Act& act, CPShared<D>& S,
                                          int qhead, int nq, int tbase, int lane) {
    const int e = lane < nq ? S.queue[(qhead + lane) & (kCPQueue - 1)] : -1;
    const int t = e >= 0 ? (e >> 16) : 0x7fffffff;
    float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (e >= 0 && Act::NC > 0) {
        const int k = e & 0xffff;
        const int i = tbase + t;
        const int j = S.cj[k];
        const float4 xj = S.cx[k];
        const int tj = S.ct[k];
        const float4 xi = CA.A.s.xh[i];
        const int ti = tag_of(CA.A.s.tagm[i]);
        PairGeo g;
        g.dx = __fsub_rn(xi.x, xj.x);
        g.dy = __fsub_rn(xi.y, xj.y);
        g.dz = D == 3 ? __fsub_rn(xi.z, xj.z) : 0.0f;
        g.dr2 = __fadd_rn(__fmul_rn(g.dx, g.dx), __fmul_rn(g.dy, g.dy));
        if (D == 3) g.dr2 = __fadd_rn(g.dr2, __fmul_rn(g.dz, g.dz));
        c = act.contrib(i, j, ti, tj, xi, xj, g, S.tc[t]);
    }
    if (Act::NC > 0) {
        const int key = t;
        const int knext = __shfl_down_sync(0xffffffffu, key, 1);
        const bool last = e >= 0 && (lane == 31 || knext != key);
        c.x = seg_scan(c.x, key, lane);
        if (Act::NC > 1) {
            c.y = seg_scan(c.y, key, lane);
            c.z = seg_scan(c.z, key, lane);
        }
        if (last) {
            float4 a = S.acc[t];
            a.x += c.x;
            if (Act::NC > 1) {
                a.y += c.y;
                a.z += c.z;
            }
            S.acc[t] = a;
        }
    }
    __syncwarp();
}

// The cell-pair kernel.  Persistent: warps stride over the occupied cells.  EPI (fused momentum):
// block 0 clears the scan state and the dead bin gets the integrate + bin epilogue.
template <int D, class Act, bool EPI>
__global__ void __launch_bounds__(kCPWarps * 32, 4) k_cellpair(CellArgs CA, Act act, unsigned long long* pairs,
                                                            unsigned long long* scan_state,
                                                            int n_scan_words) {
    extern __shared__ __align__(16) unsigned char cp_smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    CPShared<D>& S = reinterpret_cast<CPShared<D>*>(cp_smem)[warp];
    if (EPI && blockIdx.x == 0)
        for (int t = threadIdx.x; t < n_scan_words; t += blockDim.x) scan_state[t] = 0ull;
    const PairArgs& A = CA.A;
    const int n_occ = CA.meta[0];
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int nwarps = gridDim.x * kCPWarps;
    const int n0 = A.dom.n[0], n1 = A.dom.n[1];
    unsigned long long my_pairs = 0;
    unsigned st = 0;
    for (int oc = blockIdx.x * kCPWarps + warp; oc < n_occ; oc += nwarps) {
        const int c = CA.occ[oc];
        const int cs0 = max(A.start[c], 0);
        const int cs1 = min(A.start[c + 1], n_alive);
        const int cx = c % n0, cy = (c / n0) % n1, cz = c / (n0 * n1);   // 2D: cz = instance layer
        const int x0 = max(cx - 1, 0), x1 = min(cx + 1, n0 - 1);
        const int y0 = max(cy - 1, 0), y1 = min(cy + 1, n1 - 1);
        const int z0 = D == 3 ? max(cz - 1, 0) : cz, z1 = D == 3 ? min(cz + 1, A.dom.n[2] - 1) : cz;
        for (int tb = cs0; tb < cs1; tb += CPConf<D>::T) {
            const int TB = min(CPConf<D>::T, cs1 - tb);
            for (int t = lane; t < TB; t += 32) {
                S.acc[t] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                S.cnt[t] = 0;
                S.tc[t] = target_const<D>(A.s.xh[tb + t].w);
            }
            __syncwarp();
            int qhead = 0, qtail = 0;
            int KC = 0;
            // rows of the stencil, staged chunk by chunk
            int zz = z0, yy = y0;
            int pos = max(A.start[n0 * (yy + n1 * zz) + x0], 0);
            int hi = min(A.start[n0 * (yy + n1 * zz) + x1 + 1], A.n_max);
            bool rows_left = true;
            while (rows_left) {
                // fill the chunk
                while (rows_left && KC < CPConf<D>::C) {
                    const int piece = max(0, min(hi - pos, CPConf<D>::C - KC));
                    for (int k = lane; k < piece; k += 32) {
                        const int j = pos + k;
                        S.cj[KC + k] = j;
                        S.cx[KC + k] = A.s.xh[j];
                        S.ct[KC + k] = tag_of(A.s.tagm[j]);
                    }
                    KC += piece;
                    pos += piece;
                    if (piece == 0 || pos >= hi) {
                        if (++yy > y1) {
                            yy = y0;
                            if (++zz > z1) rows_left = false;
                        }
                        if (rows_left) {
                            pos = max(A.start[n0 * (yy + n1 * zz) + x0], 0);
                            hi = min(A.start[n0 * (yy + n1 * zz) + x1 + 1], A.n_max);
                        }
                    }
                }
                __syncwarp();
                // filter every target of the batch against the chunk
                for (int t = 0; t < TB; ++t) {
                    const int i = tb + t;
                    const float4 xi = A.s.xh[i];
                    const int ti = tag_of(A.s.tagm[i]);
                    if (ti < 1 || ti > A.n_tags) {
                        st |= EPP_STATUS_BAD_TAG;
                        continue;
                    }
                    if (!act.wants(ti)) continue;
                    const unsigned amask = A.adj[ti - 1];
                    const float h2sq = S.tc[t].h2sq;
                    int added = 0;
                    for (int k0 = 0; k0 < KC; k0 += 32) {
                        const int k = k0 + lane;
                        bool ok = false;
                        if (k < KC) {
                            const int j = S.cj[k];
                            if (j != i) {
                                const float4 xj = S.cx[k];
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
                                    ok = dr2 <= h2sq;
                                } else {
                                    const float h2 = harmonic2_exact(xi.w, xj.w);
                                    ok = dr2 <= __fmul_rn(h2, h2);
                                }
                                if (ok) {
                                    const int tj = S.ct[k];
                                    if (tj < 1 || tj > A.n_tags) {
                                        st |= EPP_STATUS_BAD_TAG;
                                        ok = false;
                                    } else {
                                        ok = (amask >> (tj - 1)) & 1u;
                                    }
                                }
                            }
                        }
                        const unsigned mask = __ballot_sync(0xffffffffu, ok);
                        if (ok) {
                            const int slot = qtail + __popc(mask & ((1u << lane) - 1u));
                            S.queue[slot & (kCPQueue - 1)] = (t << 16) | k;
                        }
                        const int nadd = __popc(mask);
                        qtail += nadd;
                        added += nadd;
                        __syncwarp();
                        if (qtail - qhead >= 32) {
                            cp_window<D>(CA, act, S, qhead, 32, tb, lane);
                            qhead += 32;
                        }
                    }
                    if (lane == 0) S.cnt[t] += added;
                    my_pairs += added;
                }
                // the queue refers to this chunk's staging: drain it before the next chunk
                if (qtail > qhead) {
                    cp_window<D>(CA, act, S, qhead, qtail - qhead, tb, lane);
                    qhead = qtail;
                }
                KC = 0;
                __syncwarp();
            }
            // epilogue per target
            for (int t = lane; t < TB; t += 32) {
                const int i = tb + t;
                const int ti = tag_of(A.s.tagm[i]);
                if (ti >= 1 && ti <= A.n_tags && act.wants(ti)) act.end(i, ti, S.acc[t], S.cnt[t]);
                else act.end_idle(i, ti);
            }
            __syncwarp();
        }
    }
    if (EPI) {
        for (int i = n_alive + (blockIdx.x * kCPWarps + warp) * 32 + lane; i < A.n_max; i += nwarps * 32)
            act.end_idle(i, tag_of(A.s.tagm[i]));
    }
    if (st) atomicOr(A.status, st);
    if (pairs) {
        // my_pairs is warp-uniform (sum of ballot counts)
        if (lane == 0 && my_pairs) atomicAdd(pairs, my_pairs);
    }
}

}  // namespace epp
