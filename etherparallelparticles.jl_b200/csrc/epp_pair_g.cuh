// epp_pair_g.cuh -- the fast pair passes: G lanes per particle over the cell rows of the stencil.
//
// In cell-sorted order the three cells (x-1, x, x+1) of one stencil row are contiguous, so the
// 3^D stencil is 3 (2D) or 9 (3D) contiguous candidate ranges.  G consecutive lanes share one
// particle and stride through each range together, so every candidate load is a coalesced
// 16-byte vector load shared by the group, and the partial sums of the G lanes are combined by
// a fixed xor-shuffle tree (deterministic).  Neighbour sets are identical to the reference's
// (same IEEE criterion); the summation order differs from the reference's list order, which
// changes FP32 sums at the rounding level only.
//
// Per-pair arithmetic avoids divisions: dW/dr / r is evaluated in closed form,
//   _gradient(r, hinv) / r = -sigma * 0.625 * hinv^(N+2) * (2 - q)^3      (WendlandC2.jl:38-49)
// and p/rho^2, 1/rho are precomputed once per particle (rp4).
#pragma once
#include "epp_pair.cuh"

namespace epp {

template <int D>
__device__ __forceinline__ float wc2_kdw(float hinv) {   // -sigma * 0.625 * hinv^(D+2)
    float h2 = hinv * hinv;
    float hp = D == 2 ? h2 * h2 : h2 * h2 * hinv;
    return -wc2_sigma<D>() * 0.625f * hp;
}

// Per-particle constants of the pair terms for h_j == h_i (bit-identical to the pair formula).
struct HConst {
    float h, hinv, hh, kdw, h2;
    __device__ __forceinline__ void init(float hi, int D) {
        h = hi;
        hinv = invharmonic_exact(hi, hi);
        hh = __fdiv_rn(1.0f, hinv);
        kdw = D == 2 ? wc2_kdw<2>(hinv) : wc2_kdw<3>(hinv);
        h2 = harmonic2_exact(hi, hi);
    }
};

template <int D, int G, class Act>
__device__ __forceinline__ void traverse_rows(const PairArgs& A, int i, float4 xi, int ti, int g,
                                              const Act& act, typename Act::Acc& acc) {
    const int c = A.s.cell[i];
    const int n0 = A.dom.n[0], n1 = A.dom.n[1];
    const int cx = c % n0;
    const int cy = (c / n0) % n1;
    const int cz = c / (n0 * n1);   // 2D: the instance layer (no coupling across it)
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, n0 - 1);
    const int y0 = max(cy - 1, 0), y1 = min(cy + 1, n1 - 1);
    const int z0 = D == 3 ? max(cz - 1, 0) : cz, z1 = D == 3 ? min(cz + 1, A.dom.n[2] - 1) : cz;
    const unsigned amask = A.adj[ti - 1];
    const float h2ii = acc.hc.h2;
    unsigned st = 0;
    for (int zz = z0; zz <= z1; ++zz) {
        for (int yy = y0; yy <= y1; ++yy) {
            const int base = n0 * (yy + n1 * zz);
            const int lo = max(A.start[base + x0], 0);
            const int hi = min(A.start[base + x1 + 1], A.n_max);
            for (int j = lo + g; j < hi; j += G) {
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
    if (st) atomicOr(A.status, st);
}

template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <int G>
__device__ __forceinline__ int group_sum(int v) {
#pragma unroll
    for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------------------------------
// search! with the dam-break continuity (or the count only): main.jl:74-90.
template <int D, bool CONT, bool FUSED>
struct ActContG {
    State s;
    DevPhys P;
    int* ncount;
    struct Acc {
        int cnt;
        float drho, rho_i;
        float4 vi;
        HConst hc;
    };
    __device__ __forceinline__ bool wants(int) const { return true; }
    __device__ __forceinline__ void begin(int i, int ti, float4 xi, Acc& a) const {
        a.cnt = 0;
        a.drho = 0.0f;
        a.hc.init(xi.w, D);
        if (CONT) {
            a.rho_i = s.rho[i];
            a.vi = s.vm[i];
        }
    }
    __device__ __forceinline__ void pair(int i, int j, int ti, int tj, float4 xi, float4 xj,
                                         float dx, float dy, float dz, float dr2, Acc& a) const {
        a.cnt += 1;
        if (!CONT) return;
        const bool ff = ti == P.fluid && tj == P.fluid;
        const bool fw = ti == P.fluid && tj == P.wall;
        const bool wf = ti == P.wall && tj == P.fluid;
        if (!(ff || fw || wf)) return;
        const float r = sqrtf(dr2);
        float hinv, kdw;
        if (xj.w == a.hc.h) {
            hinv = a.hc.hinv;
            kdw = a.hc.kdw;
        } else {
            hinv = invharmonic_exact(a.hc.h, xj.w);
            kdw = wc2_kdw<D>(hinv);
        }
        const float q = r * hinv;
        if (!(q < 2.0f)) return;   // W = dW = 0 (WendlandC2.jl:23,44): the term is zero
        const float u = 2.0f - q;
        const float dwr = kdw * (u * u * u);
        const float4 vj = s.vm[j];
        float vdx = dx * (a.vi.x - vj.x);
        vdx += dy * (a.vi.y - vj.y);
        if (D == 3) vdx += dz * (a.vi.z - vj.z);
        if (ff) a.drho += vj.w * vdx * dwr;                    // iClassicContinuity!
        else a.drho += a.rho_i * s.vol[j] * vdx * dwr;         // iBalancedContinuity!
    }
    template <int G>
    __device__ __forceinline__ void reduce(Acc& a) const {
        a.cnt = group_sum<G>(a.cnt);
        if (CONT) a.drho = group_sum<G>(a.drho);
    }
    __device__ __forceinline__ void end(int i, int ti, Acc& a) const {
        ncount[i] = a.cnt;
        if (!CONT) return;
        const float drho = FUSED ? a.drho : s.drho[i] + a.drho;
        s.drho[i] = drho;
        // density preview (sContinuity! of the next step, Continuity.jl:10-21, + eos)
        if (ti == P.fluid || ti == P.wall) {
            const int inst = inst_of(s.tagm[i]);
            const float rho = __fadd_rn(a.rho_i, __fmul_rn(drho, P.dt_of(inst)));
            s.rp4[i] = make_rp4(rho, eos(P, inst, rho));
        } else {
            s.rp4[i] = make_rp4(a.rho_i, s.p[i]);
        }
    }
    __device__ __forceinline__ int count(const Acc& a) const { return a.cnt; }
    __device__ __forceinline__ void zero(Acc& a) const {
        a.cnt = 0;
        a.drho = 0.0f;
        a.hc.h = a.hc.hinv = a.hc.hh = a.hc.kdw = a.hc.h2 = 0.0f;
    }
};

// ------------------------------------------------------------------------------------------
// interaction! with the dam-break momentum (main.jl:107-118: iClassicPressure! / iBalancedPressure!
// + sArtificialViscosity!).  Reads (rho, p, p/rho^2, 1/rho) from rp4.  FUSED: the epilogue
// integrates and bins (see ActMomentum::integrate_and_bin); otherwise du is added to dVelocity.
template <int D, bool FUSED>
struct ActMomG {
    State s;
    DevPhys P;
    DevDomain dom;
    FusedOut F;
    unsigned* status;
    struct Acc {
        float du[3];
        float4 rpi;
        float4 vi;
        HConst hc;
        float c0;
    };
    __device__ __forceinline__ bool wants(int ti) const { return ti == P.fluid; }
    __device__ __forceinline__ void begin(int i, int ti, float4 xi, Acc& a) const {
        a.du[0] = a.du[1] = a.du[2] = 0.0f;
        if (ti == P.fluid) {
            a.rpi = s.rp4[i];
            a.vi = s.vm[i];
            a.hc.init(xi.w, D);
            a.c0 = P.c0_of(inst_of(s.tagm[i]));
        }
    }
    __device__ __forceinline__ void pair(int i, int j, int ti, int tj, float4 xi, float4 xj,
                                         float dx, float dy, float dz, float dr2, Acc& a) const {
        const bool ff = tj == P.fluid;
        const bool fw = tj == P.wall;
        if (!(ff || fw)) return;
        const float r = sqrtf(dr2);
        float hinv, kdw, hh;
        if (xj.w == a.hc.h) {
            hinv = a.hc.hinv;
            kdw = a.hc.kdw;
            hh = a.hc.hh;
        } else {
            hinv = invharmonic_exact(a.hc.h, xj.w);
            kdw = wc2_kdw<D>(hinv);
            hh = __fdividef(1.0f, hinv);
        }
        const float q = r * hinv;
        if (!(q < 2.0f)) return;
        const float u = 2.0f - q;
        const float dwr = kdw * (u * u * u);      // dW/dr / r
        const float4 vj = s.vm[j];
        const float4 rpj = s.rp4[j];
        const float p_rho_2 = ff ? a.rpi.z + rpj.z                        // iClassicPressure!
                                 : (a.rpi.y + rpj.y) * a.rpi.w * rpj.w;    // iBalancedPressure!
        const float fp = p_rho_2 * (-vj.w * dwr);
        a.du[0] += fp * dx;
        a.du[1] += fp * dy;
        if (D == 3) a.du[2] += fp * dz;
        float vdx = dx * (a.vi.x - vj.x);
        vdx += dy * (a.vi.y - vj.y);
        if (D == 3) vdx += dz * (a.vi.z - vj.z);
        if (vdx < 0.0f) {                          // sArtificialViscosity!: approaching pairs only
            const float rhob = 0.5f * (a.rpi.x + rpj.x);
            const float az = dr2 + 0.01f * hh * hh;
            const float phi = __fdividef(vdx, hinv * az);
            float force = __fdividef((-P.alpha * a.c0 + P.beta * phi) * phi, rhob);
            if (P.visc == EPP_VISCOSITY_REFERENCE) force *= (-vj.w * a.rpi.w * rpj.w) * dwr;
            else force *= -vj.w * dwr;
            a.du[0] += force * dx;
            a.du[1] += force * dy;
            if (D == 3) a.du[2] += force * dz;
        }
    }
    template <int G>
    __device__ __forceinline__ void reduce(Acc& a) const {
        a.du[0] = group_sum<G>(a.du[0]);
        a.du[1] = group_sum<G>(a.du[1]);
        if (D == 3) a.du[2] = group_sum<G>(a.du[2]);
    }
    __device__ __forceinline__ void end(int i, int ti, Acc& a) const {
        if (!FUSED) {
            if (ti == P.fluid) {
                float4 d = s.dv[i];
                d.x += a.du[0];
                d.y += a.du[1];
                d.z += a.du[2];
                s.dv[i] = d;
            }
            return;
        }
        integrate_and_bin(i, ti, &a);
    }
    __device__ __forceinline__ int count(const Acc&) const { return 0; }
    __device__ __forceinline__ void zero(Acc& a) const { a.du[0] = a.du[1] = a.du[2] = 0.0f; }

    // sGravity! + sAccelerate! + sMove! (Motion.jl:17-51) and the binning of the new position
    // (insertParticlesIntoCells!, NeighbourSearch.jl:26-45); a == nullptr: no force (not fluid,
    // or dead).
    __device__ __forceinline__ void integrate_and_bin(int i, int ti, const Acc* a) const {
        float4 x = s.xh[i];
        float4 v = s.vm[i];
        float4 cp = s.comp[i];
        const int tm = s.tagm[i];
        int c = s.cell[i];
        const bool alive = c != dom.n_cells;
        const float dt = P.dt_of(inst_of(tm));
        if (alive && ti == P.fluid && a) {
            float du[3] = {a->du[0], a->du[1], a->du[2]};
            float vv[3] = {v.x, v.y, v.z}, xx[3] = {x.x, x.y, x.z}, cc[3] = {cp.x, cp.y, cp.z};
#pragma unroll
            for (int k = 0; k < D; ++k) du[k] = __fadd_rn(du[k], P.g[k]);
            advance<D>(P, dt, du, vv, xx, cc);
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
        if (alive && (movable_of(tm) || c < 0)) {
            c = cell_of<D>(dom, x, inst_of(tm));
            if (c < 0) {
                c = dom.n_cells;
                atomicOr(status, EPP_STATUS_KILLED);
            }
        }
        const int slot = atomicAdd(&F.count[c], 1);
        F.cs[i] = make_int2(c, slot);
    }
};

// interaction! test action (ActionTest.jl:71-75): dVelocity += 1 per neighbour.
template <int D>
struct ActCountG {
    State s;
    struct Acc {
        int n;
        HConst hc;
    };
    __device__ __forceinline__ bool wants(int) const { return true; }
    __device__ __forceinline__ void begin(int, int, float4 xi, Acc& a) const {
        a.n = 0;
        a.hc.init(xi.w, D);
    }
    __device__ __forceinline__ void pair(int, int, int, int, float4, float4, float, float, float,
                                         float, Acc& a) const {
        a.n += 1;
    }
    template <int G>
    __device__ __forceinline__ void reduce(Acc& a) const {
        a.n = group_sum<G>(a.n);
    }
    __device__ __forceinline__ void end(int i, int, Acc& a) const {
        float4 d = s.dv[i];
        d.x += (float)a.n;
        d.y += (float)a.n;
        if (D == 3) d.z += (float)a.n;
        s.dv[i] = d;
    }
    __device__ __forceinline__ int count(const Acc&) const { return 0; }
    __device__ __forceinline__ void zero(Acc& a) const {
        a.n = 0;
        a.hc.h = a.hc.hinv = a.hc.hh = a.hc.kdw = a.hc.h2 = 0.0f;
    }
};

// epilogue of a particle that had no force (non-fluid or dead); only the fused momentum has one
template <class Act>
__device__ __forceinline__ void act_epilogue_nf(const Act&, int, int) {}
template <int D>
__device__ __forceinline__ void act_epilogue_nf(const ActMomG<D, true>& act, int i, int ti) {
    act.integrate_and_bin(i, ti, nullptr);
}

// One pair pass, G lanes per particle.  With FUSED_EPI (momentum of the fused step) the grid
// covers every particle and lane 0 of each group runs the integrate + bin epilogue, also for the
// dead bin; block 0 clears the scan's look-back state.
template <int D, int G, class Act, bool FUSED_EPI>
__global__ void __launch_bounds__(128) k_pair_g(PairArgs A, Act act, unsigned long long* pairs,
                                                unsigned long long* scan_state, int n_scan_words) {
    if (FUSED_EPI && blockIdx.x == 0)
        for (int t = threadIdx.x; t < n_scan_words; t += blockDim.x) scan_state[t] = 0ull;
    const int n_alive = min(A.start[A.dom.n_cells], A.n_max);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t / G;
    const int g = threadIdx.x & (G - 1);
    const bool on = i < n_alive;
    typename Act::Acc acc;
    int ti = 0;
    bool go = false;
    if (on) {
        const float4 xi = A.s.xh[i];
        ti = tag_of(A.s.tagm[i]);
        act.begin(i, ti, xi, acc);
        const bool bad = ti < 1 || ti > A.n_tags;
        if (bad && g == 0) atomicOr(A.status, EPP_STATUS_BAD_TAG);
        go = !bad && act.wants(ti);
        if (go) traverse_rows<D, G>(A, i, xi, ti, g, act, acc);
    } else {
        act.zero(acc);
    }
    act.template reduce<G>(acc);
    if (g == 0) {
        if (on) {
            if (FUSED_EPI) {
                if (go) act.end(i, ti, acc);
                else act_epilogue_nf(act, i, ti);
            } else {
                act.end(i, ti, acc);
            }
        } else if (FUSED_EPI && i < A.n_max) {
            act_epilogue_nf(act, i, tag_of(A.s.tagm[i]));
        }
    }
    count_pairs(pairs, (on && g == 0) ? act.count(acc) : 0);
}

// rp4 from the current density and pressure (per-call momentum after a density selfaction!).
__global__ void k_prep_rp4(const int* start, int n_cells, int n_max, State s) {
    const int n_alive = min(start[n_cells], n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_alive) return;
    s.rp4[i] = make_rp4(s.rho[i], s.p[i]);
}

}  // namespace epp
