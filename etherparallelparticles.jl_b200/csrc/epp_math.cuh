// epp_math.cuh -- device-side state layout, constants and SPH formulas.
//
// Formulas follow the reference's Julia sources (paths relative to the EtherParallelParticles.jl
// root); the operation order is kept so that FP32 results agree with a literal evaluation:
//   Wendland C2           src/SPH/Kernel/WendlandC2.jl:10-49
//   power                 src/Math/OptimizedFunction.jl:10-42
//   Mean                  src/Math/Mean.jl:12-34
//   criteria              src/Algorithm/NeighbourSearch.jl:141-164 (IEEE, no contraction: exact)
//   cell arithmetic       src/Class/Domain/Domain2D.jl:110-137, AbstractDomain.jl:12-19 (exact)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/epp.h"

namespace epp {

constexpr int kMaxTags = EPP_MAX_TAGS;

// Domain in FP32 (as Domain2D{Int32, Float32}); n[a] cells per axis, x fastest.
struct DevDomain {
    int dim;
    int n[3];
    int n_cells;          // all instances
    int cells_per_inst;   // n[0] * n[1] * n[2]
    int n_inst;           // instances stacked as independent layers (2D only)
    float gap_square;
    float first[3], last[3], gap_inv[3];
};

// Per-instance constants of a batch (each instance has its own column height, so its own c0
// and time step).
struct InstPhys {
    float dt, c0, B, pad;
};

// Physics constants rounded to FP32 the way `parallel(x)` converts them (Parallel.jl:62-74).
// `ip` (batches only) overrides dt, c0 and B per instance.
struct DevPhys {
    float dt, rho0, c0, p0, B;
    float g[3];
    float alpha, beta, mu;
    int gamma, visc, fluid, wall, kahan;
    int kernel, eos, motion;   // EPP_KERNEL_*, EPP_EOS_*, EPP_MOTION_*
    int pff, pfw;              // EPP_PRESSURE_* of fluid-fluid and fluid-wall pairs (DEFAULT resolved)
    int tensile, wallp;        // iPressureCorrection on / off, EPP_WALL_PRESSURE_*
    const InstPhys* ip;
    const float* gap;          // Gap per caller row (indexed by State::id); tensile correction only
    __device__ __forceinline__ float dt_of(int inst) const { return ip ? ip[inst].dt : dt; }
    __device__ __forceinline__ float c0_of(int inst) const { return ip ? ip[inst].c0 : c0; }
    __device__ __forceinline__ float B_of(int inst) const { return ip ? ip[inst].B : B; }
};

// Cell-sorted particle state.  Positions and velocities carry h and m in their w lanes so that
// one 16-byte load gives what the neighbour filter (x, h) or the pair term (v, m) needs.
struct State {
    float4* xh;      // (x, y, z, h)      z = 0 in 2D
    float4* vm;      // (vx, vy, vz, m)
    float4* dv;      // dVelocity accumulator (interaction! / selfaction! calls)
    float4* comp;    // Kahan compensation of x
    float* rho;
    float* drho;
    float* vol;
    float* p;
    int* tagm;       // tag | movable << 8 | instance << 9
    int* id;         // 0-based row of the particle in the caller's matrices
    int* cell;       // 0-based cell (n_cells = dead bin)
    float4* rp4;     // (rho, p, p/rho^2, 1/rho) that the next momentum pass reads
};

struct NeighbourList {   // EPP_SEARCH_EMIT_LIST output, column-major [k * cap + i]
    int* idx;            // sorted index of the neighbour
    float* rvec;         // [(D*k + a) * cap + i]
    float* r;
    float* w;
    float* dw;
    float* hinv;
    int max_nb;
    int cap;
};

// tagm = tag | movable << 8 | instance << 9
// EPP_CHECKED builds: every index read from the cell offsets and lists is checked before
// the access; a bad one is recorded (site, index) in epp_check_slot and the access is skipped.
#ifdef EPP_CHECKED
__device__ int epp_check_slot[4];
#define EPP_CHECK(cond, site, idx)                                    \
    do {                                                              \
        if (!(cond)) {                                                \
            if (atomicCAS(&epp_check_slot[0], 0, (site)) == 0) {      \
                epp_check_slot[1] = (int)(idx);                       \
                epp_check_slot[2] = (int)(blockIdx.x);                \
                epp_check_slot[3] = (int)(threadIdx.x);               \
            }                                                         \
            return;                                                   \
        }                                                             \
    } while (0)
#else
#define EPP_CHECK(cond, site, idx) do {} while (0)
#endif

__host__ __device__ inline int tag_of(int tm) { return tm & 0xff; }
__host__ __device__ inline int movable_of(int tm) { return (tm >> 8) & 1; }
__host__ __device__ inline int inst_of(int tm) { return (int)((unsigned)tm >> 9); }
__host__ __device__ inline int make_tagm(int tag, int movable, int inst) {
    return (tag & 0xff) | ((movable != 0) << 8) | (inst << 9);
}

// power(x, Val(N)) of OptimizedFunction.jl:10-42, same association.
__device__ __forceinline__ float powi(float x, int n) {
    float t;
    switch (n) {
        case 0: return 1.0f;
        case 1: return x;
        case 2: return x * x;
        case 3: return x * x * x;
        case 4: t = x * x; return t * t;
        case 5: t = x * x; return t * t * x;
        case 6: t = x * x * x; return t * t;
        case 7: t = x * x * x; return t * t * x;
        case 8: t = x * x; t = t * t; return t * t;
        default: {
            float e = x;
            for (int i = 2; i <= n; ++i) e = e * x;
            return e;
        }
    }
}

// Division used by the physics terms.  The reference's pair functions use IEEE division; the
// fast form differs by at most 2 ulp and stays well inside the 1e-5 parity tolerance.
__device__ __forceinline__ float fdiv(float a, float b) {
#ifdef EPP_IEEE_DIV
    return __fdiv_rn(a, b);
#else
    return __fdividef(a, b);
#endif
}

// Mean.harmonic(a, b) * 2 with IEEE operations, as the symmetric criterion evaluates it.
__device__ __forceinline__ float harmonic2_exact(float a, float b) {
    return __fmul_rn(__fdiv_rn(__fmul_rn(__fmul_rn(2.0f, a), b), __fadd_rn(a, b)), 2.0f);
}
// Mean.invharmonic(a, b) = (a + b) / (2 a b), IEEE (it is cached per particle when h_i == h_j).
__device__ __forceinline__ float invharmonic_exact(float a, float b) {
    return __fdiv_rn(__fadd_rn(a, b), __fmul_rn(__fmul_rn(2.0f, a), b));
}

template <int D>
__device__ __forceinline__ float wc2_sigma() {
    return D == 2 ? 0.55704230082163f /* 7/(4 pi) */ : 0.41778172561623f /* 21/(16 pi) */;
}

// _value(r, hinv), WendlandC2.jl:17-28
template <int D>
__device__ __forceinline__ float wc2_value(float r, float hinv) {
    float q = r * hinv;
    if (q < 2.0f)
        return wc2_sigma<D>() * powi(2.0f - q, 4) * powi(hinv, D) * (1.0f + 2.0f * q) * 0.0625f;
    return 0.0f;
}

// _gradient(r, hinv), WendlandC2.jl:38-49
template <int D>
__device__ __forceinline__ float wc2_gradient(float r, float hinv) {
    float q = r * hinv;
    if (q < 2.0f) return -wc2_sigma<D>() * powi(hinv, D + 1) * 0.625f * q * powi(2.0f - q, 3);
    return 0.0f;
}

// Tait EOS: p = B ((rho / rho0)^gamma - 1) + p0 (the benchmark's, replacing main.jl:64), or the
// example's linear EOS p = c0^2 (rho - rho0) + p0 (main.jl:58,64; c0^2 rounded once).
__device__ __forceinline__ float eos(const DevPhys& P, int inst, float rho) {
    if (P.eos == EPP_EOS_LINEAR) {
        const float c0 = P.c0_of(inst);
        return __fadd_rn(__fmul_rn(__fmul_rn(c0, c0), __fsub_rn(rho, P.rho0)), P.p0);
    }
    return P.B_of(inst) * (powi(__fdiv_rn(rho, P.rho0), P.gamma) - 1.0f) + P.p0;
}

// One fluid particle's velocity and position update from du (gravity already added), IEEE in the
// reference's order.  EPP_MOTION_SYMPLECTIC: sAccelerate! then sMove! (Motion.jl:17-51),
// u += du dt, x += u dt.  EPP_MOTION_ACCELERATE_MOVE: sAccelerateMove! (Motion.jl:61-75),
// x += (u + du dt 0.5) dt with the old u, then u += du dt.  With P.kahan the position increment is
// added with compensated (Kahan) summation (new; no reference counterpart).
template <int D>
__device__ __forceinline__ void advance(const DevPhys& P, float dt, const float (&du)[3], float (&vv)[3],
                                        float (&xx)[3], float (&cc)[3]) {
#pragma unroll
    for (int k = 0; k < D; ++k) {
        float inc;
        if (P.motion == EPP_MOTION_ACCELERATE_MOVE) {
            inc = __fmul_rn(__fadd_rn(vv[k], __fmul_rn(__fmul_rn(du[k], dt), 0.5f)), dt);
            vv[k] = __fadd_rn(vv[k], __fmul_rn(du[k], dt));
        } else {
            vv[k] = __fadd_rn(vv[k], __fmul_rn(du[k], dt));
            inc = __fmul_rn(vv[k], dt);
        }
        if (P.kahan) {
            const float y = __fsub_rn(inc, cc[k]);
            const float t = __fadd_rn(xx[k], y);
            cc[k] = __fsub_rn(__fsub_rn(t, xx[k]), y);
            xx[k] = t;
        } else {
            xx[k] = __fadd_rn(xx[k], inc);
        }
    }
}

// (rho, p, p / rho^2, 1 / rho): what a momentum pass needs of a neighbour (Pressure.jl:24-60).
__device__ __forceinline__ float4 make_rp4(float rho, float p) {
    return make_float4(rho, p, __fdiv_rn(p, __fmul_rn(rho, rho)), __fdiv_rn(1.0f, rho));
}

// The cell grid of a domain, on the host, in FP32 as the Domain2D constructor computes it
// (Domain2D.jl:28-67): n_a = floor(span_a / gap) cells per axis, gap_a = span_a / n_a and
// gap_inv_a = 1 / gap_a.  `n_inst` copies of the grid are stacked as independent layers (batches).
// Returns EPP_ERR_INVALID_ARGUMENT for a non-positive or non-finite gap or extent (fewer than one
// cell on an axis) or more than 2^22 layers, and EPP_ERR_CAPACITY when all layers together hold
// more than `max_cells` (at most 2^30) cells; the count is checked after every axis, so the
// product cannot overflow, and a per-axis count is checked against 2^31 before the conversion
// to int.
inline int plan_domain(const epp_domain& in, int n_inst, long long max_cells, DevDomain& d) {
    const int D = in.dim;
    if (D != 2 && D != 3) return EPP_ERR_INVALID_ARGUMENT;
    if (n_inst < 1) n_inst = 1;
    if (n_inst > (1 << 22) || max_cells > (1ll << 30)) return EPP_ERR_INVALID_ARGUMENT;
    const float gap = in.gap;
    if (!(gap > 0.0f) || !(gap < 3.0e38f)) return EPP_ERR_INVALID_ARGUMENT;
    d.dim = D;
    d.gap_square = gap * gap;
    long long ncell = 1;
    for (int a = 0; a < 3; ++a) {
        d.n[a] = 1;
        d.first[a] = d.last[a] = 0.0f;
        d.gap_inv[a] = 1.0f;
    }
    for (int a = 0; a < D; ++a) {
        d.first[a] = in.first[a];
        d.last[a] = in.last[a];
        volatile float span = d.last[a] - d.first[a];
        volatile float q = span / gap;
        const float fq = floorf(q);
        if (!(fq >= 1.0f)) return EPP_ERR_INVALID_ARGUMENT;   // also NaN
        if (!(fq < 2147483648.0f)) return EPP_ERR_CAPACITY;
        const int na = (int)fq;
        d.n[a] = na;
        volatile float ga = span / (float)na;
        d.gap_inv[a] = 1.0f / ga;
        ncell *= na;   // <= 2^30 * 2^31 before the check below: no overflow
        if (ncell > max_cells) return EPP_ERR_CAPACITY;
    }
    if (ncell * n_inst > max_cells) return EPP_ERR_CAPACITY;   // <= 2^30 * 2^22
    d.cells_per_inst = (int)ncell;
    d.n_inst = n_inst;
    d.n_cells = (int)(ncell * n_inst);
    return EPP_OK;
}

// Cell of a position: indexCartesianFromPosition + indexCartesianToLinear (Domain2D.jl:92-137),
// 0-based.  Returns -1 when the position is outside the domain (the particle is then killed,
// NeighbourSearch.jl:41-43).
template <int D>
__device__ __forceinline__ int cell_of(const DevDomain& dom, float4 x, int inst) {
    float xs[3] = {x.x, x.y, x.z};
#pragma unroll
    for (int a = 0; a < D; ++a)
        if (!(dom.first[a] <= xs[a] && xs[a] <= dom.last[a])) return -1;
    int lin = 0, stride = 1;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        float f = floorf(__fmul_rn(__fsub_rn(xs[a], dom.first[a]), dom.gap_inv[a]));
        int i = (int)f;   // unsafe_trunc(Int32, floor(.)), 0-based here
        i = min(dom.n[a] - 1, i);
        i = max(0, i);
        lin += i * stride;
        stride *= dom.n[a];
    }
    return lin + inst * dom.cells_per_inst;
}

}  // namespace epp
