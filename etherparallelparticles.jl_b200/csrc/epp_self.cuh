// epp_self.cuh -- per-particle passes: selfaction! actions, the fused-step gather, FP64
// integrals, and the pack/unpack kernels between the reference layout and the sorted state.
#pragma once
#include "epp_tile.cuh"

namespace epp {

// selfaction! (Action.jl:39-51) bodies.  Alive particles are the first start[n_cells] rows.
// DAMBREAK_DENSITY: sContinuity! wrapper of main.jl:92-105 (Continuity.jl:10-21, State.jl:10-19).
// DAMBREAK_INTEGRATE: sMomentum! of main.jl:120-126: sGravity!, then sAccelerate! + sMove! or
// sAccelerateMove! (Motion.jl:17-75) by P.motion.
// KERNEL_FILTER_SELF: sFilter of main.jl:136-144 (Filter.jl:25-38, State.jl:10-19).
template <int D>
__global__ void k_self(int action, const int* start, int n_cells, int n_max, State s, DevPhys P,
                       unsigned* status, float4* accel) {
    const int n_alive = min(start[n_cells], n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_alive) return;
    const int tm = s.tagm[i];
    const int ti = tag_of(tm);
    const int inst = inst_of(tm);
    const float dt = P.dt_of(inst);
    if (action == EPP_ACTION_ZERO_DVELOCITY) {
        s.dv[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else if (action == EPP_ACTION_DAMBREAK_DENSITY) {
        if (ti == P.fluid || ti == P.wall) {
            const float rho = __fadd_rn(s.rho[i], __fmul_rn(s.drho[i], dt));
            s.rho[i] = rho;
            s.drho[i] = 0.0f;
            s.vol[i] = __fdiv_rn(s.vm[i].w, rho);
            s.p[i] = eos(P, inst, rho);
            if (!isfinite(rho)) atomicOr(status, EPP_STATUS_NONFINITE);
        }
    } else if (action == EPP_ACTION_DAMBREAK_INTEGRATE) {
        if (ti == P.fluid) {
            float4 d = s.dv[i], v = s.vm[i], x = s.xh[i], c = s.comp[i];
            float du[3] = {d.x, d.y, d.z}, vv[3] = {v.x, v.y, v.z}, xx[3] = {x.x, x.y, x.z};
            float cc[3] = {c.x, c.y, c.z};
#pragma unroll
            for (int k = 0; k < D; ++k) du[k] = __fadd_rn(du[k], P.g[k]);
            advance<D>(P, dt, du, vv, xx, cc);
            if (accel) accel[i] = make_float4(du[0], du[1], du[2], 0.0f);
            s.dv[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            s.vm[i] = make_float4(vv[0], vv[1], vv[2], v.w);
            s.xh[i] = make_float4(xx[0], xx[1], xx[2], x.w);
            s.comp[i] = make_float4(cc[0], cc[1], cc[2], 0.0f);
            if (!(isfinite(vv[0]) && isfinite(vv[1]) && isfinite(vv[2])))
                atomicOr(status, EPP_STATUS_NONFINITE);
        }
    }
}

// sFilter (main.jl:136-144: sKernelFilter!, Filter.jl:25-38; sVolume!; eos) for the fluid:
// rho = (wv_rho + W0 m) / (wv + W0 V) with W0 = sigma (1/h)^N, the sums reset to zero, V = m / rho,
// p = eos(rho).  `preview`: also refresh the next fused step's density preview (rp4) of fluid and
// wall particles, which the filtered density changes.
template <int D>
__global__ void k_filter_finish(const int* start, int n_cells, int n_max, State s, DevPhys P, float* wv,
                                float* wvr, int preview) {
    const int n_alive = min(start[n_cells], n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_alive) return;
    const int tm = s.tagm[i];
    const int ti = tag_of(tm);
    const int inst = inst_of(tm);
    if (ti == P.fluid) {
        const float m = s.vm[i].w;
        const float w0 = kern_value0<D>(P.kernel, __fdiv_rn(1.0f, s.xh[i].w));
        const float a = __fadd_rn(wv[i], __fmul_rn(w0, s.vol[i]));
        const float b = __fadd_rn(wvr[i], __fmul_rn(w0, m));
        const float rho = __fdiv_rn(b, a);
        wv[i] = 0.0f;
        wvr[i] = 0.0f;
        s.rho[i] = rho;
        s.vol[i] = __fdiv_rn(m, rho);
        s.p[i] = eos(P, inst, rho);
    }
    if (preview && (ti == P.fluid || ti == P.wall)) {
        const float rn = __fadd_rn(s.rho[i], __fmul_rn(s.drho[i], P.dt_of(inst)));
        s.rp4[i] = make_rp4(rn, eos(P, inst, rn));
    }
}

// sExtrapolatePressure! (Pressure.jl:133-150) on wall particles: p = wv_p / wv and the sums
// cleared, or p = p0 when no fluid neighbour contributed.
__global__ void k_extrap_finish(const int* start, int n_cells, int n_max, State s, DevPhys P, float* wv,
                                float* wvp) {
    const int n_alive = min(start[n_cells], n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_alive || tag_of(s.tagm[i]) != P.wall) return;
    const float a = wv[i];
    if (a > 0.0f) {
        s.p[i] = __fdiv_rn(wvp[i], a);
        wv[i] = 0.0f;
        wvp[i] = 0.0f;
    } else {
        s.p[i] = P.p0;
    }
}

// Density preview used when the fused step starts from a state whose rpn is not current.
__global__ void k_density_preview(const int* start, int n_cells, int n_max, State s, DevPhys P) {
    const int n_alive = min(start[n_cells], n_max);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_alive) return;
    const int ti = tag_of(s.tagm[i]);
    if (ti == P.fluid || ti == P.wall) {
        const int inst = inst_of(s.tagm[i]);
        const float rho = __fadd_rn(s.rho[i], __fmul_rn(s.drho[i], P.dt_of(inst)));
        s.rp4[i] = make_rp4(rho, eos(P, inst, rho));
    } else {
        s.rp4[i] = make_rp4(s.rho[i], s.p[i]);
    }
}

// Gather of the fused step: positions / velocities / compensation from the momentum pass's
// output, density and pressure from the preview (what sContinuity! left), volume = m / rho.
// Particles that were dead before this step keep their stored values.
struct MoverFused {
    State a, b;
    FusedOut F;
    const int* start_old;
    int n_cells;
    int fluid, wall;
    __device__ __forceinline__ void operator()(int src, int dst, int c) const {
        const float4 vm = F.vm[src];
        b.xh[dst] = F.xh[src];
        b.vm[dst] = vm;
        b.comp[dst] = F.comp[src];
        const int tm = a.tagm[src];
        b.tagm[dst] = tm;
        b.id[dst] = a.id[src];
        b.cell[dst] = c;
        const int t = tag_of(tm);
        if (src < start_old[n_cells] && (t == fluid || t == wall)) {
            const float4 rp = a.rp4[src];
            b.rho[dst] = rp.x;
            b.p[dst] = rp.y;
            b.vol[dst] = __fdiv_rn(vm.w, rp.x);
        } else {
            b.rho[dst] = a.rho[src];
            b.p[dst] = a.p[src];
            b.vol[dst] = a.vol[src];
        }
    }
};

// FP64 integrals: per-block partials, the last block folds them in block order (deterministic).
struct IntegralsOut {
    double* partial;       // [n_blocks * 8]: the 6 results, min h and the pair count of each block
    double* result;        // [8]: mass_total, mass_fluid, kinetic, potential, internal, max|v|, min h,
                           //      directed pairs of the last search (sum of nCount, exact in FP64)
    unsigned* ticket;
};

// x^n for an integer n >= 0 in FP64 (binary exponentiation; the Tait exponent is an integer).
__device__ __forceinline__ double powi_d(double x, int n) {
    double r = 1.0;
    while (n > 0) {
        if (n & 1) r *= x;
        x *= x;
        n >>= 1;
    }
    return r;
}

// Internal energy per unit mass of the EOS, zero at rho0 (as the oracle): the integral of p / rho^2.
// Tait: (B / rho0) ((rho/rho0)^(gamma-1) / (gamma-1) + rho0/rho - gamma/(gamma-1)) + p0 (1/rho0 - 1/rho);
// linear: c0^2 (ln(rho/rho0) + rho0/rho - 1) + p0 (1/rho0 - 1/rho).
__device__ __forceinline__ double eos_energy(int eos_kind, double r, double rho0, double B, int gam, double p0,
                                             double c0) {
    if (eos_kind == EPP_EOS_LINEAR) return c0 * c0 * (log(r / rho0) + rho0 / r - 1.0) + p0 * (1.0 / rho0 - 1.0 / r);
    const double g1 = (double)(gam - 1);
    return (B / rho0) * (powi_d(r / rho0, gam - 1) / g1 + rho0 / r - (double)gam / g1) + p0 * (1.0 / rho0 - 1.0 / r);
}

template <int D>
__global__ void __launch_bounds__(256) k_integrals(const int* start, int n_cells, int n_max, State s,
                                                   const int* ncount, DevPhys P, double rho0, double c0,
                                                   int gam, double p0, double g0, double g1,
                                                   double g2, IntegralsOut O) {
    __shared__ double sh[8][256 / 32];
    __shared__ bool last;
    const int n_alive = min(start[n_cells], n_max);
    const double B = rho0 * c0 * c0 / (double)gam;
    // v: mass, fluid mass, kinetic, potential, internal, max |v| (max), min h (min), pairs
    double v[8] = {0, 0, 0, 0, 0, 0, 1e300, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_alive; i += gridDim.x * blockDim.x) {
        const float4 vm = s.vm[i];
        const double m = (double)vm.w;
        v[0] += m;
        v[7] += (double)ncount[i];
        if (tag_of(s.tagm[i]) != P.fluid) continue;
        const float4 xh = s.xh[i];
        v[1] += m;
        const double u2 = (double)vm.x * vm.x + (double)vm.y * vm.y + (D == 3 ? (double)vm.z * vm.z : 0.0);
        v[2] += 0.5 * m * u2;
        v[3] += -m * (g0 * xh.x + g1 * xh.y + (D == 3 ? g2 * xh.z : 0.0));
        v[4] += m * eos_energy(P.eos, (double)s.rho[i], rho0, B, gam, p0, c0);
        v[5] = fmax(v[5], sqrt(u2));
        v[6] = fmin(v[6], (double)xh.w);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto combine = [](int k, double a, double b) { return k == 5 ? fmax(a, b) : k == 6 ? fmin(a, b) : a + b; };
    auto block_reduce = [&](double (&x)[8]) {   // fixed tree: deterministic
#pragma unroll
        for (int k = 0; k < 8; ++k) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x[k] = combine(k, x[k], __shfl_down_sync(0xffffffffu, x[k], o));
            if (lane == 0) sh[k][warp] = x[k];
        }
        __syncthreads();
        if (threadIdx.x < 8) {
            const int k = threadIdx.x;
            double a = sh[k][0];
            for (int w = 1; w < 256 / 32; ++w) a = combine(k, a, sh[k][w]);
            x[k] = a;
        }
    };
    block_reduce(v);
    if (threadIdx.x < 8) O.partial[blockIdx.x * 8 + threadIdx.x] = v[threadIdx.x];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(O.ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last block combines the partials: thread t takes blocks t, t + 256, ... in order
    double w[8] = {0, 0, 0, 0, 0, 0, 1e300, 0};
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < 8; ++k) w[k] = combine(k, w[k], __ldcg(&O.partial[b * 8 + k]));
    block_reduce(w);
    if (threadIdx.x < 8) O.result[threadIdx.x] = w[threadIdx.x];
    if (threadIdx.x == 0) *O.ticket = 0;
}

// FP64 integrals of every instance of a batch: block k reduces instance k's particles, which are
// contiguous in cell order (cells of instance k are [k * cells_per_inst, (k + 1) * cells_per_inst)).
// out[k * 9 + ...] = mass_total, mass_fluid, kinetic, potential, internal, max|v|, h_min,
// n_alive, n_pairs (the last two as doubles).
template <int D>
__global__ void __launch_bounds__(256) k_integrals_inst(const int* start, DevDomain dom, int n_max, State s,
                                                        const int* ncount, DevPhys P, double rho0, int gam,
                                                        double p0, double g0, double g1, double g2, double* out) {
    __shared__ double sh[8][256 / 32];
    const int k = blockIdx.x;
    const int lo = max(start[k * dom.cells_per_inst], 0);
    const int hi = min(start[(k + 1) * dom.cells_per_inst], n_max);
    const double c0 = (double)P.c0_of(k);
    const double B = rho0 * c0 * c0 / (double)gam;
    double v[8] = {0, 0, 0, 0, 0, 0, 1e300, 0};
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const float4 vm = s.vm[i];
        const double m = (double)vm.w;
        v[0] += m;
        v[7] += (double)ncount[i];
        if (tag_of(s.tagm[i]) != P.fluid) continue;
        const float4 xh = s.xh[i];
        v[1] += m;
        const double u2 = (double)vm.x * vm.x + (double)vm.y * vm.y + (D == 3 ? (double)vm.z * vm.z : 0.0);
        v[2] += 0.5 * m * u2;
        v[3] += -m * (g0 * xh.x + g1 * xh.y + (D == 3 ? g2 * xh.z : 0.0));
        v[4] += m * eos_energy(P.eos, (double)s.rho[i], rho0, B, gam, p0, c0);
        v[5] = fmax(v[5], sqrt(u2));
        v[6] = fmin(v[6], (double)xh.w);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double t = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = q == 5 ? fmax(v[q], t) : (q == 6 ? fmin(v[q], t) : v[q] + t);
        }
        if (lane == 0) sh[q][warp] = v[q];
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        const int q = threadIdx.x;
        double a = sh[q][0];
        for (int w = 1; w < 256 / 32; ++w) a = q == 5 ? fmax(a, sh[q][w]) : (q == 6 ? fmin(a, sh[q][w]) : a + sh[q][w]);
        out[k * 9 + (q < 7 ? q : 8)] = a;
        if (q == 0) out[k * 9 + 7] = (double)(hi - lo);
    }
}

// CFL time step of every instance (new; the reference's dt is fixed, main.jl:68):
//   dt_k = (float)(cfl h_min / (c0_k + sqrt(max |v|^2)))
// with |v|^2 in FP64 from the FP32 components, max and h_min over the alive fluid particles of
// instance k.  Instance k's particles are the contiguous range [start[k cells], start[(k+1) cells])
// of the sorted order; block b reduces chunk b % chunks of instance b / chunks into partial[b],
// and the last block to finish combines the chunks of every instance (max and min do not depend
// on the order: the result is deterministic), writes next[k].dt, adds used[k].dt (the dt of the
// step just taken) to time[k] when `used` is set, and re-arms the ticket.  FUSED reads the
// momentum pass's output (velocities and positions of the new state, in the order of `start`;
// particles its bin killed are skipped); otherwise the sorted state itself.
struct CflArgs {
    const int* start;       // cell offsets of the order the arrays are in
    int cells_per_inst, n_inst, n_cells, n_max, chunks;
    const float4* vm;       // (vx, vy, vz, m)
    const float4* xh;       // (x, y, z, h)
    const int* tagm;
    const int2* cs;         // FUSED: (cell, slot) of the bin; cell n_cells = killed
    int fluid;
    float cfl;
    const InstPhys* used;   // dt of the step just taken (added to time), or null
    InstPhys* next;         // dt written here; c0 read here
    double2* partial;       // [n_inst * chunks]: (max |v|^2, min h)
    double* time;           // [n_inst]
    unsigned* ticket;
};

template <int D, bool FUSED>
__global__ void __launch_bounds__(256) k_cfl(const __grid_constant__ CflArgs A) {
    __shared__ double sh_v[256 / 32], sh_h[256 / 32];
    __shared__ bool last;
    const int k = blockIdx.x / A.chunks, chunk = blockIdx.x % A.chunks;
    const int lo = max(A.start[k * A.cells_per_inst], 0);
    const int hi = min(A.start[(k + 1) * A.cells_per_inst], A.n_max);
    double v2 = 0.0, hm = 1e300;
    for (int i = lo + chunk * blockDim.x + threadIdx.x; i < hi; i += A.chunks * blockDim.x) {
        if (tag_of(A.tagm[i]) != A.fluid) continue;
        if (FUSED && A.cs[i].x >= A.n_cells) continue;   // left the domain in this step
        const float4 v = A.vm[i];
        const double u2 = (double)v.x * v.x + (double)v.y * v.y + (D == 3 ? (double)v.z * v.z : 0.0);
        v2 = fmax(v2, u2);
        hm = fmin(hm, (double)A.xh[i].w);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v2 = fmax(v2, __shfl_down_sync(0xffffffffu, v2, o));
        hm = fmin(hm, __shfl_down_sync(0xffffffffu, hm, o));
    }
    if (lane == 0) {
        sh_v[warp] = v2;
        sh_h[warp] = hm;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 256 / 32; ++w) {
            v2 = fmax(v2, sh_v[w]);
            hm = fmin(hm, sh_h[w]);
        }
        A.partial[blockIdx.x] = make_double2(v2, hm);
        __threadfence();
        last = atomicAdd(A.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int q = threadIdx.x; q < A.n_inst; q += blockDim.x) {
        double vq = 0.0, hq = 1e300;
        for (int c = 0; c < A.chunks; ++c) {
            const double2 p = __ldcg(&A.partial[q * A.chunks + c]);
            vq = fmax(vq, p.x);
            hq = fmin(hq, p.y);
        }
        if (A.used) A.time[q] += (double)A.used[q].dt;
        if (hq < 1e300) A.next[q].dt = (float)((double)A.cfl * hq / ((double)A.next[q].c0 + sqrt(vq)));
    }
    if (threadIdx.x == 0) *A.ticket = 0;
}

// time[k] += table[k].dt: the simulated time of a step taken through the per-call kernels.
__global__ void k_advance_time(int n_inst, const InstPhys* table, double* time) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n_inst) time[k] += (double)table[k].dt;
}

// Staging columns (by particle row), used by upload and download:
//   float: position[D], velocity[D], dvelocity[D], mass, volume, density, ddensity, pressure, h
//   int:   tag, movable, ncount, alive, cell
enum { SF_POS = 0 };
__host__ __device__ inline int sf_vel(int D) { return D; }
__host__ __device__ inline int sf_dvel(int D) { return 2 * D; }
__host__ __device__ inline int sf_mass(int D) { return 3 * D; }
__host__ __device__ inline int sf_vol(int D) { return 3 * D + 1; }
__host__ __device__ inline int sf_rho(int D) { return 3 * D + 2; }
__host__ __device__ inline int sf_drho(int D) { return 3 * D + 3; }
__host__ __device__ inline int sf_p(int D) { return 3 * D + 4; }
__host__ __device__ inline int sf_h(int D) { return 3 * D + 5; }
__host__ __device__ inline int sf_count(int D) { return 3 * D + 6; }
enum { SI_TAG = 0, SI_MOV = 1, SI_NCOUNT = 2, SI_ALIVE = 3, SI_CELL = 4, SI_INST = 5, SI_COUNT = 6 };

// Rows of the caller's matrices -> state in row order (a search sorts it afterwards).
template <int D>
__global__ void k_unpack(int n, int n_cells, const float* sf, const int* si, State s, int* ncount) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    auto F = [&](int col) { return sf[(size_t)col * n + i]; };
    auto I = [&](int col) { return si[(size_t)col * n + i]; };
    s.xh[i] = make_float4(F(0), F(1), D == 3 ? F(2) : 0.0f, F(sf_h(D)));
    s.vm[i] = make_float4(F(sf_vel(D)), F(sf_vel(D) + 1), D == 3 ? F(sf_vel(D) + 2) : 0.0f, F(sf_mass(D)));
    s.dv[i] = make_float4(F(sf_dvel(D)), F(sf_dvel(D) + 1), D == 3 ? F(sf_dvel(D) + 2) : 0.0f, 0.0f);
    s.comp[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    s.rho[i] = F(sf_rho(D));
    s.drho[i] = F(sf_drho(D));
    s.vol[i] = F(sf_vol(D));
    s.p[i] = F(sf_p(D));
    s.tagm[i] = make_tagm(I(SI_TAG), I(SI_MOV), I(SI_INST));
    s.id[i] = i;
    const int cell1 = I(SI_CELL);
    s.cell[i] = I(SI_ALIVE) == 1 ? (cell1 >= 1 && cell1 <= n_cells ? cell1 - 1 : -1) : n_cells;
    ncount[i] = I(SI_NCOUNT);
}

// Sorted state -> staging columns by particle row.
template <int D>
__global__ void k_pack(int n, int n_cells, float* sf, int* si, State s, const int* ncount) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = s.id[k];
    auto F = [&](int col, float v) { sf[(size_t)col * n + i] = v; };
    auto I = [&](int col, int v) { si[(size_t)col * n + i] = v; };
    const float4 x = s.xh[k], v = s.vm[k], d = s.dv[k];
    F(0, x.x); F(1, x.y); if (D == 3) F(2, x.z);
    F(sf_vel(D), v.x); F(sf_vel(D) + 1, v.y); if (D == 3) F(sf_vel(D) + 2, v.z);
    F(sf_dvel(D), d.x); F(sf_dvel(D) + 1, d.y); if (D == 3) F(sf_dvel(D) + 2, d.z);
    F(sf_mass(D), v.w);
    F(sf_vol(D), s.vol[k]);
    F(sf_rho(D), s.rho[k]);
    F(sf_drho(D), s.drho[k]);
    F(sf_p(D), s.p[k]);
    F(sf_h(D), x.w);
    const int tm = s.tagm[k];
    I(SI_TAG, tag_of(tm));
    I(SI_MOV, movable_of(tm));
    I(SI_NCOUNT, ncount[k]);
    const int c = s.cell[k];
    const bool alive = c != n_cells;
    I(SI_ALIVE, alive ? 1 : 0);
    I(SI_CELL, alive && c >= 0 ? c + 1 : 0);
    I(SI_INST, inst_of(tm));
}

// Emitted neighbour lists -> reference columns by particle row: nIndex (1-based ids), nRVec,
// nR, nW, nDW, nHInv.  Staging blocks are [max_nb * n] (nRVec [D * max_nb * n]).
template <int D>
__global__ void k_pack_lists(int n, NeighbourList L, const int* sorted_id, const int* ncount,
                             int* nidx, float* nrvec, float* nr, float* nw, float* ndw,
                             float* nhinv) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = sorted_id[k];
    const int cnt = min(ncount[k], L.max_nb);
    for (int q = 0; q < L.max_nb; ++q) {
        const bool on = q < cnt;
        const size_t src = (size_t)q * L.cap + k;
        const size_t dst = (size_t)q * n + i;
        nidx[dst] = on ? sorted_id[L.idx[src]] + 1 : 0;
        nr[dst] = on ? L.r[src] : 0.0f;
        nw[dst] = on ? L.w[src] : 0.0f;
        ndw[dst] = on ? L.dw[src] : 0.0f;
        nhinv[dst] = on ? L.hinv[src] : 0.0f;
        for (int a = 0; a < D; ++a)
            nrvec[((size_t)D * q + a) * n + i] = on ? L.rvec[((size_t)D * q + a) * L.cap + k] : 0.0f;
    }
}

}  // namespace epp
