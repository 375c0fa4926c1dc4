/*
 * oracle.cpp -- CPU restatement of EtherParallelParticles.jl's SPH time step.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Compiled with -ffp-contract=off and without
 * -ffast-math so that every FP32 expression rounds exactly as written; the order of the
 * operations follows the Julia source that each function cites (Julia evaluates a * b * c
 * as (a * b) * c).  Paths are relative to the EtherParallelParticles.jl project root.
 *
 * Data layout (as the reference, src/Class/ParticleSystem/ParticleSystemBase.jl:12-18):
 *   int_properties_   column-major, columns Tag, IsMovable, nCount, nIndex[max_nb]
 *   float_properties_ column-major, columns Position[D], Velocity[D], dVelocity[D], Mass,
 *                     Volume, Density, dDensity, Pressure, Gap, H, nW, nDW, nHInv,
 *                     nRVec[D*max_nb], nR  (the layout of example/collapse_dry/same/casegen.jl:47-69)
 * Cell buckets (src/Class/NeighbourSystem/NeighbourSystemBase.jl:12-18): a count per cell and a
 * fixed-capacity list per cell, column-major (cell, slot).
 *
 * 3D has no reference implementation (src/Class/Domain/AbstractDomain.jl:117-119 is a TODO);
 * the 3D code here is the natural extension of the 2D code and is marked as such.
 */
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

/* ------------------------------------------------------------------------------------ */
/* Domain: src/Class/Domain/Domain2D.jl:28-67 (ctor), :92-137 (index math),              */
/* src/Class/Domain/AbstractDomain.jl:12-19 (device_floor)                               */
/* ------------------------------------------------------------------------------------ */
template <typename T>
struct Domain {
    int dim = 2;
    T gap = 1, gap_square = 1;
    int32_t n[3] = {1, 1, 1};
    int64_t n_cells = 1;
    T first[3] = {0, 0, 0}, last[3] = {0, 0, 0}, span[3] = {0, 0, 0};
    T gap_axis[3] = {1, 1, 1}, gap_inv[3] = {1, 1, 1};
};

template <typename T>
Domain<T> make_domain(const epp_domain& d) {
    Domain<T> o;
    o.dim = d.dim;
    o.gap = T(d.gap);
    o.gap_square = o.gap * o.gap;              // Domain2D.jl:36
    o.n_cells = 1;
    for (int a = 0; a < d.dim; ++a) {
        o.first[a] = T(d.first[a]);
        o.last[a] = T(d.last[a]);
        o.span[a] = o.last[a] - o.first[a];    // Domain2D.jl:41-42
        o.n[a] = (int32_t)std::floor(o.span[a] / o.gap);   // floor(IT, span / gap) :43-44
        o.gap_axis[a] = o.span[a] / T(o.n[a]);  // :46-47
        o.gap_inv[a] = T(1) / o.gap_axis[a];    // :48-49
        o.n_cells *= o.n[a];
    }
    return o;
}

/* indexCartesianFromPosition, Domain2D.jl:118-128: clamp(unsafe_trunc(floor((x-x0)*inv))+1) */
template <typename T>
inline int32_t axis_index(const Domain<T>& D, int a, T x) {
    T f = std::floor((x - D.first[a]) * D.gap_inv[a]);
    int32_t i = (int32_t)f + 1;
    i = std::min(D.n[a], i);
    i = std::max(int32_t(1), i);
    return i;
}

/* indexCartesianToLinear, Domain2D.jl:92-98 (1-based, x fastest); 3D extends it by k. */
template <typename T>
inline int32_t linear_index(const Domain<T>& D, int32_t i, int32_t j, int32_t k) {
    return i + D.n[0] * (j - 1) + D.n[0] * D.n[1] * (k - 1);
}

/* inside, Domain2D.jl:110-116 */
template <typename T>
inline bool inside(const Domain<T>& D, const T* x) {
    for (int a = 0; a < D.dim; ++a)
        if (!(D.first[a] <= x[a] && x[a] <= D.last[a])) return false;
    return true;
}

/* device_initializeNeighbourSystem!, NeighbourSystemBase.jl:28-48: di outer, dj inner.
 * 3D (no reference): di outer, dj, dk inner. */
void neighbour_cells(int dim, const int32_t* n, std::vector<int32_t>& count,
                     std::vector<int32_t>& list) {
    int64_t nc = (int64_t)n[0] * n[1] * (dim == 3 ? n[2] : 1);
    int stencil = dim == 3 ? 27 : 9;
    count.assign(nc, 0);
    list.assign(nc * stencil, 0);
    for (int64_t c = 0; c < nc; ++c) {
        int32_t I = (int32_t)c + 1;
        int32_t i = (I - 1) % n[0] + 1;                // mod1(index, n_x)  :100-108
        int32_t j = ((I - 1) / n[0]) % n[1] + 1;
        int32_t k = dim == 3 ? (int32_t)((I - 1) / ((int64_t)n[0] * n[1])) + 1 : 1;
        int dkmin = dim == 3 ? -1 : 0, dkmax = dim == 3 ? 1 : 0;
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
                for (int dk = dkmin; dk <= dkmax; ++dk) {
                    int32_t ii = i + di, jj = j + dj, kk = k + dk;
                    if (ii >= 1 && ii <= n[0] && jj >= 1 && jj <= n[1] &&
                        (dim == 2 || (kk >= 1 && kk <= n[2]))) {
                        int32_t id = ii + n[0] * (jj - 1) + n[0] * n[1] * (kk - 1);
                        list[c * stencil + count[c]] = id;
                        count[c] += 1;
                    }
                }
    }
}

/* ------------------------------------------------------------------------------------ */
/* Math: power (src/Math/OptimizedFunction.jl:10-42), Mean (src/Math/Mean.jl:12-34)      */
/* ------------------------------------------------------------------------------------ */
template <typename T>
inline T power(T x, int n) {
    T t;
    switch (n) {
        case 0: return T(1);
        case 1: return x;
        case 2: return x * x;
        case 3: return x * x * x;
        case 4: t = x * x; return t * t;
        case 5: t = x * x; return t * t * x;
        case 6: t = x * x * x; return t * t;
        case 7: t = x * x * x; return t * t * x;
        case 8: t = x * x; t = t * t; return t * t;
        default: {
            T e = x;
            for (int i = 2; i <= n; ++i) e = e * x;
            return e;
        }
    }
}
template <typename T> inline T harmonic(T a, T b) { return T(2) * a * b / (a + b); }      // :28-30
template <typename T> inline T invharmonic(T a, T b) { return (a + b) / (T(2) * a * b); } // :32-34
template <typename T> inline T arithmetic(T a, T b) { return T(0.5) * (a + b); }          // :12-14

/* Wendland C2, src/SPH/Kernel/WendlandC2.jl:10-57 */
template <typename T>
inline T wc2_sigma(int dim) {
    return dim == 2 ? T(7.0 / 4.0 / M_PI) : T(21.0 / 16.0 / M_PI);   // :14-15
}
template <typename T>
inline T wc2_value(T r, T hinv, int dim) {   // _value :17-28
    T q = r * hinv;
    if (q < T(2.0))
        return wc2_sigma<T>(dim) * power<T>(T(2) - q, 4) * power<T>(hinv, dim) *
               (T(1) + T(2) * q) * T(0.0625);
    return T(0.0);
}
template <typename T>
inline T wc2_gradient(T r, T hinv, int dim) {   // _gradient :38-49
    T q = r * hinv;
    if (q < T(2.0))
        return -wc2_sigma<T>(dim) * power<T>(hinv, dim + 1) * T(0.625) * q *
               power<T>(T(2) - q, 3);
    return T(0.0);
}

/* The other kernels of src/SPH/Kernel/: CubicSpline.jl, Gaussian.jl, WendlandC4.jl (sigma, _value,
 * _gradient), and _value0 = sigma hinv^N (Kernel.jl:16-22). */
template <typename T>
inline T kern_sigma(int kind, int dim) {
    switch (kind) {
        case EPP_KERNEL_CUBIC_SPLINE: return dim == 2 ? T(10.0 / 7.0 / M_PI) : T(1.0 / M_PI);
        case EPP_KERNEL_GAUSSIAN: return dim == 2 ? T(1.0 / M_PI) : T(1.0 / std::sqrt(M_PI * M_PI * M_PI));
        case EPP_KERNEL_WENDLAND_C4: return dim == 2 ? T(9.0 / 4.0 / M_PI) : T(495.0 / 256.0 / M_PI);
        default: return wc2_sigma<T>(dim);
    }
}
template <typename T>
inline T kern_value(int kind, T r, T hinv, int dim) {
    T q = r * hinv;
    switch (kind) {
        case EPP_KERNEL_CUBIC_SPLINE:
            if (q < T(1.0)) return kern_sigma<T>(kind, dim) * power<T>(hinv, dim) * (3 * q * q * (q - 2) + 4) * T(0.25);
            if (q < T(2.0)) return kern_sigma<T>(kind, dim) * power<T>(hinv, dim) * power<T>(T(2) - q, 3) * T(0.25);
            return T(0.0);
        case EPP_KERNEL_GAUSSIAN:
            return q < T(3.0) ? kern_sigma<T>(kind, dim) * power<T>(hinv, dim) * std::exp(-q * q) : T(0.0);
        case EPP_KERNEL_WENDLAND_C4:
            return q < T(2.0) ? kern_sigma<T>(kind, dim) * power<T>(hinv, dim) * power<T>(T(2) - q, 6) *
                                    (q * (35 * q + 36) + 12) * T(0.0013020833333333333)
                              : T(0.0);
        default: return wc2_value<T>(r, hinv, dim);
    }
}
template <typename T>
inline T kern_gradient(int kind, T r, T hinv, int dim) {
    T q = r * hinv;
    switch (kind) {
        case EPP_KERNEL_CUBIC_SPLINE:
            if (q < T(1.0)) return kern_sigma<T>(kind, dim) * power<T>(hinv, dim + 1) * q * (3 * q - 4) * T(0.75);
            if (q < T(2.0)) {
                T to_2 = T(2) - q;
                return -kern_sigma<T>(kind, dim) * power<T>(hinv, dim + 1) * to_2 * to_2 * T(0.75);
            }
            return T(0.0);
        case EPP_KERNEL_GAUSSIAN:
            return q < T(3.0) ? -2 * kern_sigma<T>(kind, dim) * power<T>(hinv, dim + 1) * q * std::exp(-q * q) : T(0.0);
        case EPP_KERNEL_WENDLAND_C4:
            return q < T(2.0) ? -kern_sigma<T>(kind, dim) * power<T>(hinv, dim + 1) * q *
                                    (T(0.3645833333333333) * q + T(0.14583333333333334)) * power<T>(T(2) - q, 5)
                              : T(0.0);
        default: return wc2_gradient<T>(r, hinv, dim);
    }
}
template <typename T>
inline T kern_value0(int kind, T hinv, int dim) { return kern_sigma<T>(kind, dim) * power<T>(hinv, dim); }

/* Physics constants converted to FT as `parallel(x)` does (src/Environment/Parallel.jl:62-74). */
template <typename T>
struct Phys {
    T dt, rho0, c0, p0, B, g[3], alpha, beta, coef, mu, c02;
    double cfl;   // 0: fixed dt; > 0: the CFL time step of each step's starting state
    int gamma, visc, fluid, wall, kahan, kernel, eos, motion, filter_interval;
    int pff, pfw, tensile, wallp;   // resolved EPP_PRESSURE_* per pair type, tensile flag, EPP_WALL_PRESSURE_*
};
template <typename T>
Phys<T> make_phys(const epp_physics& p) {
    Phys<T> o;
    o.dt = T(p.dt);
    o.cfl = (double)p.cfl;
    o.rho0 = T(p.rho0);
    o.c0 = T(p.c0);
    o.p0 = T(p.p0);
    /* Tait stiffness B = rho0 c0^2 / gamma, evaluated in double and rounded once. */
    o.B = T((double)p.rho0 * (double)p.c0 * (double)p.c0 / (double)p.gamma);
    for (int a = 0; a < 3; ++a) o.g[a] = T(p.gravity[a]);
    o.alpha = T(p.alpha);
    o.beta = T(p.beta);
    o.coef = T(0);
    o.gamma = p.gamma;
    o.visc = p.viscosity;
    o.fluid = p.fluid_tag;
    o.wall = p.wall_tag;
    o.kahan = p.kahan;
    o.kernel = p.kernel;
    o.eos = p.eos;
    o.mu = T(p.mu);
    o.c02 = o.c0 * o.c0;   // main.jl:58 const c02 = c0 * c0
    o.motion = p.motion;
    o.filter_interval = p.filter_interval;
    o.pff = p.pressure_ff == EPP_PRESSURE_DEFAULT ? EPP_PRESSURE_CLASSIC : p.pressure_ff;    // main.jl:109
    o.pfw = p.pressure_fw == EPP_PRESSURE_DEFAULT ? EPP_PRESSURE_BALANCED : p.pressure_fw;   // main.jl:113
    o.tensile = p.tensile;
    o.wallp = p.wall_pressure;
    return o;
}

/* Tait EOS (the benchmark cases replace the linear eos of main.jl:64):
 * p = B ((rho / rho0)^gamma - 1) + p0; or the example's linear eos p = c0^2 (rho - rho0) + p0 */
template <typename T>
inline T eos(const Phys<T>& P, T rho) {
    if (P.eos == EPP_EOS_LINEAR) return P.c02 * (rho - P.rho0) + P.p0;
    return P.B * (power<T>(rho / P.rho0, P.gamma) - T(1)) + P.p0;
}

/* ------------------------------------------------------------------------------------ */
/* System in the reference layout                                                        */
/* ------------------------------------------------------------------------------------ */
struct SysBase {
    virtual ~SysBase() {}
    int precision = 32;
    uint32_t status = 0;
    bool deterministic = true;
};

template <typename T>
struct System : SysBase {
    int D = 2;
    int n_cap = 0, n = 0, max_nb = 50, max_cell = 50;
    Domain<T> dom;
    int n_tags = 1;
    std::vector<int32_t> adj;
    /* base_ */
    std::vector<int32_t> alive, cell;
    /* int_properties_ columns */
    std::vector<int32_t> tag, movable, ncount, nindex;
    /* float_properties_ columns */
    std::vector<T> pos, vel, dvel, comp, accel, accel_abs, drho_abs;
    std::vector<T> mass, vol, rho, drho, p, gapc, h;
    std::vector<T> wv, wv_rho;   // kernel-filter sums (Filter.jl: SumWeight, SumWeightedDensity)
    std::vector<T> wv_p;         // SumWeightedPressure of the wall-pressure extrapolation (Pressure.jl:85-131)
    long long step_count = 0;    // steps since upload (main.jl:165 step += 1)
    double sim_time = 0.0;       // sum of the dt of the steps since upload
    std::vector<T> nw, ndw, nhinv, nr, nrvec;
    /* neighbour system */
    std::vector<int32_t> ccount, clist, nccount, nclist;
    std::vector<std::atomic<int32_t>> acount;
    bool searched = false;
    int last_criterion = EPP_CRITERION_DEFAULT;

    T& X(int a, int I) { return pos[(size_t)a * n_cap + I]; }
    T& U(int a, int I) { return vel[(size_t)a * n_cap + I]; }
    T& DU(int a, int I) { return dvel[(size_t)a * n_cap + I]; }
    T& RV(int ni, int a, int I) { return nrvec[((size_t)D * ni + a) * n_cap + I]; }
    int32_t& NIDX(int ni, int I) { return nindex[(size_t)ni * n_cap + I]; }
    T& NR(int ni, int I) { return nr[(size_t)ni * n_cap + I]; }
    T& NW(int ni, int I) { return nw[(size_t)ni * n_cap + I]; }
    T& NDW(int ni, int I) { return ndw[(size_t)ni * n_cap + I]; }
    T& NH(int ni, int I) { return nhinv[(size_t)ni * n_cap + I]; }

    bool active(int32_t ti, int32_t tj, uint32_t& st) {
        if (ti < 1 || ti > n_tags || tj < 1 || tj > n_tags) {
            st |= EPP_STATUS_BAD_TAG;
            return false;
        }
        return adj[(size_t)(ti - 1) * n_tags + (tj - 1)] == 1;
    }

    int init(const epp_config& c) {
        D = c.domain.dim;
        if (D != 2 && D != 3) return EPP_ERR_INVALID_ARGUMENT;
        n_cap = c.n_capacity;
        max_nb = c.max_neighbour_number > 0 ? c.max_neighbour_number : 50;
        max_cell = c.max_cell_particles > 0 ? c.max_cell_particles : 64;
        dom = make_domain<T>(c.domain);
        n_tags = c.n_tags;
        adj.assign((size_t)n_tags * n_tags, 0);
        for (int a = 0; a < n_tags; ++a)
            for (int b = 0; b < n_tags; ++b)
                adj[(size_t)a * n_tags + b] = c.adjacency[a * EPP_MAX_TAGS + b];
        size_t N = n_cap;
        alive.assign(N, 0); cell.assign(N, 0);
        tag.assign(N, 0); movable.assign(N, 0); ncount.assign(N, 0);
        nindex.assign(N * max_nb, 0);
        pos.assign(N * D, 0); vel.assign(N * D, 0); dvel.assign(N * D, 0);
        comp.assign(N * D, 0); accel.assign(N * D, 0); accel_abs.assign(N * D, 0);
        drho_abs.assign(N, 0);
        mass.assign(N, 0); vol.assign(N, 0); rho.assign(N, 0); drho.assign(N, 0);
        p.assign(N, 0); gapc.assign(N, 0); h.assign(N, 0);
        wv.assign(N, 0); wv_rho.assign(N, 0); wv_p.assign(N, 0);
        nw.assign(N * max_nb, 0); ndw.assign(N * max_nb, 0); nhinv.assign(N * max_nb, 0);
        nr.assign(N * max_nb, 0); nrvec.assign(N * max_nb * D, 0);
        ccount.assign(dom.n_cells, 0);
        clist.assign((size_t)dom.n_cells * max_cell, 0);
        acount = std::vector<std::atomic<int32_t>>(dom.n_cells);
        neighbour_cells(D, dom.n, nccount, nclist);
        return EPP_OK;
    }

    /* --- clean! + insertParticlesIntoCells!  NeighbourSystem.jl:43-54, NeighbourSearch.jl:12-47 */
    void insert_one(int I, int32_t c1, std::vector<int32_t>* slots) {
        int32_t slot;
        if (slots) slot = acount[c1 - 1].fetch_add(1, std::memory_order_relaxed);
        else slot = ccount[c1 - 1]++;
        if (slot < max_cell) clist[(size_t)(c1 - 1) + (size_t)dom.n_cells * slot] = I + 1;
        else status |= EPP_STATUS_CELL_OVERFLOW;   // the reference writes out of bounds here
    }
    int32_t bin(int I) {   // returns 1-based cell or 0 (killed)
        if (!movable[I] && cell[I] != 0) return cell[I];
        T x[3] = {X(0, I), X(1, I), D == 3 ? X(2, I) : T(0)};
        if (inside(dom, x)) {
            int32_t i = axis_index(dom, 0, x[0]);
            int32_t j = axis_index(dom, 1, x[1]);
            int32_t k = D == 3 ? axis_index(dom, 2, x[2]) : 1;
            cell[I] = linear_index(dom, i, j, k);
            return cell[I];
        }
        alive[I] = 0;
        cell[I] = 0;
        status |= EPP_STATUS_KILLED;
        return 0;
    }
    void insert() {
        std::fill(ccount.begin(), ccount.end(), 0);   // clean!
        if (deterministic) {
            for (int I = 0; I < n; ++I) {   // particle-id order stands in for atomic arrival
                if (alive[I] != 1) continue;
                int32_t c = bin(I);
                if (c) insert_one(I, c, nullptr);
            }
        } else {
            for (auto& a : acount) a.store(0, std::memory_order_relaxed);
            uint32_t st = 0;
#pragma omp parallel for schedule(static) reduction(| : st)
            for (int I = 0; I < n; ++I) {
                if (alive[I] != 1) continue;
                int32_t c;
                if (!movable[I] && cell[I] != 0) c = cell[I];
                else {
                    T x[3] = {X(0, I), X(1, I), D == 3 ? X(2, I) : T(0)};
                    if (inside(dom, x)) {
                        int32_t i = axis_index(dom, 0, x[0]);
                        int32_t j = axis_index(dom, 1, x[1]);
                        int32_t k = D == 3 ? axis_index(dom, 2, x[2]) : 1;
                        c = cell[I] = linear_index(dom, i, j, k);
                    } else {
                        alive[I] = 0; cell[I] = 0; st |= EPP_STATUS_KILLED; c = 0;
                    }
                }
                if (c) {
                    int32_t slot = acount[c - 1].fetch_add(1, std::memory_order_relaxed);
                    if (slot < max_cell) clist[(size_t)(c - 1) + (size_t)dom.n_cells * slot] = I + 1;
                    else st |= EPP_STATUS_CELL_OVERFLOW;
                }
            }
            status |= st;
            for (int64_t c = 0; c < dom.n_cells; ++c) ccount[c] = acount[c].load();
        }
    }

    /* --- criteria, NeighbourSearch.jl:141-164 */
    bool criterion(int crit, int I, int J, T dr2) {
        if (crit == EPP_CRITERION_DEFAULT) return dr2 <= dom.gap_square;
        T h2 = harmonic<T>(h[I], h[J]) * T(2);
        return dr2 <= h2 * h2;
    }

    /* --- findNeighbourParticlesFromCells!, NeighbourSearch.jl:166-227 */
    void find(int crit, int action, const Phys<T>& P) {
        uint32_t st = 0;
        int stencil = D == 3 ? 27 : 9;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : st)
        for (int I = 0; I < n; ++I) {
            if (alive[I] != 1) continue;
            int32_t cnt = 0;
            int32_t c = cell[I];
            int32_t ncells = nccount[c - 1];
            for (int ic = 0; ic < ncells; ++ic) {
                int32_t nc = nclist[(size_t)(c - 1) * stencil + ic];
                int32_t m = std::min(ccount[nc - 1], max_cell);
                for (int s = 0; s < m; ++s) {
                    int32_t J1 = clist[(size_t)(nc - 1) + (size_t)dom.n_cells * s];
                    int J = J1 - 1;
                    if (I == J) continue;
                    if (!active(tag[I], tag[J], st)) continue;
                    T d[3] = {T(0), T(0), T(0)};
                    for (int a = 0; a < D; ++a) d[a] = X(a, I) - X(a, J);
                    T dr2 = d[0] * d[0] + d[1] * d[1];
                    if (D == 3) dr2 = dr2 + d[2] * d[2];
                    if (!criterion(crit, I, J, dr2)) continue;
                    if (cnt >= max_nb) {   // the reference writes past the columns here
                        st |= EPP_STATUS_NEIGHBOUR_OVERFLOW;
                        continue;
                    }
                    NIDX(cnt, I) = J1;
                    for (int a = 0; a < D; ++a) RV(cnt, a, I) = d[a];
                    NR(cnt, I) = std::sqrt(dr2);
                    cnt += 1;
                }
            }
            ncount[I] = cnt;
            search_action(action, I, P);
        }
        status |= st;
        last_criterion = crit;
        searched = true;
    }

    T vdotx(int I, int ni, int J) {   // Library.jl:21-34
        T v = T(0.0);
        for (int a = 0; a < D; ++a) v += RV(ni, a, I) * (U(a, I) - U(a, J));
        return v;
    }

    /* sComputeKernelAndiContinuity!, main.jl:74-90, with iValueGradient! (SPH/Library/Kernel.jl:114-128),
     * iClassicContinuity! / iBalancedContinuity! (Continuity.jl:23-47) */
    void search_action(int action, int I, const Phys<T>& P) {
        if (action != EPP_ACTION_DAMBREAK_CONTINUITY) return;
        drho_abs[I] = T(0);
        for (int ni = 0; ni < ncount[I]; ++ni) {
            int J = NIDX(ni, I) - 1;
            bool ff = tag[I] == P.fluid && tag[J] == P.fluid;
            bool fw = tag[I] == P.fluid && tag[J] == P.wall;
            bool wf = tag[I] == P.wall && tag[J] == P.fluid;
            if (!(ff || fw || wf)) continue;
            T hinv = invharmonic<T>(h[I], h[J]);
            NH(ni, I) = hinv;
            NW(ni, I) = kern_value<T>(P.kernel, NR(ni, I), hinv, D);
            NDW(ni, I) = kern_gradient<T>(P.kernel, NR(ni, I), hinv, D);
            T dw = NDW(ni, I);
            T term;
            if (ff) term = mass[J] * vdotx(I, ni, J) * dw / NR(ni, I);
            else term = rho[I] * vol[J] * vdotx(I, ni, J) * dw / NR(ni, I);
            drho[I] += term;
            drho_abs[I] += std::fabs(term);
        }
    }

    /* --- interaction!, Action.jl:121-138 */
    int interaction(int action, const Phys<T>& P) {
        if (!searched) return EPP_ERR_STATE;
        if (action != EPP_ACTION_DAMBREAK_MOMENTUM && action != EPP_ACTION_COUNT_NEIGHBOURS &&
            action != EPP_ACTION_NONE && action != EPP_ACTION_KERNEL_FILTER &&
            action != EPP_ACTION_EXTRAPOLATE_PRESSURE)
            return EPP_ERR_UNSUPPORTED_ACTION;
#pragma omp parallel for schedule(dynamic, 256)
        for (int I = 0; I < n; ++I) {
            if (alive[I] != 1) continue;
            for (int a = 0; a < D; ++a) accel_abs[(size_t)a * n_cap + I] = T(0);
            for (int ni = 0; ni < ncount[I]; ++ni) {
                if (action == EPP_ACTION_COUNT_NEIGHBOURS) {
                    for (int a = 0; a < D; ++a) DU(a, I) += T(1.0);
                } else if (action == EPP_ACTION_DAMBREAK_MOMENTUM) {
                    momentum_pair(I, ni, P);
                } else if (action == EPP_ACTION_KERNEL_FILTER) {
                    /* iFilter, main.jl:128-134: iKernelFilter! (Filter.jl:10-23) on fluid-fluid pairs
                     * with the kernel value cached by the search */
                    int J = NIDX(ni, I) - 1;
                    if (tag[I] == P.fluid && tag[J] == P.fluid) {
                        wv[I] += NW(ni, I) * vol[J];
                        wv_rho[I] += NW(ni, I) * mass[J];
                    }
                } else if (action == EPP_ACTION_EXTRAPOLATE_PRESSURE) {
                    /* iExtrapolatePressure!, Pressure.jl:85-131, on wall-fluid pairs with the kernel
                     * value cached by the search; p0 and g of the physics */
                    int J = NIDX(ni, I) - 1;
                    if (tag[I] == P.wall && tag[J] == P.fluid) {
                        T g_dot_x = T(0.0);
                        for (int a = 0; a < D; ++a) g_dot_x += RV(ni, a, I) * P.g[a];
                        T w_v = NW(ni, I) * vol[J];
                        wv[I] += w_v;
                        wv_p[I] += w_v * (std::max(p[J], P.p0) + std::max(rho[J] * g_dot_x, P.p0));
                    }
                }
            }
        }
        return EPP_OK;
    }

    /* iMomentum!, main.jl:107-118, with the benchmark's artificial viscosity in place of
     * iClassicViscosity!: fluid-fluid iClassicPressure! (Pressure.jl:24-41), fluid-wall
     * iBalancedPressure! (:43-60), both followed by sArtificialViscosity! (Viscosity.jl:28-52). */
    void momentum_pair(int I, int ni, const Phys<T>& P) {
        int J = NIDX(ni, I) - 1;
        bool ff = tag[I] == P.fluid && tag[J] == P.fluid;
        bool fw = tag[I] == P.fluid && tag[J] == P.wall;
        if (!(ff || fw)) return;
        T dw = NDW(ni, I);
        T r = NR(ni, I);
        T p_rho_2;
        const int form = ff ? P.pff : P.pfw;
        if (form == EPP_PRESSURE_CLASSIC)   // iClassicPressure!, Pressure.jl:24-41
            p_rho_2 = p[I] / (rho[I] * rho[I]) + p[J] / (rho[J] * rho[J]);
        else if (form == EPP_PRESSURE_BALANCED)   // iBalancedPressure!, :43-60
            p_rho_2 = (p[I] + p[J]) / (rho[I] * rho[J]);
        else   // iDensityWeightedPressure!, :62-79
            p_rho_2 = 2 * (p[I] * rho[I] + p[J] * rho[J]) / ((rho[I] + rho[J]) * rho[I] * rho[J]);
        T coef = P.coef;
        if (P.tensile)   // iPressureCorrection, :10-22: 0.01 w / W(mean gap, hinv), w = W(r) of the pair
            coef = T(0.01) * kern_value<T>(P.kernel, r, NH(ni, I), D) /
                   kern_value<T>(P.kernel, arithmetic<T>(gapc[I], gapc[J]), NH(ni, I), D);
        p_rho_2 += std::fabs(p_rho_2) * coef;
        p_rho_2 *= -mass[J] * dw / r;
        for (int a = 0; a < D; ++a) {
            DU(a, I) += p_rho_2 * RV(ni, a, I);
            accel_abs[(size_t)a * n_cap + I] += std::fabs(p_rho_2 * RV(ni, a, I));
        }
        if (P.visc == EPP_VISCOSITY_CLASSIC) {
            /* iClassicViscosity!, Viscosity.jl:10-26 (the example's viscosity, main.jl:110,114) */
            T hinv = NH(ni, I);
            T hh = T(1) / hinv;
            T force = 2 * P.mu * mass[J] * r * dw / (rho[I] * rho[J] * (r * r + T(0.01) * hh * hh));
            for (int a = 0; a < D; ++a) {
                DU(a, I) += force * (U(a, I) - U(a, J));
                accel_abs[(size_t)a * n_cap + I] += std::fabs(force * (U(a, I) - U(a, J)));
            }
            return;
        }
        /* sArtificialViscosity! */
        T v_dot_x = vdotx(I, ni, J);
        if (v_dot_x > 0) return;
        T rhob = arithmetic<T>(rho[I], rho[J]);
        T hinv = NH(ni, I);
        T hh = T(1) / hinv;
        T az = r * r + T(0.01) * hh * hh;   // avoidzero, Library.jl:17-19
        T phi = v_dot_x / (hinv * az);
        T force = (-P.alpha * P.c0 + P.beta * phi) * phi / rhob;
        if (P.visc == EPP_VISCOSITY_REFERENCE) force *= -mass[J] / (rho[I] * rho[J] * r) * dw;
        else force *= -mass[J] / r * dw;
        for (int a = 0; a < D; ++a) {
            DU(a, I) += force * RV(ni, a, I);
            accel_abs[(size_t)a * n_cap + I] += std::fabs(force * RV(ni, a, I));
        }
    }

    /* --- selfaction!, Action.jl:39-51 */
    int selfaction(int action, const Phys<T>& P) {
        if (action == EPP_ACTION_NONE) return EPP_OK;
        if (action != EPP_ACTION_DAMBREAK_DENSITY && action != EPP_ACTION_DAMBREAK_INTEGRATE &&
            action != EPP_ACTION_ZERO_DVELOCITY && action != EPP_ACTION_KERNEL_FILTER_SELF &&
            action != EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF)
            return EPP_ERR_UNSUPPORTED_ACTION;
#pragma omp parallel for schedule(static)
        for (int I = 0; I < n; ++I) {
            if (alive[I] != 1) continue;
            if (action == EPP_ACTION_ZERO_DVELOCITY) {
                for (int a = 0; a < D; ++a) DU(a, I) = T(0.0);
            } else if (action == EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF) {
                /* sExtrapolatePressure!, Pressure.jl:133-150, on wall particles */
                if (tag[I] == P.wall) {
                    if (wv[I] > T(0.0)) {
                        p[I] = wv_p[I] / wv[I];
                        wv[I] = T(0.0);
                        wv_p[I] = T(0.0);
                    } else {
                        p[I] = P.p0;
                    }
                }
            } else if (action == EPP_ACTION_KERNEL_FILTER_SELF) {
                /* sFilter, main.jl:136-144: sKernelFilter! (Filter.jl:25-38), sVolume!, eos */
                if (tag[I] == P.fluid) {
                    T w0 = kern_value0<T>(P.kernel, T(1) / h[I], D);
                    wv[I] += w0 * vol[I];
                    wv_rho[I] += w0 * mass[I];
                    rho[I] = wv_rho[I] / wv[I];
                    wv[I] = T(0.0);
                    wv_rho[I] = T(0.0);
                    vol[I] = mass[I] / rho[I];
                    p[I] = eos(P, rho[I]);
                }
            } else if (action == EPP_ACTION_DAMBREAK_DENSITY) {
                /* sContinuity! wrapper, main.jl:92-105: Continuity.jl:10-21, State.jl:10-19 */
                if (tag[I] == P.fluid || tag[I] == P.wall) {
                    rho[I] += drho[I] * P.dt;
                    drho[I] = T(0.0);
                    vol[I] = mass[I] / rho[I];
                    p[I] = eos(P, rho[I]);
                }
            } else {
                /* sMomentum!, main.jl:120-126 with sAccelerate! + sMove! (Motion.jl:17-51) in
                 * place of sAccelerateMove!; sGravity! State.jl:35-62 */
                if (tag[I] == P.fluid) {
                    for (int a = 0; a < D; ++a) {
                        DU(a, I) += P.g[a];
                        accel_abs[(size_t)a * n_cap + I] += std::fabs(P.g[a]);
                    }
                    T dx[3];
                    for (int a = 0; a < D; ++a) {
                        accel[(size_t)a * n_cap + I] = DU(a, I);
                        if (P.motion == EPP_MOTION_ACCELERATE_MOVE) {
                            /* sAccelerateMove!, Motion.jl:61-75: x += (u + du dt / 2) dt with the
                             * old u, then u += du dt */
                            dx[a] = (U(a, I) + DU(a, I) * P.dt * T(0.5)) * P.dt;
                            U(a, I) += DU(a, I) * P.dt;
                        } else {
                            U(a, I) += DU(a, I) * P.dt;
                            dx[a] = U(a, I) * P.dt;
                        }
                        DU(a, I) = T(0.0);
                    }
                    for (int a = 0; a < D; ++a) {
                        if (P.kahan) {   // compensated summation (new; no reference counterpart)
                            T& c = comp[(size_t)a * n_cap + I];
                            T y = dx[a] - c;
                            T t = X(a, I) + y;
                            c = (t - X(a, I)) - y;
                            X(a, I) = t;
                        } else {
                            X(a, I) += dx[a];
                        }
                    }
                }
            }
        }
        return EPP_OK;
    }

    int search(int crit, int action, const Phys<T>& P) {
        if (crit != EPP_CRITERION_DEFAULT && crit != EPP_CRITERION_SYMMETRY)
            return EPP_ERR_UNSUPPORTED_CRITERION;
        if (action != EPP_ACTION_NONE && action != EPP_ACTION_DAMBREAK_CONTINUITY)
            return EPP_ERR_UNSUPPORTED_ACTION;
        insert();
        find(crit, action, P);
        return EPP_OK;
    }

    /* CFL time step of the current state (new; the reference's dt is fixed, main.jl:68):
     * cfl h_min / (c0 + max|v|) over the alive fluid particles, |v|^2 summed in FP64 from the
     * stored components, h_min the smallest H, rounded once to FT.  Without fluid: P.dt. */
    T cfl_dt(const Phys<T>& P) const {
        double v2max = 0.0, hmin = 1e300;
        for (int I = 0; I < n; ++I) {
            if (alive[I] != 1 || tag[I] != P.fluid) continue;
            double v2 = 0.0;
            for (int a = 0; a < D; ++a) {
                const double u = (double)vel[(size_t)a * n_cap + I];
                v2 += u * u;
            }
            v2max = std::max(v2max, v2);
            hmin = std::min(hmin, (double)h[I]);
        }
        if (!(hmin < 1e300)) return P.dt;
        return T(P.cfl * hmin / ((double)P.c0 + std::sqrt(v2max)));
    }

    /* main.jl:166-182; with P.cfl > 0 each step takes the CFL dt of the state it starts from */
    int step(int nsteps, const Phys<T>& P0) {
        if (!searched) return EPP_ERR_STATE;
        for (int s = 0; s < nsteps; ++s) {
            Phys<T> P = P0;
            if (P0.cfl > 0.0) P.dt = cfl_dt(P0);
            sim_time += (double)P.dt;
            ++step_count;
            selfaction(EPP_ACTION_DAMBREAK_DENSITY, P);
            if (P.wallp == EPP_WALL_PRESSURE_EXTRAPOLATE) {   // wall pressure from the fluid around it
                interaction(EPP_ACTION_EXTRAPOLATE_PRESSURE, P);
                selfaction(EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF, P);
            }
            interaction(EPP_ACTION_DAMBREAK_MOMENTUM, P);
            selfaction(EPP_ACTION_DAMBREAK_INTEGRATE, P);
            search(EPP_CRITERION_SYMMETRY, EPP_ACTION_DAMBREAK_CONTINUITY, P);
            if (P.filter_interval > 0 && step_count % P.filter_interval == 0) {   // main.jl:180-183
                interaction(EPP_ACTION_KERNEL_FILTER, P);
                selfaction(EPP_ACTION_KERNEL_FILTER_SELF, P);
            }
        }
        return EPP_OK;
    }
};

template <typename T>
T* field_ptr(System<T>* s, int field, int k, bool& vec) {
    vec = false;
    switch (field) {
        case ORC_FIELD_POSITION: vec = true; return &s->pos[(size_t)k * s->n_cap];
        case ORC_FIELD_VELOCITY: vec = true; return &s->vel[(size_t)k * s->n_cap];
        case ORC_FIELD_DVELOCITY: vec = true; return &s->dvel[(size_t)k * s->n_cap];
        case ORC_FIELD_ACCEL: vec = true; return &s->accel[(size_t)k * s->n_cap];
        case ORC_FIELD_ACCEL_ABS: vec = true; return &s->accel_abs[(size_t)k * s->n_cap];
        case ORC_FIELD_DDENSITY_ABS: return s->drho_abs.data();
        case ORC_FIELD_DENSITY: return s->rho.data();
        case ORC_FIELD_DDENSITY: return s->drho.data();
        case ORC_FIELD_PRESSURE: return s->p.data();
        case ORC_FIELD_VOLUME: return s->vol.data();
        case ORC_FIELD_MASS: return s->mass.data();
        default: return nullptr;
    }
}

template <typename T>
int upload(System<T>* s, int32_t n, const int32_t* alive, const int32_t* cell, const int32_t* ip,
           int64_t ldi, const float* fp, int64_t ldf, const epp_column_map* m) {
    if (n < 0 || n > s->n_cap || !alive || !ip || !fp || !m) return EPP_ERR_INVALID_ARGUMENT;
    if (m->tag < 0 || m->position < 0) return EPP_ERR_INVALID_ARGUMENT;
    s->n = n;
    int D = s->D;
    auto icol = [&](int c, int I) { return ip[(size_t)c * ldi + I]; };
    auto fcol = [&](int c, int I) { return fp[(size_t)c * ldf + I]; };
    for (int I = 0; I < n; ++I) {
        s->alive[I] = alive[I];
        s->cell[I] = cell ? cell[I] : 0;
        s->tag[I] = icol(m->tag, I);
        s->movable[I] = m->is_movable >= 0 ? icol(m->is_movable, I) : 1;
        s->ncount[I] = m->n_count >= 0 ? icol(m->n_count, I) : 0;
        for (int a = 0; a < D; ++a) {
            s->X(a, I) = T(fcol(m->position + a, I));
            s->U(a, I) = m->velocity >= 0 ? T(fcol(m->velocity + a, I)) : T(0);
            s->DU(a, I) = m->dvelocity >= 0 ? T(fcol(m->dvelocity + a, I)) : T(0);
            s->comp[(size_t)a * s->n_cap + I] = T(0);
        }
        s->mass[I] = m->mass >= 0 ? T(fcol(m->mass, I)) : T(0);
        s->vol[I] = m->volume >= 0 ? T(fcol(m->volume, I)) : T(0);
        s->rho[I] = m->density >= 0 ? T(fcol(m->density, I)) : T(0);
        s->drho[I] = m->ddensity >= 0 ? T(fcol(m->ddensity, I)) : T(0);
        s->p[I] = m->pressure >= 0 ? T(fcol(m->pressure, I)) : T(0);
        s->gapc[I] = m->gap >= 0 ? T(fcol(m->gap, I)) : T(0);
        s->h[I] = m->h >= 0 ? T(fcol(m->h, I)) : T(0);
    }
    for (int I = n; I < s->n_cap; ++I) s->alive[I] = 0;
    s->searched = false;
    s->step_count = 0;
    s->sim_time = 0.0;
    std::fill(s->wv.begin(), s->wv.end(), T(0));       // filter sums start at zero (not uploaded)
    std::fill(s->wv_rho.begin(), s->wv_rho.end(), T(0));
    std::fill(s->wv_p.begin(), s->wv_p.end(), T(0));
    return EPP_OK;
}

template <typename T>
int download(System<T>* s, int32_t* alive, int32_t* cell, int32_t* ip, int64_t ldi, float* fp,
             int64_t ldf, const epp_column_map* m) {
    if (!m) return EPP_ERR_INVALID_ARGUMENT;
    int D = s->D;
    for (int I = 0; I < s->n; ++I) {
        if (alive) alive[I] = s->alive[I];
        if (cell) cell[I] = s->cell[I];
        if (ip) {
            auto put = [&](int c, int32_t v) { if (c >= 0) ip[(size_t)c * ldi + I] = v; };
            put(m->tag, s->tag[I]);
            put(m->is_movable, s->movable[I]);
            put(m->n_count, s->ncount[I]);
            if (m->n_index >= 0)
                for (int k = 0; k < s->max_nb; ++k) ip[(size_t)(m->n_index + k) * ldi + I] = s->NIDX(k, I);
        }
        if (fp) {
            auto put = [&](int c, T v) { if (c >= 0) fp[(size_t)c * ldf + I] = (float)v; };
            for (int a = 0; a < D; ++a) {
                if (m->position >= 0) put(m->position + a, s->X(a, I));
                if (m->velocity >= 0) put(m->velocity + a, s->U(a, I));
                if (m->dvelocity >= 0) put(m->dvelocity + a, s->DU(a, I));
            }
            put(m->mass, s->mass[I]); put(m->volume, s->vol[I]); put(m->density, s->rho[I]);
            put(m->ddensity, s->drho[I]); put(m->pressure, s->p[I]); put(m->gap, s->gapc[I]);
            put(m->h, s->h[I]);
            for (int k = 0; k < s->max_nb; ++k) {
                if (m->n_r >= 0) put(m->n_r + k, s->NR(k, I));
                if (m->n_w >= 0) put(m->n_w + k, s->NW(k, I));
                if (m->n_dw >= 0) put(m->n_dw + k, s->NDW(k, I));
                if (m->n_hinv >= 0) put(m->n_hinv + k, s->NH(k, I));
                if (m->n_rvec >= 0)
                    for (int a = 0; a < D; ++a) put(m->n_rvec + D * k + a, s->RV(k, a, I));
            }
        }
    }
    return EPP_OK;
}

template <typename T>
int integrals(System<T>* s, const epp_physics* ph, epp_integrals* out) {
    double mt = 0, mf = 0, ke = 0, pe = 0, ie = 0, vmax = 0, hmin = 1e300;
    int64_t na = 0, np = 0;
    double rho0 = ph->rho0, c0 = ph->c0, gam = ph->gamma, p0 = ph->p0;
    double B = rho0 * c0 * c0 / gam;
    for (int I = 0; I < s->n; ++I) {
        if (s->alive[I] != 1) continue;
        na += 1;
        np += s->ncount[I];
        double m = (double)s->mass[I];
        mt += m;
        if (s->tag[I] != ph->fluid_tag) continue;
        mf += m;
        double v2 = 0, gx = 0;
        for (int a = 0; a < s->D; ++a) {
            double u = (double)s->U(a, I);
            v2 += u * u;
            gx += (double)ph->gravity[a] * (double)s->X(a, I);
        }
        ke += 0.5 * m * v2;
        pe += -m * gx;
        double r = (double)s->rho[I];
        double e = ph->eos == EPP_EOS_LINEAR
                       ? c0 * c0 * (std::log(r / rho0) + rho0 / r - 1.0) + p0 * (1.0 / rho0 - 1.0 / r)
                       : (B / rho0) * (std::pow(r / rho0, gam - 1.0) / (gam - 1.0) + rho0 / r - gam / (gam - 1.0)) +
                             p0 * (1.0 / rho0 - 1.0 / r);
        ie += m * e;
        vmax = std::max(vmax, std::sqrt(v2));
        hmin = std::min(hmin, (double)s->h[I]);
    }
    out->mass_total = mt; out->mass_fluid = mf; out->kinetic = ke; out->potential = pe;
    out->internal = ie; out->max_speed = vmax;
    out->cfl_dt = hmin < 1e300 ? (ph->cfl > 0.0f ? (double)ph->cfl : 0.1) * hmin / (c0 + vmax) : 0.0;
    out->n_alive = na; out->n_pairs = np;
    return EPP_OK;
}

template <typename T>
int cell_stats(System<T>* s, int32_t* counts, int32_t* offsets, int32_t* ids, int32_t* n_cells) {
    int64_t nc = s->dom.n_cells;
    if (n_cells) *n_cells = (int32_t)nc;
    int64_t acc = 0;
    for (int64_t c = 0; c < nc; ++c) {
        int32_t k = s->ccount[c];
        if (counts) counts[c] = k;
        if (offsets) offsets[c] = (int32_t)acc;
        if (ids) {
            int32_t m = std::min(k, s->max_cell);
            std::vector<int32_t> b(m);
            for (int i = 0; i < m; ++i) b[i] = s->clist[(size_t)c + (size_t)nc * i];
            std::sort(b.begin(), b.end());
            for (int i = 0; i < m; ++i) ids[acc + i] = b[i];
        }
        acc += k;
    }
    if (offsets) offsets[nc] = (int32_t)acc;
    return EPP_OK;
}

#define DISPATCH(s, expr)                                                 \
    do {                                                                  \
        if ((s)->precision == 64) {                                       \
            auto* S = static_cast<System<double>*>(s);                    \
            auto P = phys ? make_phys<double>(*phys) : Phys<double>{};    \
            (void)P;                                                      \
            return expr;                                                  \
        } else {                                                          \
            auto* S = static_cast<System<float>*>(s);                     \
            auto P = phys ? make_phys<float>(*phys) : Phys<float>{};      \
            (void)P;                                                      \
            return expr;                                                  \
        }                                                                 \
    } while (0)

}  // namespace

struct orc_sys : SysBase {};

extern "C" {

int32_t orc_domain_info(const epp_domain* d, int32_t precision, int32_t n_out[3],
                        double gap_axis[3], double gap_inv[3]) {
    if (!d || (d->dim != 2 && d->dim != 3)) return EPP_ERR_INVALID_ARGUMENT;
    auto fill = [&](auto D) {
        for (int a = 0; a < 3; ++a) {
            if (n_out) n_out[a] = D.n[a];
            if (gap_axis) gap_axis[a] = (double)D.gap_axis[a];
            if (gap_inv) gap_inv[a] = (double)D.gap_inv[a];
        }
    };
    if (precision == 64) fill(make_domain<double>(*d));
    else fill(make_domain<float>(*d));
    return EPP_OK;
}

int32_t orc_cell_of(const epp_domain* d, int32_t precision, const float* x, int32_t cart_out[3],
                    int32_t* linear_out, int32_t* inside_out) {
    if (!d || !x) return EPP_ERR_INVALID_ARGUMENT;
    auto go = [&](auto D, auto zero) {
        using T = decltype(zero);
        T xx[3] = {T(x[0]), T(x[1]), d->dim == 3 ? T(x[2]) : T(0)};
        int32_t c[3] = {axis_index(D, 0, xx[0]), axis_index(D, 1, xx[1]),
                        d->dim == 3 ? axis_index(D, 2, xx[2]) : 1};
        if (cart_out) for (int a = 0; a < 3; ++a) cart_out[a] = c[a];
        if (linear_out) *linear_out = linear_index(D, c[0], c[1], c[2]);
        if (inside_out) *inside_out = inside(D, xx) ? 1 : 0;
    };
    if (precision == 64) go(make_domain<double>(*d), 0.0);
    else go(make_domain<float>(*d), 0.0f);
    return EPP_OK;
}

int32_t orc_neighbour_cell_table(const epp_domain* d, int32_t* counts, int32_t* lists) {
    if (!d) return EPP_ERR_INVALID_ARGUMENT;
    auto D = make_domain<float>(*d);
    std::vector<int32_t> c, l;
    neighbour_cells(d->dim, D.n, c, l);
    if (counts) std::copy(c.begin(), c.end(), counts);
    if (lists) std::copy(l.begin(), l.end(), lists);
    return EPP_OK;
}

int32_t orc_kernel(int32_t kind, int32_t dim, double r, double hinv, double* w, double* dw) {
    if ((dim != 2 && dim != 3) || kind < EPP_KERNEL_WENDLAND_C2 || kind > EPP_KERNEL_WENDLAND_C4 || !w || !dw)
        return EPP_ERR_INVALID_ARGUMENT;
    *w = kern_value<double>(kind, r, hinv, dim);
    *dw = kern_gradient<double>(kind, r, hinv, dim);
    return EPP_OK;
}

orc_sys* orc_create(int32_t precision, const epp_config* cfg) {
    if (!cfg) return nullptr;
    SysBase* s;
    int rc;
    if (precision == 64) {
        auto* t = new System<double>();
        t->precision = 64;
        rc = t->init(*cfg);
        s = t;
    } else {
        auto* t = new System<float>();
        t->precision = 32;
        rc = t->init(*cfg);
        s = t;
    }
    if (rc != EPP_OK) {
        delete s;
        return nullptr;
    }
    return reinterpret_cast<orc_sys*>(s);
}

void orc_destroy(orc_sys* s) { delete reinterpret_cast<SysBase*>(s); }

int32_t orc_set_threads(int32_t n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
    return EPP_OK;
}

int32_t orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int32_t orc_set_deterministic(orc_sys* s, int32_t det) {
    reinterpret_cast<SysBase*>(s)->deterministic = det != 0;
    return EPP_OK;
}

int32_t orc_upload(orc_sys* s0, int32_t n, const int32_t* alive, const int32_t* cell,
                   const int32_t* ip, int64_t ldi, const float* fp, int64_t ldf,
                   const epp_column_map* m) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    const epp_physics* phys = nullptr;
    DISPATCH(s, upload(S, n, alive, cell, ip, ldi, fp, ldf, m));
}

int32_t orc_download(orc_sys* s0, int32_t* alive, int32_t* cell, int32_t* ip, int64_t ldi,
                     float* fp, int64_t ldf, const epp_column_map* m) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    const epp_physics* phys = nullptr;
    DISPATCH(s, download(S, alive, cell, ip, ldi, fp, ldf, m));
}

int32_t orc_get_field(orc_sys* s0, int32_t field, int32_t k, double* out) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    if (!out) return EPP_ERR_INVALID_ARGUMENT;
    auto go = [&](auto* S) -> int32_t {
        if (field == ORC_FIELD_NCOUNT) {
            for (int I = 0; I < S->n; ++I) out[I] = S->ncount[I];
            return EPP_OK;
        }
        bool vec;
        if (k < 0 || k >= S->D) return EPP_ERR_INVALID_ARGUMENT;
        auto* p = field_ptr(S, field, k, vec);
        if (!p) return EPP_ERR_INVALID_ARGUMENT;
        if (!vec && k != 0) return EPP_ERR_INVALID_ARGUMENT;
        for (int I = 0; I < S->n; ++I) out[I] = (double)p[I];
        return EPP_OK;
    };
    if (s->precision == 64) return go(static_cast<System<double>*>(s));
    return go(static_cast<System<float>*>(s));
}

int32_t orc_set_field(orc_sys* s0, int32_t field, int32_t k, const double* in) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    if (!in) return EPP_ERR_INVALID_ARGUMENT;
    auto go = [&](auto* S) -> int32_t {
        using T = typename std::remove_reference<decltype(S->rho[0])>::type;
        bool vec;
        if (k < 0 || k >= S->D) return EPP_ERR_INVALID_ARGUMENT;
        auto* p = field_ptr(S, field, k, vec);
        if (!p || field == ORC_FIELD_ACCEL || field == ORC_FIELD_ACCEL_ABS ||
            field == ORC_FIELD_DDENSITY_ABS || (!vec && k != 0))
            return EPP_ERR_INVALID_ARGUMENT;
        for (int I = 0; I < S->n; ++I) p[I] = (T)in[I];
        return EPP_OK;
    };
    if (s->precision == 64) return go(static_cast<System<double>*>(s));
    return go(static_cast<System<float>*>(s));
}

int32_t orc_search(orc_sys* s0, int32_t criterion, int32_t action, const epp_physics* phys,
                   int32_t flags) {
    (void)flags;
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    if (action == EPP_ACTION_DAMBREAK_CONTINUITY && !phys) return EPP_ERR_INVALID_ARGUMENT;
    DISPATCH(s, S->search(criterion, action, P));
}

int32_t orc_interaction(orc_sys* s0, int32_t action, const epp_physics* phys) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    if ((action == EPP_ACTION_DAMBREAK_MOMENTUM || action == EPP_ACTION_KERNEL_FILTER) && !phys)
        return EPP_ERR_INVALID_ARGUMENT;
    DISPATCH(s, S->interaction(action, P));
}

int32_t orc_selfaction(orc_sys* s0, int32_t action, const epp_physics* phys) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    if ((action == EPP_ACTION_DAMBREAK_DENSITY || action == EPP_ACTION_DAMBREAK_INTEGRATE ||
         action == EPP_ACTION_KERNEL_FILTER_SELF) && !phys)
        return EPP_ERR_INVALID_ARGUMENT;
    DISPATCH(s, S->selfaction(action, P));
}

int32_t orc_step(orc_sys* s0, int32_t n_steps, const epp_physics* phys) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    if (!phys) return EPP_ERR_INVALID_ARGUMENT;
    DISPATCH(s, S->step(n_steps, P));
}

int32_t orc_integrals(orc_sys* s0, const epp_physics* phys, epp_integrals* out) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    if (!phys || !out) return EPP_ERR_INVALID_ARGUMENT;
    DISPATCH(s, integrals(S, phys, out));
}

int32_t orc_cell_stats(orc_sys* s0, int32_t* counts, int32_t* offsets, int32_t* ids,
                       int32_t* n_cells) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    const epp_physics* phys = nullptr;
    DISPATCH(s, cell_stats(S, counts, offsets, ids, n_cells));
}

int32_t orc_step_dt(orc_sys* s0, const epp_physics* phys, double* next_dt, double* sim_time) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    if (!phys) return EPP_ERR_INVALID_ARGUMENT;
    auto go = [&](auto* S) -> int32_t {
        using T = typename std::remove_reference<decltype(S->rho[0])>::type;
        const Phys<T> P = make_phys<T>(*phys);
        if (next_dt) *next_dt = (double)(P.cfl > 0.0 ? S->cfl_dt(P) : P.dt);
        if (sim_time) *sim_time = S->sim_time;
        return EPP_OK;
    };
    if (s->precision == 64) return go(static_cast<System<double>*>(s));
    return go(static_cast<System<float>*>(s));
}

uint32_t orc_status(orc_sys* s0) {
    SysBase* s = reinterpret_cast<SysBase*>(s0);
    uint32_t v = s->status;
    s->status = 0;
    return v;
}

}  // extern "C"
