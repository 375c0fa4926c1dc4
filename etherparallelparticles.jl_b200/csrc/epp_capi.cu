// epp_capi.cu -- the C ABI of libepp.so (include/epp.h): context, device arena, reference-layout
// upload/download, the search! / interaction! / selfaction! entry points and the fused,
// graph-captured dam-break step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "epp_window.cuh"
#include "epp_self.cuh"

using namespace epp;

namespace {

constexpr int kThreads = 128;
constexpr int kProfileStages = EPP_PROFILE_STAGES;
constexpr int kIntegralBlocks = 592;   // 4 x 148 SMs

inline int blocks_for(long long n, int t = kThreads) { return (int)((n + t - 1) / t); }

struct Arena {
    char* base = nullptr;
    size_t size = 0, off = 0;
    template <class T>
    T* take(size_t count) {
        size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
        if (off + bytes > size) return nullptr;
        T* p = reinterpret_cast<T*>(base + off);
        off += bytes;
        return p;
    }
};

DevPhys to_dev(const epp_physics& p) {
    DevPhys d;
    d.ip = nullptr;
    d.dt = p.dt;
    d.rho0 = p.rho0;
    d.c0 = p.c0;
    d.p0 = p.p0;
    d.B = (float)((double)p.rho0 * (double)p.c0 * (double)p.c0 / (double)p.gamma);
    for (int a = 0; a < 3; ++a) d.g[a] = p.gravity[a];
    d.alpha = p.alpha;
    d.beta = p.beta;
    d.mu = p.mu;
    d.kernel = p.kernel;
    d.eos = p.eos;
    d.motion = p.motion;
    d.gamma = p.gamma;
    d.visc = p.viscosity;
    d.fluid = p.fluid_tag;
    d.wall = p.wall_tag;
    d.kahan = p.kahan;
    d.pff = p.pressure_ff == EPP_PRESSURE_DEFAULT ? EPP_PRESSURE_CLASSIC : p.pressure_ff;    // main.jl:109
    d.pfw = p.pressure_fw == EPP_PRESSURE_DEFAULT ? EPP_PRESSURE_BALANCED : p.pressure_fw;   // main.jl:113
    d.tensile = p.tensile;
    d.wallp = p.wall_pressure;
    d.gap = nullptr;
    return d;
}

bool same_phys(const epp_physics& a, const epp_physics& b) { return std::memcmp(&a, &b, sizeof a) == 0; }

}  // namespace

struct epp_ctx {
    epp_config cfg{};
    int D = 2;
    int dev = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    DevDomain dom{};
    int n = 0;        // particles uploaded (rows)
    int cap = 0;
    int n_cells = 0;
    int n_tiles = 0;
    Arena arena;
    State S[2]{};
    int* start[2]{};
    int* occ[2]{};             // occupied cells of each buffer set (cell order)
    int* meta[2]{};            // meta[set][0] = number of occupied cells
    int sms = 148;
    int cur = 0;
    FusedOut tmp{};       // xh/vm/comp of the fused momentum pass
    int* count = nullptr;
    int2* cs = nullptr;
    int2* perm = nullptr;
    unsigned long long* scan_state = nullptr;
    unsigned* status = nullptr;
    unsigned long long* pairs = nullptr;
    int* ncnt[2] = {nullptr, nullptr};   // nCount of each state set (what the last search of that set found)
    float* stage_f = nullptr;
    int* stage_i = nullptr;
    double* ipartial = nullptr;
    double* iresult = nullptr;
    unsigned* iticket = nullptr;
    float4* accel = nullptr;   // optional dv/dt output of the fused momentum pass
    // lazily allocated neighbour lists (EPP_SEARCH_EMIT_LIST)
    NeighbourList L{};
    void* list_mem = nullptr;
    void* list_stage = nullptr;
    // host state flags
    bool searched = false;      // cells match the current positions
    bool sorted_once = false;   // the state is cell-ordered with a valid alive count
    bool lists_valid = false;
    bool dv_dirty = true;       // dVelocity may be non-zero (fused step assumes zero)
    bool rpn_valid = false;     // density preview matches rho, drho and rpn_phys
    float* fwv = nullptr;       // kernel-filter sums (SumWeight, SumWeightedDensity) per sorted particle
    float* fwr = nullptr;
    float* fwp = nullptr;       // SumWeightedPressure of the wall-pressure extrapolation (SumWeight: fwv)
    float* gap = nullptr;       // Gap column per caller row (tensile correction)
    bool has_gap = false;       // the last upload mapped the Gap column
    bool filter_pending = false;   // interaction!(KERNEL_FILTER) done, selfaction!(KERNEL_FILTER_SELF) not yet
    bool extrap_pending = false;   // interaction!(EXTRAPOLATE_PRESSURE) done, its selfaction! not yet
    bool rpn_walls = false;        // the density preview carries the extrapolated wall pressure
    long long step_count = 0;      // epp_step steps since upload (the filter runs after every k-th)
    epp_physics rpn_phys{};
    int last_crit = EPP_CRITERION_SYMMETRY;
    unsigned adj[kMaxTags]{};
    int lanes = 0;             // pair-pass family: 0 warp tiles + lists, 1 cell-centric, 2..32 lane groups
    int store = 0;             // family 0: 0 = default (2D window search), EPP_TUNING_LISTS (lockstep list search)
    int pass_threads = 128;    // threads per block of the family-0 search and list passes (32, 64, 128)
    int* nlist = nullptr;      // neighbour lists of the last search ([LCAP * cap])
    bool nlist_valid = false;   // the lists match the current order, positions and criterion
    int n_inst = 1;            // batch instances (independent layers of the cell grid)
    InstPhys* inst_table = nullptr;     // device [n_inst]; null when no per-instance physics is set
    std::vector<float> inst_dt, inst_c0;
    bool inst_dirty = false;
    float inst_rho0 = 0.0f;
    int inst_gamma = 0;
    double* inst_out = nullptr;         // device [n_inst * 9] integrals
    // CFL time stepping (epp_physics.cfl > 0): tbl[set][k] holds instance k's dt (and c0, B) for the
    // step that starts from the state in buffer set `set`; the fused step of parity c reads tbl[c]
    // and its k_cfl writes tbl[1 - c] for the state it produces
    InstPhys* tbl[2]{};
    double2* cfl_partial = nullptr;     // [n_inst * cfl_chunks]
    unsigned* cfl_ticket = nullptr;
    double* sim_time = nullptr;         // [n_inst] simulated time of steps taken with a CFL dt
    int cfl_chunks = 1;
    int graph_fluid = 1;                // fluid tag k_cfl reduces over
    bool cfl_tables_ok = false;         // c0 and B of both tables match tbl_c0 / tbl_key
    bool cfl_valid = false;             // tbl[cur].dt is the CFL dt of the current state
    float tbl_rho0 = 0.0f, tbl_c0 = 0.0f;
    int tbl_gamma = 0;
    std::vector<double> time_fixed;     // simulated time of steps taken with a fixed dt, per instance
    // fused step graphs, one per ping-pong parity
    cudaGraphExec_t graph[2]{};
    cudaGraphExec_t graph_f[2]{};   // the same step followed by the kernel filter
    epp_physics graph_phys{};
    bool graph_accel = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // epp_integrals_async: pinned host slots (8 results + n_alive each), their events and tickets
    double* ihost = nullptr;
    cudaEvent_t iev[EPP_INTEGRALS_SLOTS]{};
    long long iticket_next = 0;
    long long islot_ticket[EPP_INTEGRALS_SLOTS]{-1, -1, -1, -1};
    float islot_c0[EPP_INTEGRALS_SLOTS]{};
    float islot_cfl[EPP_INTEGRALS_SLOTS]{};
    // ... which run on a second stream beside the next epp_step: they read only the state set they
    // were asked for (positions, velocities, density, tags, its nCount and cell offsets), which the
    // next step reads but does not write; `idone[k]` marks the integrals of set k done
    cudaStream_t istream = nullptr;
    cudaEvent_t iready = nullptr;
    cudaEvent_t idone[2]{};
    bool ipending[2]{};
    bool timed = false;
    std::string err;
};

namespace {

int fail(epp_ctx* c, int code, const char* fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(ctx, EPP_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                               \
    } while (0)

#define CK_LAUNCH() CK(cudaGetLastError())

// Makes the context's stream wait for integrals still running beside it on set k (both sets when
// k < 0).  Every entry point that may overwrite a state set, or run the integrals' reduction
// itself, calls it before enqueueing work.
int join_integrals(epp_ctx* ctx, int k = -1) {
    for (int s = 0; s < 2; ++s)
        if (ctx->ipending[s] && (k < 0 || k == s)) {
            CK(cudaStreamWaitEvent(ctx->stream, ctx->idone[s], 0));
            ctx->ipending[s] = false;
        }
    return EPP_OK;
}

size_t state_bytes(int cap) {
    // xh, vm, dv, comp, rp4 (float4) + rho, drho, vol, p, tagm, id, cell (4 B), aligned
    return (size_t)cap * (5 * 16 + 7 * 4) + 12 * 256;
}

size_t arena_bytes(int cap, int n_cells, int D, int n_tiles) {
    size_t b = 2 * state_bytes(cap);
    b += (size_t)cap * 3 * 16 + 3 * 256;                 // fused temp
    b += (size_t)(n_cells + 2) * 4 + 256;                // count
    b += 2 * ((size_t)(n_cells + 2) * 4 + 256);          // start[2]
    b += (size_t)cap * 8 * 2 + 512;                      // cs, perm
    b += (size_t)(n_tiles + 1) * 8 + 256;                // scan state
    b += 2 * ((size_t)(n_cells + 1) * 4 + 256 + 256);    // occ[2], meta[2]
    b += 256 * 3;                                        // status, pairs
    b += 2 * ((size_t)cap * 4 + 256);                    // nCount of each set
    b += (size_t)cap * 4 * (3 * D + 6) + 256;            // stage_f
    b += (size_t)cap * 4 * SI_COUNT + 256;               // stage_i
    b += (size_t)kIntegralBlocks * 8 * 8 + 8 * 8 + 4 * 256;
    b += 4 * ((size_t)cap * 4 + 256);                    // filter / extrapolation sums, gap by row
    b += 2 * 256;                                                                  // instance tables (small)
    return b + (1 << 20);
}

// Device memory of a context comes from the stream-ordered allocator on the context's stream:
// creating or destroying one context never synchronises the device, so a server can admit and
// retire simulations while others keep running.
template <class T>
cudaError_t dev_alloc(epp_ctx* ctx, T** p, size_t bytes) {
    return cudaMallocAsync(reinterpret_cast<void**>(p), bytes, ctx->stream);
}
template <class T>
void dev_free(epp_ctx* ctx, T*& p) {
    if (p) cudaFreeAsync(p, ctx->stream);
    p = nullptr;
}

// Cells of the grid (all instances) of a configuration: EPP_OK, or the status that rejects it.
int plan_cells(const epp_config* cfg, DevDomain& d) {
    const int n_inst = cfg->n_instances > 1 ? cfg->n_instances : 1;
    if (cfg->domain.dim == 3 && n_inst > 1) return EPP_ERR_INVALID_ARGUMENT;   // batches are 2D
    return plan_domain(cfg->domain, n_inst, 1ll << 30, d);
}

size_t nlist_bytes(int D, int cap) {
    return sizeof(int) * (size_t)(D == 2 ? ListConf<2>::LCAP : ListConf<3>::LCAP) * cap;
}

template <int D>
int run_search(epp_ctx* ctx, int crit, int action, const epp_physics* phys, bool emit);

void fill_state(Arena& a, State& s, int cap) {
    s.xh = a.take<float4>(cap);
    s.vm = a.take<float4>(cap);
    s.dv = a.take<float4>(cap);
    s.comp = a.take<float4>(cap);
    s.rho = a.take<float>(cap);
    s.drho = a.take<float>(cap);
    s.vol = a.take<float>(cap);
    s.p = a.take<float>(cap);
    s.tagm = a.take<int>(cap);
    s.id = a.take<int>(cap);
    s.cell = a.take<int>(cap);
    s.rp4 = a.take<float4>(cap);
}

// The CFL tables (epp_physics.cfl > 0): c0 and B of every instance (its own c0 in a batch with
// instance physics, phys.c0 otherwise) in both buffer sets; their dt fields are written on the
// device by k_cfl.  Re-uploading them invalidates the current CFL dt.
void ensure_cfl_tables(epp_ctx* ctx, const epp_physics& p) {
    if (ctx->cfl_tables_ok && ctx->tbl_rho0 == p.rho0 && ctx->tbl_gamma == p.gamma &&
        (!ctx->inst_c0.empty() || ctx->tbl_c0 == p.c0))
        return;
    std::vector<InstPhys> t(ctx->n_inst);
    for (int k = 0; k < ctx->n_inst; ++k) {
        const float c0 = ctx->inst_c0.empty() ? p.c0 : ctx->inst_c0[k];
        t[k].dt = ctx->inst_dt.empty() ? p.dt : ctx->inst_dt[k];
        t[k].c0 = c0;
        t[k].B = (float)((double)p.rho0 * (double)c0 * (double)c0 / (double)p.gamma);
        t[k].pad = 0.0f;
    }
    for (int b = 0; b < 2; ++b)
        cudaMemcpyAsync(ctx->tbl[b], t.data(), sizeof(InstPhys) * ctx->n_inst, cudaMemcpyHostToDevice, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    ctx->cfl_tables_ok = true;
    ctx->tbl_rho0 = p.rho0;
    ctx->tbl_gamma = p.gamma;
    ctx->tbl_c0 = p.c0;
    ctx->cfl_valid = false;
}

// Device physics of a call: the per-instance table (uploaded when it changed) overrides dt, c0, B;
// with a CFL physics, the CFL table of the current buffer set does.
DevPhys dev_phys(epp_ctx* ctx, const epp_physics& p) {
    DevPhys d = to_dev(p);
    if (p.cfl > 0.0f) {
        ensure_cfl_tables(ctx, p);
        d.ip = ctx->tbl[ctx->cur];
        d.gap = ctx->gap;
        return d;
    }
    if (!ctx->inst_dt.empty()) {
        if (ctx->inst_dirty || ctx->inst_rho0 != p.rho0 || ctx->inst_gamma != p.gamma) {
            std::vector<InstPhys> t(ctx->n_inst);
            for (int k = 0; k < ctx->n_inst; ++k) {
                t[k].dt = ctx->inst_dt[k];
                t[k].c0 = ctx->inst_c0[k];
                t[k].B = (float)((double)p.rho0 * (double)ctx->inst_c0[k] * (double)ctx->inst_c0[k] / (double)p.gamma);
                t[k].pad = 0.0f;
            }
            cudaMemcpyAsync(ctx->inst_table, t.data(), sizeof(InstPhys) * ctx->n_inst, cudaMemcpyHostToDevice,
                            ctx->stream);
            cudaStreamSynchronize(ctx->stream);
            ctx->inst_dirty = false;
            ctx->inst_rho0 = p.rho0;
            ctx->inst_gamma = p.gamma;
        }
        d.ip = ctx->inst_table;
    }
    d.gap = ctx->gap;
    return d;
}

PairArgs pair_args(epp_ctx* ctx, int set, int crit) {
    PairArgs A;
    A.dom = ctx->dom;
    A.s = ctx->S[set];
    A.start = ctx->start[set];
    for (int t = 0; t < kMaxTags; ++t) A.adj[t] = ctx->adj[t];
    A.n_tags = ctx->cfg.n_tags;
    A.crit = crit;
    A.n_max = ctx->n;
    A.status = ctx->status;
    return A;
}

int lanes_of(const epp_ctx* ctx) { return ctx->lanes; }

// k_cfl over the state in buffer set `set` (FUSED: the momentum pass's output of a step from set
// `set`), writing `next`; `used` (or null) is the table of the step just taken, added to the time.
template <int D, bool FUSED>
int launch_cfl(epp_ctx* ctx, int set, float cfl, const InstPhys* used, InstPhys* next) {
    CflArgs a;
    a.start = ctx->start[set];
    a.cells_per_inst = ctx->dom.cells_per_inst;
    a.n_inst = ctx->n_inst;
    a.n_cells = ctx->n_cells;
    a.n_max = ctx->n;
    a.chunks = ctx->cfl_chunks;
    a.vm = FUSED ? ctx->tmp.vm : ctx->S[set].vm;
    a.xh = FUSED ? ctx->tmp.xh : ctx->S[set].xh;
    a.tagm = ctx->S[set].tagm;
    a.cs = ctx->cs;
    a.fluid = ctx->graph_fluid;
    a.cfl = cfl;
    a.used = used;
    a.next = next;
    a.partial = ctx->cfl_partial;
    a.time = ctx->sim_time;
    a.ticket = ctx->cfl_ticket;
    k_cfl<D, FUSED><<<ctx->n_inst * ctx->cfl_chunks, 256, 0, ctx->stream>>>(a);
    CK_LAUNCH();
    return EPP_OK;
}

// The CFL dt of the current state into its table (tbl[cur]).
template <int D>
int cfl_update(epp_ctx* ctx, const epp_physics& p) {
    ensure_cfl_tables(ctx, p);
    ctx->graph_fluid = p.fluid_tag;
    const int rc = launch_cfl<D, false>(ctx, ctx->cur, p.cfl, nullptr, ctx->tbl[ctx->cur]);
    if (rc == EPP_OK) ctx->cfl_valid = true;
    return rc;
}

// Physics that needs the generic pair terms (any kernel, classic viscosity); the benchmark physics
// (Wendland C2, artificial viscosity) runs the specialised ones.
bool generic_physics(const epp_physics* p) {
    return p && (p->kernel != EPP_KERNEL_WENDLAND_C2 || p->viscosity == EPP_VISCOSITY_CLASSIC ||
                 (p->pressure_ff != EPP_PRESSURE_DEFAULT && p->pressure_ff != EPP_PRESSURE_CLASSIC) ||
                 (p->pressure_fw != EPP_PRESSURE_DEFAULT && p->pressure_fw != EPP_PRESSURE_BALANCED) ||
                 p->tensile != 0);
}

// Family 0 in 2D searches each particle's own stencil-row windows with the search action folded in
// (epp_window.cuh), unless the context was set to the lockstep list search and a separate
// continuity pass (epp_set_tuning EPP_TUNING_LISTS); 3D always uses the latter.
bool uses_windows(const epp_ctx* ctx) { return ctx->D == 2 && ctx->store != EPP_TUNING_LISTS; }

// The 2D window search pass with search action `act` (CPCount: lists and nCount only).
template <class Act>
int launch_win_build(epp_ctx* ctx, int set, int crit, const Act& act, unsigned long long* pairs) {
    PairArgs A = pair_args(ctx, set, crit);
    TileMask M{ctx->cap, ctx->nlist};
    k_win_build<Act><<<blocks_for(ctx->n, ctx->pass_threads), ctx->pass_threads, 0, ctx->stream>>>(A, M, act, pairs);
    CK_LAUNCH();
    return EPP_OK;
}

// Family 0, the search pass: neighbour lists and nCount of set `set` under `crit`.
template <int D>
int launch_build(epp_ctx* ctx, int set, int crit, unsigned long long* pairs) {
    if constexpr (D == 2) {
        if (uses_windows(ctx)) return launch_win_build(ctx, set, crit, CPCount<2>{ctx->ncnt[set]}, pairs);
    }
    PairArgs A = pair_args(ctx, set, crit);
    TileMask M{ctx->cap, ctx->nlist};
    k_build<D><<<blocks_for(ctx->n, ctx->pass_threads), ctx->pass_threads, 0, ctx->stream>>>(A, M, ctx->ncnt[set], pairs);
    CK_LAUNCH();
    return EPP_OK;
}

// Family 0, a pair action over the lists of the last search pass (same order and positions).
template <int D, class Act, bool EPI = false>
int launch_list(epp_ctx* ctx, int set, int crit, const Act& act) {
    PairArgs A = pair_args(ctx, set, crit);
    TileMask M{ctx->cap, ctx->nlist};
    k_list<D, Act, EPI><<<blocks_for(ctx->n, ctx->pass_threads), ctx->pass_threads, 0, ctx->stream>>>(
        A, M, ctx->ncnt[set], act, ctx->scan_state, ctx->n_tiles + 1);
    CK_LAUNCH();
    return EPP_OK;
}

// A pair pass of family 0.  BUILD: the search pass first (new lists at the current positions);
// then the action over the lists (none for the count-only action: the search wrote nCount).  In
// 2D with the window search, the search pass runs the search action itself (one kernel).
template <int D, bool BUILD, class Act, bool EPI = false>
int launch_pass(epp_ctx* ctx, int set, int crit, const Act& act, unsigned long long* pairs) {
    if constexpr (D == 2 && BUILD && !EPI) {
        if (uses_windows(ctx)) return launch_win_build(ctx, set, crit, act, pairs);
    }
    if (BUILD) {
        int rc = launch_build<D>(ctx, set, crit, pairs);
        if (rc) return rc;
    }
    if constexpr (std::is_same<Act, CPCount<D>>::value) return EPP_OK;
    else return launch_list<D, Act, EPI>(ctx, set, crit, act);
}

// Launch a G-lane pair pass over `groups` particles (G from the context's tuning).
template <int D, class Act, bool EPI>
int launch_pair_g(epp_ctx* ctx, const PairArgs& A, const Act& act, unsigned long long* pairs, long long groups) {
    const int G = lanes_of(ctx);
    const int nw = ctx->n_tiles + 1;
#define EPP_G(GG)                                                                                 \
    case GG:                                                                                      \
        k_pair_g<D, GG, Act, EPI><<<blocks_for(groups * GG), kThreads, 0, ctx->stream>>>(          \
            A, act, pairs, ctx->scan_state, nw);                                                  \
        break;
    switch (G) {
        EPP_G(2)
        EPP_G(4)
        EPP_G(8)
        EPP_G(16)
        EPP_G(32)
        default:
            return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "lanes per particle %d not in {2,4,8,16,32}", G);
    }
#undef EPP_G
    CK_LAUNCH();
    return EPP_OK;
}

// Persistent grid of a cell-pair kernel: resident blocks per SM x SMs (computed once per
// instantiation, with the dynamic shared memory opt-in set outside any graph capture).
template <int D, class Act, bool EPI>
int cellpair_grid(epp_ctx* ctx) {   // -1 on a CUDA error (recorded in the context)
    static int grid = 0;
    if (grid) return grid;
    const size_t smem = sizeof(CPShared<D>) * kCPWarps;
    cudaError_t e = cudaFuncSetAttribute(k_cellpair<D, Act, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    int per_sm = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cellpair<D, Act, EPI>, kCPWarps * 32, smem);
    if (e != cudaSuccess) {
        fail(ctx, EPP_ERR_CUDA, "cell-pair kernel setup: %s", cudaGetErrorString(e));
        return -1;
    }
    grid = (per_sm > 0 ? per_sm : 1) * ctx->sms;
    return grid;
}

template <int D, class Act, bool EPI = false>
int launch_cellpair(epp_ctx* ctx, int set, int crit, const Act& act, unsigned long long* pairs) {
    CellArgs CA{pair_args(ctx, set, crit), ctx->occ[set], ctx->meta[set]};
    const int grid = cellpair_grid<D, Act, EPI>(ctx);
    if (grid < 0) return EPP_ERR_CUDA;
    const size_t smem = sizeof(CPShared<D>) * kCPWarps;
    k_cellpair<D, Act, EPI><<<grid, kCPWarps * 32, smem, ctx->stream>>>(CA, act, pairs, ctx->scan_state,
                                                                         ctx->n_tiles + 1);
    CK_LAUNCH();
    return EPP_OK;
}

template <int D>
int prepare_kernels(epp_ctx* ctx) {
    int g = 0;
    g |= cellpair_grid<D, CPCont<D, true>, false>(ctx) < 0;
    g |= cellpair_grid<D, CPCont<D, false>, false>(ctx) < 0;
    g |= cellpair_grid<D, CPCount<D>, false>(ctx) < 0;
    g |= cellpair_grid<D, CPCountDv<D>, false>(ctx) < 0;
    g |= cellpair_grid<D, CPMom<D, true>, true>(ctx) < 0;
    g |= cellpair_grid<D, CPMom<D, false>, false>(ctx) < 0;
    g |= cellpair_grid<D, CPCont<D, true, true>, false>(ctx) < 0;
    g |= cellpair_grid<D, CPCont<D, false, true>, false>(ctx) < 0;
    g |= cellpair_grid<D, CPMom<D, true, true>, true>(ctx) < 0;
    g |= cellpair_grid<D, CPMom<D, false, true>, false>(ctx) < 0;
    return g ? EPP_ERR_CUDA : EPP_OK;
}

// clean! + insert (bin, count, scan, scatter, rank-by-id gather) from set `from` into 1-from.
template <int D>
int sort_cells(epp_ctx* ctx) {
    const int from = ctx->cur, to = 1 - ctx->cur;
    const int n = ctx->n;
    k_bin_count<D><<<blocks_for(n), kThreads, 0, ctx->stream>>>(
        n, ctx->dom, ctx->S[from], ctx->count, ctx->cs, ctx->cfg.max_cell_particles, ctx->status,
        ctx->scan_state, ctx->n_tiles + 1);
    CK_LAUNCH();
    k_scan<<<ctx->n_tiles, kScanThreads, 0, ctx->stream>>>(ctx->n_cells + 1, ctx->count, ctx->start[to],
                                                          ctx->occ[to], ctx->meta[to], ctx->scan_state,
                                                          ctx->status);
    CK_LAUNCH();
    k_scatter<<<blocks_for(n), kThreads, 0, ctx->stream>>>(n, ctx->cs, ctx->start[to], ctx->S[from].id,
                                                           ctx->perm, ctx->status);
    CK_LAUNCH();
    ctx->nlist_valid = false;
    MoverAll mv{ctx->S[from], ctx->S[to]};
    k_rank_gather<<<blocks_for(n), kThreads, 0, ctx->stream>>>(n, ctx->n_cells, ctx->perm, ctx->cs,
                                                               ctx->start[to], mv, ctx->status);
    CK_LAUNCH();
    ctx->cur = to;
    return EPP_OK;
}

int ensure_lists(epp_ctx* ctx) {
    if (ctx->list_mem) return EPP_OK;
    const size_t cap = ctx->cap, nb = ctx->cfg.max_neighbour_number, D = ctx->D;
    const size_t words = cap * nb * (1 + D + 4);
    CK(dev_alloc(ctx, &ctx->list_mem, words * 4));
    CK(cudaMemsetAsync(ctx->list_mem, 0, words * 4, ctx->stream));
    CK(dev_alloc(ctx, &ctx->list_stage, words * 4));
    char* p = (char*)ctx->list_mem;
    ctx->L.idx = (int*)p; p += cap * nb * 4;
    ctx->L.rvec = (float*)p; p += cap * nb * D * 4;
    ctx->L.r = (float*)p; p += cap * nb * 4;
    ctx->L.w = (float*)p; p += cap * nb * 4;
    ctx->L.dw = (float*)p; p += cap * nb * 4;
    ctx->L.hinv = (float*)p;
    ctx->L.max_nb = (int)nb;
    ctx->L.cap = (int)cap;
    return EPP_OK;
}

template <int D>
int launch_search_pass(epp_ctx* ctx, int set, int crit, int action, const epp_physics* phys, bool emit,
                       bool fused) {
    PairArgs A = pair_args(ctx, set, crit);
    DevPhys P = phys ? dev_phys(ctx, *phys) : DevPhys{};
    const bool cont = action == EPP_ACTION_DAMBREAK_CONTINUITY;
    if (emit) {
        ctx->nlist_valid = false;
        // the emitted list keeps the reference's neighbour order: one thread per particle
        const int grid = blocks_for(ctx->n);
        if (cont) {
            ActSearch<D, true, true, false> act{ctx->S[set], ctx->L, P, ctx->ncnt[set], ctx->status};
            k_pair<D><<<grid, kThreads, 0, ctx->stream>>>(A, act, ctx->pairs);
        } else {
            ActSearch<D, true, false, false> act{ctx->S[set], ctx->L, P, ctx->ncnt[set], ctx->status};
            k_pair<D><<<grid, kThreads, 0, ctx->stream>>>(A, act, ctx->pairs);
        }
        CK_LAUNCH();
        return EPP_OK;
    }
    const bool gen = generic_physics(phys);
    if (ctx->lanes == 0) {
        int rc;
        auto cont_pass = [&](auto G) {
            constexpr bool GG = decltype(G)::value;
            if (fused) return launch_pass<D, true>(ctx, set, crit, CPCont<D, true, GG>{ctx->S[set], P, ctx->ncnt[set]}, ctx->pairs);
            return launch_pass<D, true>(ctx, set, crit, CPCont<D, false, GG>{ctx->S[set], P, ctx->ncnt[set]}, ctx->pairs);
        };
        if (fused || cont) rc = gen ? cont_pass(std::true_type{}) : cont_pass(std::false_type{});
        else rc = launch_pass<D, true>(ctx, set, crit, CPCount<D>{ctx->ncnt[set]}, ctx->pairs);
        ctx->nlist_valid = rc == EPP_OK;
        return rc;
    }
    ctx->nlist_valid = false;
    if (ctx->lanes >= 2) {   // lane-group kernels (tuning alternative)
        if (fused) {
            ActContG<D, true, true> act{ctx->S[set], P, ctx->ncnt[set]};
            return launch_pair_g<D, decltype(act), false>(ctx, A, act, ctx->pairs, ctx->n);
        }
        if (cont) {
            ActContG<D, true, false> act{ctx->S[set], P, ctx->ncnt[set]};
            return launch_pair_g<D, decltype(act), false>(ctx, A, act, ctx->pairs, ctx->n);
        }
        ActContG<D, false, false> act{ctx->S[set], P, ctx->ncnt[set]};
        return launch_pair_g<D, decltype(act), false>(ctx, A, act, ctx->pairs, ctx->n);
    }
    if (gen) {
        if (fused) return launch_cellpair<D>(ctx, set, crit, CPCont<D, true, true>{ctx->S[set], P, ctx->ncnt[set]}, ctx->pairs);
        if (cont) return launch_cellpair<D>(ctx, set, crit, CPCont<D, false, true>{ctx->S[set], P, ctx->ncnt[set]}, ctx->pairs);
    }
    if (fused) return launch_cellpair<D>(ctx, set, crit, CPCont<D, true>{ctx->S[set], P, ctx->ncnt[set]}, ctx->pairs);
    if (cont) return launch_cellpair<D>(ctx, set, crit, CPCont<D, false>{ctx->S[set], P, ctx->ncnt[set]}, ctx->pairs);
    return launch_cellpair<D>(ctx, set, crit, CPCount<D>{ctx->ncnt[set]}, ctx->pairs);
}

template <int D>
int run_search(epp_ctx* ctx, int crit, int action, const epp_physics* phys, bool emit) {
    if (emit) {
        int rc = ensure_lists(ctx);
        if (rc) return rc;
    }
    int rc = sort_cells<D>(ctx);
    if (rc) return rc;
    ctx->cfl_valid = false;   // a new buffer set
    if (phys && phys->cfl > 0.0f && action == EPP_ACTION_DAMBREAK_CONTINUITY) {
        rc = cfl_update<D>(ctx, *phys);   // the continuity pass previews the next step's density
        if (rc) return rc;
    }
    rc = launch_search_pass<D>(ctx, ctx->cur, crit, action, phys, emit, false);
    if (rc) return rc;
    ctx->searched = true;
    ctx->sorted_once = true;
    ctx->lists_valid = emit;
    ctx->last_crit = crit;
    if (action == EPP_ACTION_DAMBREAK_CONTINUITY) {
        ctx->rpn_valid = true;
        ctx->rpn_phys = *phys;
    } else {
        ctx->rpn_valid = false;
    }
    ctx->rpn_walls = false;
    return EPP_OK;
}

// One fused step from set c to 1 - c (captured into a graph by the caller).  With `ev`, an
// event is recorded before the first and after every kernel (profiling, no graph).
template <int D>
int enqueue_fused_step(epp_ctx* ctx, int c, const epp_physics& phys, cudaEvent_t* ev = nullptr, bool filter = false) {
#define EPP_MARK(k) do { if (ev) CK(cudaEventRecord(ev[k], ctx->stream)); } while (0)
    EPP_MARK(0);
    const int to = 1 - c;
    const int n = ctx->n;
    PairArgs A = pair_args(ctx, c, EPP_CRITERION_SYMMETRY);
    ActMomG<D, true> mom;
    mom.s = ctx->S[c];
    mom.P = dev_phys(ctx, phys);
    mom.dom = ctx->dom;
    mom.F = ctx->tmp;
    mom.F.n = n;
    mom.F.accel = ctx->graph_accel ? ctx->accel : nullptr;
    mom.status = ctx->status;
    const bool gen = generic_physics(&phys);
    const bool cfl = phys.cfl > 0.0f;
    // passes after the momentum pass preview the next step's density: the next step's dt
    DevPhys Pn = mom.P;
    if (cfl) {   // this step takes tbl[c]; its k_cfl writes tbl[1 - c] for the state it produces
        mom.P.ip = ctx->tbl[c];
        Pn.ip = ctx->tbl[to];
    }
    {
        auto mom_pass = [&](auto G) {
            constexpr bool GG = decltype(G)::value;
            using M = CPMom<D, true, GG>;
            return ctx->lanes >= 2 ? launch_pair_g<D, ActMomG<D, true>, true>(ctx, A, mom, nullptr, n)
                   : ctx->lanes == 1 ? launch_cellpair<D, M, true>(ctx, c, EPP_CRITERION_SYMMETRY, M{mom}, nullptr)
                                     : launch_list<D, M, true>(ctx, c, EPP_CRITERION_SYMMETRY, M{mom});
        };
        const int rc0 = gen ? mom_pass(std::true_type{}) : mom_pass(std::false_type{});
        if (rc0) return rc0;
        if (cfl) {
            ctx->graph_fluid = phys.fluid_tag;
            const int rc1 = launch_cfl<D, true>(ctx, c, phys.cfl, ctx->tbl[c], ctx->tbl[to]);
            if (rc1) return rc1;
        }
    }
    EPP_MARK(1);
    k_scan<<<ctx->n_tiles, kScanThreads, 0, ctx->stream>>>(ctx->n_cells + 1, ctx->count, ctx->start[to],
                                                          ctx->occ[to], ctx->meta[to], ctx->scan_state,
                                                          ctx->status);
    CK_LAUNCH();
    EPP_MARK(2);
    k_scatter<<<blocks_for(n), kThreads, 0, ctx->stream>>>(n, ctx->cs, ctx->start[to], ctx->S[c].id,
                                                           ctx->perm, ctx->status);
    CK_LAUNCH();
    EPP_MARK(3);
    MoverFused mv{ctx->S[c], ctx->S[to], mom.F, ctx->start[c], ctx->n_cells, phys.fluid_tag, phys.wall_tag};
    k_rank_gather<<<blocks_for(n), kThreads, 0, ctx->stream>>>(n, ctx->n_cells, ctx->perm, ctx->cs,
                                                               ctx->start[to], mv, ctx->status);
    CK_LAUNCH();
    EPP_MARK(4);
    int rc;
    if (ctx->lanes == 0 && uses_windows(ctx)) {   // 2D windows: one search pass with the continuity action
        rc = gen ? launch_pass<D, true>(ctx, to, EPP_CRITERION_SYMMETRY, CPCont<D, true, true>{ctx->S[to], Pn, ctx->ncnt[to]},
                                        ctx->pairs)
                 : launch_pass<D, true>(ctx, to, EPP_CRITERION_SYMMETRY, CPCont<D, true>{ctx->S[to], Pn, ctx->ncnt[to]},
                                        ctx->pairs);
        if (rc) return rc;
        EPP_MARK(5);
    } else if (ctx->lanes == 0) {   // search pass, then continuity over the new lists
        rc = launch_build<D>(ctx, to, EPP_CRITERION_SYMMETRY, ctx->pairs);
        if (rc) return rc;
        EPP_MARK(5);
        rc = gen ? launch_list<D>(ctx, to, EPP_CRITERION_SYMMETRY, CPCont<D, true, true>{ctx->S[to], Pn, ctx->ncnt[to]})
                 : launch_list<D>(ctx, to, EPP_CRITERION_SYMMETRY, CPCont<D, true>{ctx->S[to], Pn, ctx->ncnt[to]});
        if (rc) return rc;
    } else {
        rc = launch_search_pass<D>(ctx, to, EPP_CRITERION_SYMMETRY, EPP_ACTION_DAMBREAK_CONTINUITY, &phys, false,
                                   true);
        if (rc) return rc;
        EPP_MARK(5);
    }
    EPP_MARK(6);
    if (filter) {   // the kernel filter after this step's search (main.jl:180-183), family 0
        rc = launch_list<D>(ctx, to, EPP_CRITERION_SYMMETRY, CPFilter<D>{ctx->S[to], Pn, ctx->fwv, ctx->fwr});
        if (rc) return rc;
        k_filter_finish<D><<<blocks_for(n), kThreads, 0, ctx->stream>>>(ctx->start[to], ctx->n_cells, n, ctx->S[to],
                                                                        Pn, ctx->fwv, ctx->fwr, 1);
        CK_LAUNCH();
    }
    if (phys.wall_pressure == EPP_WALL_PRESSURE_EXTRAPOLATE) {   // wall pressure of the previewed density
        rc = launch_list<D>(ctx, to, EPP_CRITERION_SYMMETRY, CPExtrap<D, true>{ctx->S[to], Pn, nullptr, nullptr});
        if (rc) return rc;
    }
#undef EPP_MARK
    return EPP_OK;
}

// The fused momentum pass reads the neighbour lists of the last search: rebuild them (count-only
// search pass at the current positions) when the last search did not leave one.
template <int D>
int ensure_nlist(epp_ctx* ctx) {
    if (ctx->lanes != 0 || ctx->nlist_valid) return EPP_OK;
    int rc = launch_build<D>(ctx, ctx->cur, EPP_CRITERION_SYMMETRY, nullptr);
    if (rc == EPP_OK) ctx->nlist_valid = true;
    return rc;
}

void drop_graphs(epp_ctx* ctx) {
    for (int c = 0; c < 2; ++c) {
        if (ctx->graph[c]) {
            cudaGraphExecDestroy(ctx->graph[c]);
            ctx->graph[c] = nullptr;
        }
        if (ctx->graph_f[c]) {
            cudaGraphExecDestroy(ctx->graph_f[c]);
            ctx->graph_f[c] = nullptr;
        }
    }
}

template <int D>
int build_graphs(epp_ctx* ctx, const epp_physics& phys) {
    drop_graphs(ctx);
    for (int f = 0; f < (phys.filter_interval > 0 ? 2 : 1); ++f) {
        for (int c = 0; c < 2; ++c) {
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue_fused_step<D>(ctx, c, phys, nullptr, f == 1);
            cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
            if (rc) return rc;
            if (e != cudaSuccess) return fail(ctx, EPP_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
            e = cudaGraphInstantiate(f ? &ctx->graph_f[c] : &ctx->graph[c], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail(ctx, EPP_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        }
    }
    ctx->graph_phys = phys;
    return EPP_OK;
}

template <int D>
int run_selfaction(epp_ctx* ctx, int action, const epp_physics* phys) {
    if (phys && phys->cfl > 0.0f && !ctx->cfl_valid &&
        (action == EPP_ACTION_DAMBREAK_DENSITY || action == EPP_ACTION_DAMBREAK_INTEGRATE)) {
        const int rc = cfl_update<D>(ctx, *phys);   // the dt of the step that starts from this state
        if (rc) return rc;
    }
    DevPhys P = phys ? dev_phys(ctx, *phys) : DevPhys{};
    if (action == EPP_ACTION_KERNEL_FILTER_SELF) {
        k_filter_finish<D><<<blocks_for(ctx->n), kThreads, 0, ctx->stream>>>(
            ctx->start[ctx->cur], ctx->n_cells, ctx->n, ctx->S[ctx->cur], P, ctx->fwv, ctx->fwr, 0);
        CK_LAUNCH();
        ctx->filter_pending = false;
        return EPP_OK;
    }
    if (action == EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF) {
        k_extrap_finish<<<blocks_for(ctx->n), kThreads, 0, ctx->stream>>>(
            ctx->start[ctx->cur], ctx->n_cells, ctx->n, ctx->S[ctx->cur], P, ctx->fwv, ctx->fwp);
        CK_LAUNCH();
        ctx->extrap_pending = false;
        return EPP_OK;
    }
    k_self<D><<<blocks_for(ctx->n), kThreads, 0, ctx->stream>>>(action, ctx->start[ctx->cur], ctx->n_cells,
                                                                ctx->n, ctx->S[ctx->cur], P, ctx->status,
                                                                ctx->accel);
    CK_LAUNCH();
    return EPP_OK;
}

// interaction! with family 0: over the lists of the last search, rebuilt first when this order,
// these positions or the criterion no longer match them.
template <int D, class Act>
int launch_interaction_pass(epp_ctx* ctx, const Act& act) {
    if (!ctx->nlist_valid) {
        int rc = launch_build<D>(ctx, ctx->cur, ctx->last_crit, nullptr);
        if (rc) return rc;
        ctx->nlist_valid = true;
    }
    return launch_list<D>(ctx, ctx->cur, ctx->last_crit, act);
}

template <int D>
int run_interaction(epp_ctx* ctx, int action, const epp_physics* phys) {
    PairArgs A = pair_args(ctx, ctx->cur, ctx->last_crit);
    if (action == EPP_ACTION_KERNEL_FILTER) {
        if (ctx->lanes != 0) return fail(ctx, EPP_ERR_UNSUPPORTED_ACTION, "the kernel filter runs on pair-pass family 0");
        const int rc = launch_interaction_pass<D>(ctx, CPFilter<D>{ctx->S[ctx->cur], dev_phys(ctx, *phys), ctx->fwv, ctx->fwr});
        if (rc == EPP_OK) ctx->filter_pending = true;
        return rc;
    }
    if (action == EPP_ACTION_EXTRAPOLATE_PRESSURE) {
        if (ctx->lanes != 0)
            return fail(ctx, EPP_ERR_UNSUPPORTED_ACTION, "the pressure extrapolation runs on pair-pass family 0");
        const int rc = launch_interaction_pass<D>(
            ctx, CPExtrap<D, false>{ctx->S[ctx->cur], dev_phys(ctx, *phys), ctx->fwv, ctx->fwp});
        if (rc == EPP_OK) ctx->extrap_pending = true;
        return rc;
    }
    if (action == EPP_ACTION_DAMBREAK_MOMENTUM) {
        k_prep_rp4<<<blocks_for(ctx->n), kThreads, 0, ctx->stream>>>(ctx->start[ctx->cur], ctx->n_cells, ctx->n,
                                                                      ctx->S[ctx->cur]);
        CK_LAUNCH();
        ActMomG<D, false> act;
        act.s = ctx->S[ctx->cur];
        act.P = dev_phys(ctx, *phys);
        act.dom = ctx->dom;
        act.F = FusedOut{};
        act.status = ctx->status;
        if (ctx->lanes >= 2) return launch_pair_g<D, decltype(act), false>(ctx, A, act, nullptr, ctx->n);
        if (generic_physics(phys)) {
            if (ctx->lanes == 1) return launch_cellpair<D>(ctx, ctx->cur, ctx->last_crit, CPMom<D, false, true>{act}, nullptr);
            return launch_interaction_pass<D>(ctx, CPMom<D, false, true>{act});
        }
        if (ctx->lanes == 1) return launch_cellpair<D>(ctx, ctx->cur, ctx->last_crit, CPMom<D, false>{act}, nullptr);
        return launch_interaction_pass<D>(ctx, CPMom<D, false>{act});
    }
    if (ctx->lanes >= 2) {
        ActCountG<D> act{ctx->S[ctx->cur]};
        return launch_pair_g<D, decltype(act), false>(ctx, A, act, nullptr, ctx->n);
    }
    if (ctx->lanes == 1) return launch_cellpair<D>(ctx, ctx->cur, ctx->last_crit, CPCountDv<D>{ctx->S[ctx->cur]}, nullptr);
    return launch_interaction_pass<D>(ctx, CPCountDv<D>{ctx->S[ctx->cur]});
}

// Simulated time of `n` steps with a fixed dt (host bookkeeping; CFL steps add on the device).
void advance_fixed_time(epp_ctx* ctx, const epp_physics& phys, long long n) {
    for (int k = 0; k < ctx->n_inst; ++k)
        ctx->time_fixed[k] += (double)n * (double)(ctx->inst_dt.empty() ? phys.dt : ctx->inst_dt[k]);
}

template <int D>
int run_step(epp_ctx* ctx, int n_steps, const epp_physics& phys, bool accel) {
    int rc;
    const bool cfl = phys.cfl > 0.0f;
    if (ctx->inst_dirty) dev_phys(ctx, phys);   // upload the per-instance table the graphs read
    if (cfl) ensure_cfl_tables(ctx, phys);
    if (ctx->dv_dirty) {
        // the first step goes through the per-call kernels, which honour a non-zero dVelocity
        if ((rc = join_integrals(ctx))) return rc;
        rc = run_selfaction<D>(ctx, EPP_ACTION_DAMBREAK_DENSITY, &phys);
        if (!rc && phys.wall_pressure == EPP_WALL_PRESSURE_EXTRAPOLATE) {
            rc = run_interaction<D>(ctx, EPP_ACTION_EXTRAPOLATE_PRESSURE, &phys);
            if (!rc) rc = run_selfaction<D>(ctx, EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF, &phys);
        }
        if (!rc) rc = run_interaction<D>(ctx, EPP_ACTION_DAMBREAK_MOMENTUM, &phys);
        if (!rc) rc = run_selfaction<D>(ctx, EPP_ACTION_DAMBREAK_INTEGRATE, &phys);
        if (!rc) {
            ctx->cfl_valid = false;   // the velocities moved on
            if (cfl) {
                k_advance_time<<<1, 256, 0, ctx->stream>>>(ctx->n_inst, ctx->tbl[ctx->cur], ctx->sim_time);
                CK_LAUNCH();
            } else {
                advance_fixed_time(ctx, phys, 1);
            }
        }
        if (!rc) rc = run_search<D>(ctx, EPP_CRITERION_SYMMETRY, EPP_ACTION_DAMBREAK_CONTINUITY, &phys, false);
        if (rc) return rc;
        ++ctx->step_count;
        if (phys.filter_interval > 0 && ctx->step_count % phys.filter_interval == 0) {
            rc = run_interaction<D>(ctx, EPP_ACTION_KERNEL_FILTER, &phys);
            if (!rc) rc = run_selfaction<D>(ctx, EPP_ACTION_KERNEL_FILTER_SELF, &phys);
            if (rc) return rc;
            ctx->filter_pending = false;
            ctx->rpn_valid = false;
        }
        CK(cudaMemsetAsync(ctx->S[0].dv, 0, sizeof(float4) * ctx->cap, ctx->stream));
        CK(cudaMemsetAsync(ctx->S[1].dv, 0, sizeof(float4) * ctx->cap, ctx->stream));
        ctx->dv_dirty = false;
        --n_steps;
        if (n_steps == 0) return EPP_OK;
    }
    const bool extrap = phys.wall_pressure == EPP_WALL_PRESSURE_EXTRAPOLATE;
    if (cfl && !ctx->cfl_valid) {   // the graph's first step takes the CFL dt of this state
        rc = cfl_update<D>(ctx, phys);
        if (rc) return rc;
        ctx->rpn_valid = false;
    }
    if (!ctx->rpn_valid || !same_phys(ctx->rpn_phys, phys)) {
        k_density_preview<<<blocks_for(ctx->n), kThreads, 0, ctx->stream>>>(
            ctx->start[ctx->cur], ctx->n_cells, ctx->n, ctx->S[ctx->cur], dev_phys(ctx, phys));
        CK_LAUNCH();
        ctx->rpn_walls = false;
    }
    if (ctx->last_crit != EPP_CRITERION_SYMMETRY) ctx->nlist_valid = false;
    if (ctx->lanes == 0 && !ctx->nlist_valid && (rc = join_integrals(ctx, ctx->cur))) return rc;   // rewrites nCount
    rc = ensure_nlist<D>(ctx);
    if (rc) return rc;
    if (extrap && !ctx->rpn_walls) {   // the first step's wall pressure (later steps: the graph's tail)
        rc = launch_list<D>(ctx, ctx->cur, EPP_CRITERION_SYMMETRY,
                            CPExtrap<D, true>{ctx->S[ctx->cur], dev_phys(ctx, phys), nullptr, nullptr});
        if (rc) return rc;
    }
    if (!ctx->graph[0] || !same_phys(ctx->graph_phys, phys) || ctx->graph_accel != accel) {
        ctx->graph_accel = accel;
        rc = build_graphs<D>(ctx, phys);
        if (rc) return rc;
    }
    for (int s = 0; s < n_steps; ++s) {
        ++ctx->step_count;
        const bool f = phys.filter_interval > 0 && ctx->step_count % phys.filter_interval == 0;
        // a step reads set cur and writes set 1 - cur: integrals still reading set cur run on
        if ((rc = join_integrals(ctx, 1 - ctx->cur))) return rc;
        CK(cudaGraphLaunch(f ? ctx->graph_f[ctx->cur] : ctx->graph[ctx->cur], ctx->stream));
        ctx->cur = 1 - ctx->cur;
    }
    if (!cfl) advance_fixed_time(ctx, phys, n_steps);
    ctx->cfl_valid = cfl;   // each step's k_cfl left the dt of the state it produced
    ctx->rpn_valid = true;
    ctx->rpn_walls = extrap;
    ctx->rpn_phys = phys;
    ctx->searched = true;
    ctx->lists_valid = false;
    ctx->last_crit = EPP_CRITERION_SYMMETRY;
    ctx->nlist_valid = ctx->lanes == 0;
    return EPP_OK;
}

// The physics options a call may use with this context's pair-pass family.
int check_physics(epp_ctx* ctx, const epp_physics* p) {
    if (!p) return EPP_OK;
    if (p->kernel < EPP_KERNEL_WENDLAND_C2 || p->kernel > EPP_KERNEL_WENDLAND_C4 || p->eos < EPP_EOS_TAIT ||
        p->eos > EPP_EOS_LINEAR || p->motion < EPP_MOTION_SYMPLECTIC || p->motion > EPP_MOTION_ACCELERATE_MOVE ||
        p->viscosity < EPP_VISCOSITY_REFERENCE || p->viscosity > EPP_VISCOSITY_CLASSIC || p->filter_interval < 0)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "physics option out of range (kernel %d, eos %d, motion %d, "
                    "viscosity %d, filter_interval %d)", p->kernel, p->eos, p->motion, p->viscosity, p->filter_interval);
    if (ctx->lanes >= 2 && (p->kernel != EPP_KERNEL_WENDLAND_C2 || p->viscosity == EPP_VISCOSITY_CLASSIC))
        return fail(ctx, EPP_ERR_UNSUPPORTED_ACTION,
                    "the lane-group pair passes run Wendland C2 with artificial viscosity; use family 0 or 1");
    if (ctx->lanes != 0 && p->filter_interval > 0)
        return fail(ctx, EPP_ERR_UNSUPPORTED_ACTION, "the kernel filter runs on pair-pass family 0");
    if (p->pressure_ff < EPP_PRESSURE_DEFAULT || p->pressure_ff > EPP_PRESSURE_DENSITY_WEIGHTED ||
        p->pressure_fw < EPP_PRESSURE_DEFAULT || p->pressure_fw > EPP_PRESSURE_DENSITY_WEIGHTED ||
        (p->tensile != 0 && p->tensile != 1) || p->wall_pressure < EPP_WALL_PRESSURE_EOS ||
        p->wall_pressure > EPP_WALL_PRESSURE_EXTRAPOLATE)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "pressure option out of range (ff %d, fw %d, tensile %d, wall %d)",
                    p->pressure_ff, p->pressure_fw, p->tensile, p->wall_pressure);
    if (p->tensile && !ctx->has_gap)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "the tensile correction needs the Gap column (epp_column_map.gap)");
    if (ctx->lanes >= 2 && generic_physics(p))
        return fail(ctx, EPP_ERR_UNSUPPORTED_ACTION,
                    "the lane-group pair passes run the dam break's pressure terms; use family 0 or 1");
    if (ctx->lanes != 0 && p->wall_pressure == EPP_WALL_PRESSURE_EXTRAPOLATE)
        return fail(ctx, EPP_ERR_UNSUPPORTED_ACTION, "the pressure extrapolation runs on pair-pass family 0");
    if (!(p->cfl >= 0.0f && p->cfl < 1e30f))
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "cfl %g out of range", (double)p->cfl);
    if (ctx->lanes != 0 && p->cfl > 0.0f)
        return fail(ctx, EPP_ERR_UNSUPPORTED_ACTION, "the CFL time step runs on pair-pass family 0");
    return EPP_OK;
}

}  // namespace


// =========================================================================================
extern "C" {

int32_t epp_abi_version(void) { return EPP_ABI_VERSION; }

int32_t epp_device_count(int32_t* count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (count) *count = e == cudaSuccess ? n : 0;
    return e == cudaSuccess && n > 0 ? EPP_OK : EPP_ERR_NO_DEVICE;
}

const char* epp_last_error(const epp_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int32_t epp_create(const epp_config* cfg, epp_ctx** out) {
    if (!cfg || !out) return EPP_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    const int D = cfg->domain.dim;
    if ((D != 2 && D != 3) || cfg->n_capacity < 1 || cfg->n_tags < 1 || cfg->n_tags > EPP_MAX_TAGS ||
        !(cfg->domain.gap > 0.0f))
        return EPP_ERR_INVALID_ARGUMENT;
    if (cfg->n_capacity > (1 << kEntryBits)) return EPP_ERR_CAPACITY;   // list entries hold 28-bit indices
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return EPP_ERR_NO_DEVICE;
    if (cfg->device < 0 || cfg->device >= ndev) return EPP_ERR_INVALID_ARGUMENT;
    epp_ctx* ctx = new (std::nothrow) epp_ctx();
    if (!ctx) return EPP_ERR_OUT_OF_MEMORY;
    ctx->cfg = *cfg;
    if (ctx->cfg.max_neighbour_number <= 0) ctx->cfg.max_neighbour_number = 50;
    ctx->D = D;
    ctx->dev = cfg->device;
    ctx->cap = cfg->n_capacity;
    // domain in FP32 exactly as Domain2D (Domain2D.jl:34-66)
    DevDomain& d = ctx->dom;
    if (const int prc = plan_cells(cfg, d)) {
        delete ctx;
        return prc;
    }
    const int n_inst = d.n_inst;
    ctx->n_inst = n_inst;
    ctx->n_cells = d.n_cells;
    ctx->n_tiles = (ctx->n_cells + 1 + kScanTile - 1) / kScanTile;
    for (int a = 0; a < cfg->n_tags; ++a) {
        unsigned m = 0;
        for (int b = 0; b < cfg->n_tags; ++b)
            if (cfg->adjacency[a * EPP_MAX_TAGS + b] == 1) m |= 1u << b;
        ctx->adj[a] = m;
    }
    const size_t need = arena_bytes(ctx->cap, ctx->n_cells, D, ctx->n_tiles);
    if (cfg->hbm_budget_bytes > 0 && (long long)need > cfg->hbm_budget_bytes) {
        delete ctx;
        return EPP_ERR_BUDGET;
    }
    if (cudaSetDevice(ctx->dev) != cudaSuccess) {
        delete ctx;
        return EPP_ERR_CUDA;
    }
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        cudaGetLastError();
        return EPP_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, ctx->dev);
    if (dev_alloc(ctx, &ctx->arena.base, need) != cudaSuccess) {
        cudaGetLastError();
        epp_destroy(ctx);
        return EPP_ERR_OUT_OF_MEMORY;
    }
    ctx->arena.size = need;
    Arena& a = ctx->arena;
    fill_state(a, ctx->S[0], ctx->cap);
    fill_state(a, ctx->S[1], ctx->cap);
    ctx->tmp.xh = a.take<float4>(ctx->cap);
    ctx->tmp.vm = a.take<float4>(ctx->cap);
    ctx->tmp.comp = a.take<float4>(ctx->cap);
    ctx->count = a.take<int>(ctx->n_cells + 2);
    ctx->start[0] = a.take<int>(ctx->n_cells + 2);
    ctx->start[1] = a.take<int>(ctx->n_cells + 2);
    ctx->occ[0] = a.take<int>(ctx->n_cells + 1);
    ctx->occ[1] = a.take<int>(ctx->n_cells + 1);
    ctx->meta[0] = a.take<int>(64);
    ctx->meta[1] = a.take<int>(64);
    ctx->cs = a.take<int2>(ctx->cap);
    ctx->perm = a.take<int2>(ctx->cap);
    ctx->scan_state = a.take<unsigned long long>(ctx->n_tiles + 1);
    ctx->status = a.take<unsigned>(1);
    ctx->pairs = a.take<unsigned long long>(1);
    ctx->ncnt[0] = a.take<int>(ctx->cap);
    ctx->ncnt[1] = a.take<int>(ctx->cap);
    ctx->stage_f = a.take<float>((size_t)ctx->cap * (3 * D + 6));
    ctx->stage_i = a.take<int>((size_t)ctx->cap * SI_COUNT);
    ctx->ipartial = a.take<double>(kIntegralBlocks * 8);
    ctx->iresult = a.take<double>(8);
    ctx->iticket = a.take<unsigned>(1);
    ctx->fwv = a.take<float>(ctx->cap);
    ctx->fwp = a.take<float>(ctx->cap);
    ctx->gap = a.take<float>(ctx->cap);
    ctx->fwr = a.take<float>(ctx->cap);
    ctx->tmp.count = ctx->count;
    ctx->tmp.cs = ctx->cs;
    ctx->tmp.scan_state = ctx->scan_state;
    ctx->tmp.n_scan_words = ctx->n_tiles + 1;
    ctx->tmp.accel = nullptr;
    if (!ctx->fwr) {   // the last part taken: the arena held everything
        epp_destroy(ctx);
        return EPP_ERR_OUT_OF_MEMORY;
    }
    if (cfg->hbm_budget_bytes > 0 && (long long)(need + nlist_bytes(D, ctx->cap)) > cfg->hbm_budget_bytes) {
        epp_destroy(ctx);
        return EPP_ERR_BUDGET;
    }
    ctx->cfl_chunks = std::max(1, (4 * ctx->sms) / n_inst);
    ctx->time_fixed.assign(n_inst, 0.0);
    if (dev_alloc(ctx, &ctx->nlist, nlist_bytes(D, ctx->cap)) != cudaSuccess ||
        dev_alloc(ctx, &ctx->inst_table, sizeof(InstPhys) * n_inst) != cudaSuccess ||
        dev_alloc(ctx, &ctx->inst_out, sizeof(double) * 9 * n_inst) != cudaSuccess ||
        dev_alloc(ctx, &ctx->tbl[0], sizeof(InstPhys) * n_inst) != cudaSuccess ||
        dev_alloc(ctx, &ctx->tbl[1], sizeof(InstPhys) * n_inst) != cudaSuccess ||
        dev_alloc(ctx, &ctx->cfl_partial, sizeof(double2) * n_inst * ctx->cfl_chunks) != cudaSuccess ||
        dev_alloc(ctx, &ctx->cfl_ticket, sizeof(unsigned)) != cudaSuccess ||
        dev_alloc(ctx, &ctx->sim_time, sizeof(double) * n_inst) != cudaSuccess) {
        cudaGetLastError();
        epp_destroy(ctx);
        return EPP_ERR_OUT_OF_MEMORY;
    }
    // zeroed lists: a list slot read before any search wrote it holds index 0, in bounds
    if (cudaMemsetAsync(ctx->arena.base, 0, need, ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(ctx->nlist, 0, nlist_bytes(D, ctx->cap), ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(ctx->cfl_ticket, 0, sizeof(unsigned), ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(ctx->sim_time, 0, sizeof(double) * n_inst, ctx->stream) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        epp_destroy(ctx);
        return EPP_ERR_CUDA;
    }
    if ((D == 2 ? prepare_kernels<2>(ctx) : prepare_kernels<3>(ctx)) != EPP_OK) {
        epp_destroy(ctx);
        return EPP_ERR_CUDA;
    }
    *out = ctx;
    return EPP_OK;
}

int32_t epp_destroy(epp_ctx* ctx) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->dev);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->istream) cudaStreamSynchronize(ctx->istream);
    ctx->stream = ctx->own_stream;   // the frees below are ordered on the context's own stream
    drop_graphs(ctx);
    dev_free(ctx, ctx->accel);
    dev_free(ctx, ctx->inst_table);
    dev_free(ctx, ctx->nlist);
    dev_free(ctx, ctx->inst_out);
    dev_free(ctx, ctx->tbl[0]);
    dev_free(ctx, ctx->tbl[1]);
    dev_free(ctx, ctx->cfl_partial);
    dev_free(ctx, ctx->cfl_ticket);
    dev_free(ctx, ctx->sim_time);
    dev_free(ctx, ctx->list_mem);
    dev_free(ctx, ctx->list_stage);
    dev_free(ctx, ctx->arena.base);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    for (int k = 0; k < EPP_INTEGRALS_SLOTS; ++k)
        if (ctx->iev[k]) cudaEventDestroy(ctx->iev[k]);
    if (ctx->ihost) cudaFreeHost(ctx->ihost);
    if (ctx->iready) cudaEventDestroy(ctx->iready);
    for (int k = 0; k < 2; ++k)
        if (ctx->idone[k]) cudaEventDestroy(ctx->idone[k]);
    if (ctx->istream) cudaStreamDestroy(ctx->istream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return EPP_OK;
}

int32_t epp_upload(epp_ctx* ctx, int32_t n, const int32_t* is_alive, const int32_t* cell_index,
                   const int32_t* ip, int64_t ldi, const float* fp, int64_t ldf,
                   const epp_column_map* m) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    if (!is_alive || !ip || !fp || !m || n < 0) return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "null argument");
    if (n > ctx->cap) return fail(ctx, EPP_ERR_CAPACITY, "%d particles > capacity %d", n, ctx->cap);
    if (m->tag < 0 || m->position < 0)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "Tag and PositionVec columns are required");
    if (ldi < n || ldf < n) return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "leading dimension < n");
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    const int D = ctx->D;
    const bool same_n = n == ctx->n;
    ctx->n = n;
    if (n == 0) {
        drop_graphs(ctx);
        ctx->searched = false;
        return EPP_OK;
    }
    auto fcol = [&](int stage_col, int user_col, int width, float fill) -> int {
        for (int k = 0; k < width; ++k) {
            float* dst = ctx->stage_f + (size_t)(stage_col + k) * n;
            if (user_col >= 0) {
                CK(cudaMemcpyAsync(dst, fp + (size_t)(user_col + k) * ldf, (size_t)n * 4,
                                   cudaMemcpyHostToDevice, ctx->stream));
            } else if (fill == 0.0f) {
                CK(cudaMemsetAsync(dst, 0, (size_t)n * 4, ctx->stream));
            } else {
                std::vector<float> h(n, fill);
                CK(cudaMemcpyAsync(dst, h.data(), (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
                CK(cudaStreamSynchronize(ctx->stream));
            }
        }
        return EPP_OK;
    };
    auto icol = [&](int stage_col, const int32_t* src, int fill) -> int {
        int* dst = ctx->stage_i + (size_t)stage_col * n;
        if (src) {
            CK(cudaMemcpyAsync(dst, src, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
        } else if (fill == 0) {
            CK(cudaMemsetAsync(dst, 0, (size_t)n * 4, ctx->stream));
        } else {
            std::vector<int> h(n, fill);
            CK(cudaMemcpyAsync(dst, h.data(), (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
        }
        return EPP_OK;
    };
    int rc = 0;
    rc |= fcol(0, m->position, D, 0.0f);
    rc |= fcol(sf_vel(D), m->velocity, D, 0.0f);
    rc |= fcol(sf_dvel(D), m->dvelocity, D, 0.0f);
    rc |= fcol(sf_mass(D), m->mass, 1, 0.0f);
    rc |= fcol(sf_vol(D), m->volume, 1, 0.0f);
    rc |= fcol(sf_rho(D), m->density, 1, 0.0f);
    rc |= fcol(sf_drho(D), m->ddensity, 1, 0.0f);
    rc |= fcol(sf_p(D), m->pressure, 1, 0.0f);
    rc |= fcol(sf_h(D), m->h, 1, 0.0f);
    rc |= icol(SI_TAG, ip + (size_t)m->tag * ldi, 0);
    rc |= icol(SI_MOV, m->is_movable >= 0 ? ip + (size_t)m->is_movable * ldi : nullptr, 1);
    rc |= icol(SI_NCOUNT, m->n_count >= 0 ? ip + (size_t)m->n_count * ldi : nullptr, 0);
    rc |= icol(SI_ALIVE, is_alive, 0);
    rc |= icol(SI_CELL, cell_index, 0);
    if (m->instance >= 0) {
        const int32_t* ic = ip + (size_t)m->instance * ldi;
        for (int k = 0; k < n; ++k)
            if (ic[k] < 0 || ic[k] >= ctx->n_inst)
                return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "particle %d: instance %d outside 0..%d", k, ic[k],
                            ctx->n_inst - 1);
        rc |= icol(SI_INST, ic, 0);
    } else {
        rc |= icol(SI_INST, nullptr, 0);
    }
    {
        const int32_t* tc = ip + (size_t)m->tag * ldi;
        for (int k = 0; k < n; ++k)
            if (tc[k] < 0 || tc[k] > 255) return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "tag %d out of range", tc[k]);
    }
    if (rc) return rc;
    ctx->cur = 0;
    auto launch = [&](auto Dt) {
        constexpr int DD = decltype(Dt)::value;
        k_unpack<DD><<<blocks_for(n), kThreads, 0, ctx->stream>>>(n, ctx->n_cells, ctx->stage_f, ctx->stage_i,
                                                                  ctx->S[0], ctx->ncnt[0]);
    };
    if (D == 2) launch(std::integral_constant<int, 2>{});
    else launch(std::integral_constant<int, 3>{});
    CK_LAUNCH();
    // the captured step graphs hold the particle count (grid sizes, bounds) and otherwise only the
    // context's own buffers: they stay valid for an upload of the same count
    if (!same_n) drop_graphs(ctx);
    CK(cudaMemsetAsync(ctx->fwv, 0, sizeof(float) * ctx->cap, ctx->stream));
    CK(cudaMemsetAsync(ctx->fwr, 0, sizeof(float) * ctx->cap, ctx->stream));
    CK(cudaMemsetAsync(ctx->fwp, 0, sizeof(float) * ctx->cap, ctx->stream));
    ctx->has_gap = m->gap >= 0;   // Gap per caller row: the pair passes index it by State::id
    if (ctx->has_gap)
        CK(cudaMemcpyAsync(ctx->gap, fp + (size_t)m->gap * ldf, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
    else
        CK(cudaMemsetAsync(ctx->gap, 0, sizeof(float) * ctx->cap, ctx->stream));
    ctx->filter_pending = false;
    ctx->extrap_pending = false;
    ctx->rpn_walls = false;
    ctx->step_count = 0;
    ctx->cfl_valid = false;
    ctx->time_fixed.assign(ctx->n_inst, 0.0);
    CK(cudaMemsetAsync(ctx->sim_time, 0, sizeof(double) * ctx->n_inst, ctx->stream));
    ctx->searched = false;
    ctx->sorted_once = false;
    ctx->nlist_valid = false;
    ctx->lists_valid = false;
    ctx->rpn_valid = false;
    ctx->dv_dirty = true;
    return EPP_OK;
}

int32_t epp_download(epp_ctx* ctx, int32_t* is_alive, int32_t* cell_index, int32_t* ip, int64_t ldi,
                     float* fp, int64_t ldf, const epp_column_map* m) {
    if (!ctx || !m) return EPP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    const int D = ctx->D, n = ctx->n;
    if (n == 0) return EPP_OK;
    if ((ip && ldi < n) || (fp && ldf < n)) return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "leading dimension < n");
    auto launch = [&](auto Dt) {
        constexpr int DD = decltype(Dt)::value;
        k_pack<DD><<<blocks_for(n), kThreads, 0, ctx->stream>>>(n, ctx->n_cells, ctx->stage_f, ctx->stage_i,
                                                                ctx->S[ctx->cur], ctx->ncnt[ctx->cur]);
    };
    if (D == 2) launch(std::integral_constant<int, 2>{});
    else launch(std::integral_constant<int, 3>{});
    CK_LAUNCH();
    auto fget = [&](int stage_col, int user_col, int width) -> int {
        if (!fp || user_col < 0) return EPP_OK;
        for (int k = 0; k < width; ++k)
            CK(cudaMemcpyAsync(fp + (size_t)(user_col + k) * ldf, ctx->stage_f + (size_t)(stage_col + k) * n,
                               (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream));
        return EPP_OK;
    };
    auto iget = [&](int stage_col, int32_t* dst) -> int {
        if (!dst) return EPP_OK;
        CK(cudaMemcpyAsync(dst, ctx->stage_i + (size_t)stage_col * n, (size_t)n * 4, cudaMemcpyDeviceToHost,
                           ctx->stream));
        return EPP_OK;
    };
    int rc = 0;
    rc |= fget(0, m->position, D);
    rc |= fget(sf_vel(D), m->velocity, D);
    rc |= fget(sf_dvel(D), m->dvelocity, D);
    rc |= fget(sf_mass(D), m->mass, 1);
    rc |= fget(sf_vol(D), m->volume, 1);
    rc |= fget(sf_rho(D), m->density, 1);
    rc |= fget(sf_drho(D), m->ddensity, 1);
    rc |= fget(sf_p(D), m->pressure, 1);
    rc |= fget(sf_h(D), m->h, 1);
    rc |= iget(SI_ALIVE, is_alive);
    rc |= iget(SI_CELL, cell_index);
    if (ip) {
        if (m->tag >= 0) rc |= iget(SI_TAG, ip + (size_t)m->tag * ldi);
        if (m->is_movable >= 0) rc |= iget(SI_MOV, ip + (size_t)m->is_movable * ldi);
        if (m->n_count >= 0) rc |= iget(SI_NCOUNT, ip + (size_t)m->n_count * ldi);
        if (m->instance >= 0) rc |= iget(SI_INST, ip + (size_t)m->instance * ldi);
    }
    if (rc) return rc;
    const bool want_lists = ctx->lists_valid && ((ip && m->n_index >= 0) ||
                            (fp && (m->n_rvec >= 0 || m->n_r >= 0 || m->n_w >= 0 || m->n_dw >= 0 || m->n_hinv >= 0)));
    if (want_lists) {
        const size_t nb = ctx->L.max_nb;
        int* nidx = (int*)ctx->list_stage;
        float* nrvec = (float*)(nidx + nb * n);
        float* nr = nrvec + nb * D * n;
        float* nw = nr + nb * n;
        float* ndw = nw + nb * n;
        float* nh = ndw + nb * n;
        auto launch2 = [&](auto Dt) {
            constexpr int DD = decltype(Dt)::value;
            k_pack_lists<DD><<<blocks_for(n), kThreads, 0, ctx->stream>>>(n, ctx->L, ctx->S[ctx->cur].id,
                                                                          ctx->ncnt[ctx->cur], nidx, nrvec, nr, nw, ndw, nh);
        };
        if (D == 2) launch2(std::integral_constant<int, 2>{});
        else launch2(std::integral_constant<int, 3>{});
        CK_LAUNCH();
        auto cols = [&](const void* src, void* dstbase, int user_col, int64_t ld, int ncols) -> int {
            if (user_col < 0 || !dstbase) return EPP_OK;
            for (int k = 0; k < ncols; ++k)
                CK(cudaMemcpyAsync((char*)dstbase + ((size_t)(user_col + k) * ld) * 4,
                                   (const char*)src + (size_t)k * n * 4, (size_t)n * 4,
                                   cudaMemcpyDeviceToHost, ctx->stream));
            return EPP_OK;
        };
        rc |= cols(nidx, ip, ip ? m->n_index : -1, ldi, (int)nb);
        rc |= cols(nrvec, fp, fp ? m->n_rvec : -1, ldf, (int)(nb * D));
        rc |= cols(nr, fp, fp ? m->n_r : -1, ldf, (int)nb);
        rc |= cols(nw, fp, fp ? m->n_w : -1, ldf, (int)nb);
        rc |= cols(ndw, fp, fp ? m->n_dw : -1, ldf, (int)nb);
        rc |= cols(nh, fp, fp ? m->n_hinv : -1, ldf, (int)nb);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return EPP_OK;
}

int32_t epp_search(epp_ctx* ctx, int32_t criterion, int32_t action, const epp_physics* phys, int32_t flags) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    if (criterion != EPP_CRITERION_DEFAULT && criterion != EPP_CRITERION_SYMMETRY)
        return fail(ctx, EPP_ERR_UNSUPPORTED_CRITERION, "criterion %d", criterion);
    if (action != EPP_ACTION_NONE && action != EPP_ACTION_DAMBREAK_CONTINUITY)
        return fail(ctx, EPP_ERR_UNSUPPORTED_ACTION, "search action %d", action);
    if (action == EPP_ACTION_DAMBREAK_CONTINUITY && !phys)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "physics required");
    if (const int prc = check_physics(ctx, phys)) return prc;
    if (ctx->filter_pending)
        return fail(ctx, EPP_ERR_STATE, "kernel-filter sums pending: selfaction!(KERNEL_FILTER_SELF) first");
    if (ctx->extrap_pending)
        return fail(ctx, EPP_ERR_STATE, "extrapolation sums pending: selfaction!(EXTRAPOLATE_PRESSURE_SELF) first");
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    if (ctx->n == 0) return EPP_OK;
    const bool emit = (flags & EPP_SEARCH_EMIT_LIST) != 0;
    return ctx->D == 2 ? run_search<2>(ctx, criterion, action, phys, emit)
                       : run_search<3>(ctx, criterion, action, phys, emit);
}

int32_t epp_interaction(epp_ctx* ctx, int32_t action, const epp_physics* phys) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    if (action == EPP_ACTION_NONE) return EPP_OK;
    if (action != EPP_ACTION_DAMBREAK_MOMENTUM && action != EPP_ACTION_COUNT_NEIGHBOURS &&
        action != EPP_ACTION_KERNEL_FILTER && action != EPP_ACTION_EXTRAPOLATE_PRESSURE)
        return fail(ctx, EPP_ERR_UNSUPPORTED_ACTION, "interaction action %d", action);
    if (action != EPP_ACTION_COUNT_NEIGHBOURS && !phys)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "physics required");
    if (const int prc = check_physics(ctx, phys)) return prc;
    if (!ctx->searched)
        return fail(ctx, EPP_ERR_STATE, "interaction! needs a search! at the current positions");
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    if (ctx->n == 0) return EPP_OK;
    ctx->dv_dirty = true;
    return ctx->D == 2 ? run_interaction<2>(ctx, action, phys) : run_interaction<3>(ctx, action, phys);
}

int32_t epp_selfaction(epp_ctx* ctx, int32_t action, const epp_physics* phys) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    if (action == EPP_ACTION_NONE) return EPP_OK;
    if (action != EPP_ACTION_DAMBREAK_DENSITY && action != EPP_ACTION_DAMBREAK_INTEGRATE &&
        action != EPP_ACTION_ZERO_DVELOCITY && action != EPP_ACTION_KERNEL_FILTER_SELF &&
        action != EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF)
        return fail(ctx, EPP_ERR_UNSUPPORTED_ACTION, "selfaction action %d", action);
    if (action != EPP_ACTION_ZERO_DVELOCITY && !phys)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "physics required");
    if (const int prc = check_physics(ctx, phys)) return prc;
    if (!ctx->sorted_once)
        return fail(ctx, EPP_ERR_STATE, "selfaction! runs on the cell-sorted state: call search! first");
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    if (ctx->n == 0) return EPP_OK;
    int rc = ctx->D == 2 ? run_selfaction<2>(ctx, action, phys) : run_selfaction<3>(ctx, action, phys);
    if (action == EPP_ACTION_DAMBREAK_INTEGRATE) {
        ctx->nlist_valid = false;
        ctx->searched = false;   // positions moved: the next pass needs a search!
        ctx->rpn_valid = false;
        ctx->cfl_valid = false;
    }
    if (action == EPP_ACTION_DAMBREAK_DENSITY || action == EPP_ACTION_KERNEL_FILTER_SELF ||
        action == EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF)
        ctx->rpn_valid = false;
    if (action == EPP_ACTION_ZERO_DVELOCITY) ctx->dv_dirty = true;
    ctx->lists_valid = ctx->lists_valid && action != EPP_ACTION_DAMBREAK_INTEGRATE;
    return rc;
}

int32_t epp_step(epp_ctx* ctx, int32_t n_steps, const epp_physics* phys) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    if (!phys || n_steps < 0) return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "bad arguments");
    if (const int prc = check_physics(ctx, phys)) return prc;
    if (ctx->filter_pending)
        return fail(ctx, EPP_ERR_STATE, "kernel-filter sums pending: selfaction!(KERNEL_FILTER_SELF) first");
    if (ctx->extrap_pending)
        return fail(ctx, EPP_ERR_STATE, "extrapolation sums pending: selfaction!(EXTRAPOLATE_PRESSURE_SELF) first");
    if (!ctx->searched)
        return fail(ctx, EPP_ERR_STATE, "epp_step needs an initial search! (main.jl:157-164)");
    cudaSetDevice(ctx->dev);
    if (n_steps == 0 || ctx->n == 0) return EPP_OK;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    int rc = ctx->D == 2 ? run_step<2>(ctx, n_steps, *phys, ctx->accel != nullptr)
                         : run_step<3>(ctx, n_steps, *phys, ctx->accel != nullptr);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->timed = true;
    return EPP_OK;
}

namespace {

// k_integrals of the current set on stream `st`: the 8 results land in ctx->iresult.
int launch_integrals(epp_ctx* ctx, const epp_physics* phys, cudaStream_t st) {
    IntegralsOut O{ctx->ipartial, ctx->iresult, ctx->iticket};
    DevPhys P = dev_phys(ctx, *phys);
    auto launch = [&](auto Dt) {
        constexpr int DD = decltype(Dt)::value;
        k_integrals<DD><<<kIntegralBlocks, 256, 0, st>>>(
            ctx->start[ctx->cur], ctx->n_cells, ctx->n, ctx->S[ctx->cur], ctx->ncnt[ctx->cur], P, phys->rho0, phys->c0,
            phys->gamma, phys->p0,
            phys->gravity[0], phys->gravity[1], phys->gravity[2], O);
    };
    if (ctx->D == 2) launch(std::integral_constant<int, 2>{});
    else launch(std::integral_constant<int, 3>{});
    CK_LAUNCH();
    return EPP_OK;
}

void fill_integrals(epp_integrals* out, const double* r, int n_alive, float c0, float cfl) {
    out->mass_total = r[0];
    out->mass_fluid = r[1];
    out->kinetic = r[2];
    out->potential = r[3];
    out->internal = r[4];
    out->max_speed = r[5];
    out->cfl_dt = r[6] < 1e300 ? (cfl > 0.0f ? (double)cfl : 0.1) * r[6] / ((double)c0 + r[5]) : 0.0;
    out->n_alive = n_alive;
    out->n_pairs = (int64_t)r[7];   // directed pairs of the last search = sum of nCount over alive particles
}

}  // namespace

int32_t epp_get_integrals(epp_ctx* ctx, const epp_physics* phys, epp_integrals* out) {
    if (!ctx || !phys || !out) return EPP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    std::memset(out, 0, sizeof *out);
    if (ctx->n == 0) return EPP_OK;
    if (!ctx->sorted_once) return fail(ctx, EPP_ERR_STATE, "integrals need a search! first");
    if (const int rc = launch_integrals(ctx, phys, ctx->stream)) return rc;
    double r[8];
    int n_alive = 0;
    CK(cudaMemcpyAsync(r, ctx->iresult, 8 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&n_alive, ctx->start[ctx->cur] + ctx->n_cells, sizeof(int), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    fill_integrals(out, r, n_alive, phys->c0, phys->cfl);
    return EPP_OK;
}

int32_t epp_integrals_async(epp_ctx* ctx, const epp_physics* phys, int64_t* ticket) {
    if (!ctx || !phys || !ticket) return EPP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->dev);
    if (ctx->n > 0 && !ctx->sorted_once) return fail(ctx, EPP_ERR_STATE, "integrals need a search! first");
    const long long t = ctx->iticket_next;
    const int slot = (int)(t % EPP_INTEGRALS_SLOTS);
    if (ctx->islot_ticket[slot] >= 0)
        return fail(ctx, EPP_ERR_STATE, "%d integrals tickets outstanding: wait for one first", EPP_INTEGRALS_SLOTS);
    if (!ctx->ihost) {   // pinned slots, the second stream and its events on first use
        CK(cudaMallocHost(reinterpret_cast<void**>(&ctx->ihost), sizeof(double) * 9 * EPP_INTEGRALS_SLOTS));
        for (int k = 0; k < EPP_INTEGRALS_SLOTS; ++k) CK(cudaEventCreateWithFlags(&ctx->iev[k], cudaEventDisableTiming));
        int prio = 0;
        CK(cudaStreamGetPriority(ctx->stream, &prio));
        CK(cudaStreamCreateWithPriority(&ctx->istream, cudaStreamNonBlocking, prio));
        CK(cudaEventCreateWithFlags(&ctx->iready, cudaEventDisableTiming));
        for (int k = 0; k < 2; ++k) CK(cudaEventCreateWithFlags(&ctx->idone[k], cudaEventDisableTiming));
    }
    double* h = ctx->ihost + 9 * slot;
    // the second stream starts once the state is complete on the context's stream, and the next
    // epp_step runs meanwhile (it reads this set and writes the other)
    dev_phys(ctx, *phys);   // any table upload it needs goes first, on the context's stream
    CK(cudaEventRecord(ctx->iready, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->istream, ctx->iready, 0));
    if (ctx->n == 0) {
        for (int k = 0; k < 9; ++k) h[k] = 0.0;
        h[6] = 1e300;
    } else {
        if (const int rc = launch_integrals(ctx, phys, ctx->istream)) return rc;
        CK(cudaMemcpyAsync(h, ctx->iresult, 8 * sizeof(double), cudaMemcpyDeviceToHost, ctx->istream));
        CK(cudaMemcpyAsync(h + 8, ctx->start[ctx->cur] + ctx->n_cells, sizeof(int), cudaMemcpyDeviceToHost,
                           ctx->istream));
        CK(cudaEventRecord(ctx->idone[ctx->cur], ctx->istream));
        ctx->ipending[ctx->cur] = true;
    }
    CK(cudaEventRecord(ctx->iev[slot], ctx->istream));
    ctx->islot_ticket[slot] = t;
    ctx->islot_c0[slot] = phys->c0;
    ctx->islot_cfl[slot] = phys->cfl;
    ctx->iticket_next = t + 1;
    *ticket = t;
    return EPP_OK;
}

int32_t epp_integrals_wait(epp_ctx* ctx, int64_t ticket, epp_integrals* out) {
    if (!ctx || !out) return EPP_ERR_INVALID_ARGUMENT;
    const int slot = ticket >= 0 ? (int)(ticket % EPP_INTEGRALS_SLOTS) : 0;
    if (ticket < 0 || ctx->islot_ticket[slot] != ticket)
        return fail(ctx, EPP_ERR_STATE, "integrals ticket %lld is not outstanding", (long long)ticket);
    cudaSetDevice(ctx->dev);
    CK(cudaEventSynchronize(ctx->iev[slot]));
    const double* h = ctx->ihost + 9 * slot;
    int n_alive = 0;
    std::memcpy(&n_alive, h + 8, sizeof n_alive);
    std::memset(out, 0, sizeof *out);
    fill_integrals(out, h, n_alive, ctx->islot_c0[slot], ctx->islot_cfl[slot]);
    ctx->islot_ticket[slot] = -1;
    return EPP_OK;
}

int32_t epp_cell_stats(epp_ctx* ctx, int32_t* counts, int32_t* offsets, int32_t* sorted_ids, int32_t* n_cells) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    if (n_cells) *n_cells = ctx->n_cells;
    if (!counts && !offsets && !sorted_ids) return EPP_OK;
    if (!ctx->searched) return fail(ctx, EPP_ERR_STATE, "no cell list: call search! first");
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    std::vector<int> st(ctx->n_cells + 2);
    CK(cudaMemcpyAsync(st.data(), ctx->start[ctx->cur], sizeof(int) * (ctx->n_cells + 1), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const int n_alive = st[ctx->n_cells];
    if (counts)
        for (int c = 0; c < ctx->n_cells; ++c) counts[c] = st[c + 1] - st[c];
    if (offsets)
        for (int c = 0; c <= ctx->n_cells; ++c) offsets[c] = st[c];
    if (sorted_ids && n_alive > 0) {
        CK(cudaMemcpy(sorted_ids, ctx->S[ctx->cur].id, sizeof(int) * n_alive, cudaMemcpyDeviceToHost));
        for (int k = 0; k < n_alive; ++k) sorted_ids[k] += 1;
    }
    return EPP_OK;
}

int32_t epp_neighbour_lists(epp_ctx* ctx, int32_t* counts, int32_t* ids, int64_t ld, int32_t max_nb) {
    if (!ctx || !counts) return EPP_ERR_INVALID_ARGUMENT;
    if (ids && (max_nb < 0 || ld < ctx->n)) return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "ld < n or max_nb < 0");
    if (ctx->lanes != 0 || !ctx->nlist_valid)
        return fail(ctx, EPP_ERR_STATE, "no neighbour lists of the search pass (family 0, after a search or step)");
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    const int n = ctx->n;
    if (n == 0) return EPP_OK;
    const int lcap = ctx->D == 2 ? ListConf<2>::LCAP : ListConf<3>::LCAP;
    const bool row_major = ctx->D == 2 ? ListConf<2>::ROW : ListConf<3>::ROW;
    int n_alive = 0;
    CK(cudaMemcpyAsync(&n_alive, ctx->start[ctx->cur] + ctx->n_cells, sizeof(int), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    n_alive = n_alive < 0 ? 0 : n_alive > n ? n : n_alive;
    std::vector<int> id(n_alive > 0 ? n_alive : 1), cnt(n_alive > 0 ? n_alive : 1);
    std::vector<int> list((size_t)lcap * ctx->cap);
    if (n_alive > 0) {
        CK(cudaMemcpyAsync(id.data(), ctx->S[ctx->cur].id, sizeof(int) * n_alive, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(cnt.data(), ctx->ncnt[ctx->cur], sizeof(int) * n_alive, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(list.data(), ctx->nlist, sizeof(int) * list.size(), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    for (int r = 0; r < n; ++r) counts[r] = 0;   // particles not alive have no list
    for (int i = 0; i < n_alive; ++i) {
        const int row = id[i];
        if (row < 0 || row >= n) return fail(ctx, EPP_ERR_DEVICE_STATUS, "sorted particle %d has id %d", i, row);
        counts[row] = cnt[i];
        if (!ids) continue;
        if (cnt[i] > lcap) continue;   // beyond the list's capacity: read from its stencil, not stored
        const int kept = std::min(cnt[i], (int)max_nb);
        for (int k = 0; k < kept; ++k) {
            const int e = row_major ? list[(size_t)i * lcap + k] : list[(size_t)k * ctx->cap + i];
            const int j = e & ((1 << kEntryBits) - 1);
            if (j >= n_alive) return fail(ctx, EPP_ERR_DEVICE_STATUS, "list entry %d of particle %d: index %d", k, i, j);
            ids[(size_t)k * ld + row] = id[j] + 1;
        }
    }
    return EPP_OK;
}

int32_t epp_synchronize(epp_ctx* ctx, uint32_t* device_status) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned st = 0;
    CK(cudaMemcpy(&st, ctx->status, sizeof st, cudaMemcpyDeviceToHost));
    CK(cudaMemset(ctx->status, 0, sizeof st));
    if (device_status) *device_status = st;
    if (st & ~(unsigned)EPP_STATUS_KILLED)
        return fail(ctx, EPP_ERR_DEVICE_STATUS, "device status 0x%x", st);
    return EPP_OK;
}

int32_t epp_step_dt(epp_ctx* ctx, const epp_physics* phys, int32_t n, float* next_dt, double* sim_time) {
    if (!ctx || !phys) return EPP_ERR_INVALID_ARGUMENT;
    if (n != ctx->n_inst) return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "n = %d, context has %d instances", n, ctx->n_inst);
    if (const int prc = check_physics(ctx, phys)) return prc;
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    if (next_dt) {
        if (phys->cfl > 0.0f && ctx->n > 0) {
            if (!ctx->sorted_once) return fail(ctx, EPP_ERR_STATE, "the CFL time step needs a search! first");
            ensure_cfl_tables(ctx, *phys);
            if (!ctx->cfl_valid) {
                const int rc = ctx->D == 2 ? cfl_update<2>(ctx, *phys) : cfl_update<3>(ctx, *phys);
                if (rc) return rc;
            }
            std::vector<InstPhys> t(n);
            CK(cudaMemcpyAsync(t.data(), ctx->tbl[ctx->cur], sizeof(InstPhys) * n, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            for (int k = 0; k < n; ++k) next_dt[k] = t[k].dt;
        } else {
            for (int k = 0; k < n; ++k) next_dt[k] = ctx->inst_dt.empty() ? phys->dt : ctx->inst_dt[k];
        }
    }
    if (sim_time) {
        std::vector<double> t(n);
        CK(cudaMemcpyAsync(t.data(), ctx->sim_time, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (int k = 0; k < n; ++k) sim_time[k] = t[k] + ctx->time_fixed[k];
    }
    return EPP_OK;
}

int32_t epp_last_step_timing(epp_ctx* ctx, float* ms_total) {
    if (!ctx || !ms_total) return EPP_ERR_INVALID_ARGUMENT;
    if (!ctx->timed) return fail(ctx, EPP_ERR_STATE, "no timed step");
    CK(cudaEventSynchronize(ctx->ev1));
    CK(cudaEventElapsedTime(ms_total, ctx->ev0, ctx->ev1));
    return EPP_OK;
}

int32_t epp_pairs_total(epp_ctx* ctx, int64_t* out) {
    if (!ctx || !out) return EPP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->dev);
    unsigned long long v = 0;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(&v, ctx->pairs, sizeof v, cudaMemcpyDeviceToHost));
    *out = (int64_t)v;
    return EPP_OK;
}

int32_t epp_set_instance_physics(epp_ctx* ctx, int32_t n, const float* dt, const float* c0) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    if (n != ctx->n_inst || !dt || !c0)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "need dt and c0 for all %d instances", ctx->n_inst);
    ctx->inst_dt.assign(dt, dt + n);
    ctx->inst_c0.assign(c0, c0 + n);
    ctx->inst_dirty = true;
    ctx->cfl_tables_ok = false;
    ctx->rpn_valid = false;   // the density preview used the previous time steps
    return EPP_OK;
}

int32_t epp_get_instance_integrals(epp_ctx* ctx, const epp_physics* phys, epp_integrals* out, int32_t n) {
    if (!ctx || !phys || !out) return EPP_ERR_INVALID_ARGUMENT;
    if (n != ctx->n_inst) return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "n = %d, context has %d instances", n, ctx->n_inst);
    if (!ctx->sorted_once) return fail(ctx, EPP_ERR_STATE, "integrals need a search! first");
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    DevPhys P = dev_phys(ctx, *phys);
    auto launch = [&](auto Dt) {
        constexpr int DD = decltype(Dt)::value;
        k_integrals_inst<DD><<<ctx->n_inst, 256, 0, ctx->stream>>>(
            ctx->start[ctx->cur], ctx->dom, ctx->n, ctx->S[ctx->cur], ctx->ncnt[ctx->cur], P, phys->rho0, phys->gamma,
            phys->p0, phys->gravity[0], phys->gravity[1], phys->gravity[2], ctx->inst_out);
    };
    if (ctx->D == 2) launch(std::integral_constant<int, 2>{});
    else launch(std::integral_constant<int, 3>{});
    CK_LAUNCH();
    std::vector<double> r((size_t)9 * n);
    CK(cudaMemcpyAsync(r.data(), ctx->inst_out, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < n; ++k) {
        const double* v = &r[(size_t)9 * k];
        const double c0 = ctx->inst_c0.empty() ? (double)phys->c0 : (double)ctx->inst_c0[k];
        out[k].mass_total = v[0];
        out[k].mass_fluid = v[1];
        out[k].kinetic = v[2];
        out[k].potential = v[3];
        out[k].internal = v[4];
        out[k].max_speed = v[5];
        out[k].cfl_dt = v[6] < 1e300 ? (phys->cfl > 0.0f ? (double)phys->cfl : 0.1) * v[6] / (c0 + v[5]) : 0.0;
        out[k].n_alive = (int64_t)v[7];
        out[k].n_pairs = (int64_t)v[8];
    }
    return EPP_OK;
}

int32_t epp_set_tuning(epp_ctx* ctx, int32_t lanes_per_particle) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    const int g0 = lanes_per_particle;
    if (g0 != 0 && g0 != 1 && g0 != 2 && g0 != 4 && g0 != 8 && g0 != 16 && g0 != 32 && g0 != EPP_TUNING_LISTS)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "pair-pass family %d not in {0,1,2,4,8,16,32,64}", g0);
    const bool fam0 = g0 == EPP_TUNING_LISTS;
    const int g = fam0 ? 0 : g0;
    const int store = fam0 ? g0 : 0;
    if (g != 0 && ctx->n_inst > 1)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "batches of %d instances use pair-pass family 0", ctx->n_inst);
    if (g != ctx->lanes || store != ctx->store) {
        ctx->lanes = g;
        ctx->store = store;
        ctx->nlist_valid = false;
        drop_graphs(ctx);
    }
    return EPP_OK;
}

#ifdef EPP_CHECKED
extern "C" int32_t epp_checked_slot(int32_t* out4) {
    return cudaMemcpyFromSymbol(out4, epp_check_slot, sizeof(int) * 4) == cudaSuccess ? EPP_OK : EPP_ERR_CUDA;
}
#endif

int32_t epp_set_block_threads(epp_ctx* ctx, int32_t threads) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    if (threads != 32 && threads != 64 && threads != 128)
        return fail(ctx, EPP_ERR_INVALID_ARGUMENT, "threads per block %d not in {32, 64, 128}", threads);
    if (threads != ctx->pass_threads) {
        ctx->pass_threads = threads;
        drop_graphs(ctx);
    }
    return EPP_OK;
}

int32_t epp_context_bytes(const epp_config* cfg, int64_t* bytes) {
    if (!cfg || !bytes) return EPP_ERR_INVALID_ARGUMENT;
    const int D = cfg->domain.dim;
    if ((D != 2 && D != 3) || cfg->n_capacity < 1 || !(cfg->domain.gap > 0.0f)) return EPP_ERR_INVALID_ARGUMENT;
    if (cfg->n_capacity > (1 << kEntryBits)) return EPP_ERR_CAPACITY;
    DevDomain d;
    if (const int prc = plan_cells(cfg, d)) return prc;
    const int n_tiles = (d.n_cells + 1 + kScanTile - 1) / kScanTile;
    // + per instance: instance table, integrals, two CFL tables, CFL partials (at most 4 x 148 chunks
    // per instance), simulated time
    const size_t b = arena_bytes(cfg->n_capacity, d.n_cells, D, n_tiles) + nlist_bytes(D, cfg->n_capacity) +
                     (3 * sizeof(InstPhys) + sizeof(double) * 10) * (size_t)d.n_inst +
                     sizeof(double2) * (size_t)std::max(d.n_inst, 4 * 148) + 8 * 256;
    *bytes = (int64_t)b;
    return EPP_OK;
}

int32_t epp_query(epp_ctx* ctx, int32_t* done) {
    if (!ctx || !done) return EPP_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaStreamQuery(ctx->stream);
    if (e == cudaSuccess && ctx->istream) e = cudaStreamQuery(ctx->istream);   // integrals beside the step
    if (e == cudaErrorNotReady) {
        *done = 0;
        return EPP_OK;
    }
    *done = 1;
    if (e != cudaSuccess) return fail(ctx, EPP_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
    return EPP_OK;
}

int32_t epp_set_priority(epp_ctx* ctx, int32_t priority, int32_t* applied) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    int lo = 0, hi = 0;   // numerically: hi (greatest priority) <= lo
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    const int p = priority < hi ? hi : priority > lo ? lo : priority;
    cudaStream_t s = nullptr;
    CK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, p));
    CK(cudaStreamSynchronize(ctx->stream));
    const bool was_own = ctx->stream == ctx->own_stream;
    cudaStreamDestroy(ctx->own_stream);
    ctx->own_stream = s;
    if (was_own) ctx->stream = s;
    if (applied) *applied = p;
    return EPP_OK;
}

int32_t epp_set_stream(epp_ctx* ctx, void* stream) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return EPP_OK;
}

int32_t epp_profile_step(epp_ctx* ctx, const epp_physics* phys, float* stage_ms) {
    if (!ctx || !phys || !stage_ms) return EPP_ERR_INVALID_ARGUMENT;
    if (!ctx->searched) return fail(ctx, EPP_ERR_STATE, "epp_profile_step needs an initial search!");
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    if (ctx->n == 0) return EPP_OK;
    if (ctx->dv_dirty) {
        int rc = epp_step(ctx, 1, phys);   // settles dVelocity through the per-call path
        if (rc) return rc;
    }
    if (phys->cfl > 0.0f && !ctx->cfl_valid) {
        const int rc = ctx->D == 2 ? cfl_update<2>(ctx, *phys) : cfl_update<3>(ctx, *phys);
        if (rc) return rc;
        ctx->rpn_valid = false;
    }
    if (!ctx->rpn_valid || !same_phys(ctx->rpn_phys, *phys)) {
        k_density_preview<<<blocks_for(ctx->n), kThreads, 0, ctx->stream>>>(
            ctx->start[ctx->cur], ctx->n_cells, ctx->n, ctx->S[ctx->cur], dev_phys(ctx, *phys));
        CK_LAUNCH();
    }
    if (ctx->last_crit != EPP_CRITERION_SYMMETRY) ctx->nlist_valid = false;
    {
        int rc0 = ctx->D == 2 ? ensure_nlist<2>(ctx) : ensure_nlist<3>(ctx);
        if (rc0) return rc0;
    }
    cudaEvent_t ev[kProfileStages + 1];
    for (int k = 0; k <= kProfileStages; ++k) CK(cudaEventCreate(&ev[k]));
    int rc = ctx->D == 2 ? enqueue_fused_step<2>(ctx, ctx->cur, *phys, ev)
                         : enqueue_fused_step<3>(ctx, ctx->cur, *phys, ev);
    if (!rc) {
        ctx->cur = 1 - ctx->cur;
        ctx->cfl_valid = phys->cfl > 0.0f;
        if (phys->cfl <= 0.0f) advance_fixed_time(ctx, *phys, 1);
        ctx->rpn_valid = true;
        ctx->rpn_phys = *phys;
        ctx->lists_valid = false;
        ctx->nlist_valid = ctx->lanes == 0;
        cudaError_t e = cudaEventSynchronize(ev[kProfileStages]);
        for (int k = 0; k < kProfileStages && e == cudaSuccess; ++k)
            e = cudaEventElapsedTime(&stage_ms[k], ev[k], ev[k + 1]);
        if (e != cudaSuccess) rc = fail(ctx, EPP_ERR_CUDA, "profile events: %s", cudaGetErrorString(e));
    }
    for (int k = 0; k <= kProfileStages; ++k) cudaEventDestroy(ev[k]);
    return rc;
}

int32_t epp_set_accel_output(epp_ctx* ctx, int32_t enable) {
    if (!ctx) return EPP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    if (enable && !ctx->accel) {
        CK(dev_alloc(ctx, &ctx->accel, sizeof(float4) * ctx->cap));
        CK(cudaMemsetAsync(ctx->accel, 0, sizeof(float4) * ctx->cap, ctx->stream));
    } else if (!enable && ctx->accel) {
        dev_free(ctx, ctx->accel);
    }
    return EPP_OK;
}

int32_t epp_get_accel(epp_ctx* ctx, float* out, int32_t n) {
    // dv/dt (momentum + gravity) of the last fused step, per particle row, dim components each
    // stored as out[a * n + row]; rows of non-fluid particles are 0.
    if (!ctx || !out || n != ctx->n) return EPP_ERR_INVALID_ARGUMENT;
    if (!ctx->accel) return fail(ctx, EPP_ERR_STATE, "accel output disabled");
    cudaSetDevice(ctx->dev);
    if (const int rc_ = join_integrals(ctx)) return rc_;
    // accel is indexed by the order before the last gather; the permutation is cs/perm.  Copy
    // with the id array of that order (the other ping-pong set).
    std::vector<float4> a(ctx->n);
    std::vector<int> ids(ctx->n);
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(a.data(), ctx->accel, sizeof(float4) * ctx->n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ids.data(), ctx->S[1 - ctx->cur].id, sizeof(int) * ctx->n, cudaMemcpyDeviceToHost));
    for (int k = 0; k < ctx->n; ++k) {
        const int i = ids[k];
        out[i] = a[k].x;
        out[(size_t)n + i] = a[k].y;
        if (ctx->D == 3) out[(size_t)2 * n + i] = a[k].z;
    }
    return EPP_OK;
}

}  // extern "C"
