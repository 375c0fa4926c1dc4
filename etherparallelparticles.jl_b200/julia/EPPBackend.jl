#=
  EPPBackend.jl -- the B200 backend of EtherParallelParticles.jl: the reference's own
  Algorithm.search! / interaction! / selfaction! and Class.syncto! / asyncto! calls, dispatched on a
  particle system whose Backend type parameter is `kB200`, run through `ccall` into libepp.so
  (include/epp.h).

  Use (example/collapse_dry/same/main.jl with only the set-up lines changed):

      include("EPPBackend.jl"); using .EPPBackend
      const parallel = Environment.Parallel{Int32, Float32, Array, EPPBackend.kB200}()  # the backend line
      ...                                  # domain, particle systems, neighbour system as before
      EPPBackend.attach!(device_particle_system, domain, neighbour_system;
                         physics = EPPBackend.example_physics(dt, ...),
                         actions = (sContinuity! => EPPBackend.DamBreakDensity,
                                    iMomentum! => EPPBackend.DamBreakMomentum,
                                    sMomentum! => EPPBackend.DamBreakIntegrate,
                                    sComputeKernelAndiContinuity! => EPPBackend.DamBreakContinuity,
                                    iFilter => EPPBackend.KernelFilter, sFilter => EPPBackend.KernelFilterSelf))
      # the time loop of main.jl:166-206 runs unchanged; or EPPBackend.step!(device_particle_system, n)

  Closures cannot cross a C ABI, so each Julia action function is registered once as one of the
  library's named bundles (EPP_ACTION_*); an unregistered function raises
  EPP_ERR_UNSUPPORTED_ACTION (there is no CPU fallback).  The particle system's arrays stay host
  Arrays (the mirror the reference keeps in `base_`); the state itself lives on the GPU in the
  epp context, as it would in a CuArray backend: asyncto!/syncto! move it.
=#
module EPPBackend

using EtherParallelParticles
using EtherParallelParticles: Environment, Class, Algorithm

const libepp = get(ENV, "EPP_LIB", joinpath(@__DIR__, "..", "epp", "libepp.so"))
const ABI_VERSION = Int32(4)
const MAX_TAGS = 16

# -------------------------------------------------------------------- backend and named bundles

"The backend value of `Environment.Parallel{IT, FT, Array, kB200}`."
struct B200 end
const kB200 = B200()

# EPP_CRITERION_* and EPP_ACTION_* of include/epp.h
const CriterionDefault = Int32(0)       # defaultSearchCriterion   NeighbourSearch.jl:141-151
const CriterionSymmetry = Int32(1)      # symmetrySearchCriterion  NeighbourSearch.jl:153-164
const ActionNone = Int32(0)             # defaultSelfaction!       Action.jl:27-35
const DamBreakContinuity = Int32(1)     # search! action: kernel cache + continuity  main.jl:74-90
const DamBreakDensity = Int32(2)        # selfaction!: sContinuity!  main.jl:92-105
const DamBreakMomentum = Int32(3)       # interaction!: iMomentum!   main.jl:107-118
const DamBreakIntegrate = Int32(4)      # selfaction!: sMomentum!    main.jl:120-126
const ZeroDVelocity = Int32(5)
const CountNeighbours = Int32(6)
const KernelFilter = Int32(7)           # interaction!: iFilter      main.jl:128-134
const KernelFilterSelf = Int32(8)       # selfaction!: sFilter       main.jl:136-144
const ExtrapolatePressure = Int32(9)
const ExtrapolatePressureSelf = Int32(10)
const SearchEmitList = Int32(1)         # epp_search flag: keep nIndex/nRVec/nR/nW/nDW/nHInv

# ------------------------------------------------------------- C structs (layout of include/epp.h)

struct EppDomain
    dim::Int32
    gap::Float32
    first::NTuple{3, Float32}
    last::NTuple{3, Float32}
end

struct EppPhysics
    dt::Float32
    rho0::Float32
    c0::Float32
    p0::Float32
    gamma::Int32
    gravity::NTuple{3, Float32}
    alpha::Float32
    beta::Float32
    viscosity::Int32
    fluid_tag::Int32
    wall_tag::Int32
    kahan::Int32
    kernel::Int32
    eos::Int32
    mu::Float32
    motion::Int32
    filter_interval::Int32
    pressure_ff::Int32
    pressure_fw::Int32
    tensile::Int32
    wall_pressure::Int32
    cfl::Float32
end

struct EppConfig
    domain::EppDomain
    n_capacity::Int32
    max_neighbour_number::Int32
    max_cell_particles::Int32
    n_tags::Int32
    adjacency::NTuple{256, Int32}
    device::Int32
    hbm_budget_bytes::Int64
    n_instances::Int32
end

struct EppColumnMap
    tag::Int32
    is_movable::Int32
    n_count::Int32
    n_index::Int32
    position::Int32
    velocity::Int32
    dvelocity::Int32
    mass::Int32
    volume::Int32
    density::Int32
    ddensity::Int32
    pressure::Int32
    gap::Int32
    h::Int32
    n_rvec::Int32
    n_r::Int32
    n_w::Int32
    n_dw::Int32
    n_hinv::Int32
    instance::Int32
end

struct EppIntegrals
    mass_total::Float64
    mass_fluid::Float64
    kinetic::Float64
    potential::Float64
    internal::Float64
    max_speed::Float64
    cfl_dt::Float64
    n_alive::Int64
    n_pairs::Int64
end

# ------------------------------------------------------------------------------- ccall wrappers

epp_abi_version() = ccall((:epp_abi_version, libepp), Int32, ())
epp_last_error(ctx::Ptr{Cvoid}) = unsafe_string(ccall((:epp_last_error, libepp), Cstring, (Ptr{Cvoid},), ctx))
epp_create(cfg::EppConfig, out::Ref{Ptr{Cvoid}}) =
    ccall((:epp_create, libepp), Int32, (Ref{EppConfig}, Ref{Ptr{Cvoid}}), cfg, out)
epp_destroy(ctx::Ptr{Cvoid}) = ccall((:epp_destroy, libepp), Int32, (Ptr{Cvoid},), ctx)
epp_upload(ctx, n, is_alive, cell_index, ip, ld_int, fp, ld_float, cmap::EppColumnMap) =
    ccall((:epp_upload, libepp), Int32,
          (Ptr{Cvoid}, Int32, Ptr{Int32}, Ptr{Int32}, Ptr{Int32}, Int64, Ptr{Float32}, Int64, Ref{EppColumnMap}),
          ctx, n, is_alive, cell_index, ip, ld_int, fp, ld_float, cmap)
epp_download(ctx, is_alive, cell_index, ip, ld_int, fp, ld_float, cmap::EppColumnMap) =
    ccall((:epp_download, libepp), Int32,
          (Ptr{Cvoid}, Ptr{Int32}, Ptr{Int32}, Ptr{Int32}, Int64, Ptr{Float32}, Int64, Ref{EppColumnMap}),
          ctx, is_alive, cell_index, ip, ld_int, fp, ld_float, cmap)
epp_search(ctx, criterion, action, phys::EppPhysics, flags) =
    ccall((:epp_search, libepp), Int32, (Ptr{Cvoid}, Int32, Int32, Ref{EppPhysics}, Int32),
          ctx, criterion, action, phys, flags)
epp_interaction(ctx, action, phys::EppPhysics) =
    ccall((:epp_interaction, libepp), Int32, (Ptr{Cvoid}, Int32, Ref{EppPhysics}), ctx, action, phys)
epp_selfaction(ctx, action, phys::EppPhysics) =
    ccall((:epp_selfaction, libepp), Int32, (Ptr{Cvoid}, Int32, Ref{EppPhysics}), ctx, action, phys)
epp_step(ctx, n_steps, phys::EppPhysics) =
    ccall((:epp_step, libepp), Int32, (Ptr{Cvoid}, Int32, Ref{EppPhysics}), ctx, n_steps, phys)
epp_get_integrals(ctx, phys::EppPhysics, out::Ref{EppIntegrals}) =
    ccall((:epp_get_integrals, libepp), Int32, (Ptr{Cvoid}, Ref{EppPhysics}, Ref{EppIntegrals}), ctx, phys, out)
epp_synchronize(ctx, status::Ref{UInt32}) =
    ccall((:epp_synchronize, libepp), Int32, (Ptr{Cvoid}, Ref{UInt32}), ctx, status)
epp_step_dt(ctx, phys::EppPhysics, n, next_dt, sim_time) =
    ccall((:epp_step_dt, libepp), Int32, (Ptr{Cvoid}, Ref{EppPhysics}, Int32, Ptr{Float32}, Ptr{Float64}),
          ctx, phys, n, next_dt, sim_time)
epp_context_bytes(cfg::EppConfig, out::Ref{Int64}) =
    ccall((:epp_context_bytes, libepp), Int32, (Ref{EppConfig}, Ref{Int64}), cfg, out)

struct EppError <: Exception
    code::Int32
    what::String
end
Base.showerror(io::IO, e::EppError) = print(io, "libepp status ", e.code, ": ", e.what)

check(rc::Int32, ctx::Ptr{Cvoid}, what) =
    rc == 0 || throw(EppError(rc, what * (ctx == C_NULL ? "" : ": " * epp_last_error(ctx))))

# ------------------------------------------------------------------------- physics constructors

"""The benchmark physics (Wendland C2, Tait EOS, artificial viscosity, symplectic Euler with
Kahan positions); zeros in the option fields select it."""
benchmark_physics(dt; rho0 = 1000.0f0, c0, p0 = 0.0f0, gamma = 7, gravity = (0.0f0, -9.81f0, 0.0f0),
                  alpha = 0.1f0, beta = 0.1f0, fluid_tag = 1, wall_tag = 2, kahan = 1, cfl = 0.0f0) =
    EppPhysics(dt, rho0, c0, p0, gamma, Float32.(gravity), alpha, beta, 0, fluid_tag, wall_tag, kahan,
               0, 0, 0.0f0, 0, 0, 0, 0, 0, 0, cfl)

"""The physics of example/collapse_dry/same/main.jl:53-144: CubicSpline, linear EOS, classic
viscosity with mu, sAccelerateMove!, kernel filter every `filter_interval` steps."""
example_physics(dt; rho0, c0, p0, mu, gravity, filter_interval = 20, fluid_tag = 1, wall_tag = 2) =
    EppPhysics(dt, rho0, c0, p0, 7, Float32.(gravity), 0.0f0, 0.0f0, 2, fluid_tag, wall_tag, 0,
               1, 1, mu, 1, filter_interval, 0, 0, 0, 0, 0.0f0)

# ------------------------------------------------------------------ device state of a system

mutable struct DeviceState
    ctx::Ptr{Cvoid}
    cmap::EppColumnMap
    physics::EppPhysics
    actions::IdDict{Any, Int32}
end

# one context per particle system (keyed by identity); finalised with the system
const STATES = IdDict{Any, DeviceState}()

state(ps) = haskey(STATES, ps) ? STATES[ps] :
    error("EPPBackend: call EPPBackend.attach!(particle_system, domain, neighbour_system; physics) first")

column(nt::NamedTuple, name::Symbol) = haskey(nt, name) ? Int32(nt[name] - 1) : Int32(-1)

"""The epp_column_map of a particle system: 0-based columns of its NamedIndex
(ParticleSystem.jl:28-41, NamedIndex.jl:95-110, BasicIndex.jl:10-44); `names` renames columns
(e.g. `Dict(:Density => :rho)`); absent columns are -1."""
function column_map(ps; names = Dict{Symbol, Symbol}())
    idx = Class.get_index_named_tuple(ps.named_index_)
    b = ps.basic_index_
    nm(s) = get(names, s, s)
    c(s) = column(idx, nm(s))
    return EppColumnMap(Int32(b.Tag - 1), Int32(b.IsMovable - 1), Int32(b.nCount - 1), Int32(b.nIndex - 1),
                        Int32(b.PositionVec - 1), c(:VelocityVec), c(:dVelocityVec), c(:Mass), c(:Volume),
                        c(:Density), c(:dDensity), c(:Pressure), c(:Gap), c(:H), Int32(b.nRVec - 1),
                        Int32(b.nR - 1), c(:nW), c(:nDW), c(:nHInv), c(:Instance))
end

"""epp_config of a domain, neighbour system and particle system: the cell grid of the Domain2D
(Domain2D.jl:28-67), the active-pair matrix (ActivePair.jl:12-33), the bucket capacity of the
neighbour system (NeighbourSystemBase.jl:77-96), the width of the nIndex column group and the
capacity of the particle system."""
function config(ps, domain, ns; device = 0, hbm_budget_bytes = 0)
    Class.dimension(domain) == 2 || error("EPPBackend: the reference's domain type is Domain2D")
    gap = Float32(Class.get_gap(domain))
    first = (Float32(Class.get_first_x(domain)), Float32(Class.get_first_y(domain)), 0.0f0)
    last = (Float32(Class.get_last_x(domain)), Float32(Class.get_last_y(domain)), 0.0f0)
    adj = Array(ns.active_pair_.adjacency_matrix_)
    n_tags = size(adj, 1)
    n_tags <= MAX_TAGS || error("EPPBackend: $(n_tags) tags > $(MAX_TAGS)")
    flat = zeros(Int32, MAX_TAGS * MAX_TAGS)
    for a in 1:n_tags, b in 1:n_tags
        flat[(a - 1) * MAX_TAGS + b] = Int32(adj[a, b])
    end
    ints = ps.named_index_.int_named_index_table_
    nindex = findfirst(==(ps.basic_index_.nIndex), ints.index_named_tuple_)
    max_nb = Int32(ints.capacity_named_tuple_[nindex])
    max_cell = Int32(size(ns.base_.contained_particle_index_list_, 2))
    return EppConfig(EppDomain(Int32(2), gap, first, last), Int32(Class.get_n_capacity(ps)), max_nb, max_cell,
                     Int32(n_tags), Tuple(flat), Int32(device), Int64(hbm_budget_bytes), Int32(1))
end

"""Create the device context of a B200-backed particle system, register the action functions
(`Pair`s of a Julia function and an EPP action id) and upload the state."""
function attach!(ps, domain, ns; physics::EppPhysics, actions = (), device = 0, names = Dict{Symbol, Symbol}(),
                 hbm_budget_bytes = 0)
    epp_abi_version() == ABI_VERSION || error("EPPBackend: libepp ABI $(epp_abi_version()) != $(ABI_VERSION)")
    haskey(STATES, ps) && detach!(ps)
    cfg = config(ps, domain, ns; device = device, hbm_budget_bytes = hbm_budget_bytes)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    check(epp_create(cfg, out), C_NULL, "epp_create")
    st = DeviceState(out[], column_map(ps; names = names), physics, IdDict{Any, Int32}())
    st.actions[Algorithm.defaultSelfaction!] = ActionNone
    for (f, id) in actions
        st.actions[f] = Int32(id)
    end
    STATES[ps] = st
    upload!(ps)
    return st
end

function detach!(ps)
    st = pop!(STATES, ps, nothing)
    st === nothing || epp_destroy(st.ctx)
    return nothing
end

action_id(st::DeviceState, f) = haskey(st.actions, f) ? st.actions[f] :
    throw(EppError(Int32(4), "EPP_ERR_UNSUPPORTED_ACTION: $(f) is not registered with EPPBackend.attach!"))
criterion_id(::typeof(Algorithm.defaultSearchCriterion)) = CriterionDefault
criterion_id(::typeof(Algorithm.symmetrySearchCriterion)) = CriterionSymmetry
criterion_id(f) = throw(EppError(Int32(5), "EPP_ERR_UNSUPPORTED_CRITERION: $(f)"))

function sync!(st::DeviceState)
    status = Ref{UInt32}(0)
    check(epp_synchronize(st.ctx, status), st.ctx, "epp_synchronize")
    return status[]
end

"The host arrays of the particle system -> the device (Class.asyncto!(device, host))."
function upload!(ps)
    st = state(ps)
    b = ps.base_
    check(epp_upload(st.ctx, Int32(Class.get_n_particles(ps)), b.is_alive_, b.cell_index_, b.int_properties_,
                     Int64(size(b.int_properties_, 1)), b.float_properties_, Int64(size(b.float_properties_, 1)),
                     st.cmap), st.ctx, "epp_upload")
end

"The device -> the host arrays of the particle system (Class.asyncto!(host, device))."
function download!(ps)
    st = state(ps)
    b = ps.base_
    check(epp_download(st.ctx, b.is_alive_, b.cell_index_, b.int_properties_, Int64(size(b.int_properties_, 1)),
                       b.float_properties_, Int64(size(b.float_properties_, 1)), st.cmap), st.ctx, "epp_download")
end

"The whole time step of main.jl:166-182, fused and replayed as a CUDA graph, `n` times."
function step!(ps, n::Integer = 1; physics::EppPhysics = state(ps).physics)
    st = state(ps)
    check(epp_step(st.ctx, Int32(n), physics), st.ctx, "epp_step")
    return nothing
end

"FP64 mass, energy, max |v|, CFL dt and pair count of the current state."
function integrals(ps; physics::EppPhysics = state(ps).physics)
    st = state(ps)
    out = Ref{EppIntegrals}()
    check(epp_get_integrals(st.ctx, physics, out), st.ctx, "epp_get_integrals")
    return out[]
end

# ------------------------------------------- the reference's API, dispatched on the B200 backend

const B200System{IT, FT, Dimension} = Class.AbstractParticleSystem{IT, FT, Array, kB200, Dimension}

# NeighbourSearch.jl:323-347 (search!), :349-377 (static_search!), dynamic_search!
function Algorithm.search!(ps::B200System{IT, FT, Dimension}, domain::Class.AbstractDomain{IT, FT, Dimension},
                           ns::Class.AbstractNeighbourSystem; criterion::Function = Algorithm.defaultSearchCriterion,
                           action!::Function = Algorithm.defaultSelfaction!, n_threads::Integer = 0,
                           emit_list::Bool = false) where {IT <: Integer, FT <: AbstractFloat, Dimension}
    st = state(ps)
    check(epp_search(st.ctx, criterion_id(criterion), action_id(st, action!), st.physics,
                     emit_list ? SearchEmitList : Int32(0)), st.ctx, "epp_search")
    sync!(st)   # the reference synchronises after each launch (Action.jl:91)
    return nothing
end
Algorithm.static_search!(ps::B200System, domain, ns; kwargs...) = Algorithm.search!(ps, domain, ns; kwargs...)
Algorithm.dynamic_search!(ps::B200System, domain, ns; kwargs...) = Algorithm.search!(ps, domain, ns; kwargs...)

# Action.jl:140-152 (interaction!), :154-181
function Algorithm.interaction!(ps::B200System, action!::Function; n_threads::Integer = 0)
    st = state(ps)
    check(epp_interaction(st.ctx, action_id(st, action!), st.physics), st.ctx, "epp_interaction")
    sync!(st)
    return nothing
end
Algorithm.static_interaction!(ps::B200System, action!::Function; kwargs...) = Algorithm.interaction!(ps, action!; kwargs...)
Algorithm.dynamic_interaction!(ps::B200System, action!::Function; kwargs...) = Algorithm.interaction!(ps, action!; kwargs...)

# Action.jl:53-67 (selfaction!), :69-93
function Algorithm.selfaction!(ps::B200System, action!::Function; n_threads::Integer = 0)
    st = state(ps)
    check(epp_selfaction(st.ctx, action_id(st, action!), st.physics), st.ctx, "epp_selfaction")
    sync!(st)
    return nothing
end
Algorithm.static_selfaction!(ps::B200System, action!::Function; kwargs...) = Algorithm.selfaction!(ps, action!; kwargs...)
Algorithm.dynamic_selfaction!(ps::B200System, action!::Function; kwargs...) = Algorithm.selfaction!(ps, action!; kwargs...)

# ParticleSystem.jl:275-307: the host mirror <-> the device state
function Class.syncto!(dst::B200System, src::Class.AbstractParticleSystem)
    @inbounds dst.n_particles_[1] = src.n_particles_[1]
    Class.syncto!(dst.base_, src.base_)
    haskey(STATES, dst) && upload!(dst)
    return nothing
end
function Class.syncto!(dst::Class.AbstractParticleSystem, src::B200System)
    haskey(STATES, src) && download!(src)
    @inbounds dst.n_particles_[1] = src.n_particles_[1]
    Class.syncto!(dst.base_, src.base_)
    return nothing
end
Class.asyncto!(dst::B200System, src::Class.AbstractParticleSystem) = Class.syncto!(dst, src)
Class.asyncto!(dst::Class.AbstractParticleSystem, src::B200System) = Class.syncto!(dst, src)

# NeighbourSystemBase.jl:50-64 launches a KernelAbstractions kernel on the backend; the
# neighbour-cell table of a B200 system is built on the host (the library does not read it)
function Class.host_initializeNeighbourSystem!(::Environment.AbstractParallel{IT, FT, CT, kB200}, domain,
                                               neighbour_cell_index_count, neighbour_cell_index_list;
                                               n_threads::Integer = 1) where {IT, FT, CT}
    cpu = Environment.Parallel{IT, FT, Environment.kCPUContainerType, Environment.kCPUBackend}()
    Class.host_initializeNeighbourSystem!(cpu, domain, neighbour_cell_index_count, neighbour_cell_index_list;
                                          n_threads = max(n_threads, 1))
end

end # module
