"""Algorithm-layer mirror: search!, interaction!, selfaction! on the B200 backend.

Same call shape as the reference (src/Algorithm/NeighbourSearch.jl:323-413,
src/Algorithm/Action.jl:53-206): each call runs on the device and returns after the device has
finished (the reference synchronises after every launch, Action.jl:91).  Julia closures cannot
cross the C ABI, so `action` and `criterion` are the named bundles of include/epp.h.

A DeviceParticleSystem pairs a host ParticleSystem (reference layout) with a device context;
`syncto`/`asyncto` mirror Class.syncto!/asyncto! (ParticleSystem.jl:275-307).
"""
from . import abi
from .lib import Context

defaultSearchCriterion = abi.EPP_CRITERION_DEFAULT
symmetrySearchCriterion = abi.EPP_CRITERION_SYMMETRY
defaultSelfaction = abi.EPP_ACTION_NONE


class DeviceParticleSystem:
    """The device side of a particle system: an epp context sized for the host system."""

    def __init__(self, host_ps, neighbour_system, device=0, hbm_budget_bytes=0, column_names=None,
                 n_instances=1):
        self.host = host_ps
        self.ns = neighbour_system
        adj = neighbour_system.active_pair.adjacency_matrix.tolist()
        self.config = abi.make_config(host_ps.domain.to_abi(), host_ps.n_capacity, adj,
                                      max_neighbour_number=neighbour_system.max_neighbour_number,
                                      max_cell_particles=neighbour_system.max_cell_particles,
                                      device=device, hbm_budget_bytes=hbm_budget_bytes,
                                      n_instances=n_instances)
        self.ctx = Context(self.config)
        self.cmap = host_ps.column_map(column_names)
        self.physics = None

    def syncto(self):
        """host -> device (Class.asyncto!(device, host))."""
        h = self.host
        self.ctx.upload(h.n_particles, h.is_alive, h.cell_index, h.int_properties, h.float_properties,
                        self.cmap)

    def asyncto(self):
        """device -> host (Class.asyncto!(host, device)); waits for the device."""
        h = self.host
        self.ctx.download(h.is_alive, h.cell_index, h.int_properties, h.float_properties, self.cmap)

    def close(self):
        self.ctx.close()


def search(dps, criterion=defaultSearchCriterion, action=defaultSelfaction, physics=None,
           emit_list=True, sync=True):
    """Algorithm.search! -- clean!, insert, find neighbours, fused self-action."""
    dps.ctx.search(criterion, action, physics or dps.physics,
                   abi.EPP_SEARCH_EMIT_LIST if emit_list else 0)
    if sync:
        dps.ctx.synchronize()


def interaction(dps, action, physics=None, sync=True):
    """Algorithm.interaction! -- action per (particle, neighbour) of the last search."""
    dps.ctx.interaction(action, physics or dps.physics)
    if sync:
        dps.ctx.synchronize()


def selfaction(dps, action, physics=None, sync=True):
    """Algorithm.selfaction! -- action per alive particle."""
    dps.ctx.selfaction(action, physics or dps.physics)
    if sync:
        dps.ctx.synchronize()


def step(dps, n_steps=1, physics=None, sync=True):
    """The dam-break loop body of main.jl:166-182 as one fused, graph-replayed device step."""
    dps.ctx.step(n_steps, physics or dps.physics)
    if sync:
        dps.ctx.synchronize()


# Reference spellings
dynamic_search = search
static_search = search
dynamic_interaction = interaction
static_interaction = interaction
dynamic_selfaction = selfaction
static_selfaction = selfaction
