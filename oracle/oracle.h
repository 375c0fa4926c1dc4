/*
 * oracle.h -- C ABI of the CPU oracle (liboracle.so).
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle restates EtherParallelParticles.jl's SPH time step on
 * the CPU so that the CUDA path can be checked against it.  Only tests/, the smoke check in
 * __graft_entry__.py and the cpu_baseline / reference legs of bench.py may load it.  The
 * product (libepp.so and the epp package) never links, imports or calls it.
 *
 * It keeps the reference's own data layout and algorithm: column-major property matrices
 * with one column per scalar and per-neighbour columns (nIndex, nRVec, nR, nW, nDW, nHInv),
 * fixed-capacity cell buckets filled by particle id, and stored neighbour lists that the
 * interaction pass walks.  Two precisions: 32 (Float32, reference order) and 64 (Float64).
 * Parity is pinned against the reference's own known-answer tests (test/Algorithm,
 * test/Class); the physics has no reference assertions and is pinned by closed forms.
 */
#ifndef EPP_ORACLE_H
#define EPP_ORACLE_H

#include <stdint.h>
#include "../include/epp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sys orc_sys;

/* Fields readable in FP64 with orc_get_field (component k for vectors). */
#define ORC_FIELD_POSITION   0
#define ORC_FIELD_VELOCITY   1
#define ORC_FIELD_DVELOCITY  2
#define ORC_FIELD_DENSITY    3
#define ORC_FIELD_DDENSITY   4
#define ORC_FIELD_PRESSURE   5
#define ORC_FIELD_VOLUME     6
#define ORC_FIELD_MASS       7
#define ORC_FIELD_ACCEL      8 /* dv/dt of the last DAMBREAK_INTEGRATE (momentum sum + gravity) */
#define ORC_FIELD_NCOUNT     9
/* Sum of |terms| of the last momentum interaction (vector, + |g| after integrate) and of the last
 * continuity search: the scale against which an FP32 sum's rounding error is measured. */
#define ORC_FIELD_ACCEL_ABS  10
#define ORC_FIELD_DDENSITY_ABS 11

int32_t orc_domain_info(const epp_domain* d, int32_t precision, int32_t n_out[3],
                        double gap_axis[3], double gap_inv[3]);
int32_t orc_cell_of(const epp_domain* d, int32_t precision, const float* x, int32_t cart_out[3],
                    int32_t* linear_out, int32_t* inside_out);
/* counts[n_cells]; lists[n_cells * 3^dim] (row per cell, 1-based cell ids) or NULL */
int32_t orc_neighbour_cell_table(const epp_domain* d, int32_t* counts, int32_t* lists);

/* Kernel value W and gradient dW/dr of EPP_KERNEL_* `kind` in `dim` dimensions (FP64). */
int32_t orc_kernel(int32_t kind, int32_t dim, double r, double hinv, double* w, double* dw);
orc_sys* orc_create(int32_t precision, const epp_config* cfg);
void orc_destroy(orc_sys* s);
int32_t orc_set_threads(int32_t n);
int32_t orc_get_threads(void);
/* 1 (default): cell buckets filled in particle-id order; 0: parallel atomic insert whose
 * within-bucket order is arrival order, as the reference's threaded CPU backend. */
int32_t orc_set_deterministic(orc_sys* s, int32_t det);

int32_t orc_upload(orc_sys* s, int32_t n_particles, const int32_t* is_alive,
                   const int32_t* cell_index, const int32_t* int_props, int64_t ld_int,
                   const float* float_props, int64_t ld_float, const epp_column_map* map);
int32_t orc_download(orc_sys* s, int32_t* is_alive, int32_t* cell_index, int32_t* int_props,
                     int64_t ld_int, float* float_props, int64_t ld_float,
                     const epp_column_map* map);
int32_t orc_get_field(orc_sys* s, int32_t field, int32_t component, double* out);
/* Overwrite a state field (position, velocity, dvelocity, density, ddensity, pressure, volume). */
int32_t orc_set_field(orc_sys* s, int32_t field, int32_t component, const double* in);

int32_t orc_search(orc_sys* s, int32_t criterion, int32_t action, const epp_physics* phys,
                   int32_t flags);
int32_t orc_interaction(orc_sys* s, int32_t action, const epp_physics* phys);
int32_t orc_selfaction(orc_sys* s, int32_t action, const epp_physics* phys);
/* main.jl:166-182: density update, momentum, integrate, search + continuity */
int32_t orc_step(orc_sys* s, int32_t n_steps, const epp_physics* phys);
int32_t orc_integrals(orc_sys* s, const epp_physics* phys, epp_integrals* out);
int32_t orc_cell_stats(orc_sys* s, int32_t* counts, int32_t* offsets, int32_t* sorted_ids,
                       int32_t* n_cells);
/* returns and clears the accumulated EPP_STATUS_* bits */
/* dt of the next step under phys (the CFL dt of the current state when phys->cfl > 0) and the
 * simulated time of the steps since upload. */
int32_t orc_step_dt(orc_sys* s, const epp_physics* phys, double* next_dt, double* sim_time);
uint32_t orc_status(orc_sys* s);

#ifdef __cplusplus
}
#endif

#endif
