/*
 * lbm_oracle.h — CPU restatement of the LBM3D_BB single-domain time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for liblbm3d.so
 * and the timed CPU baseline; nothing in the product links, imports or calls it.
 *
 * Parity status: UNPINNED.  The reference (Julia + CUDA.jl, GPU-only, FP32-only)
 * ships no golden vectors, known-answer tests or fixtures, and julia is absent on
 * every machine available here, so no reference output could be generated.  The
 * restatement follows the reference source line by line (citations in
 * lbm_oracle.cpp) and is cross-checked in tests against an independent numpy
 * transliteration of the reference's table-driven code (Utilities.jl list
 * builders + the per-kernel updates) and against analytic solutions.
 *
 * The API mirrors include/lbm3d.h one-for-one so tests compare the two directly.
 * All population arrays are SoA (f[d*N + node]) FP64 on the host.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H
#include <stdint.h>
#include "../include/lbm3d.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

/* precision: 0 = FP32 arithmetic and storage, 1 = FP64. */
orc_sim* orc_create(const lbm_config* cfg, int32_t precision);
void orc_destroy(orc_sim* s);
const char* orc_last_error(const orc_sim* s);
int32_t orc_set_threads(int32_t n);

int32_t orc_add_body(orc_sim* s, const lbm_body* body);
int32_t orc_add_spheres(orc_sim* s, int32_t count, const double* xyzr);
int32_t orc_update_body(orc_sim* s, const lbm_pose* pose_n, const lbm_pose* pose_half);
int32_t orc_init_equilibrium(orc_sim* s, const double* rho, const double* u, const double* v,
                             const double* w);
int32_t orc_set_populations(orc_sim* s, const double* f_soa);
int32_t orc_step(orc_sim* s, int32_t nsteps);
int64_t orc_step_count(const orc_sim* s);

int32_t orc_get_force(orc_sim* s, int64_t step, double out[6]);
int32_t orc_get_macros(orc_sim* s, double* rho, double* u, double* v, double* w);
int32_t orc_get_populations(orc_sim* s, double* f_soa);
int32_t orc_get_flags(orc_sim* s, uint8_t* mask_s, uint8_t* mask_bb);
int32_t orc_get_links(orc_sim* s, int32_t* bb_ptr, int32_t* bb_lidxs, int8_t* bb_dirs, int64_t cap,
                      int64_t* nnz);
int32_t orc_mass(orc_sim* s, double* out);

#ifdef __cplusplus
}
#endif
#endif
