/*
 * kinetic_oracle.h — CPU restatement of the reference kinetic backend (TEST INFRASTRUCTURE: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it; the product never links it).
 *
 * Same entry points and argument meaning as include/gsis_b200.h with the prefix orc_ instead of kin_.
 * The arithmetic follows the reference CPU backend (src/kinetic/kinetic_backend_cpu.cpp) and its per-point
 * headers (src/kinetic/kinetic_kernels.hpp, discrete_equilibrium.hpp, src/physics/maxwell.hpp, limiter.hpp):
 * f and all per-point arithmetic in the storage precision, velocity sums in double, LU-SGS sweeps walking each
 * block's cells one by one in the reference sweep order, velocities in the reference storage order.
 */
#ifndef KINETIC_ORACLE_H
#define KINETIC_ORACLE_H

#include "../include/gsis_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcHandle OrcHandle;

int orc_create(const KinSetupDesc* desc, OrcHandle** out);
void orc_destroy(OrcHandle* h);
const char* orc_last_error(const OrcHandle* h);
int orc_chunk_width(OrcHandle* h, int32_t* out);
int orc_set_equilibrium(OrcHandle* h, const double* states, int64_t n);
int orc_set_distribution(OrcHandle* h, const double* f, int64_t n);
int orc_get_distribution(OrcHandle* h, double* f, int64_t n);
int orc_compute_moments(OrcHandle* h, double* out, int64_t n);
int orc_scale_distribution(OrcHandle* h, double s);
int orc_update_cell_params(OrcHandle* h);
int orc_set_inflow(OrcHandle* h, const KinInflowState* inflow, int64_t n);
int orc_boundary_sums(OrcHandle* h, double* out, int64_t n);
int orc_sweep(OrcHandle* h, double* residual_cell, int64_t n);
int orc_gsis_correction(OrcHandle* h, const double* w_half, const double* w_new, int64_t n, int32_t* flags,
                        int64_t* replaced);
int orc_internal_face_mass_flux(OrcHandle* h, const int32_t* cells, const int32_t* entries, int64_t n, double* out);
int orc_deq_counts(OrcHandle* h, KinDeqCounts* out);
int orc_moment_sums(OrcHandle* h, double* out, int64_t n);
int orc_set_moments(OrcHandle* h, const double* m, int64_t n);
int orc_gsis_correction_extrema(OrcHandle* h, const double* wh, const double* wn, int64_t n, double* ext,
                                int64_t n_ext);
int orc_gsis_correction_apply(OrcHandle* h, const double* wh, const double* wn, int64_t n, const double* ext,
                              int64_t n_ext, int32_t* flags, int64_t* replaced);
/* test support: the LU-SGS block passes on a given steady residual (storage order), f += the update */
int orc_passes_given(OrcHandle* h, const double* R, int64_t n);
int orc_discrete_maxwell(OrcHandle* h, const double* states, int64_t n, double tolerance, double* out,
                         int32_t* result);

#ifdef __cplusplus
}
#endif

#endif
