/*
 * gsis_b200.h — C ABI of the B200 kinetic backend (discrete-velocity Shakhov CIS / LU-SGS).
 *
 * This library is a drop-in for the reference's `gsis::kinetic::KineticBackend` CUDA implementation
 * (src/kinetic/kinetic_backend.hpp:59-105, factory `make_cuda_backend` at src/kinetic/kinetic_backend.hpp:105,
 * defined in src/kinetic/kinetic_backend_cuda.cpp:506-509). Every entry point below replaces one virtual method
 * of that interface; the C++ shim that wraps them into a `KineticBackend` lives in
 * gsis_sim_b200/integration/b200_backend.cpp.
 *
 * Conventions (identical to the reference backend interface):
 *   - every host array is FP64 (or int32) in the solver's INTERNAL numbering: cells and boundary faces as
 *     renumbered by `build_kinetic_setup` (src/kinetic/kinetic_setup.cpp:293-514), velocities in the reference
 *     storage order (`VelocityLayout`, src/kinetic/kinetic_setup.hpp:29-38);
 *   - f is addressed as f[cell * nv + p] with p the reference storage position (kinetic_kernels.hpp:64-67);
 *   - moments: 15 per cell, rho, ux, uy, uz, T, p, sxx, syy, szz, sxy, syz, sxz, qx, qy, qz
 *     (src/kinetic/kinetic_types.hpp:107-109);
 *   - boundary sums: 20 per face (src/kinetic/kinetic_types.hpp:111-116);
 *   - arrays passed in are owned by the caller and only read during the call.
 *
 * Every function returns KIN_OK (0) on success and a negative KIN_E* code on failure; the message of the last
 * failure on a handle is returned by kin_last_error(handle) (kin_last_error(NULL) for kin_create failures).
 * Errors replace the reference's `GSIS_CHECK` / `GSIS_CUDA_CHECK` exceptions (src/core/error.hpp:1-47,
 * src/gpu/cuda_check.hpp:16-24); the C++ shim turns them back into `gsis::Error`.
 */
#ifndef GSIS_B200_H
#define GSIS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KIN_ABI_VERSION 2

/* status codes */
#define KIN_OK 0
#define KIN_E_ARG (-1)      /* invalid argument or size mismatch (reference: GSIS_CHECK) */
#define KIN_E_CUDA (-2)     /* CUDA runtime error (reference: GSIS_CUDA_CHECK) */
#define KIN_E_MEMORY (-3)   /* f or the work arrays do not fit in device memory */
#define KIN_E_STATE (-4)    /* call out of order (e.g. boundary sums before set_inflow) */
#define KIN_E_TIMEOUT (-5)  /* a bounded device-side wait gave up (the LU-SGS block pass's staging waits, read back
                               from the device after kin_sweep / kin_adjoint_update) */

/* storage / arithmetic precision of the distribution function */
#define KIN_PREC_FP32 0  /* reference precision = "fp32": f and all per-point arithmetic in FP32 */
#define KIN_PREC_FP64 1  /* reference precision = "fp64" */
#define KIN_PREC_MIXED 2 /* f stored in FP32; limited gradients and LU-SGS passes in FP32 arithmetic; steady residual,
                            moments, boundary sums, equilibrium and GSIS correction in FP64 arithmetic (the FP32
                            sweeps are a defect correction of the FP64 residual); no reference counterpart */

/* BoundaryKind (src/kinetic/kinetic_types.hpp:19-26) */
#define KIN_BC_DIFFUSE_WALL 0
#define KIN_BC_PRESSURE 1
#define KIN_BC_VACUUM 2
#define KIN_BC_SYMMETRY 3
#define KIN_BC_PERIODIC 4
#define KIN_BC_MAXWELL_WALL 5

/* LimiterMode (src/kinetic/kinetic_types.hpp:101-105) */
#define KIN_LIMITER_NONE 0
#define KIN_LIMITER_VENKAT_ABSOLUTE 1
#define KIN_LIMITER_VENKAT_RELATIVE 2

/* gsis_negative_check (src/kinetic/kinetic_kernels.hpp:584-587) */
#define KIN_NEGATIVE_ALL 0
#define KIN_NEGATIVE_CREATED 1
#define KIN_NEGATIVE_LIMIT 2
#define KIN_NEGATIVE_BLEND 3

/* number of values per cell / face in the host arrays */
#define KIN_MOMENTS_PER_CELL 15
#define KIN_BOUNDARY_SUMS_PER_FACE 20
#define KIN_CSR_GEOM 12  /* sx sy sz  dsx dsy dsz  dox doy doz  cx cy cz   (CsrEntry<F>, kinetic_types.hpp:35-42) */
#define KIN_BFACE_GEOM 7 /* nx ny nz  area  dx dy dz                       (BoundaryFaceInfo<F>, :46-54) */

typedef struct KinHandle KinHandle;

/*
 * Everything the backend needs from the reference's `KineticSetup` (src/kinetic/kinetic_setup.hpp:56-115) as
 * flat arrays. The nondimensional geometry is the FP64 value that the reference casts to F in
 * make_csr_entries / make_bface_infos / make_eps2 (src/kinetic/kinetic_setup.cpp:516-599).
 */
typedef struct KinSetupDesc {
  int32_t abi_version; /* KIN_ABI_VERSION */
  int32_t precision;   /* KIN_PREC_* */
  int32_t device;      /* CUDA device ordinal */
  int32_t n_cells;
  int32_t nv;
  int32_t n_bfaces;
  int32_t n_blocks;

  /* velocity grid in storage order (VelocityLayout::xi_*, ::weight) */
  const double* xi_x;
  const double* xi_y;
  const double* xi_z;
  const double* weights; /* optional per-velocity quadrature weights (NULL: every point has `weight`) */
  double weight;         /* uniform weight (used when weights == NULL) */

  /* cell -> face CSR, faces of a cell in ascending face order (CellFaceCsr, src/mesh/fv_geometry.hpp:180-190) */
  const int32_t* csr_offsets; /* n_cells + 1 */
  const int32_t* csr_other;   /* neighbour cell or -1 */
  const int32_t* csr_bface;   /* boundary face index or -1 */
  const double* csr_geom;     /* n_csr * KIN_CSR_GEOM */
  const double* eps2;         /* n_cells: K^3 V */

  /* boundary faces */
  const int32_t* bface_owner;
  const int32_t* bface_kind;       /* KIN_BC_* */
  const int32_t* bface_mirror_xor; /* symmetry / Maxwell wall: mirrored storage position p ^ mirror_xor */
  const int32_t* bface_patch;
  const double* bface_geom; /* n_bfaces * KIN_BFACE_GEOM */

  /* per-cell nondimensional volume and V / dt */
  const double* volume;
  const double* vdt;

  /* LU-SGS blocks and per-direction sweep orders (kinetic_setup.hpp:80-96) */
  const int32_t* block_offsets; /* n_blocks + 1 */
  int32_t n_sweep_dirs;         /* 0: "block" order (internal numbering) */
  const int32_t* sweep_order;   /* n_sweep_dirs * n_cells */
  const int32_t* sweep_pos;     /* n_sweep_dirs * n_cells */
  const uint8_t* sweep_dir_of;  /* nv */

  /* scheme parameters (KineticParams, src/kinetic/kinetic_params.hpp:11-117) */
  int32_t limiter_mode; /* KIN_LIMITER_* */
  int32_t positivity;   /* positivity_limiter */
  double diag_scale;
  double interface_damping;
  int32_t block_passes;
  int32_t negative_check_mode; /* KIN_NEGATIVE_* */
  int64_t velocity_chunk;      /* 0: as large as device memory allows */

  /* gas: mu = mu0 T^omega, Shakhov Prandtl number */
  double mu0;
  double omega;
  double Pr;
  double cold_bgk_temperature;

  /* conservative discrete equilibrium (DeqGrid, src/kinetic/discrete_equilibrium.hpp:25-32) */
  int32_t discrete_eq;
  int32_t deq_fallback_collisionless;
  double deq_lo[3];
  double deq_hi[3];
  double deq_d[3];
  double deq_criterion;
  double deq_tolerance;
  int32_t deq_max_iterations;

  /* partially accommodating walls (MaxwellFace, src/kinetic/kinetic_types.hpp:28-31) */
  int32_t n_maxwell_faces;
  const int64_t* maxwell_offset;             /* n_bfaces, -1 for non-Maxwell faces (NULL if none) */
  const double* maxwell_specular_fraction;   /* n_bfaces */
  const int32_t* grid_to_storage;            /* nv (NULL if no Maxwell walls) */
  int32_t grid_n[3];

  /* velocity sharding (no reference counterpart): when the handle stores only a subset of the velocities (one shard
     of the grid, the others on other GPUs), the discrete equilibrium is still solved on the full grid given here.
     deq_nv == 0: the stored velocities are the full grid. */
  int32_t deq_nv;
  const double* deq_xi_x;
  const double* deq_xi_y;
  const double* deq_xi_z;
  const double* deq_weights; /* NULL: every point has `weight` */
} KinSetupDesc;

/* InflowState (src/kinetic/kinetic_backend.hpp:45-50): scale * f_eq(rho, u, T); same memory layout */
typedef struct KinInflowState {
  double scale;
  double rho;
  double ux, uy, uz;
  double T;
} KinInflowState;

/* StepTimings (src/kinetic/kinetic_backend.hpp:19-41), seconds. The B200 block-pass kernels run the forward and the
   backward sweep of a pass in one launch: sweep_forward holds those launches, sweep_backward the kernel that couples
   a later pass to the previous one across block boundaries. */
typedef struct KinStepTimings {
  double moments;
  double boundary;
  double gradient;
  double residual;
  double sweep_forward;
  double sweep_backward;
  double other;
} KinStepTimings;

/* DeqCounts (src/kinetic/kinetic_backend.hpp:53-57) */
typedef struct KinDeqCounts {
  int64_t corrected;
  int64_t failed;
  int32_t max_iterations;
} KinDeqCounts;

/* make_cuda_backend (src/kinetic/kinetic_backend_cuda.cpp:506-509): uploads the setup, allocates f and the
   velocity-chunk work arrays (CudaBackend ctor, kinetic_backend_cuda.cpp:92-175) */
int kin_create(const KinSetupDesc* desc, KinHandle** out);
/* ~CudaBackend */
void kin_destroy(KinHandle* h);
/* message of the last failure (NULL handle: the last kin_create failure of this thread) */
const char* kin_last_error(const KinHandle* h);

/* KineticBackend::name / chunk_width / memory_bytes (kinetic_backend.hpp:63-65) */
const char* kin_name(const KinHandle* h);
int kin_chunk_width(const KinHandle* h, int32_t* out);
int kin_memory_bytes(const KinHandle* h, uint64_t* out);

/* KineticBackend::set_equilibrium (kinetic_backend.hpp:68); states: 5 * n_cells (rho, ux, uy, uz, T) */
int kin_set_equilibrium(KinHandle* h, const double* states, int64_t n);
/* KineticBackend::set_distribution / get_distribution (:69-70); f: n_cells * nv */
int kin_set_distribution(KinHandle* h, const double* f, int64_t n);
int kin_get_distribution(KinHandle* h, double* f, int64_t n);
/* KineticBackend::compute_moments (:73); out: 15 * n_cells */
int kin_compute_moments(KinHandle* h, double* out, int64_t n);
/* KineticBackend::scale_distribution (:75) */
int kin_scale_distribution(KinHandle* h, double s);
/* KineticBackend::update_cell_params (:77) */
int kin_update_cell_params(KinHandle* h);
/* KineticBackend::set_inflow (:79); n = n_bfaces */
int kin_set_inflow(KinHandle* h, const KinInflowState* inflow, int64_t n);
/* KineticBackend::boundary_sums (:81); out: 20 * n_bfaces */
int kin_boundary_sums(KinHandle* h, double* out, int64_t n);
/* KineticBackend::sweep (:83); residual_cell: n_cells, sum over velocities of R^2 */
int kin_sweep(KinHandle* h, double* residual_cell, int64_t n);
/* KineticBackend::gsis_correction (:86-87); w_half, w_new: 5 * n_cells; replaced_flags: NULL or n_cells */
int kin_gsis_correction(KinHandle* h, const double* w_half, const double* w_new, int64_t n,
                        int32_t* replaced_flags, int64_t* replaced);
/* KineticBackend::internal_face_mass_flux (:92-93) */
int kin_internal_face_mass_flux(KinHandle* h, const int32_t* cells, const int32_t* entries, int64_t n,
                                double* out);
/* KineticBackend::take_timings (:96) */
int kin_take_timings(KinHandle* h, KinStepTimings* out);
/* KineticBackend::deq_counts (:99) */
int kin_deq_counts(KinHandle* h, KinDeqCounts* out);

/* ---- B200 additions (no reference counterpart) ---------------------------------------------------------- */

/* Run every subsequent kernel of this handle on `stream` (a cudaStream_t; NULL: the legacy default stream). */
int kin_set_stream(KinHandle* h, void* stream);
/* Number of kernels this handle has launched since creation. */
int kin_launch_count(const KinHandle* h, int64_t* out);
/* Device pointer of f (storage order of the handle, see kin_velocity_permutation) and its element size. */
int kin_device_f(KinHandle* h, void** f, int32_t* elem_bytes);
/* The handle stores velocities in its own order (grouped by sweep direction): perm[q] = reference storage
   position of the handle's velocity q. */
int kin_velocity_permutation(const KinHandle* h, int32_t* perm, int64_t n);
/* Conservative discrete Maxwellian of n macroscopic states (rho, ux, uy, uz, T), FP64 on the velocity grid with
   the given Newton tolerance: the host-side correction of inflow states (correct_inflow,
   src/kinetic/kinetic_solver.cpp:103-114) batched on the device. out: the corrected states (unchanged where
   result <= 0); result: Newton iterations (0: resolved, no correction; -1: no convergence). */
int kin_discrete_maxwell(KinHandle* h, const double* states, int64_t n, double tolerance, double* out,
                         int32_t* result);

/* Largest batch kin_discrete_maxwell_noalloc accepts, in states. */
#define KIN_NOALLOC_MAX_STATES 4096
/* kin_discrete_maxwell without allocating anything (no reference counterpart): same arguments, same results.
   kin_discrete_maxwell allocates (and frees) device buffers for the states on every call. That does not suit two
   kinds of caller: one that has given nearly all of the device memory to f and the sweep work arrays (a handle sizes
   its velocity chunk to the memory that is free when it is created), for which even a small cudaMalloc can fail;
   and one that keeps other streams of the device busy, which cudaFree would stall because it waits for the whole
   device. This entry point works in a fixed scratch area in the library's static device memory (about 336 KB per
   device: the input states, the corrected states and the Newton results of KIN_NOALLOC_MAX_STATES states), so it
   only copies, launches one kernel and waits for the handle's stream.
   - n > KIN_NOALLOC_MAX_STATES is refused with KIN_E_ARG and a message (split the batch); n == 0 does nothing.
   - Creating a handle looks up the scratch address on its device (cudaGetSymbolAddress, which also makes the
     static array resident) before f and the velocity chunk are sized to the free memory, and keeps it; a call
     therefore only copies, launches and waits, and changes no device memory use.
   - There is ONE scratch per device, shared by every handle on it: calls whose copies or kernels overlap on the
     GPU (from different host threads, or handles on different streams) race and overwrite each other's states.
     Calls made one after another from one thread do not overlap: each returns after its stream is done. */
int kin_discrete_maxwell_noalloc(KinHandle* h, const double* states, int64_t n, double tolerance, double* out,
                                 int32_t* result);
/* LU-SGS level schedule statistics: number of levels of the longest (direction, block) chain and the total
   number of (direction, block) chains. */
int kin_schedule_info(const KinHandle* h, int32_t* max_levels, int32_t* n_chains);

/* Velocity sharding (no reference counterpart; kin_compute_moments is the unsharded form): the 13 velocity sums of
   every cell (sum of w f {1, c, c c (6), |c|^2 c}, c = xi - shift, with the handle's current shift) over the
   velocities this handle stores, not finalised, so that the shards' sums can be added before finalising. */
int kin_moment_sums(KinHandle* h, double* out, int64_t n);
/* Velocity sharding: install the finalised moments (15 per cell, reduced over all shards) as the handle's moments
   (they feed kin_update_cell_params) and move the shift to their velocity, as kin_compute_moments does. */
int kin_set_moments(KinHandle* h, const double* moments, int64_t n);
/* Velocity sharding with the reductions in device memory (no reference counterpart). kin_moment_sums,
   kin_boundary_sums and kin_sweep accept out == NULL: the sums then stay in the handle's device buffer, which
   kin_device_sums returns (pointer and length in doubles), for a multi-GPU caller to reduce IN PLACE across the
   shards (a sum all-reduce of the same buffer on every rank, e.g. NCCL over NVLink) before the call that consumes it:
     KIN_SUMS_MOMENTS   13 * n_cells, consumed by kin_finalize_moments (the moments finalised, installed and the
                        shift moved on the device; out: NULL or 15 * n_cells host doubles)
     KIN_SUMS_BOUNDARY  20 * n_bfaces, read back with kin_read_sums
     KIN_SUMS_RESIDUAL  n_cells, read back with kin_read_sums
   Every call returns with the handle's stream idle; the caller's reduction must be complete before the next call
   on the handle. */
#define KIN_SUMS_MOMENTS 0
#define KIN_SUMS_BOUNDARY 1
#define KIN_SUMS_RESIDUAL 2
int kin_device_sums(KinHandle* h, int32_t which, double** ptr, int64_t* n);
int kin_finalize_moments(KinHandle* h, double* out, int64_t n);
int kin_read_sums(KinHandle* h, int32_t which, double* out, int64_t n);
/* Velocity sharding of the GSIS correction (no reference counterpart; kin_gsis_correction is the unsharded form,
   KineticBackend::gsis_correction :86-87). The negativity rule of a cell reduces over all its velocities, so a
   sharded correction runs in two phases. kin_gsis_correction_extrema writes, per cell (n_ext = n_cells), this
   handle's part of that reduction: the minimum of the limit factor ("limit"), the negated maximum of the blend
   factor ("blend"), or the minimum of the check value (the replacing rules); it changes nothing. The caller reduces
   the shards' arrays with an element-wise MINIMUM and passes the result to kin_gsis_correction_apply, which applies
   the correction exactly as kin_gsis_correction would on the whole grid (flags and replaced as there). */
int kin_gsis_correction_extrema(KinHandle* h, const double* w_half, const double* w_new, int64_t n, double* ext,
                                int64_t n_ext);
int kin_gsis_correction_apply(KinHandle* h, const double* w_half, const double* w_new, int64_t n, const double* ext,
                              int64_t n_ext, int32_t* replaced_flags, int64_t* replaced);

/* ---- discrete adjoint of the converged fixed point (no reference counterpart; FP64 or mixed-precision handles, one
   velocity chunk, no Maxwell walls) --------------------------------------------------------------------------------
   On a mixed-precision handle lambda, the transport seeds and O_f are stored in FP32 and the block passes run in
   FP32 arithmetic (as the forward's sweeps), while O(y) is evaluated in FP64 arithmetic from the stored values (as
   the forward's residual); all sums returned to the host are FP64. FP32 handles are refused (KIN_E_ARG).
   The adjoint y = (lambda [cell][velocity], nu [diffuse wall face]) of an objective J solves O(y) = 0 with
   O(y) = y^T dF/dx - dJ/dx, F = (steady residual R of residual_value, rho_Gamma - Phi of the wall densities). The
   handle evaluates O in pieces; the host finishes the per-cell and per-face algebra (gsis_sim_b200/adjoint.py).
   Prerequisites: the forward state installed (f, moments, cell parameters and inflow of the last prepare).

   kin_adjoint_begin: allocate the adjoint arrays, lambda = 0. rev_velocity[p] = storage position of -xi_p (a
   symmetric grid); rev_entry[e] = for an internal CSR entry of cell j pointing at cell i, the entry of cell i that
   points back at j (-1 for boundary entries). Optional (NULL: no accommodation sums): flip_velocity[a * nv + p] =
   storage position of xi_p with component a negated, face_axis[b] = the axis boundary face b's normal is aligned with
   (-1 none); they give the specular sums of axis-aligned diffuse walls. */
int kin_adjoint_begin(KinHandle* h, const int32_t* rev_velocity, const int32_t* rev_entry, int64_t n_entries,
                      const int32_t* flip_velocity, const int32_t* face_axis);
/* lambda in the storage order of kin_set_distribution (n = n_cells * nv). */
int kin_adjoint_set(KinHandle* h, const double* lambda, int64_t n);
int kin_adjoint_get(KinHandle* h, double* lambda, int64_t n);
/* Transposed transport and the per-cell / per-face sums. mu[b] (n_bfaces): weight of the seed w_q a_q mu[b] on the
   outgoing face values of boundary face b (diffuse walls: nu_b / (area_b sm5_b); inlet / outlet faces: the objective's
   -dJ/d(patch flow) factor), also applied to the incoming values of pressure faces. Outputs, per cell (19): the sums
   of lambda against f^S - f and d f^S / d(rho, u, T, q); where the cell's equilibrium is the discrete one (the
   Newton solve of the cell parameters succeeded) those derivatives are taken at fixed (beta, gamma) and the cell adds
   sum lambda E F psi (5) and sum lambda E psi (5), psi = (1, c, c^2 / 2), F = the Shakhov factor (zeros for the
   other cells); per boundary face: S0, S1 (3), S2 of the seeds on the incoming inflow values against the inflow
   Maxwellian (M, M c, M c^2) and S5, S6 = sum_in w an M {c^2, 1} / area; A1 = sum_in a lambda f_spec,
   A2 = sum_in s_grad f_owner(reflected velocity), S_spec = sum_in w an f_spec (axis-aligned diffuse walls,
   f_spec = the owner's reconstructed face value at the reflected velocity; zero elsewhere); sum_in w an M c / area
   (3); and (18 in all) sum_in w psi f_spec (5, psi = (1, xi, |xi|^2 / 2), axis-aligned diffuse walls). cell_sums = NULL with n_cell = 0 skips the per-cell sums, face_sums = NULL
   with n_face = 0 the per-face sums; the transposed transport (the seeds that kin_adjoint_update gathers) always
   runs, on every cell, except with cell_sums = NULL and face_sums given: then it runs on the owner cells of wall and
   pressure faces only (all the per-face sums read) and the other cells keep their seeds of the previous call, so a
   kin_adjoint_update must follow a call that ran the full transport. */
int kin_adjoint_reduce(KinHandle* h, const double* mu, int64_t n_mu, double* cell_sums, int64_t n_cell,
                       double* face_sums, int64_t n_face);
/* Seeds on the moment sums of the boundary faces' distributions (the face states of the boundary sums, which the
   "limited" pressure-boundary reconstruction reads: src/kinetic/kinetic_solver.cpp:172-260, 280-335): seeds[5 b + k]
   (n = 5 n_bfaces) is the weight of the seed w_q psi_k(xi_q) on the outgoing reconstructed face value of boundary face
   b at velocity q, psi = (1, xi_x, xi_y, xi_z, |xi|^2 / 2); at a symmetry face the value also carries the incoming
   half at the mirrored velocity. Kept for the following kin_adjoint_reduce calls; seeds = NULL with n = 0 removes
   them. Extends the adjoint of the "cell" reconstruction, which needs none; no reference counterpart. */
int kin_adjoint_face_moment_seeds(KinHandle* h, const double* seeds, int64_t n);
/* Finish O_f(y) with the per-cell moment-expansion coefficients coef (8 per cell: a0, a (3), a2, b (3); the term
   w_q (a0 + a.c + a2 c^2 + b.c c^2), c = xi_q - u_cell), return sum_q O_f^2 per cell in res_cell and, if op_out is not
   NULL, O_f(y) itself (storage order); with run_passes != 0 then update lambda by the LU-SGS block passes of the
   reversed velocities (the transposed preconditioner): lambda -= P^-T O_f(y). */
int kin_adjoint_update(KinHandle* h, const double* coef, int64_t n_coef, double* res_cell, int64_t n_res,
                       int32_t run_passes, double* op_out, int64_t n_op);
/* Free the adjoint arrays. */
int kin_adjoint_end(KinHandle* h);

#ifdef __cplusplus
}
#endif

#endif /* GSIS_B200_H */
