/*
 * CPU restatement of the reference kinetic backend — TEST INFRASTRUCTURE ONLY (see kinetic_oracle.h).
 * Shared FP64 pieces (discrete-equilibrium Newton, moment finalisation) are here; the per-precision body is
 * kinetic_oracle_impl.h, included once per (storage, arithmetic) pair.
 */
#define _POSIX_C_SOURCE 200809L
#include "kinetic_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846

static double* orc_dup_d(const double* a, int64_t n) {
  double* o = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  if (n > 0) memcpy(o, a, sizeof(double) * n);
  return o;
}
static int32_t* orc_dup_i(const int32_t* a, int64_t n) {
  int32_t* o = (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
  if (n > 0) memcpy(o, a, sizeof(int32_t) * n);
  return o;
}
static double orc_max(double a, double b) { return a < b ? b : a; }

/* deq_resolved (src/kinetic/discrete_equilibrium.hpp:35-48) */
static int orc_deq_resolved(const double* lo, const double* hi, const double* d, double crit, double ux, double uy,
                            double uz, double T) {
  if (!(T > 0.0)) return 0;
  const double u[3] = {ux, uy, uz};
  for (int a = 0; a < 3; ++a) {
    if (2.0 * ORC_PI * ORC_PI * T / (d[a] * d[a]) < crit) return 0;
    const double m1 = hi[a] - u[a], m2 = u[a] - lo[a];
    if (!(m1 > 0.0 && m2 > 0.0)) return 0;
    if (m1 * m1 < 2.0 * T * crit || m2 * m2 < 2.0 * T * crit) return 0;
  }
  return 1;
}

/* deq_initial_beta (:134-141) */
static void orc_deq_initial_beta(double rho, double T, double* beta) {
  const double tp = 2.0 * ORC_PI * T;
  beta[0] = log(rho / (tp * sqrt(tp)));
  beta[1] = beta[2] = beta[3] = 0.0;
  beta[4] = -1.0 / T;
}

/* deq_jacobian (:83-94) */
static void orc_jac(const double* s, double w, double J[5][5]) {
  int k = 0;
  for (int a = 0; a < 5; ++a)
    for (int b = a; b < 5; ++b) {
      J[a][b] = w * s[k];
      J[b][a] = J[a][b];
      ++k;
    }
}

/* deq_solve5 (:97-131) */
static int orc_solve5(double A[5][5], double* b, double* x) {
  for (int k = 0; k < 5; ++k) {
    int piv = k;
    double best = fabs(A[k][k]);
    for (int r = k + 1; r < 5; ++r)
      if (fabs(A[r][k]) > best) {
        best = fabs(A[r][k]);
        piv = r;
      }
    if (!(best > 0.0)) return 0;
    if (piv != k) {
      for (int c = 0; c < 5; ++c) {
        const double t = A[k][c];
        A[k][c] = A[piv][c];
        A[piv][c] = t;
      }
      const double t = b[k];
      b[k] = b[piv];
      b[piv] = t;
    }
    for (int r = k + 1; r < 5; ++r) {
      const double f = A[r][k] / A[k][k];
      for (int c = k; c < 5; ++c) A[r][c] -= f * A[k][c];
      b[r] -= f * b[k];
    }
  }
  for (int k = 4; k >= 0; --k) {
    double sum = b[k];
    for (int c = k + 1; c < 5; ++c) sum -= A[k][c] * x[c];
    x[k] = sum / A[k][k];
    if (!(x[k] == x[k])) return 0;
  }
  return 1;
}

/* deq_newton_step (:159-180) */
static int orc_deq_newton_step(const double* s, double w, double rho, double T, double tol, double* beta, double* rel) {
  const double G[5] = {w * s[0] - rho, w * s[1], w * s[2], w * s[3], w * s[4] - 1.5 * rho * T};
  const double su = rho * sqrt(T);
  *rel = orc_max(fabs(G[0]) / rho,
                 orc_max(orc_max(fabs(G[1]), orc_max(fabs(G[2]), fabs(G[3]))) / su, fabs(G[4]) / (rho * T)));
  if (!(*rel == *rel)) return -1;
  if (*rel < tol) return 1;
  double J[5][5];
  orc_jac(s, w, J);
  double rhs[5] = {-G[0], -G[1], -G[2], -G[3], -G[4]};
  double d[5] = {0, 0, 0, 0, 0};
  if (!orc_solve5(J, rhs, d)) return -1;
  double scale = 1.0;
  if (fabs(d[4]) > 0.5 * fabs(beta[4])) scale = 0.5 * fabs(beta[4]) / fabs(d[4]);
  if (fabs(d[0]) * scale > 1.0) scale = 1.0 / fabs(d[0]);
  for (int k = 0; k < 5; ++k) beta[k] += scale * d[k];
  if (!(beta[4] < 0.0)) return -1;
  return 0;
}

/* deq_accept (src/kinetic/kinetic_kernels.hpp:489-493) */
static int orc_deq_accept(int r, double rel, double rel_prev, int last) {
  if (r == 1) return 1;
  if (r == 0 && rel < 1e-4 && (rel > 0.5 * rel_prev || last)) return 1;
  return 0;
}

/* deq_shakhov_correction (:183-188) */
static int orc_deq_shakhov_correction(const double* s, double w, double* gamma) {
  double J[5][5];
  orc_jac(s, w, J);
  double rhs[5] = {-w * s[15], -w * s[16], -w * s[17], -w * s[18], -w * s[19]};
  return orc_solve5(J, rhs, gamma);
}

/* finalize_moments (src/kinetic/kinetic_kernels.hpp:401-442) */
static void orc_finalize_moments(const double* s, double weight, double u0x, double u0y, double u0z, double* out) {
  const double s0 = s[0];
  if (!(s0 > 0.0)) {
    out[0] = weight * s0;
    for (int k = 1; k < 15; ++k) out[k] = 0.0;
    return;
  }
  const double dx = s[1] / s0, dy = s[2] / s0, dz = s[3] / s0;
  const double rho = weight * s0;
  const double pxx = weight * (s[4] - s0 * dx * dx), pyy = weight * (s[5] - s0 * dy * dy),
               pzz = weight * (s[6] - s0 * dz * dz), pxy = weight * (s[7] - s0 * dx * dy),
               pyz = weight * (s[8] - s0 * dy * dz), pxz = weight * (s[9] - s0 * dx * dz);
  const double p = (pxx + pyy + pzz) / 3.0;
  const double tr2 = s[4] + s[5] + s[6], du2 = dx * dx + dy * dy + dz * dz;
  const double s2dx = s[4] * dx + s[7] * dy + s[9] * dz, s2dy = s[7] * dx + s[5] * dy + s[8] * dz,
               s2dz = s[9] * dx + s[8] * dy + s[6] * dz;
  out[0] = rho;
  out[1] = u0x + dx;
  out[2] = u0y + dy;
  out[3] = u0z + dz;
  out[4] = p / rho;
  out[5] = p;
  out[6] = pxx - p;
  out[7] = pyy - p;
  out[8] = pzz - p;
  out[9] = pxy;
  out[10] = pyz;
  out[11] = pxz;
  out[12] = 0.5 * weight * (s[10] - dx * tr2 - 2.0 * s2dx + 2.0 * s0 * du2 * dx);
  out[13] = 0.5 * weight * (s[11] - dy * tr2 - 2.0 * s2dy + 2.0 * s0 * du2 * dy);
  out[14] = 0.5 * weight * (s[12] - dz * tr2 - 2.0 * s2dz + 2.0 * s0 * du2 * dz);
}


/* discrete_maxwell_seq<double> + maxwell_params_to_state (src/kinetic/kinetic_kernels.hpp:499-552) on the FP64
   velocity grid: the host-side correction of inflow states (correct_inflow, src/kinetic/kinetic_solver.cpp:103-114) */
static int orc_deq_state_f64(const double* xx, const double* xy, const double* xz, const double* w8, int nv, double weight,
                             const double* lo, const double* hi, const double* dd, double crit, int maxit, double tol,
                             const double* st, double* out) {
  for (int k = 0; k < 5; ++k) out[k] = st[k];
  const double rho = st[0], ux = st[1], uy = st[2], uz = st[3], T = st[4];
  if (orc_deq_resolved(lo, hi, dd, crit, ux, uy, uz, T)) return 0;
  double beta[5];
  orc_deq_initial_beta(rho, T, beta);
  const double w = w8 ? 1.0 : weight;
  double rel_prev = 1e300;
  for (int it = 0; it < maxit; ++it) {
    const double B = -0.5 * beta[4];
    const double dx = -beta[1] / beta[4], dy = -beta[2] / beta[4], dz = -beta[3] / beta[4];
    const double mux = ux + dx, muy = uy + dy, muz = uz + dz;
    const double A = exp(beta[0] + B * (dx * dx + dy * dy + dz * dz));
    double sums[20] = {0};
    for (int p = 0; p < nv; ++p) {
      const double cx = xx[p] - ux, cy = xy[p] - uy, cz = xz[p] - uz;
      const double ex = xx[p] - mux, ey = xy[p] - muy, ez = xz[p] - muz;
      double e = A * exp(-B * (ex * ex + ey * ey + ez * ez));
      if (w8) e *= w8[p];
      const double h = 0.5 * (cx * cx + cy * cy + cz * cz);
      double t[20];
      t[0] = e; t[1] = e * cx; t[2] = e * cy; t[3] = e * cz; t[4] = e * h;
      t[5] = t[1] * cx; t[6] = t[1] * cy; t[7] = t[1] * cz; t[8] = t[1] * h;
      t[9] = t[2] * cy; t[10] = t[2] * cz; t[11] = t[2] * h;
      t[12] = t[3] * cz; t[13] = t[3] * h; t[14] = t[4] * h;
      for (int k = 15; k < 20; ++k) t[k] = 0.0;
      for (int k = 0; k < 20; ++k) sums[k] += t[k];
    }
    double b[5] = {beta[0], beta[1], beta[2], beta[3], beta[4]};
    double rel = 0.0;
    const int r = orc_deq_newton_step(sums, w, rho, T, tol, b, &rel);
    if (orc_deq_accept(r, rel, rel_prev, it + 1 == maxit)) {
      const double Tn = 1.0 / (2.0 * B);
      const double tp = 2.0 * ORC_PI * Tn;
      out[0] = A * tp * sqrt(tp);
      out[1] = mux;
      out[2] = muy;
      out[3] = muz;
      out[4] = Tn;
      return it + 1;
    }
    if (r < 0) break;
    for (int k = 0; k < 5; ++k) beta[k] = b[k];
    rel_prev = rel;
  }
  for (int k = 0; k < 5; ++k) out[k] = st[k];
  return -1;
}

#define S float
#define M float
#define SFX _f32
#include "kinetic_oracle_impl.h"
#undef S
#undef M
#undef SFX

#define S double
#define M double
#define SFX _f64
#include "kinetic_oracle_impl.h"
#undef S
#undef M
#undef SFX

#define S float
#define M double
#define SFX _mix
#include "kinetic_oracle_impl.h"
#undef S
#undef M
#undef SFX

struct OrcHandle {
  int precision;
  void* state;
  /* mixed precision: an FP32-arithmetic state that shares f and the chunk work arrays with the FP64-arithmetic
     state; it runs the gradient and the LU-SGS passes, the FP64 state everything else (residual included) */
  State_f32* fast;
  /* mixed precision: defect of the FP32 residual against the FP64 one, taken at the first sweep after the cell
     parameters (or f) changed; the inner sweeps after it run the FP32 residual plus this defect */
  float* defect;
  int defect_valid;
  int defect_scheme; /* KIN_MIXED_RESIDUAL=defect at creation; else the FP64 residual at every sweep */
  char err[512];
};

/* mixed precision: share the FP32 storage of the FP64-arithmetic state with the FP32-arithmetic state */
static State_f32* mixed_fast_state(const KinSetupDesc* d, State_mix* m) {
  State_f32* f = create_f32(d);
  free(f->f);
  free(f->gx);
  free(f->gy);
  free(f->gz);
  free(f->r);
  f->f = m->f;
  f->gx = m->gx;
  f->gy = m->gy;
  f->gz = m->gz;
  f->r = m->r;
  return f;
}

static void mixed_fast_destroy(State_f32* f) {
  f->f = f->gx = f->gy = f->gz = f->r = NULL;
  destroy_f32(f);
}

/* FP32 copy of the FP64 cell parameters (the LU-SGS diagonal and the Maxwell-wall reconstruction use them) */
static void mixed_cast_cell_params(State_f32* f, const State_mix* m) {
  for (int c = 0; c < m->nc; ++c) {
    const Cp_mix* a = &m->cp[c];
    Cp_f32* b = &f->cp[c];
    b->eq.ux = (float)a->eq.ux;
    b->eq.uy = (float)a->eq.uy;
    b->eq.uz = (float)a->eq.uz;
    b->eq.A = (float)a->eq.A;
    b->eq.B = (float)a->eq.B;
    b->ucx = (float)a->ucx;
    b->ucy = (float)a->ucy;
    b->ucz = (float)a->ucz;
    b->qx = (float)a->qx;
    b->qy = (float)a->qy;
    b->qz = (float)a->qz;
    b->theta = (float)a->theta;
    b->coef = (float)a->coef;
    b->g0 = (float)a->g0;
    b->g4 = (float)a->g4;
    b->gx = (float)a->gx;
    b->gy = (float)a->gy;
    b->gz = (float)a->gz;
    b->coll = (float)a->coll;
    b->diag = (float)a->diag;
  }
}

#define DISPATCH(h, fn, ...)                                      \
  do {                                                            \
    switch ((h)->precision) {                                     \
      case KIN_PREC_FP32: fn##_f32((State_f32*)(h)->state, ##__VA_ARGS__); break; \
      case KIN_PREC_FP64: fn##_f64((State_f64*)(h)->state, ##__VA_ARGS__); break; \
      default: fn##_mix((State_mix*)(h)->state, ##__VA_ARGS__); break;            \
    }                                                             \
  } while (0)

static int orc_fail(OrcHandle* h, const char* msg) {
  snprintf(h->err, sizeof(h->err), "%s", msg);
  return KIN_E_ARG;
}

static int orc_nc(OrcHandle* h) { return *(int32_t*)h->state; } /* nc is the first member of every State */
static int orc_nv(OrcHandle* h) { return ((int32_t*)h->state)[1]; }
static int orc_nb(OrcHandle* h) { return ((int32_t*)h->state)[2]; }

int orc_create(const KinSetupDesc* d, OrcHandle** out) {
  OrcHandle* h = (OrcHandle*)calloc(1, sizeof(OrcHandle));
  h->precision = d->precision;
  if (d->precision == KIN_PREC_FP32) h->state = create_f32(d);
  else if (d->precision == KIN_PREC_FP64) h->state = create_f64(d);
  else {
    h->state = create_mix(d);
    h->fast = mixed_fast_state(d, (State_mix*)h->state);
    const char* mode = getenv("KIN_MIXED_RESIDUAL");
    h->defect_scheme = mode != NULL && strcmp(mode, "defect") == 0;
    if (h->defect_scheme) h->defect = (float*)calloc((size_t)d->n_cells * (size_t)d->nv, sizeof(float));
  }
  *out = h;
  return KIN_OK;
}

void orc_destroy(OrcHandle* h) {
  if (!h) return;
  if (h->precision == KIN_PREC_FP32) destroy_f32((State_f32*)h->state);
  else if (h->precision == KIN_PREC_FP64) destroy_f64((State_f64*)h->state);
  else {
    mixed_fast_destroy(h->fast);
    destroy_mix((State_mix*)h->state);
    free(h->defect);
  }
  free(h);
}

const char* orc_last_error(const OrcHandle* h) { return h ? h->err : ""; }

int orc_chunk_width(OrcHandle* h, int32_t* out) {
  if (h->precision == KIN_PREC_FP32) *out = ((State_f32*)h->state)->chunk;
  else if (h->precision == KIN_PREC_FP64) *out = ((State_f64*)h->state)->chunk;
  else *out = ((State_mix*)h->state)->chunk;
  return KIN_OK;
}

int orc_set_equilibrium(OrcHandle* h, const double* st, int64_t n) {
  if (n != 5LL * orc_nc(h)) return orc_fail(h, "length of the initial states does not match the number of cells");
  h->defect_valid = 0;
  DISPATCH(h, set_equilibrium, st);
  return KIN_OK;
}

#define SETGET(SF)                                                                  \
  static void set_dist##SF(State##SF* s, const double* f) {                         \
    for (int64_t i = 0; i < (int64_t)s->nc * s->nv; ++i) s->f[i] = f[i];            \
  }                                                                                 \
  static void get_dist##SF(State##SF* s, double* f) {                               \
    for (int64_t i = 0; i < (int64_t)s->nc * s->nv; ++i) f[i] = (double)s->f[i];    \
  }
SETGET(_f32)
SETGET(_f64)
SETGET(_mix)

int orc_set_distribution(OrcHandle* h, const double* f, int64_t n) {
  if (n != (int64_t)orc_nc(h) * orc_nv(h)) return orc_fail(h, "length of the distribution function does not match");
  h->defect_valid = 0;
  DISPATCH(h, set_dist, f);
  return KIN_OK;
}
int orc_get_distribution(OrcHandle* h, double* f, int64_t n) {
  if (n != (int64_t)orc_nc(h) * orc_nv(h)) return orc_fail(h, "length of the distribution function does not match");
  DISPATCH(h, get_dist, f);
  return KIN_OK;
}
int orc_compute_moments(OrcHandle* h, double* out, int64_t n) {
  if (n != 15LL * orc_nc(h)) return orc_fail(h, "length of the moment output does not match");
  DISPATCH(h, compute_moments, out);
  return KIN_OK;
}
int orc_scale_distribution(OrcHandle* h, double s) {
  h->defect_valid = 0;
  DISPATCH(h, scale, s);
  return KIN_OK;
}
int orc_update_cell_params(OrcHandle* h) {
  h->defect_valid = 0;
  DISPATCH(h, update_cell_params);
  if (h->fast) mixed_cast_cell_params(h->fast, (State_mix*)h->state);
  return KIN_OK;
}
int orc_set_inflow(OrcHandle* h, const KinInflowState* in, int64_t n) {
  if (n != orc_nb(h)) return orc_fail(h, "length of the inflow states does not match the number of boundary faces");
  DISPATCH(h, set_inflow, in);
  if (h->fast) set_inflow_f32(h->fast, in);
  return KIN_OK;
}
int orc_boundary_sums(OrcHandle* h, double* out, int64_t n) {
  if (n != 20LL * orc_nb(h)) return orc_fail(h, "length of the boundary-sum output does not match");
  DISPATCH(h, boundary_sums, out);
  if (h->fast) reflect_f32(h->fast);
  return KIN_OK;
}
int orc_sweep(OrcHandle* h, double* res, int64_t n) {
  if (n != orc_nc(h)) return orc_fail(h, "length of the residual output does not match the number of cells");
  if (h->fast) {
    State_mix* m = (State_mix*)h->state;
    for (int c = 0; c < m->nc; ++c) res[c] = 0.0;
    for (int k0 = 0; k0 < m->nv; k0 += m->chunk) {
      const int kc = m->chunk < m->nv - k0 ? m->chunk : m->nv - k0;
      sweep_gradient_f32(h->fast, k0, kc);
      if (!h->defect_scheme) {
        sweep_residual_mix(m, k0, kc, res);
      } else if (!h->defect_valid) {
        /* first sweep of the iteration: the FP64 residual, and the defect of the FP32 one at the same f */
        sweep_residual_mix(m, k0, kc, res);
        sweep_residual_defect_f32(h->fast, k0, kc, res, h->defect, 1);
      } else {
        sweep_residual_defect_f32(h->fast, k0, kc, res, h->defect, 2);
      }
      sweep_passes_f32(h->fast, k0, kc);
    }
    h->defect_valid = 1;
    return KIN_OK;
  }
  DISPATCH(h, sweep, res);
  return KIN_OK;
}
int orc_gsis_correction(OrcHandle* h, const double* wh, const double* wn, int64_t n, int32_t* flags,
                        int64_t* replaced) {
  if (n != 5LL * orc_nc(h)) return orc_fail(h, "length of the GSIS macroscopic states does not match");
  h->defect_valid = 0;
  if (h->precision == KIN_PREC_FP32) *replaced = gsis_correction_f32((State_f32*)h->state, wh, wn, flags);
  else if (h->precision == KIN_PREC_FP64) *replaced = gsis_correction_f64((State_f64*)h->state, wh, wn, flags);
  else *replaced = gsis_correction_mix((State_mix*)h->state, wh, wn, flags);
  return KIN_OK;
}
int orc_gsis_correction_extrema(OrcHandle* h, const double* wh, const double* wn, int64_t n, double* ext,
                                int64_t n_ext) {
  if (n != 5LL * orc_nc(h) || n_ext != orc_nc(h)) return orc_fail(h, "length of the GSIS correction arrays");
  if (h->precision == KIN_PREC_FP32) gsis_correction_phase_f32((State_f32*)h->state, wh, wn, NULL, ext, 1);
  else if (h->precision == KIN_PREC_FP64) gsis_correction_phase_f64((State_f64*)h->state, wh, wn, NULL, ext, 1);
  else gsis_correction_phase_mix((State_mix*)h->state, wh, wn, NULL, ext, 1);
  return KIN_OK;
}
int orc_gsis_correction_apply(OrcHandle* h, const double* wh, const double* wn, int64_t n, const double* ext,
                              int64_t n_ext, int32_t* flags, int64_t* replaced) {
  if (n != 5LL * orc_nc(h) || n_ext != orc_nc(h)) return orc_fail(h, "length of the GSIS correction arrays");
  h->defect_valid = 0;
  double* e = (double*)ext;
  if (h->precision == KIN_PREC_FP32) *replaced = gsis_correction_phase_f32((State_f32*)h->state, wh, wn, flags, e, 2);
  else if (h->precision == KIN_PREC_FP64) *replaced = gsis_correction_phase_f64((State_f64*)h->state, wh, wn, flags, e, 2);
  else *replaced = gsis_correction_phase_mix((State_mix*)h->state, wh, wn, flags, e, 2);
  return KIN_OK;
}
int orc_internal_face_mass_flux(OrcHandle* h, const int32_t* cells, const int32_t* entries, int64_t n, double* out) {
  DISPATCH(h, internal_flux, cells, entries, n, out);
  return KIN_OK;
}
int orc_deq_counts(OrcHandle* h, KinDeqCounts* out) {
  out->corrected = out->failed = 0;
  out->max_iterations = 0;
  const int32_t* fl;
  int valid, nc = orc_nc(h);
  if (h->precision == KIN_PREC_FP32) { fl = ((State_f32*)h->state)->deq_flags; valid = ((State_f32*)h->state)->deq_valid; }
  else if (h->precision == KIN_PREC_FP64) { fl = ((State_f64*)h->state)->deq_flags; valid = ((State_f64*)h->state)->deq_valid; }
  else { fl = ((State_mix*)h->state)->deq_flags; valid = ((State_mix*)h->state)->deq_valid; }
  if (!valid) return KIN_OK;
  for (int c = 0; c < nc; ++c) {
    if (fl[c] > 0) ++out->corrected;
    if (fl[c] < 0) ++out->failed;
    if (fl[c] > out->max_iterations) out->max_iterations = fl[c];
  }
  return KIN_OK;
}

#define DEQ_STATES(SF)                                                                                         \
  static void deq_states##SF(State##SF* s, const double* st, int64_t n, double tol, double* out, int32_t* res) { \
    _Pragma("omp parallel for schedule(dynamic, 1)")                                                           \
    for (int64_t i = 0; i < n; ++i)                                                                            \
      res[i] = orc_deq_state_f64(s->dq_xd, s->dq_yd, s->dq_zd, s->dq_w, s->dq_nv, s->weight, s->deq_lo,         \
                                 s->deq_hi, s->deq_d, s->deq_crit, s->deq_maxit, tol, st + 5 * i, out + 5 * i); \
  }
DEQ_STATES(_f32)
DEQ_STATES(_f64)
DEQ_STATES(_mix)

int orc_discrete_maxwell(OrcHandle* h, const double* states, int64_t n, double tol, double* out, int32_t* result) {
  DISPATCH(h, deq_states, states, n, tol, out, result);
  return KIN_OK;
}

int orc_moment_sums(OrcHandle* h, double* out, int64_t n) {
  if (n != 13LL * orc_nc(h)) return orc_fail(h, "length of the moment-sum output does not match");
  DISPATCH(h, moment_sums, out);
  return KIN_OK;
}
int orc_passes_given(OrcHandle* h, const double* R, int64_t n) {
  if (n != (int64_t)orc_nc(h) * orc_nv(h)) return orc_fail(h, "length of the residual does not match");
  DISPATCH(h, passes_given, R);
  return KIN_OK;
}
int orc_set_moments(OrcHandle* h, const double* m, int64_t n) {
  if (n != 15LL * orc_nc(h)) return orc_fail(h, "length of the moments does not match");
  h->defect_valid = 0;
  DISPATCH(h, set_moments, m);
  return KIN_OK;
}
