/*
 * Body of the CPU oracle for one (storage S, arithmetic M) pair; included by kinetic_oracle.c three times
 * (fp32: float/float, fp64: double/double, mixed: float/double). TEST INFRASTRUCTURE ONLY.
 * Each routine cites the reference routine it restates.
 */
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define N(x) CAT(x, SFX)

typedef struct { int32_t other, bface; M s[3], ds[3], dn[3], c[3]; } N(Csr);
typedef struct { int32_t owner, kind, mirror_xor, patch; M n[3]; M area; M d[3]; } N(BFace);
typedef struct { M ux, uy, uz, A, B; } N(Mx);
typedef struct { N(Mx) eq; M ucx, ucy, ucz, qx, qy, qz, theta, coef, g0, g4, gx, gy, gz, coll, diag; } N(Cp);
typedef struct { N(Mx) m; M scale; } N(In);

typedef struct {
  int32_t nc, nv, nb, n_blocks, n_dirs, chunk, passes, limiter, positivity, discrete, collisionless, negmode;
  int32_t n_maxwell, grid_n[3];
  double weight, mu0, omega, Pr, cold_T, deq_lo[3], deq_hi[3], deq_d[3], deq_crit, deq_tol;
  int32_t deq_maxit;
  M diag_scale, damping;
  M *xi_x, *xi_y, *xi_z;     /* storage order, precision M */
  double *xd_x, *xd_y, *xd_z; /* FP64 velocities */
  double* w;                  /* per-velocity weights or NULL */
  int32_t* csr_off;
  N(Csr) * csr;
  M* eps2;
  N(BFace) * bf;
  double *volume, *vdt;
  int32_t* block_off;
  int32_t *order, *pos;
  uint8_t* dir_of;
  int64_t* mw_off;
  double* mw_frac;
  int32_t* g2s;
  M *spec, *spec_first;
  N(In) * in;
  N(Cp) * cp;
  S* f;
  double *moments, *shift;
  S *gx, *gy, *gz, *r;
  int32_t* deq_flags;
  int deq_valid;
  /* velocity grid of the discrete equilibrium: the stored velocities, or the full grid of a velocity shard */
  M *dq_x, *dq_y, *dq_z;
  double *dq_xd, *dq_yd, *dq_zd, *dq_w;
  int dq_nv, dq_own;
} N(State);

static inline M N(mexp)(M x) { return (sizeof(M) == sizeof(float)) ? (M)expf((float)x) : (M)exp((double)x); }
static inline M N(mabs)(M x) { return x < (M)0 ? -x : x; }
static inline M N(mmin)(M a, M b) { return b < a ? b : a; }
static inline M N(mmax)(M a, M b) { return a < b ? b : a; }

/* maxwellian (src/physics/maxwell.hpp:25-29) */
static inline M N(maxw)(const N(Mx) * m, M x, M y, M z) {
  const M cx = x - m->ux, cy = y - m->uy, cz = z - m->uz;
  return m->A * N(mexp)(-m->B * (cx * cx + cy * cy + cz * cz));
}

/* maxwell_params_from (src/kinetic/kinetic_kernels.hpp:475-482) */
static N(Mx) N(mx_from)(double rho, double ux, double uy, double uz, double T) {
  const double tp = 2.0 * ORC_PI * T;
  N(Mx) m;
  m.ux = (M)ux;
  m.uy = (M)uy;
  m.uz = (M)uz;
  m.A = (M)(rho / (tp * sqrt(tp)));
  m.B = (M)(1.0 / (2.0 * T));
  return m;
}

/* shakhov_poly / shakhov_target (src/kinetic/kinetic_types.hpp:79-90) */
static inline M N(spoly)(const N(Cp) * s, M cx, M cy, M cz, M c2) {
  return s->coef * (cx * s->qx + cy * s->qy + cz * s->qz) * (c2 / s->theta - (M)5);
}
static inline M N(starget)(const N(Cp) * s, M x, M y, M z) {
  const M cx = x - s->ucx, cy = y - s->ucy, cz = z - s->ucz;
  const M c2 = cx * cx + cy * cy + cz * cz;
  const M m = N(maxw)(&s->eq, x, y, z);
  return m * ((M)1 + N(spoly)(s, cx, cy, cz, c2) + (s->g0 + (s->gx * cx + s->gy * cy + s->gz * cz) + (M)0.5 * s->g4 * c2));
}

/* make_cell_params (src/kinetic/kinetic_kernels.hpp:451-471) */
static N(Cp) N(make_cp)(const double* m, double V, double vdt, double mu0, double omega, double Pr, double cold) {
  const double rho = m[0], T = m[4], tp = 2.0 * ORC_PI * T;
  N(Cp) cp;
  memset(&cp, 0, sizeof(cp));
  cp.eq.ux = (M)m[1];
  cp.eq.uy = (M)m[2];
  cp.eq.uz = (M)m[3];
  cp.eq.A = (M)(rho / (tp * sqrt(tp)));
  cp.eq.B = (M)(1.0 / (2.0 * T));
  cp.ucx = cp.eq.ux;
  cp.ucy = cp.eq.uy;
  cp.ucz = cp.eq.uz;
  cp.qx = (M)m[12];
  cp.qy = (M)m[13];
  cp.qz = (M)m[14];
  cp.theta = (M)T;
  cp.coef = T < cold ? (M)0 : (M)((1.0 - Pr) / (5.0 * (rho * T) * T));
  const double mu = mu0 * pow(T, omega);
  const double coll = V * m[5] / mu;
  cp.coll = (M)coll;
  cp.diag = (M)(coll + vdt);
  return cp;
}

/* venkatakrishnan_face (src/physics/limiter.hpp:17-31) */
static inline M N(venkat)(M d2, M dmax, M dmin, M eps2) {
  M d1;
  if (d2 > (M)0) d1 = dmax;
  else if (d2 < (M)0) d1 = dmin;
  else return (M)1;
  const M num = (d1 * d1 + eps2) + (M)2 * d1 * d2;
  const M den = d1 * d1 + (M)2 * d2 * d2 + d1 * d2 + eps2;
  if (!(den > (M)0)) return (M)0;
  M v = num / den;
  return v < (M)0 ? (M)0 : ((M)1 < v ? (M)1 : v);
}

static inline M N(fat)(const N(State) * s, int c, int p) { return (M)s->f[(int64_t)c * s->nv + p]; }
static inline M N(inflow_value)(const N(State) * s, int b, M x, M y, M z) {
  return s->in[b].scale * N(maxw)(&s->in[b].m, x, y, z);
}

/* boundary_value_first_order (src/kinetic/kinetic_kernels.hpp:145-157) */
static M N(bvalue)(const N(State) * s, const N(Csr) * c, int cell, int p, M x, M y, M z, M fi) {
  const N(BFace)* b = &s->bf[c->bface];
  if (b->kind == KIN_BC_PERIODIC) return fi;
  if (b->kind == KIN_BC_SYMMETRY) return (M)0.5 * (fi + N(fat)(s, cell, p ^ b->mirror_xor));
  const M a = x * c->s[0] + y * c->s[1] + z * c->s[2];
  if (a >= (M)0) return fi;
  if (b->kind == KIN_BC_MAXWELL_WALL)
    return N(inflow_value)(s, c->bface, x, y, z) + (M)s->mw_frac[c->bface] * s->spec_first[s->mw_off[c->bface] + p];
  return N(inflow_value)(s, c->bface, x, y, z);
}

/* limited_gradient (src/kinetic/kinetic_kernels.hpp:161-201) */
static void N(lgrad)(const N(State) * s, int cell, int p, M x, M y, M z, M fi, M* g) {
  const int e0 = s->csr_off[cell], e1 = s->csr_off[cell + 1];
  M gx = 0, gy = 0, gz = 0, fmax = fi, fmin = fi;
  for (int e = e0; e < e1; ++e) {
    const N(Csr)* c = &s->csr[e];
    const M fk = c->other >= 0 ? N(fat)(s, c->other, p) : N(bvalue)(s, c, cell, p, x, y, z, fi);
    const M d = fk - fi;
    gx += c->c[0] * d;
    gy += c->c[1] * d;
    gz += c->c[2] * d;
    fmax = N(mmax)(fmax, fk);
    fmin = N(mmin)(fmin, fk);
  }
  if (s->limiter == KIN_LIMITER_NONE && s->positivity == 0) {
    g[0] = gx; g[1] = gy; g[2] = gz;
    return;
  }
  if (s->positivity != 0 && !(fi > (M)0)) {
    g[0] = g[1] = g[2] = 0;
    return;
  }
  M eps2 = s->eps2[cell];
  if (s->limiter == KIN_LIMITER_VENKAT_RELATIVE) {
    const M sc = N(mmax)(N(mabs)(fmax), N(mabs)(fmin));
    eps2 *= sc * sc;
  }
  M phi = 1, proj_min = 0;
  for (int e = e0; e < e1; ++e) {
    const N(Csr)* c = &s->csr[e];
    if (c->other < 0 && s->bf[c->bface].kind == KIN_BC_PERIODIC) continue;
    const M proj = gx * c->ds[0] + gy * c->ds[1] + gz * c->ds[2];
    if (s->limiter != KIN_LIMITER_NONE) phi = N(mmin)(phi, N(venkat)(proj, fmax - fi, fmin - fi, eps2));
    proj_min = N(mmin)(proj_min, proj);
  }
  if (s->positivity != 0 && proj_min < (M)0) phi = fi > (M)0 ? N(mmin)(phi, fi / (-proj_min)) : (M)0;
  g[0] = phi * gx;
  g[1] = phi * gy;
  g[2] = phi * gz;
}

/* reconstruct_at_boundary (src/kinetic/kinetic_kernels.hpp:205-211) */
static M N(recon_b)(const N(State) * s, const N(BFace) * b, int p) {
  const M fi = N(fat)(s, b->owner, p);
  if (b->kind == KIN_BC_PERIODIC) return fi;
  M g[3];
  N(lgrad)(s, b->owner, p, s->xi_x[p], s->xi_y[p], s->xi_z[p], fi, g);
  return fi + g[0] * b->d[0] + g[1] * b->d[1] + g[2] * b->d[2];
}

static inline M N(maxwell_inflow)(const N(State) * s, int b, int p, M x, M y, M z) {
  return N(inflow_value)(s, b, x, y, z) + (M)s->mw_frac[b] * s->spec[s->mw_off[b] + p];
}

/* reflected_value (src/kinetic/kinetic_kernels.hpp:86-127) */
static M N(reflected)(const N(State) * s, const N(BFace) * b, int p, M x, M y, M z, int reconstruct) {
  if (b->mirror_xor != 0) {
    const int q = p ^ b->mirror_xor;
    return reconstruct ? N(recon_b)(s, b, q) : N(fat)(s, b->owner, q);
  }
  const M un = x * b->n[0] + y * b->n[1] + z * b->n[2];
  const M r[3] = {x - (M)2 * un * b->n[0], y - (M)2 * un * b->n[1], z - (M)2 * un * b->n[2]};
  int base[3];
  M t[3];
  for (int a = 0; a < 3; ++a) {
    const double zz = ((double)r[a] - s->deq_lo[a]) / s->deq_d[a] - 0.5;
    if (zz < -1e-5 || zz > s->grid_n[a] - 1.0 + 1e-5) return 0;
    double cl = zz < s->grid_n[a] - 1.0 ? zz : s->grid_n[a] - 1.0;
    cl = 0.0 < cl ? cl : 0.0;
    base[a] = (int)cl;
    if (base[a] >= s->grid_n[a] - 1) base[a] = s->grid_n[a] - 2;
    t[a] = (M)(cl - base[a]);
  }
  M result = 0;
  const N(Mx)* ref = &s->cp[b->owner].eq;
  for (int k = 0; k < 8; ++k) {
    const int ix = base[0] + (k & 1), iy = base[1] + ((k >> 1) & 1), iz = base[2] + ((k >> 2) & 1);
    const M w = ((k & 1) ? t[0] : (M)1 - t[0]) * ((k & 2) ? t[1] : (M)1 - t[1]) * ((k & 4) ? t[2] : (M)1 - t[2]);
    if (w == (M)0) continue;
    const int q = s->g2s[ix + s->grid_n[0] * (iy + s->grid_n[1] * iz)];
    const M value = reconstruct ? N(recon_b)(s, b, q) : N(fat)(s, b->owner, q);
    const double drx = (double)r[0] - ref->ux, dry = (double)r[1] - ref->uy, drz = (double)r[2] - ref->uz;
    const double dqx = (double)s->xi_x[q] - ref->ux, dqy = (double)s->xi_y[q] - ref->uy,
                 dqz = (double)s->xi_z[q] - ref->uz;
    const double ratio = exp(-(double)ref->B * (drx * drx + dry * dry + drz * drz - dqx * dqx - dqy * dqy - dqz * dqz));
    result += w * (M)((double)value * ratio);
  }
  return result;
}

/* discrete_maxwell_seq (src/kinetic/kinetic_kernels.hpp:499-540) */
static int N(deq_seq)(const N(State) * s, double rho, double ux, double uy, double uz, double T, const N(Cp) * poly,
                      N(Mx) * out, double* gamma) {
  for (int k = 0; k < 5; ++k) gamma[k] = 0.0;
  *out = N(mx_from)(rho, ux, uy, uz, T);
  if (orc_deq_resolved(s->deq_lo, s->deq_hi, s->deq_d, s->deq_crit, ux, uy, uz, T)) return 0;
  double beta[5];
  orc_deq_initial_beta(rho, T, beta);
  const M fux = (M)ux, fuy = (M)uy, fuz = (M)uz;
  const double w = s->dq_w ? 1.0 : s->weight;
  double rel_prev = 1e300;
  for (int it = 0; it < s->deq_maxit; ++it) {
    N(Mx) m;
    {
      const double B = -0.5 * beta[4];
      const double dx = -beta[1] / beta[4], dy = -beta[2] / beta[4], dz = -beta[3] / beta[4];
      m.ux = (M)(ux + dx);
      m.uy = (M)(uy + dy);
      m.uz = (M)(uz + dz);
      m.A = (M)exp(beta[0] + B * (dx * dx + dy * dy + dz * dz));
      m.B = (M)B;
    }
    double sums[20] = {0};
    for (int p = 0; p < s->dq_nv; ++p) {
      const M x = s->dq_x[p], y = s->dq_y[p], z = s->dq_z[p];
      const M cx = x - fux, cy = y - fuy, cz = z - fuz;
      M e = N(maxw)(&m, x, y, z);
      const M pm = poly ? N(spoly)(poly, cx, cy, cz, cx * cx + cy * cy + cz * cz) : (M)0;
      if (s->dq_w) e *= (M)s->dq_w[p];
      const M h = (M)0.5 * (cx * cx + cy * cy + cz * cz);
      M t[20];
      t[0] = e; t[1] = e * cx; t[2] = e * cy; t[3] = e * cz; t[4] = e * h;
      t[5] = t[1] * cx; t[6] = t[1] * cy; t[7] = t[1] * cz; t[8] = t[1] * h;
      t[9] = t[2] * cy; t[10] = t[2] * cz; t[11] = t[2] * h;
      t[12] = t[3] * cz; t[13] = t[3] * h; t[14] = t[4] * h;
      const M ep = e * pm;
      t[15] = ep; t[16] = ep * cx; t[17] = ep * cy; t[18] = ep * cz; t[19] = ep * h;
      for (int k = 0; k < 20; ++k) sums[k] += (double)t[k];
    }
    double b[5] = {beta[0], beta[1], beta[2], beta[3], beta[4]};
    double rel = 0.0;
    const int r = orc_deq_newton_step(sums, w, rho, T, s->deq_tol, b, &rel);
    if (orc_deq_accept(r, rel, rel_prev, it + 1 == s->deq_maxit)) {
      *out = m;
      if (poly && !orc_deq_shakhov_correction(sums, w, gamma))
        for (int k = 0; k < 5; ++k) gamma[k] = 0.0;
      return it + 1;
    }
    if (r < 0) break;
    for (int k = 0; k < 5; ++k) beta[k] = b[k];
    rel_prev = rel;
  }
  *out = N(mx_from)(rho, ux, uy, uz, T);
  for (int k = 0; k < 5; ++k) gamma[k] = 0.0;
  return -1;
}

static N(Mx) N(eq_params)(const N(State) * s, double rho, double ux, double uy, double uz, double T, int* result) {
  if (result) *result = 0;
  if (!s->discrete) return N(mx_from)(rho, ux, uy, uz, T);
  N(Mx) m;
  double gamma[5];
  const int r = N(deq_seq)(s, rho, ux, uy, uz, T, NULL, &m, gamma);
  if (result) *result = r;
  return m;
}

/* ---- operations (CpuBackend, src/kinetic/kinetic_backend_cpu.cpp) ----------------------------------------- */

static void N(set_equilibrium)(N(State) * s, const double* st) {
#pragma omp parallel for schedule(static)
  for (int c = 0; c < s->nc; ++c) {
    const double* w = st + 5 * (int64_t)c;
    const N(Mx) m = N(eq_params)(s, w[0], w[1], w[2], w[3], w[4], NULL);
    for (int p = 0; p < s->nv; ++p) s->f[(int64_t)c * s->nv + p] = (S)N(maxw)(&m, s->xi_x[p], s->xi_y[p], s->xi_z[p]);
    s->shift[3 * c] = w[1];
    s->shift[3 * c + 1] = w[2];
    s->shift[3 * c + 2] = w[3];
  }
}

static void N(compute_moments)(N(State) * s, double* out) {
#pragma omp parallel for schedule(static)
  for (int c = 0; c < s->nc; ++c) {
    const double u0x = s->shift[3 * c], u0y = s->shift[3 * c + 1], u0z = s->shift[3 * c + 2];
    double sums[13] = {0};
    for (int p = 0; p < s->nv; ++p) {
      double f = (double)s->f[(int64_t)c * s->nv + p];
      if (s->w) f *= s->w[p];
      const double cx = s->xd_x[p] - u0x, cy = s->xd_y[p] - u0y, cz = s->xd_z[p] - u0z;
      const double t1 = f * cx, t2 = f * cy, t3 = f * cz, fc2 = f * (cx * cx + cy * cy + cz * cz);
      sums[0] += f; sums[1] += t1; sums[2] += t2; sums[3] += t3;
      sums[4] += t1 * cx; sums[5] += t2 * cy; sums[6] += t3 * cz;
      sums[7] += t1 * cy; sums[8] += t2 * cz; sums[9] += t1 * cz;
      sums[10] += fc2 * cx; sums[11] += fc2 * cy; sums[12] += fc2 * cz;
    }
    double* m = s->moments + 15 * (int64_t)c;
    orc_finalize_moments(sums, s->w ? 1.0 : s->weight, u0x, u0y, u0z, m);
    if (m[0] > 0.0) {
      s->shift[3 * c] = m[1];
      s->shift[3 * c + 1] = m[2];
      s->shift[3 * c + 2] = m[3];
    }
  }
  memcpy(out, s->moments, sizeof(double) * 15 * (size_t)s->nc);
}

/* the 13 shifted sums of one velocity shard, not finalised (velocity sharding; no reference counterpart) */
static void N(moment_sums)(N(State) * s, double* out) {
#pragma omp parallel for schedule(static)
  for (int c = 0; c < s->nc; ++c) {
    const double u0x = s->shift[3 * c], u0y = s->shift[3 * c + 1], u0z = s->shift[3 * c + 2];
    double sums[13] = {0};
    for (int p = 0; p < s->nv; ++p) {
      double f = (double)s->f[(int64_t)c * s->nv + p];
      if (s->w) f *= s->w[p];
      const double cx = s->xd_x[p] - u0x, cy = s->xd_y[p] - u0y, cz = s->xd_z[p] - u0z;
      const double t1 = f * cx, t2 = f * cy, t3 = f * cz, fc2 = f * (cx * cx + cy * cy + cz * cz);
      sums[0] += f; sums[1] += t1; sums[2] += t2; sums[3] += t3;
      sums[4] += t1 * cx; sums[5] += t2 * cy; sums[6] += t3 * cz;
      sums[7] += t1 * cy; sums[8] += t2 * cz; sums[9] += t1 * cz;
      sums[10] += fc2 * cx; sums[11] += fc2 * cy; sums[12] += fc2 * cz;
    }
    for (int k = 0; k < 13; ++k) out[13 * (int64_t)c + k] = sums[k];
  }
}

/* install moments reduced over all shards and move the shift as compute_moments does */
static void N(set_moments)(N(State) * s, const double* m) {
  memcpy(s->moments, m, sizeof(double) * 15 * (size_t)s->nc);
  for (int c = 0; c < s->nc; ++c) {
    if (m[15 * (int64_t)c] > 0.0) {
      for (int a = 0; a < 3; ++a) s->shift[3 * c + a] = m[15 * (int64_t)c + 1 + a];
    }
  }
}

static void N(scale)(N(State) * s, double sc) {
  const S sf = (S)sc;
  const int64_t n = (int64_t)s->nc * s->nv;
  for (int64_t i = 0; i < n; ++i) s->f[i] *= sf;
  for (int c = 0; c < s->nc; ++c) {
    double* m = s->moments + 15 * (int64_t)c;
    m[0] *= sc;
    for (int k = 5; k < 15; ++k) m[k] *= sc;
  }
}

static void N(update_cell_params)(N(State) * s) {
#pragma omp parallel for schedule(static)
  for (int c = 0; c < s->nc; ++c) {
    const double* m = s->moments + 15 * (int64_t)c;
    N(Cp) cp = N(make_cp)(m, s->volume[c], s->vdt[c], s->mu0, s->omega, s->Pr, s->cold_T);
    if (s->discrete) {
      N(Mx) eq;
      double gamma[5];
      const int r = N(deq_seq)(s, m[0], m[1], m[2], m[3], m[4], &cp, &eq, gamma);
      if (r > 0) {
        cp.eq = eq;
        cp.g0 = (M)gamma[0];
        cp.gx = (M)gamma[1];
        cp.gy = (M)gamma[2];
        cp.gz = (M)gamma[3];
        cp.g4 = (M)gamma[4];
      } else if (r < 0 && s->collisionless) {
        cp.coll = 0;
        cp.diag = (M)s->vdt[c];
      }
      s->deq_flags[c] = r;
    }
    s->cp[c] = cp;
  }
  s->deq_valid = s->discrete;
}

static void N(set_inflow)(N(State) * s, const KinInflowState* in) {
  for (int b = 0; b < s->nb; ++b) {
    s->in[b].m = N(mx_from)(in[b].rho, in[b].ux, in[b].uy, in[b].uz, in[b].T);
    s->in[b].scale = (M)in[b].scale;
  }
}

static void N(add_terms)(M wf, M x, M y, M z, M an, double* flux5, double* mom5) {
  const M e = (M)0.5 * (x * x + y * y + z * z);
  const M af = an * wf;
  flux5[0] += (double)af; flux5[1] += (double)(af * x); flux5[2] += (double)(af * y);
  flux5[3] += (double)(af * z); flux5[4] += (double)(af * e);
  mom5[0] += (double)wf; mom5[1] += (double)(wf * x); mom5[2] += (double)(wf * y);
  mom5[3] += (double)(wf * z); mom5[4] += (double)(wf * e);
}

/* specular caches of partially accommodating walls (k_maxwell_reflection, kinetic_cuda_kernels.cu:262-272) */
static void N(reflect)(N(State) * s) {
  if (s->n_maxwell > 0) {
    for (int pass = 0; pass < 2; ++pass) {
#pragma omp parallel for schedule(dynamic, 1)
      for (int b = 0; b < s->nb; ++b) {
        if (s->mw_off[b] < 0) continue;
        const N(BFace)* bf = &s->bf[b];
        M* dst = pass == 0 ? s->spec_first : s->spec;
        for (int p = 0; p < s->nv; ++p) {
          const M x = s->xi_x[p], y = s->xi_y[p], z = s->xi_z[p];
          dst[s->mw_off[b] + p] = (x * bf->n[0] + y * bf->n[1] + z * bf->n[2]) < (M)0 ? N(reflected)(s, bf, p, x, y, z, pass) : (M)0;
        }
      }
    }
  }
}

static void N(boundary_sums)(N(State) * s, double* out) {
  N(reflect)(s);
  const M wu = (M)s->weight;
#pragma omp parallel for schedule(dynamic, 4)
  for (int b = 0; b < s->nb; ++b) {
    const N(BFace)* bf = &s->bf[b];
    double acc[20] = {0};
    for (int p = 0; p < s->nv; ++p) {
      const M x = s->xi_x[p], y = s->xi_y[p], z = s->xi_z[p];
      const M w = s->w ? (M)s->w[p] : wu;
      const M an = x * bf->n[0] + y * bf->n[1] + z * bf->n[2];
      if (an >= (M)0 || bf->kind == KIN_BC_PERIODIC) {
        const M fb = N(recon_b)(s, bf, p);
        N(add_terms)(w * fb, x, y, z, an, acc, acc + 10);
      } else {
        M fb;
        if (bf->kind == KIN_BC_SYMMETRY) fb = N(recon_b)(s, bf, p ^ bf->mirror_xor);
        else if (bf->kind == KIN_BC_MAXWELL_WALL) fb = N(maxwell_inflow)(s, b, p, x, y, z);
        else fb = N(maxw)(&s->in[b].m, x, y, z);
        N(add_terms)(w * fb, x, y, z, an, acc + 5, acc + 15);
      }
    }
    for (int k = 0; k < 20; ++k) out[20 * (int64_t)b + k] = acc[k];
  }
}

static void N(internal_flux)(N(State) * s, const int32_t* cells, const int32_t* entries, int64_t n, double* out) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t i = 0; i < n; ++i) {
    const int c = cells[i];
    const N(Csr)* ce = &s->csr[entries[i]];
    double acc = 0.0;
    for (int p = 0; p < s->nv; ++p) {
      const M x = s->xi_x[p], y = s->xi_y[p], z = s->xi_z[p];
      const M a = x * ce->s[0] + y * ce->s[1] + z * ce->s[2];
      M ff, g[3];
      if (a >= (M)0) {
        const M fi = N(fat)(s, c, p);
        N(lgrad)(s, c, p, x, y, z, fi, g);
        ff = fi + g[0] * ce->ds[0] + g[1] * ce->ds[1] + g[2] * ce->ds[2];
      } else {
        const M fj = N(fat)(s, ce->other, p);
        N(lgrad)(s, ce->other, p, x, y, z, fj, g);
        ff = fj + g[0] * ce->dn[0] + g[1] * ce->dn[1] + g[2] * ce->dn[2];
      }
      double term = (double)(a * ff);
      if (s->w) term *= s->w[p];
      acc += term;
    }
    out[i] = (s->w ? 1.0 : (double)(M)s->weight) * acc;
  }
}

/* residual_value (src/kinetic/kinetic_kernels.hpp:238-278); mirrored gradients recomputed */
static M N(residual)(const N(State) * s, int k0, int stride, int cell, int t) {
  const int p = k0 + t;
  const M x = s->xi_x[p], y = s->xi_y[p], z = s->xi_z[p];
  const M fi = N(fat)(s, cell, p);
  const int64_t wi = (int64_t)cell * stride + t;
  const M gix = (M)s->gx[wi], giy = (M)s->gy[wi], giz = (M)s->gz[wi];
  M R = 0;
  for (int e = s->csr_off[cell]; e < s->csr_off[cell + 1]; ++e) {
    const N(Csr)* c = &s->csr[e];
    int kind = -1;
    if (c->other < 0) {
      kind = s->bf[c->bface].kind;
      if (kind == KIN_BC_PERIODIC) continue;
    }
    const M a = x * c->s[0] + y * c->s[1] + z * c->s[2];
    M ff;
    if (a >= (M)0) {
      if (sizeof(S) < sizeof(M)) /* mixed precision: face reconstruction in the storage precision */
        ff = (M)(s->f[(int64_t)cell * s->nv + p] + s->gx[wi] * (S)c->ds[0] + s->gy[wi] * (S)c->ds[1] +
                 s->gz[wi] * (S)c->ds[2]);
      else
        ff = fi + gix * c->ds[0] + giy * c->ds[1] + giz * c->ds[2];
    } else if (c->other >= 0) {
      const int64_t wj = (int64_t)c->other * stride + t;
      if (sizeof(S) < sizeof(M))
        ff = (M)(s->f[(int64_t)c->other * s->nv + p] + s->gx[wj] * (S)c->dn[0] + s->gy[wj] * (S)c->dn[1] +
                 s->gz[wj] * (S)c->dn[2]);
      else
        ff = N(fat)(s, c->other, p) + (M)s->gx[wj] * c->dn[0] + (M)s->gy[wj] * c->dn[1] + (M)s->gz[wj] * c->dn[2];
    } else if (kind == KIN_BC_SYMMETRY) {
      const int pm = p ^ s->bf[c->bface].mirror_xor;
      const M fm = N(fat)(s, cell, pm);
      M g[3];
      N(lgrad)(s, cell, pm, s->xi_x[pm], s->xi_y[pm], s->xi_z[pm], fm, g);
      ff = fm + g[0] * c->ds[0] + g[1] * c->ds[1] + g[2] * c->ds[2];
    } else if (kind == KIN_BC_MAXWELL_WALL) {
      ff = N(maxwell_inflow)(s, c->bface, p, x, y, z);
    } else {
      ff = N(inflow_value)(s, c->bface, x, y, z);
    }
    R += a * ff;
  }
  const N(Cp)* cp = &s->cp[cell];
  R -= cp->coll * (N(starget)(cp, x, y, z) - fi);
  return R;
}

/* sweep_forward_cell / sweep_backward_cell (src/kinetic/kinetic_kernels.hpp:289-358) */
static void N(fwd_cell)(const N(State) * s, int stride, S* r, const S* r0, const S* dprev, int cell, int t, int cb,
                        int ce, M x, M y, M z, const int32_t* pos) {
  M ap = 0, am_out = 0, Lsum = 0, Lout = 0;
  const int pi = pos ? pos[cell] : cell;
  for (int e = s->csr_off[cell]; e < s->csr_off[cell + 1]; ++e) {
    const N(Csr)* c = &s->csr[e];
    if (c->other < 0 && s->bf[c->bface].kind == KIN_BC_PERIODIC) continue;
    const M a = x * c->s[0] + y * c->s[1] + z * c->s[2];
    if (a > (M)0) {
      ap += a;
    } else if (c->other >= 0) {
      if (c->other < cb || c->other >= ce) {
        if (dprev) Lout += a * (M)dprev[(int64_t)c->other * stride + t];
        else am_out -= a;
      } else if ((pos ? pos[c->other] : c->other) < pi) {
        Lsum += a * (M)r[(int64_t)c->other * stride + t];
      }
    }
  }
  const M D = s->cp[cell].diag + s->diag_scale * ap + s->damping * am_out;
  const int64_t wi = (int64_t)cell * stride + t;
  const M Ri = r0 ? (M)r0[wi] : (M)r[wi];
  r[wi] = (S)((-Ri - Lout - Lsum) / D);
}

static void N(bwd_cell)(N(State) * s, int stride, int k0, S* r, const S* dprev, int update_f, int cell, int t, int cb,
                        int ce, M x, M y, M z, const int32_t* pos) {
  M ap = 0, am_out = 0, U = 0;
  const int pi = pos ? pos[cell] : cell;
  for (int e = s->csr_off[cell]; e < s->csr_off[cell + 1]; ++e) {
    const N(Csr)* c = &s->csr[e];
    if (c->other < 0 && s->bf[c->bface].kind == KIN_BC_PERIODIC) continue;
    const M a = x * c->s[0] + y * c->s[1] + z * c->s[2];
    if (a > (M)0) {
      ap += a;
    } else if (c->other >= 0) {
      if (c->other < cb || c->other >= ce) {
        if (!dprev) am_out -= a;
      } else if ((pos ? pos[c->other] : c->other) > pi) {
        U += a * (M)r[(int64_t)c->other * stride + t];
      }
    }
  }
  const M D = s->cp[cell].diag + s->diag_scale * ap + s->damping * am_out;
  const int64_t wi = (int64_t)cell * stride + t;
  const M df = (M)r[wi] - U / D;
  r[wi] = (S)df;
  if (update_f) {
    S* fp = &s->f[(int64_t)cell * s->nv + k0 + t];
    *fp = (S)((M)*fp + df);
  }
}

/* CpuBackend::sweep (src/kinetic/kinetic_backend_cpu.cpp:262-344), in three parts per velocity chunk */
static void N(sweep_gradient)(N(State) * s, int k0, int kc) {
  const int stride = s->chunk;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < s->nc; ++c) {
    for (int t = 0; t < kc; ++t) {
      const int p = k0 + t;
      M g[3];
      N(lgrad)(s, c, p, s->xi_x[p], s->xi_y[p], s->xi_z[p], N(fat)(s, c, p), g);
      const int64_t wi = (int64_t)c * stride + t;
      s->gx[wi] = (S)g[0];
      s->gy[wi] = (S)g[1];
      s->gz[wi] = (S)g[2];
    }
  }
}

static void N(sweep_residual)(N(State) * s, int k0, int kc, double* residual_cell) {
  const int stride = s->chunk;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < s->nc; ++c) {
    double r2 = 0.0;
    for (int t = 0; t < kc; ++t) {
      const M R = N(residual)(s, k0, stride, c, t);
      s->r[(int64_t)c * stride + t] = (S)R;
      r2 += (double)R * (double)R;
    }
    residual_cell[c] += r2;
  }
}

/* mixed precision, inner sweeps (no reference counterpart): the residual in the arithmetic of this state plus the
   stored defect. mode 1 stores defect = r - R (r holds the higher-precision residual of the same f) and leaves r;
   mode 2 sets r = R + defect and adds its squares to residual_cell. defect: [cell][nv], storage order. */
__attribute__((unused)) static void N(sweep_residual_defect)(N(State) * s, int k0, int kc, double* residual_cell,
                                                              S* defect, int mode) {
  const int stride = s->chunk;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < s->nc; ++c) {
    double r2 = 0.0;
    for (int t = 0; t < kc; ++t) {
      const M R = N(residual)(s, k0, stride, c, t);
      S* d = defect + (int64_t)c * s->nv + k0 + t;
      S* rr = s->r + (int64_t)c * stride + t;
      if (mode == 1) {
        *d = (S)(*rr - (S)R);
      } else {
        const S Ru = (S)((S)R + *d);
        *rr = Ru;
        r2 += (double)Ru * (double)Ru;
      }
    }
    if (mode != 1) residual_cell[c] += r2;
  }
}

static void N(sweep_passes)(N(State) * s, int k0, int kc) {
  const int stride = s->chunk;
  const size_t work = (size_t)s->nc * (size_t)stride;
  /* block passes: gx holds R, gy the previous pass (the reference's buffer use) */
  if (s->passes > 1) memcpy(s->gx, s->r, sizeof(S) * work);
  const int n_lanes = s->n_blocks * kc;
  for (int pass = 0; pass < s->passes; ++pass) {
    const S* r0 = NULL;
    const S* dprev = NULL;
    if (pass > 0) {
      memcpy(s->gy, s->r, sizeof(S) * work);
      r0 = s->gx;
      dprev = s->gy;
    }
    const int upd = pass + 1 == s->passes;
#pragma omp parallel for schedule(static)
    for (int lane = 0; lane < n_lanes; ++lane) {
      const int b = lane / kc, t = lane % kc, p = k0 + t;
      const int cb = s->block_off[b], ce = s->block_off[b + 1];
      const int32_t* order = s->n_dirs > 0 ? s->order + (int64_t)s->dir_of[p] * s->nc : NULL;
      const int32_t* pos = s->n_dirs > 0 ? s->pos + (int64_t)s->dir_of[p] * s->nc : NULL;
      for (int k = cb; k < ce; ++k)
        N(fwd_cell)(s, stride, s->r, r0, dprev, order ? order[k] : k, t, cb, ce, s->xi_x[p], s->xi_y[p], s->xi_z[p], pos);
    }
#pragma omp parallel for schedule(static)
    for (int lane = 0; lane < n_lanes; ++lane) {
      const int b = lane / kc, t = lane % kc, p = k0 + t;
      const int cb = s->block_off[b], ce = s->block_off[b + 1];
      const int32_t* order = s->n_dirs > 0 ? s->order + (int64_t)s->dir_of[p] * s->nc : NULL;
      const int32_t* pos = s->n_dirs > 0 ? s->pos + (int64_t)s->dir_of[p] * s->nc : NULL;
      for (int k = ce - 1; k >= cb; --k)
        N(bwd_cell)(s, stride, k0, s->r, dprev, upd, order ? order[k] : k, t, cb, ce, s->xi_x[p], s->xi_y[p], s->xi_z[p], pos);
    }
  }
}

static void N(sweep)(N(State) * s, double* residual_cell) {
  for (int c = 0; c < s->nc; ++c) residual_cell[c] = 0.0;
  for (int k0 = 0; k0 < s->nv; k0 += s->chunk) {
    const int kc = s->chunk < s->nv - k0 ? s->chunk : s->nv - k0;
    N(sweep_gradient)(s, k0, kc);
    N(sweep_residual)(s, k0, kc, residual_cell);
    N(sweep_passes)(s, k0, kc);
  }
}

/* the LU-SGS block passes on a given steady residual R (storage order, all velocities): f += the pass update, as
   sweep does after its own residual (used by the adjoint tests as the transposed preconditioner on
   velocity-reversed storage) */
static void N(passes_given)(N(State) * s, const double* R) {
  for (int k0 = 0; k0 < s->nv; k0 += s->chunk) {
    const int kc = s->chunk < s->nv - k0 ? s->chunk : s->nv - k0;
    for (int c = 0; c < s->nc; ++c)
      for (int t = 0; t < kc; ++t) s->r[(int64_t)c * s->chunk + t] = (S)R[(int64_t)c * s->nv + k0 + t];
    N(sweep_passes)(s, k0, kc);
  }
}

/* CpuBackend::gsis_correction (src/kinetic/kinetic_backend_cpu.cpp:346-432).
   phase 0: the whole correction. Velocity sharding (no reference counterpart) splits it in two: phase 1 writes, per
   cell, this state's part of the negativity rule's reduction over the velocities into ext (the minimum of the limit
   factor, the negated maximum of the blend factor, or the minimum of the check value; the minimum over all shards is
   the whole grid's value) and changes nothing; phase 2 applies the correction with the reduced ext. */
static int64_t N(gsis_correction_phase)(N(State) * s, const double* w_half, const double* w_new, int32_t* flags,
                                       double* ext, int phase) {
  int64_t replaced = 0;
#pragma omp parallel for schedule(static) reduction(+ : replaced)
  for (int c = 0; c < s->nc; ++c) {
    const double* wh = w_half + 5 * (int64_t)c;
    const double* wn = w_new + 5 * (int64_t)c;
    int rh = 0, rn = 0;
    const N(Mx) mh = N(eq_params)(s, wh[0], wh[1], wh[2], wh[3], wh[4], &rh);
    const N(Mx) mn = N(eq_params)(s, wn[0], wn[1], wn[2], wn[3], wn[4], &rn);
    if (s->collisionless && (rh < 0 || rn < 0)) {
      if (phase == 1) {
        ext[c] = 1e300;
        continue;
      }
      ++replaced;
      if (flags) flags[c] = 2;
      s->shift[3 * c] = wh[1];
      s->shift[3 * c + 1] = wh[2];
      s->shift[3 * c + 2] = wh[3];
      continue;
    }
    S* fc = s->f + (int64_t)c * s->nv;
    const double threshold = -1e-8 * wn[0] / (wn[4] * sqrt(wn[4]));
    const M thr = (M)threshold;
    int replace = 0;
    if (s->negmode == KIN_NEGATIVE_LIMIT) {
      M alpha = 1;
      if (phase != 2) {
        for (int p = 0; p < s->nv; ++p) {
          const M x = s->xi_x[p], y = s->xi_y[p], z = s->xi_z[p];
          const M d = N(maxw)(&mn, x, y, z) - N(maxw)(&mh, x, y, z);
          const M old = (M)fc[p];
          M lim = 1;
          if (d < (M)0) {
            const M room = old - (N(mmin)(old, 0) + thr);
            lim = N(mmin)(1, room / (-d));
          }
          alpha = N(mmin)(alpha, lim);
        }
      }
      if (phase == 1) {
        ext[c] = (double)alpha;
        continue;
      }
      if (phase == 2) alpha = (M)ext[c];
      for (int p = 0; p < s->nv; ++p) {
        const M x = s->xi_x[p], y = s->xi_y[p], z = s->xi_z[p];
        fc[p] = (S)((M)fc[p] + alpha * (N(maxw)(&mn, x, y, z) - N(maxw)(&mh, x, y, z)));
      }
      replace = alpha < (M)1;
    } else if (s->negmode == KIN_NEGATIVE_BLEND) {
      M theta = 0;
      if (phase != 2) {
        for (int p = 0; p < s->nv; ++p) {
          const M x = s->xi_x[p], y = s->xi_y[p], z = s->xi_z[p];
          const M e = N(maxw)(&mn, x, y, z);
          const M old = (M)fc[p];
          const M d = e - N(maxw)(&mh, x, y, z);
          const M g = old + d, bound = N(mmin)(old, 0) + thr;
          M th = 0;
          if (g < bound) {
            const M den = e - g;
            th = den > (M)0 ? N(mmin)(1, (bound - g) / den) : (M)1;
          }
          theta = N(mmax)(theta, th);
        }
      }
      if (phase == 1) {
        ext[c] = -(double)theta;
        continue;
      }
      if (phase == 2) theta = (M)(-ext[c]);
      for (int p = 0; p < s->nv; ++p) {
        const M x = s->xi_x[p], y = s->xi_y[p], z = s->xi_z[p];
        const M e = N(maxw)(&mn, x, y, z);
        const M g = (M)fc[p] + (e - N(maxw)(&mh, x, y, z));
        fc[p] = (S)(((M)1 - theta) * g + theta * e);
      }
      replace = theta > (M)0;
    } else {
      M fmin = 0;
      for (int p = 0; p < s->nv; ++p) {
        const M x = s->xi_x[p], y = s->xi_y[p], z = s->xi_z[p];
        const M old = (M)fc[p];
        const M xn = old + (N(maxw)(&mn, x, y, z) - N(maxw)(&mh, x, y, z));
        if (phase != 1) fc[p] = (S)xn;
        const M chk = s->negmode == KIN_NEGATIVE_CREATED ? xn - N(mmin)(old, 0) : xn;
        fmin = p == 0 ? chk : N(mmin)(fmin, chk);
      }
      if (phase == 1) {
        ext[c] = (double)fmin;
        continue;
      }
      if (phase == 2) fmin = (M)ext[c];
      replace = (double)fmin < threshold;
      if (replace)
        for (int p = 0; p < s->nv; ++p) fc[p] = (S)N(maxw)(&mn, s->xi_x[p], s->xi_y[p], s->xi_z[p]);
    }
    if (replace) ++replaced;
    if (flags) flags[c] = replace ? 1 : 0;
    s->shift[3 * c] = wn[1];
    s->shift[3 * c + 1] = wn[2];
    s->shift[3 * c + 2] = wn[3];
  }
  if (phase != 1) s->deq_valid = 0;
  return replaced;
}

static int64_t N(gsis_correction)(N(State) * s, const double* w_half, const double* w_new, int32_t* flags) {
  return N(gsis_correction_phase)(s, w_half, w_new, flags, NULL, 0);
}

static N(State) * N(create)(const KinSetupDesc* d) {
  N(State)* s = (N(State)*)calloc(1, sizeof(N(State)));
  s->nc = d->n_cells;
  s->nv = d->nv;
  s->nb = d->n_bfaces;
  s->n_blocks = d->n_blocks;
  s->n_dirs = d->n_sweep_dirs;
  s->chunk = d->velocity_chunk > 0 && d->velocity_chunk < d->nv ? (int)d->velocity_chunk : d->nv;
  s->passes = d->block_passes > 0 ? d->block_passes : 1;
  s->limiter = d->limiter_mode;
  s->positivity = d->positivity;
  s->discrete = d->discrete_eq;
  s->collisionless = d->deq_fallback_collisionless;
  s->negmode = d->negative_check_mode;
  s->n_maxwell = d->n_maxwell_faces;
  s->weight = d->weight;
  s->mu0 = d->mu0;
  s->omega = d->omega;
  s->Pr = d->Pr;
  s->cold_T = d->cold_bgk_temperature;
  for (int a = 0; a < 3; ++a) {
    s->grid_n[a] = d->grid_n[a];
    s->deq_lo[a] = d->deq_lo[a];
    s->deq_hi[a] = d->deq_hi[a];
    s->deq_d[a] = d->deq_d[a];
  }
  s->deq_crit = d->deq_criterion;
  s->deq_tol = d->deq_tolerance;
  s->deq_maxit = d->deq_max_iterations;
  s->diag_scale = (M)d->diag_scale;
  s->damping = (M)d->interface_damping;
  const int nc = s->nc, nv = s->nv, nb = s->nb;
  s->xi_x = (M*)malloc(sizeof(M) * nv);
  s->xi_y = (M*)malloc(sizeof(M) * nv);
  s->xi_z = (M*)malloc(sizeof(M) * nv);
  s->xd_x = orc_dup_d(d->xi_x, nv);
  s->xd_y = orc_dup_d(d->xi_y, nv);
  s->xd_z = orc_dup_d(d->xi_z, nv);
  for (int p = 0; p < nv; ++p) {
    s->xi_x[p] = (M)d->xi_x[p];
    s->xi_y[p] = (M)d->xi_y[p];
    s->xi_z[p] = (M)d->xi_z[p];
  }
  s->w = d->weights ? orc_dup_d(d->weights, nv) : NULL;
  if (d->deq_nv > 0) {
    const int m = d->deq_nv;
    s->dq_own = 1;
    s->dq_nv = m;
    s->dq_xd = orc_dup_d(d->deq_xi_x, m);
    s->dq_yd = orc_dup_d(d->deq_xi_y, m);
    s->dq_zd = orc_dup_d(d->deq_xi_z, m);
    s->dq_w = d->deq_weights ? orc_dup_d(d->deq_weights, m) : NULL;
    s->dq_x = (M*)malloc(sizeof(M) * m);
    s->dq_y = (M*)malloc(sizeof(M) * m);
    s->dq_z = (M*)malloc(sizeof(M) * m);
    for (int p = 0; p < m; ++p) {
      s->dq_x[p] = (M)d->deq_xi_x[p];
      s->dq_y[p] = (M)d->deq_xi_y[p];
      s->dq_z[p] = (M)d->deq_xi_z[p];
    }
  } else {
    s->dq_own = 0;
    s->dq_nv = nv;
    s->dq_x = s->xi_x;
    s->dq_y = s->xi_y;
    s->dq_z = s->xi_z;
    s->dq_xd = s->xd_x;
    s->dq_yd = s->xd_y;
    s->dq_zd = s->xd_z;
    s->dq_w = s->w;
  }
  s->csr_off = orc_dup_i(d->csr_offsets, nc + 1);
  const int n_csr = d->csr_offsets[nc];
  s->csr = (N(Csr)*)malloc(sizeof(N(Csr)) * (n_csr > 0 ? n_csr : 1));
  for (int k = 0; k < n_csr; ++k) {
    s->csr[k].other = d->csr_other[k];
    s->csr[k].bface = d->csr_bface[k];
    for (int a = 0; a < 3; ++a) {
      s->csr[k].s[a] = (M)d->csr_geom[12 * k + a];
      s->csr[k].ds[a] = (M)d->csr_geom[12 * k + 3 + a];
      s->csr[k].dn[a] = (M)d->csr_geom[12 * k + 6 + a];
      s->csr[k].c[a] = (M)d->csr_geom[12 * k + 9 + a];
    }
  }
  s->eps2 = (M*)malloc(sizeof(M) * nc);
  for (int c = 0; c < nc; ++c) s->eps2[c] = (M)d->eps2[c];
  s->bf = (N(BFace)*)calloc(nb > 0 ? nb : 1, sizeof(N(BFace)));
  for (int b = 0; b < nb; ++b) {
    s->bf[b].owner = d->bface_owner[b];
    s->bf[b].kind = d->bface_kind[b];
    s->bf[b].mirror_xor = d->bface_mirror_xor[b];
    s->bf[b].patch = d->bface_patch ? d->bface_patch[b] : 0;
    for (int a = 0; a < 3; ++a) {
      s->bf[b].n[a] = (M)d->bface_geom[7 * b + a];
      s->bf[b].d[a] = (M)d->bface_geom[7 * b + 4 + a];
    }
    s->bf[b].area = (M)d->bface_geom[7 * b + 3];
  }
  s->volume = orc_dup_d(d->volume, nc);
  s->vdt = orc_dup_d(d->vdt, nc);
  s->block_off = orc_dup_i(d->block_offsets, d->n_blocks + 1);
  if (s->n_dirs > 0) {
    s->order = orc_dup_i(d->sweep_order, (int64_t)s->n_dirs * nc);
    s->pos = orc_dup_i(d->sweep_pos, (int64_t)s->n_dirs * nc);
    s->dir_of = (uint8_t*)malloc(nv);
    memcpy(s->dir_of, d->sweep_dir_of, nv);
  }
  if (s->n_maxwell > 0) {
    s->mw_off = (int64_t*)malloc(sizeof(int64_t) * nb);
    memcpy(s->mw_off, d->maxwell_offset, sizeof(int64_t) * nb);
    s->mw_frac = orc_dup_d(d->maxwell_specular_fraction, nb);
    s->g2s = orc_dup_i(d->grid_to_storage, nv);
    s->spec = (M*)calloc((size_t)s->n_maxwell * nv, sizeof(M));
    s->spec_first = (M*)calloc((size_t)s->n_maxwell * nv, sizeof(M));
  }
  s->in = (N(In)*)calloc(nb > 0 ? nb : 1, sizeof(N(In)));
  s->cp = (N(Cp)*)calloc(nc, sizeof(N(Cp)));
  s->f = (S*)calloc((size_t)nc * nv, sizeof(S));
  s->moments = (double*)calloc((size_t)nc * 15, sizeof(double));
  s->shift = (double*)calloc((size_t)nc * 3, sizeof(double));
  const size_t work = (size_t)nc * s->chunk;
  s->gx = (S*)calloc(work, sizeof(S));
  s->gy = (S*)calloc(work, sizeof(S));
  s->gz = (S*)calloc(work, sizeof(S));
  s->r = (S*)calloc(work, sizeof(S));
  s->deq_flags = (int32_t*)calloc(nc, sizeof(int32_t));
  return s;
}

static void N(destroy)(N(State) * s) {
  if (s->dq_own) {
    void* own[] = {s->dq_x, s->dq_y, s->dq_z, s->dq_xd, s->dq_yd, s->dq_zd, s->dq_w};
    for (size_t i = 0; i < sizeof(own) / sizeof(own[0]); ++i) free(own[i]);
  }
  void* ptrs[] = {s->xi_x, s->xi_y, s->xi_z, s->xd_x, s->xd_y, s->xd_z, s->w, s->csr_off, s->csr, s->eps2, s->bf,
                  s->volume, s->vdt, s->block_off, s->order, s->pos, s->dir_of, s->mw_off, s->mw_frac, s->g2s,
                  s->spec, s->spec_first, s->in, s->cp, s->f, s->moments, s->shift, s->gx, s->gy, s->gz, s->r,
                  s->deq_flags};
  for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
  free(s);
}

#undef N
#undef CAT
#undef CAT2
