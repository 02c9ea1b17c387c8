// Per-(cell, velocity) arithmetic of the discrete-velocity Shakhov CIS on the device.
//
// The formulas are those of the reference's shared kernel headers; each function names the one it follows:
//   src/physics/maxwell.hpp, src/physics/limiter.hpp, src/kinetic/kinetic_types.hpp,
//   src/kinetic/kinetic_kernels.hpp, src/kinetic/discrete_equilibrium.hpp.
// Types: S = storage type of f and of the work arrays, M = arithmetic type of the per-point math
// (fp32: S = M = float; fp64: S = M = double; mixed: S = float, M = double). Velocity-space sums are always
// accumulated in double (the reference CPU backend does the same, src/kinetic/kinetic_backend_cpu.cpp:92-120).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace kin {

constexpr double kPi = 3.14159265358979323846;

enum : int32_t { kDiffuseWall = 0, kPressure = 1, kVacuum = 2, kSymmetry = 3, kPeriodic = 4, kMaxwellWall = 5 };
enum : int32_t { kLimNone = 0, kLimAbs = 1, kLimRel = 2 };
enum : int32_t { kNegAll = 0, kNegCreated = 1, kNegLimit = 2, kNegBlend = 3 };
constexpr int kMomentSums = 13;
constexpr int kDeqSums = 20;
constexpr int kCorrectionSkipped = 2;

__host__ __device__ inline float kexp(float x) { return expf(x); }
__host__ __device__ inline double kexp(double x) { return exp(x); }
__host__ __device__ inline float kabs(float x) { return fabsf(x); }
__host__ __device__ inline double kabs(double x) { return fabs(x); }
__host__ __device__ inline float ksqrt(float x) { return sqrtf(x); }
__host__ __device__ inline double ksqrt(double x) { return sqrt(x); }
// min/max/clamp with the NaN behaviour of the reference (src/core/math.hpp:30-41)
template <class T>
__host__ __device__ inline T kmin(T a, T b) { return b < a ? b : a; }
template <class T>
__host__ __device__ inline T kmax(T a, T b) { return a < b ? b : a; }
template <class T>
__host__ __device__ inline T kclamp(T x, T lo, T hi) { return x < lo ? lo : (hi < x ? hi : x); }

// f_eq = A exp(-B |xi - u|^2)   (MaxwellParams, src/physics/maxwell.hpp:17-29)
template <class M>
struct Maxwell {
  M ux, uy, uz, A, B;
};

template <class M>
__host__ __device__ inline M maxwellian(const Maxwell<M>& m, M x, M y, M z) {
  const M cx = x - m.ux, cy = y - m.uy, cz = z - m.uz;
  return m.A * kexp(-m.B * (cx * cx + cy * cy + cz * cz));
}

// make_maxwell_params in double, then cast (maxwell_params_from, src/kinetic/kinetic_kernels.hpp:475-482)
template <class M>
__host__ __device__ inline Maxwell<M> maxwell_from(double rho, double ux, double uy, double uz, double T) {
  const double two_pi_T = 2.0 * kPi * T;
  Maxwell<M> m;
  m.ux = static_cast<M>(ux);
  m.uy = static_cast<M>(uy);
  m.uz = static_cast<M>(uz);
  m.A = static_cast<M>(rho / (two_pi_T * sqrt(two_pi_T)));
  m.B = static_cast<M>(1.0 / (2.0 * T));
  return m;
}

// Shakhov target f^S = eq [1 + coef (c.q)(|c|^2/theta - 5) + g0 + g.c + g4 |c|^2 / 2], c = xi - uc,
// plus the per-cell collision coefficient V/tau and the velocity-independent LU-SGS diagonal
// (ShakhovTarget + CellParams, src/kinetic/kinetic_types.hpp:67-98)
template <class M>
struct CellParams {
  Maxwell<M> eq;
  M ucx, ucy, ucz;
  M qx, qy, qz;
  M theta, coef, g0, g4, gx, gy, gz;
  M coll, diag;
  M inv_theta;  // 1 / theta: the Shakhov polynomial multiplies by it (no division per velocity)
};

// cell parameters in another precision (member by member)
template <class To, class From>
__host__ __device__ inline CellParams<To> cast_cell_params(const CellParams<From>& s) {
  CellParams<To> o;
  o.eq.ux = static_cast<To>(s.eq.ux);
  o.eq.uy = static_cast<To>(s.eq.uy);
  o.eq.uz = static_cast<To>(s.eq.uz);
  o.eq.A = static_cast<To>(s.eq.A);
  o.eq.B = static_cast<To>(s.eq.B);
  o.ucx = static_cast<To>(s.ucx);
  o.ucy = static_cast<To>(s.ucy);
  o.ucz = static_cast<To>(s.ucz);
  o.qx = static_cast<To>(s.qx);
  o.qy = static_cast<To>(s.qy);
  o.qz = static_cast<To>(s.qz);
  o.theta = static_cast<To>(s.theta);
  o.coef = static_cast<To>(s.coef);
  o.g0 = static_cast<To>(s.g0);
  o.g4 = static_cast<To>(s.g4);
  o.gx = static_cast<To>(s.gx);
  o.gy = static_cast<To>(s.gy);
  o.gz = static_cast<To>(s.gz);
  o.coll = static_cast<To>(s.coll);
  o.diag = static_cast<To>(s.diag);
  o.inv_theta = static_cast<To>(s.inv_theta);
  return o;
}

template <class M>
__host__ __device__ inline M shakhov_poly(const CellParams<M>& s, M cx, M cy, M cz, M c2) {
  return s.coef * (cx * s.qx + cy * s.qy + cz * s.qz) * (c2 * s.inv_theta - M(5));
}

template <class M>
__host__ __device__ inline M shakhov_target(const CellParams<M>& s, M x, M y, M z) {
  const M cx = x - s.ucx, cy = y - s.ucy, cz = z - s.ucz;
  const M c2 = cx * cx + cy * cy + cz * cz;
  const M m = maxwellian(s.eq, x, y, z);
  return m * (M(1) + shakhov_poly(s, cx, cy, cz, c2) + (s.g0 + (s.gx * cx + s.gy * cy + s.gz * cz) + M(0.5) * s.g4 * c2));
}

// make_cell_params (src/kinetic/kinetic_kernels.hpp:451-471): Shakhov target from the 15 moments, mu = mu0 T^omega
template <class M>
__host__ __device__ inline CellParams<M> make_cell_params(const double* m, double volume, double vdt, double mu0,
                                                          double omega, double Pr, double cold_bgk_T) {
  const double rho = m[0], T = m[4];
  const double two_pi_T = 2.0 * kPi * T;
  CellParams<M> cp;
  cp.eq.ux = static_cast<M>(m[1]);
  cp.eq.uy = static_cast<M>(m[2]);
  cp.eq.uz = static_cast<M>(m[3]);
  cp.eq.A = static_cast<M>(rho / (two_pi_T * sqrt(two_pi_T)));
  cp.eq.B = static_cast<M>(1.0 / (2.0 * T));
  cp.ucx = cp.eq.ux;
  cp.ucy = cp.eq.uy;
  cp.ucz = cp.eq.uz;
  cp.qx = static_cast<M>(m[12]);
  cp.qy = static_cast<M>(m[13]);
  cp.qz = static_cast<M>(m[14]);
  cp.theta = static_cast<M>(T);
  cp.inv_theta = static_cast<M>(1.0 / T);
  const double p = rho * T;
  const double coef = (1.0 - Pr) / (5.0 * p * T);
  cp.coef = T < cold_bgk_T ? M(0) : static_cast<M>(coef);
  cp.g0 = M(0);
  cp.g4 = M(0);
  cp.gx = cp.gy = cp.gz = M(0);
  const double mu = mu0 * pow(T, omega);
  const double coll = volume * m[5] / mu;
  cp.coll = static_cast<M>(coll);
  cp.diag = static_cast<M>(coll + vdt);
  return cp;
}

// Venkatakrishnan limiter of one face (venkatakrishnan_face, src/physics/limiter.hpp:17-31)
// num / den with subnormal operands first scaled by 2^64 (exact, so the correctly rounded quotient is unchanged):
// the FP32 limiter of states with tiny differences (far velocity tails, near-vacuum regions; d^2 below 1e-38)
// would otherwise divide subnormals, which the division handles off its fast path. Used where 0 <= num < den.
__host__ __device__ inline float limiter_quotient(float num, float den) {
  if (den < 0x1p-100f) {
    num *= 0x1p64f;
    den *= 0x1p64f;
  }
  return num / den;
}
__host__ __device__ inline double limiter_quotient(double num, double den) { return num / den; }

template <class M>
__host__ __device__ inline M venkat_face(M d2, M dmax, M dmin, M eps2) {
  M d1;
  if (d2 > M(0)) {
    d1 = dmax;
  } else if (d2 < M(0)) {
    d1 = dmin;
  } else {
    return M(1);
  }
  const M num = (d1 * d1 + eps2) + M(2) * d1 * d2;
  const M den = d1 * d1 + M(2) * d2 * d2 + d1 * d2 + eps2;
  if (!(den > M(0))) return M(0);
  // num >= den > 0: the quotient rounds to >= 1 and the clamp gives exactly 1, so the division can be skipped
  if (num >= den) return M(1);
  return kclamp(limiter_quotient(num, den), M(0), M(1));
}

// ---- discrete equilibrium (src/kinetic/discrete_equilibrium.hpp) -------------------------------------------

struct DeqGrid {
  double lo[3], hi[3], d[3];
  double criterion, tolerance;
  int max_iterations;
};

// deq_resolved (discrete_equilibrium.hpp:35-48)
__host__ __device__ inline bool deq_resolved(const DeqGrid& g, double ux, double uy, double uz, double T) {
  if (!(T > 0.0)) return false;
  const double u[3] = {ux, uy, uz};
  for (int a = 0; a < 3; ++a) {
    if (2.0 * kPi * kPi * T / (g.d[a] * g.d[a]) < g.criterion) return false;
    const double m1 = g.hi[a] - u[a];
    const double m2 = u[a] - g.lo[a];
    if (!(m1 > 0.0 && m2 > 0.0)) return false;
    if (m1 * m1 < 2.0 * T * g.criterion || m2 * m2 < 2.0 * T * g.criterion) return false;
  }
  return true;
}

// deq_terms (discrete_equilibrium.hpp:56-80)
template <class M>
__host__ __device__ inline void deq_terms(M e, M pm, M cx, M cy, M cz, M (&t)[kDeqSums]) {
  const M h = M(0.5) * (cx * cx + cy * cy + cz * cz);
  t[0] = e;
  t[1] = e * cx;
  t[2] = e * cy;
  t[3] = e * cz;
  t[4] = e * h;
  t[5] = t[1] * cx;
  t[6] = t[1] * cy;
  t[7] = t[1] * cz;
  t[8] = t[1] * h;
  t[9] = t[2] * cy;
  t[10] = t[2] * cz;
  t[11] = t[2] * h;
  t[12] = t[3] * cz;
  t[13] = t[3] * h;
  t[14] = t[4] * h;
  const M ep = e * pm;
  t[15] = ep;
  t[16] = ep * cx;
  t[17] = ep * cy;
  t[18] = ep * cz;
  t[19] = ep * h;
}

// symmetric 5x5 Jacobian from the sums (deq_jacobian, :83-94)
__host__ __device__ inline void deq_jacobian(const double* s, double w, double (&J)[5][5]) {
  int k = 0;
  for (int a = 0; a < 5; ++a) {
    for (int b = a; b < 5; ++b) {
      J[a][b] = w * s[k];
      J[b][a] = J[a][b];
      ++k;
    }
  }
}

// Gaussian elimination with partial pivoting (deq_solve5, :97-131)
__host__ __device__ inline bool deq_solve5(double (&A)[5][5], double (&b)[5], double (&x)[5]) {
  for (int k = 0; k < 5; ++k) {
    int piv = k;
    double best = fabs(A[k][k]);
    for (int r = k + 1; r < 5; ++r) {
      if (fabs(A[r][k]) > best) {
        best = fabs(A[r][k]);
        piv = r;
      }
    }
    if (!(best > 0.0)) return false;
    if (piv != k) {
      for (int cc = 0; cc < 5; ++cc) {
        const double tmp = A[k][cc];
        A[k][cc] = A[piv][cc];
        A[piv][cc] = tmp;
      }
      const double tb = b[k];
      b[k] = b[piv];
      b[piv] = tb;
    }
    for (int r = k + 1; r < 5; ++r) {
      const double f = A[r][k] / A[k][k];
      for (int cc = k; cc < 5; ++cc) A[r][cc] -= f * A[k][cc];
      b[r] -= f * b[k];
    }
  }
  for (int k = 4; k >= 0; --k) {
    double sum = b[k];
    for (int cc = k + 1; cc < 5; ++cc) sum -= A[k][cc] * x[cc];
    x[k] = sum / A[k][k];
    if (!(x[k] == x[k])) return false;
  }
  return true;
}

// initial beta: the continuous Maxwellian (deq_initial_beta, :134-141)
__host__ __device__ inline void deq_initial_beta(double rho, double T, double (&beta)[5]) {
  const double two_pi_T = 2.0 * kPi * T;
  beta[0] = log(rho / (two_pi_T * sqrt(two_pi_T)));
  beta[1] = 0.0;
  beta[2] = 0.0;
  beta[3] = 0.0;
  beta[4] = -1.0 / T;
}

// beta -> A exp(-B |xi - u'|^2) (deq_params, :144-155)
template <class M>
__host__ __device__ inline Maxwell<M> deq_params(const double (&beta)[5], double ux, double uy, double uz) {
  const double B = -0.5 * beta[4];
  const double dx = -beta[1] / beta[4];
  const double dy = -beta[2] / beta[4];
  const double dz = -beta[3] / beta[4];
  Maxwell<M> m;
  m.ux = static_cast<M>(ux + dx);
  m.uy = static_cast<M>(uy + dy);
  m.uz = static_cast<M>(uz + dz);
  m.A = static_cast<M>(exp(beta[0] + B * (dx * dx + dy * dy + dz * dz)));
  m.B = static_cast<M>(B);
  return m;
}

// one damped Newton step (deq_newton_step, :159-180): 1 converged, 0 updated, -1 failed
__host__ __device__ inline int deq_newton_step(const double* s, double w, double rho, double T, double tol,
                                               double (&beta)[5], double& rel) {
  double G[5] = {w * s[0] - rho, w * s[1], w * s[2], w * s[3], w * s[4] - 1.5 * rho * T};
  const double su = rho * sqrt(T);
  rel = kmax(fabs(G[0]) / rho, kmax(kmax(fabs(G[1]), kmax(fabs(G[2]), fabs(G[3]))) / su, fabs(G[4]) / (rho * T)));
  if (!(rel == rel)) return -1;
  if (rel < tol) return 1;
  double J[5][5];
  deq_jacobian(s, w, J);
  double rhs[5] = {-G[0], -G[1], -G[2], -G[3], -G[4]};
  double d[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (!deq_solve5(J, rhs, d)) return -1;
  double scale = 1.0;
  if (fabs(d[4]) > 0.5 * fabs(beta[4])) scale = 0.5 * fabs(beta[4]) / fabs(d[4]);
  if (fabs(d[0]) * scale > 1.0) scale = 1.0 / fabs(d[0]);
  for (int k = 0; k < 5; ++k) beta[k] += scale * d[k];
  if (!(beta[4] < 0.0)) return -1;
  return 0;
}

// Shakhov-polynomial correction gamma (deq_shakhov_correction, :183-188)
__host__ __device__ inline bool deq_shakhov_correction(const double* s, double w, double (&gamma)[5]) {
  double J[5][5];
  deq_jacobian(s, w, J);
  double rhs[5] = {-w * s[15], -w * s[16], -w * s[17], -w * s[18], -w * s[19]};
  return deq_solve5(J, rhs, gamma);
}

// stopping rule of the Newton iteration (deq_accept, src/kinetic/kinetic_kernels.hpp:489-493)
__host__ __device__ inline bool deq_accept(int r, double rel, double rel_prev, bool last) {
  if (r == 1) return true;
  if (r == 0 && rel < 1e-4 && (rel > 0.5 * rel_prev || last)) return true;
  return false;
}

// ---- GSIS correction helpers (src/kinetic/kinetic_kernels.hpp:557-581) ------------------------------------

template <class M>
__host__ __device__ inline M negative_check_value(M old, M x, bool created) {
  return created ? x - kmin(old, M(0)) : x;
}

template <class M>
__host__ __device__ inline M correction_alpha_limit(M old, M d, M thr) {
  if (!(d < M(0))) return M(1);
  const M room = old - (kmin(old, M(0)) + thr);
  return kmin(M(1), room / (-d));
}

template <class M>
__host__ __device__ inline M blend_theta(M old, M d, M e, M thr) {
  const M g = old + d;
  const M bound = kmin(old, M(0)) + thr;
  if (!(g < bound)) return M(0);
  const M den = e - g;
  if (!(den > M(0))) return M(1);
  return kmin(M(1), (bound - g) / den);
}

// ---- moments (moment_terms / finalize_moments, src/kinetic/kinetic_kernels.hpp:382-442) ----------------------

__host__ __device__ inline void finalize_moments(const double* s, double weight, double u0x, double u0y, double u0z,
                                                 double* out) {
  const double s0 = s[0];
  if (!(s0 > 0.0)) {
    out[0] = weight * s0;
    for (int k = 1; k < 15; ++k) out[k] = 0.0;
    return;
  }
  const double dx = s[1] / s0;
  const double dy = s[2] / s0;
  const double dz = s[3] / s0;
  const double rho = weight * s0;
  const double pxx = weight * (s[4] - s0 * dx * dx);
  const double pyy = weight * (s[5] - s0 * dy * dy);
  const double pzz = weight * (s[6] - s0 * dz * dz);
  const double pxy = weight * (s[7] - s0 * dx * dy);
  const double pyz = weight * (s[8] - s0 * dy * dz);
  const double pxz = weight * (s[9] - s0 * dx * dz);
  const double p = (pxx + pyy + pzz) / 3.0;
  const double tr2 = s[4] + s[5] + s[6];
  const double du2 = dx * dx + dy * dy + dz * dz;
  const double s2dx = s[4] * dx + s[7] * dy + s[9] * dz;
  const double s2dy = s[7] * dx + s[5] * dy + s[8] * dz;
  const double s2dz = s[9] * dx + s[8] * dy + s[6] * dz;
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

}  // namespace kin
