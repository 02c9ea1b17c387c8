// Discrete adjoint of the converged CIS fixed point (FP64 arithmetic, FP64 or FP32 storage; sm_100a): the transposed-Jacobian kernels of
// kin_adjoint.h. The forward map they transpose is residual_value / limited_gradient / boundary_value_first_order
// (src/kinetic/kinetic_kernels.hpp:145-278), make_cell_params (:451-471) and the boundary sums of the wall density
// (src/kinetic/kinetic_cuda_kernels.cu:275-323, src/kinetic/kinetic_solver.cpp:280-335); every derivative below is
// that of the forward arithmetic in kin_kernels.cuh / kin_math.cuh.
//
// One CTA per cell (or per boundary face) walks the velocities with consecutive threads on consecutive velocities,
// so every access to f, lambda and the seed arrays is coalesced. Every velocity sum is a fixed-order block sum (no
// atomics: results are bitwise reproducible). The neighbour terms of the transposed gradient are gathered by the
// receiving cell through the reverse CSR entry instead of being scattered.
#include "kin_adjoint.h"

namespace kin {
namespace {

constexpr int kAdjThreads = 256;

template <class S>
__device__ __forceinline__ double lam_at(const AdjView<S>& a, int nv, int cell, int q) {
  return static_cast<double>(a.lam[static_cast<int64_t>(cell) * nv + a.rev[q]]);
}

template <class S>
__device__ __forceinline__ double ld(const S* p, int64_t i) {
  return static_cast<double>(p[i]);
}

// seed weight of the face moment sums sum_q w psi(xi_q) f_b(q), psi = (1, xi, |xi|^2 / 2), at one velocity
__device__ __forceinline__ double face_moment_seed(const double* __restrict__ m, double x, double y, double z) {
  return m[0] + m[1] * x + m[2] * y + m[3] * z + m[4] * (0.5 * (x * x + y * y + z * z));
}

template <class S>
__device__ __forceinline__ double entry_value(const View<S, double>& v, const CsrE<double>& c, int cell, int q,
                                              double x, double y, double z, double fi) {
  return c.other >= 0 ? f_at(v, c.other, q) : boundary_value_first_order(v, c, cell, q, x, y, z, fi);
}

// k_adj_cell: per cell, sum_q lambda_q * {f^S_q - f_q, d f^S_q / d(rho, u, T, q)} of the Shakhov target
// (shakhov_target, src/kinetic/kinetic_types.hpp:79-90). Continuous equilibrium: f^S = M (1 + P),
// P = coef (c.q)(c^2 / T - 5). Discrete equilibrium (deq_flags > 0): f^S = E F, F = 1 + P + gamma . psi,
// psi = (1, c, c^2 / 2), E = A exp(-B |xi - u'|^2) from the Newton solve: the derivative sums at fixed (beta, gamma)
// and sum lambda E F psi, sum lambda E psi for the chain through the Newton and gamma solves (host).
template <class S>
__global__ void __launch_bounds__(kAdjThreads) k_adj_cell(View<S, double> v, AdjView<S> a, double* __restrict__ out) {
  __shared__ double sh[kAdjCellSums * (kAdjThreads / 32)];
  const int cell = blockIdx.x;
  const int nv = v.nv;
  const CellParams<double> cp = v.cp[cell];
  const double rho = a.moments[static_cast<int64_t>(cell) * 15];
  const double T = cp.theta, kap = cp.coef;
  const bool discrete = a.deq_flags != nullptr && a.deq_flags[cell] > 0;
  double s[kAdjCellSums];
#pragma unroll
  for (int k = 0; k < kAdjCellSums; ++k) s[k] = 0.0;
  for (int q = threadIdx.x; q < nv; q += kAdjThreads) {
    const double x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
    const double cx = x - cp.ucx, cy = y - cp.ucy, cz = z - cp.ucz;
    const double c2 = cx * cx + cy * cy + cz * cz;
    const double M = maxwellian(cp.eq, x, y, z);
    const double cq = cx * cp.qx + cy * cp.qy + cz * cp.qz;
    const double h = c2 / T - 5.0;
    const double P = kap * cq * h;
    const double lam = lam_at(a, nv, cell, q);
    const double fi = f_at(v, cell, q);
    const double lm = lam * M;
    if (!discrete) {
      s[0] += lam * (M * (1.0 + P) - fi);
      s[1] += lm / rho;
      const double onep = 1.0 + P;
      s[2] += lm * (cx / T * onep + kap * (-cp.qx * h - 2.0 * cq * cx / T));
      s[3] += lm * (cy / T * onep + kap * (-cp.qy * h - 2.0 * cq * cy / T));
      s[4] += lm * (cz / T * onep + kap * (-cp.qz * h - 2.0 * cq * cz / T));
      s[5] += lm * ((c2 / (2.0 * T * T) - 1.5 / T) * onep + cq * (-2.0 * kap / T * h - kap * c2 / (T * T)));
      s[6] += lm * kap * cx * h;
      s[7] += lm * kap * cy * h;
      s[8] += lm * kap * cz * h;
    } else {
      const double F = 1.0 + P + (cp.g0 + (cp.gx * cx + cp.gy * cy + cp.gz * cz) + 0.5 * cp.g4 * c2);
      const double lmf = lm * F;
      const double twoB = 2.0 * cp.eq.B;
      s[0] += lam * (M * F - fi);
      s[1] += -lm * P / rho;
      s[2] += lmf * twoB * (x - cp.eq.ux) + lm * (kap * (-cp.qx * h - 2.0 * cq * cx / T) - (cp.gx + cp.g4 * cx));
      s[3] += lmf * twoB * (y - cp.eq.uy) + lm * (kap * (-cp.qy * h - 2.0 * cq * cy / T) - (cp.gy + cp.g4 * cy));
      s[4] += lmf * twoB * (z - cp.eq.uz) + lm * (kap * (-cp.qz * h - 2.0 * cq * cz / T) - (cp.gz + cp.g4 * cz));
      s[5] += lm * cq * (-2.0 * kap / T * h - kap * c2 / (T * T));
      s[6] += lm * kap * cx * h;
      s[7] += lm * kap * cy * h;
      s[8] += lm * kap * cz * h;
      s[9] += lmf;
      s[10] += lmf * cx;
      s[11] += lmf * cy;
      s[12] += lmf * cz;
      s[13] += lmf * 0.5 * c2;
      s[14] += lm;
      s[15] += lm * cx;
      s[16] += lm * cy;
      s[17] += lm * cz;
      s[18] += lm * 0.5 * c2;
    }
  }
  block_sum<kAdjCellSums, kAdjThreads>(s, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < kAdjCellSums; ++k) out[static_cast<int64_t>(cell) * kAdjCellSums + k] = s[k];
  }
}

// k_adj_transport: the transposed upwind flux and limited gradient at (cell, q). Writes the seeds that stay in the
// cell (lfb), the gradient seed G_bar and the limiter-extremum seeds for the gathers of k_adj_gather / k_adj_faces.
template <class S>
__global__ void __launch_bounds__(kAdjThreads) k_adj_transport(View<S, double> v, AdjView<S> a,
                                                              const int32_t* __restrict__ cells) {
  const int cell = cells != nullptr ? cells[blockIdx.x] : static_cast<int>(blockIdx.x);
  const int nv = v.nv;
  const int e0 = v.csr_off[cell], e1 = v.csr_off[cell + 1];
  const double coll = v.cp[cell].coll;
  const bool lim = v.limiter_mode != kLimNone;
  for (int q = threadIdx.x; q < nv; q += kAdjThreads) {
    const double x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
    const double fi = f_at(v, cell, q);
    const double wq = v.wts != nullptr ? v.wts[q] : v.weight;
    // forward: unlimited gradient and stencil extrema (the first of equal values wins, as kmax / kmin keep it)
    double Gx = 0.0, Gy = 0.0, Gz = 0.0, fmax = fi, fmin = fi;
    int amax = -1, amin = -1;
    for (int e = e0; e < e1; ++e) {
      const CsrE<double>& c = v.csr[e];
      const double fk = entry_value(v, c, cell, q, x, y, z, fi);
      const double d = fk - fi;
      Gx += c.c[0] * d;
      Gy += c.c[1] * d;
      Gz += c.c[2] * d;
      if (fmax < fk) {
        fmax = fk;
        amax = e - e0;
      }
      if (fk < fmin) {
        fmin = fk;
        amin = e - e0;
      }
    }
    double phi = 1.0, eps2 = 0.0;
    int estar = -1;
    const double dmax = fmax - fi, dmin = fmin - fi;
    if (lim) {
      eps2 = v.eps2[cell];
      if (v.limiter_mode == kLimRel) {
        const double s = kmax(kabs(fmax), kabs(fmin));
        eps2 *= s * s;
      }
      for (int e = e0; e < e1; ++e) {
        const CsrE<double>& c = v.csr[e];
        if (c.other < 0 && v.bf[c.bface].kind == kPeriodic) continue;
        const double proj = Gx * c.ds[0] + Gy * c.ds[1] + Gz * c.ds[2];
        const double vv = venkat_face(proj, dmax, dmin, eps2);
        if (vv < phi) {
          phi = vv;
          estar = e - e0;
        }
      }
    }
    // seeds on the face values f_i + g_i . ds of the faces this cell is upwind of
    const double li = lam_at(a, nv, cell, q);
    double lf = coll * li;  // R_i contains + coll f_i
    double vx = 0.0, vy = 0.0, vz = 0.0;
    for (int e = e0; e < e1; ++e) {
      const CsrE<double>& c = v.csr[e];
      const double ae = x * c.s[0] + y * c.s[1] + z * c.s[2];
      double sig;
      if (c.other >= 0) {
        if (ae < 0.0) continue;  // the neighbour is upwind: its own thread carries this face
        sig = ae * (li - lam_at(a, nv, c.other, q));
      } else {
        const BFace<double>& b = v.bf[c.bface];
        if (b.kind == kPeriodic) continue;
        if (b.kind == kSymmetry) {
          // own outgoing term, plus the mirrored incoming term of velocity qm that reads this face value
          const int qm = v.mirror_map[b.mirror * nv + q];
          const double am = v.xi_x[qm] * c.s[0] + v.xi_y[qm] * c.s[1] + v.xi_z[qm] * c.s[2];
          sig = (ae >= 0.0 ? ae * li : 0.0) + (am < 0.0 ? am * lam_at(a, nv, cell, qm) : 0.0);
          // face moment sums: this value is the outgoing half at q and the incoming half at qm (mirror weights are
          // equal on every grid of the reference)
          if (a.mom_mu != nullptr && ae >= 0.0) {
            sig += wq * face_moment_seed(a.mom_mu + 5 * c.bface, x, y, z);
            if (am < 0.0) sig += wq * face_moment_seed(a.mom_mu + 5 * c.bface, v.xi_x[qm], v.xi_y[qm], v.xi_z[qm]);
          }
        } else {
          if (ae < 0.0) continue;  // incoming inflow value: k_adj_faces
          sig = ae * (li + (a.mu != nullptr ? wq * a.mu[c.bface] : 0.0));
          if (a.mom_mu != nullptr) sig += wq * face_moment_seed(a.mom_mu + 5 * c.bface, x, y, z);
        }
      }
      lf += sig;
      vx += sig * c.ds[0];
      vy += sig * c.ds[1];
      vz += sig * c.ds[2];
    }
    // g = phi G
    double gbx = phi * vx, gby = phi * vy, gbz = phi * vz;
    double hmx = 0.0, hmn = 0.0;
    if (lim && estar >= 0) {
      const double phibar = vx * Gx + vy * Gy + vz * Gz;
      const CsrE<double>& c = v.csr[e0 + estar];
      const double p = Gx * c.ds[0] + Gy * c.ds[1] + Gz * c.ds[2];
      const double d1 = p > 0.0 ? dmax : dmin;
      const double num = (d1 * d1 + eps2) + 2.0 * d1 * p;
      const double den = d1 * d1 + 2.0 * p * p + d1 * p + eps2;
      if (p != 0.0 && den > 0.0 && num < den && num / den > 0.0) {  // venkat_face not clamped: differentiable
        const double den2 = den * den;
        const double dv_dp = (2.0 * d1 * den - num * (4.0 * p + d1)) / den2;
        const double dv_dd1 = ((2.0 * d1 + 2.0 * p) * den - num * (2.0 * d1 + p)) / den2;
        const double dv_de = (den - num) / den2;
        const double pb = phibar * dv_dp;
        gbx += pb * c.ds[0];
        gby += pb * c.ds[1];
        gbz += pb * c.ds[2];
        const double d1b = phibar * dv_dd1;
        if (p > 0.0) hmx += d1b;
        else hmn += d1b;
        lf -= d1b;
        if (v.limiter_mode == kLimRel) {
          // eps2 = eps2_cell s^2 with s = max(|fmax|, |fmin|) (|fmin| only when |fmax| < |fmin|)
          const double e2c = v.eps2[cell];
          const bool use_min = kabs(fmax) < kabs(fmin);
          const double s = use_min ? kabs(fmin) : kabs(fmax);
          const double sb = phibar * dv_de * e2c * 2.0 * s;
          if (use_min) hmn += fmin < 0.0 ? -sb : sb;
          else hmx += fmax < 0.0 ? -sb : sb;
        }
      }
    }
    if (amax < 0) {
      lf += hmx;
      hmx = 0.0;
    }
    if (amin < 0) {
      lf += hmn;
      hmn = 0.0;
    }
    // G = sum_e c_e (f_k - f_i): the f_i part, and the boundary entries whose value is this cell's own f
    double sumc = 0.0;
    for (int e = e0; e < e1; ++e) {
      const CsrE<double>& c = v.csr[e];
      const double cg = c.c[0] * gbx + c.c[1] * gby + c.c[2] * gbz;
      sumc += cg;
      if (c.other >= 0) continue;  // gathered by the neighbour
      const int k = e - e0;
      const double s = cg + (amax == k ? hmx : 0.0) + (amin == k ? hmn : 0.0);
      const BFace<double>& b = v.bf[c.bface];
      if (b.kind == kPeriodic) {
        lf += s;
      } else if (b.kind == kSymmetry) {
        lf += 0.5 * s;  // the other half lands on the mirrored velocity (k_adj_gather)
      } else if (x * c.s[0] + y * c.s[1] + z * c.s[2] >= 0.0) {
        lf += s;
      }  // incoming wall / pressure value: k_adj_faces; vacuum: constant 0
    }
    lf -= sumc;
    const int64_t i = static_cast<int64_t>(cell) * nv + q;
    a.lfb[i] = static_cast<S>(lf);
    a.gbx[i] = static_cast<S>(gbx);
    a.gby[i] = static_cast<S>(gby);
    a.gbz[i] = static_cast<S>(gbz);
    a.hmax[i] = static_cast<S>(hmx);
    a.hmin[i] = static_cast<S>(hmn);
    a.imax[i] = static_cast<int8_t>(amax);
    a.imin[i] = static_cast<int8_t>(amin);
  }
}

// k_adj_faces: per wall / pressure face, the seeds on the incoming inflow values (residual term, gradient entry and
// limiter extremum) summed against the inflow Maxwellian m: S0 = sum s M, S1 = sum s M c, S2 = sum s M c^2 with
// c = xi - u_b; for the wall-temperature derivative of sm5 also S5 = sum_in w an M c^2, S6 = sum_in w an M. For a
// diffuse wall aligned with an axis, the partially specular inflow rho M + (1 - alpha) f_spec of a Maxwell wall
// (maxwell_inflow / reflected_value, src/kinetic/kinetic_kernels.hpp:86-133) gives the accommodation derivative at
// alpha = 1 from A1 = sum_in a lambda f_spec (f_spec: the owner's reconstructed face value at the reflected
// velocity), A2 = sum_in s_grad f_o(reflected) (the first-order specular value of the gradient),
// S_spec = sum_in w an f_spec and, for the face state of the limited pressure-boundary reconstruction,
// sum_in w psi f_spec (5).
template <class S>
__global__ void __launch_bounds__(kAdjThreads) k_adj_faces(View<S, double> v, AdjView<S> a, double* __restrict__ out) {
  __shared__ double sh[kAdjFaceSums * (kAdjThreads / 32)];
  const int b = blockIdx.x;
  const int nv = v.nv;
  const BFace<double> bf = v.bf[b];
  double s[kAdjFaceSums];
#pragma unroll
  for (int k = 0; k < kAdjFaceSums; ++k) s[k] = 0.0;
  if (bf.kind == kDiffuseWall || bf.kind == kPressure) {
    const int o = bf.owner;
    const int e0 = v.csr_off[o], e1 = v.csr_off[o + 1];
    int eb = e0;
    for (int e = e0; e < e1; ++e)
      if (v.csr[e].other < 0 && v.csr[e].bface == b) eb = e;
    const CsrE<double> c = v.csr[eb];
    const int k = eb - e0;
    const Maxwell<double> m = v.inflow[b].m;
    const double mu = (bf.kind == kPressure && a.mu != nullptr) ? a.mu[b] : 0.0;
    for (int q = threadIdx.x; q < nv; q += kAdjThreads) {
      const double x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
      const double ae = x * c.s[0] + y * c.s[1] + z * c.s[2];
      if (ae >= 0.0) continue;
      const double wq = v.wts != nullptr ? v.wts[q] : v.weight;
      const int64_t i = static_cast<int64_t>(o) * nv + q;
      const double seed = ae * (lam_at(a, nv, o, q) + wq * mu) + c.c[0] * ld(a.gbx, i) + c.c[1] * ld(a.gby, i) +
                          c.c[2] * ld(a.gbz, i) + (a.imax[i] == k ? ld(a.hmax, i) : 0.0) +
                          (a.imin[i] == k ? ld(a.hmin, i) : 0.0);
      const double M = maxwellian(m, x, y, z);
      const double cx = x - m.ux, cy = y - m.uy, cz = z - m.uz;
      const double c2 = cx * cx + cy * cy + cz * cz;
      const double sm = seed * M;
      s[0] += sm;
      s[1] += sm * cx;
      s[2] += sm * cy;
      s[3] += sm * cz;
      s[4] += sm * c2;
      const double wa = wq * ae / bf.area * M;
      s[5] += wa * c2;
      s[6] += wa;
      s[10] += wa * cx;
      s[11] += wa * cy;
      s[12] += wa * cz;
      if (bf.kind == kDiffuseWall && a.face_axis != nullptr && a.face_axis[b] >= 0) {
        const int r = a.flip[a.face_axis[b] * nv + q];
        const double xr = v.xi_x[r], yr = v.xi_y[r], zr = v.xi_z[r];
        const double fr = f_at(v, o, r);
        double gx, gy, gz;
        limited_gradient(v, o, r, xr, yr, zr, fr, gx, gy, gz);
        const double fspec = fr + gx * bf.d[0] + gy * bf.d[1] + gz * bf.d[2];
        const double sgrad = seed - ae * (lam_at(a, nv, o, q) + wq * mu);
        s[7] += ae * lam_at(a, nv, o, q) * fspec;
        s[8] += sgrad * fr;
        s[9] += wq * ae / bf.area * fspec;
        // the specular part's share of the face moment sums (the accommodation derivative of the face state)
        const double wf = wq * fspec;
        s[13] += wf;
        s[14] += wf * x;
        s[15] += wf * y;
        s[16] += wf * z;
        s[17] += wf * (0.5 * (x * x + y * y + z * z));
      }
    }
  }
  block_sum<kAdjFaceSums, kAdjThreads>(s, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < kAdjFaceSums; ++k) out[static_cast<int64_t>(b) * kAdjFaceSums + k] = s[k];
  }
}

// k_adj_gather: O_f(y) at (cell, q) = the cell's own seeds + the neighbours' gradient and extremum seeds that point at
// it + the mirrored half of the symmetry values + the moment expansion; stored at the reversed position. Per-cell
// sum of squares into res_cell.
template <class S>
__global__ void __launch_bounds__(kAdjThreads) k_adj_gather(View<S, double> v, AdjView<S> a,
                                                           double* __restrict__ res_cell) {
  __shared__ double sh[kAdjThreads / 32];
  const int cell = blockIdx.x;
  const int nv = v.nv;
  const int e0 = v.csr_off[cell], e1 = v.csr_off[cell + 1];
  const double* mo = a.moments + static_cast<int64_t>(cell) * 15;
  const double ux = mo[1], uy = mo[2], uz = mo[3];
  const double* cf = a.coef + static_cast<int64_t>(cell) * kAdjCoefs;
  const double a0 = cf[0], ax = cf[1], ay = cf[2], az = cf[3], a2 = cf[4], bx = cf[5], by = cf[6], bz = cf[7];
  double acc[1] = {0.0};
  for (int q = threadIdx.x; q < nv; q += kAdjThreads) {
    const int64_t i = static_cast<int64_t>(cell) * nv + q;
    double r = ld(a.lfb, i);
    for (int e = e0; e < e1; ++e) {
      const CsrE<double>& c = v.csr[e];
      if (c.other >= 0) {
        const int n = c.other;
        const int eb = a.rev_entry[e];
        if (eb < 0) continue;
        const CsrE<double>& cn = v.csr[eb];
        const int k = eb - v.csr_off[n];
        const int64_t j = static_cast<int64_t>(n) * nv + q;
        r += cn.c[0] * ld(a.gbx, j) + cn.c[1] * ld(a.gby, j) + cn.c[2] * ld(a.gbz, j);
        if (a.imax[j] == k) r += ld(a.hmax, j);
        if (a.imin[j] == k) r += ld(a.hmin, j);
      } else {
        const BFace<double>& b = v.bf[c.bface];
        if (b.kind != kSymmetry) continue;
        const int qm = v.mirror_map[b.mirror * nv + q];
        const int64_t j = static_cast<int64_t>(cell) * nv + qm;
        const int k = e - e0;
        const double s = c.c[0] * ld(a.gbx, j) + c.c[1] * ld(a.gby, j) + c.c[2] * ld(a.gbz, j) +
                         (a.imax[j] == k ? ld(a.hmax, j) : 0.0) + (a.imin[j] == k ? ld(a.hmin, j) : 0.0);
        r += 0.5 * s;
      }
    }
    const double x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
    const double cx = x - ux, cy = y - uy, cz = z - uz;
    const double c2 = cx * cx + cy * cy + cz * cz;
    const double wq = v.wts != nullptr ? v.wts[q] : v.weight;
    r += wq * (a0 + ax * cx + ay * cy + az * cz + a2 * c2 + (bx * cx + by * cy + bz * cz) * c2);
    a.out[static_cast<int64_t>(cell) * nv + a.rev[q]] = static_cast<S>(r);
    acc[0] += r * r;
  }
  block_sum<1, kAdjThreads>(acc, sh);
  if (threadIdx.x == 0) res_cell[cell] = acc[0];
}

}  // namespace

template <class S>
void adj_cell_sums(const View<S, double>& v, const AdjView<S>& a, double* out, cudaStream_t st) {
  k_adj_cell<S><<<v.n_cells, kAdjThreads, 0, st>>>(v, a, out);
}

template <class S>
void adj_transport(const View<S, double>& v, const AdjView<S>& a, const int32_t* cells, int n, cudaStream_t st) {
  const int grid = cells != nullptr ? n : v.n_cells;
  if (grid > 0) k_adj_transport<S><<<grid, kAdjThreads, 0, st>>>(v, a, cells);
}

template <class S>
void adj_face_sums(const View<S, double>& v, const AdjView<S>& a, double* out, cudaStream_t st) {
  if (v.n_bfaces > 0) k_adj_faces<S><<<v.n_bfaces, kAdjThreads, 0, st>>>(v, a, out);
}

template <class S>
void adj_gather(const View<S, double>& v, const AdjView<S>& a, double* res_cell, cudaStream_t st) {
  k_adj_gather<S><<<v.n_cells, kAdjThreads, 0, st>>>(v, a, res_cell);
}

#define KIN_ADJ_INSTANTIATE(S)                                                                   \
  template void adj_cell_sums<S>(const View<S, double>&, const AdjView<S>&, double*, cudaStream_t); \
  template void adj_transport<S>(const View<S, double>&, const AdjView<S>&, const int32_t*, int, cudaStream_t); \
  template void adj_face_sums<S>(const View<S, double>&, const AdjView<S>&, double*, cudaStream_t); \
  template void adj_gather<S>(const View<S, double>&, const AdjView<S>&, double*, cudaStream_t);
KIN_ADJ_INSTANTIATE(double)
KIN_ADJ_INSTANTIATE(float)
#undef KIN_ADJ_INSTANTIATE

}  // namespace kin
