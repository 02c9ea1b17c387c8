// sm_100a kernels of the B200 kinetic backend (SIMT; the path has no dense contraction, so no tensor cores).
//
// Data layout in HBM:
//   f[cell][q]            distribution function, q = the backend's velocity position (velocities grouped by LU-SGS
//                         sweep direction so that every 32-velocity tile of the sweep kernel follows one order)
//   gx/gy/gz/r[cell][t]   velocity-chunk work arrays, t = q - k0 (chunk [k0, k0 + kc))
// Consecutive threads of a warp always handle consecutive velocities of the SAME cell, so every f / work-array
// access of a warp is one contiguous, coalesced segment; per-cell tables (CSR entries, cell parameters) are
// warp-uniform broadcast loads.
//
// The LU-SGS sweep (kernel k_sweep_pass) walks each (direction group, RCB block) chain level by level: the host
// levels every block's cells so that all in-block neighbours that precede a cell in the reference sweep order
// sit on an earlier level. Cells of one level are independent, which is what turns the reference's
// one-thread-walks-2000-cells recurrence into short level loops without any inter-CTA synchronisation: a lane
// only ever reads LU-SGS values of its own velocity, so a warp needs no barrier at all.
#pragma once

#include "kin_math.cuh"

namespace kin {

template <class M>
struct CsrE {
  int32_t other;  // neighbour cell or -1
  int32_t bface;  // boundary face or -1
  M s[3];         // outward area vector S_out
  M ds[3];        // x_f - x_i
  M dn[3];        // x_f - x_j (internal faces)
  M c[3];         // LSQ coefficients
};

template <class M>
struct BFace {
  int32_t owner, kind, mirror, patch;  // mirror: slot of the mirror map (-1 none)
  M n[3];
  M area;
  M d[3];
};

template <class M>
struct Inflow {
  Maxwell<M> m;
  M scale;
};

// The velocity set of the discrete equilibrium as a tensor grid: node x_a[i] per axis and separable weights
// w(q) = w_x[i] w_y[j] w_z[k] (all 1 for a uniform grid, whose scalar weight the Newton step applies). Every sum of
// the Newton iteration is a sum over the grid of A exp(-B |xi - u'|^2) times a polynomial in c = xi - u, so it
// factors into products of per-axis sums sum_i w_a[i] exp(-B (x_a[i] - u'_a)^2) (x_a[i] - u_a)^k, k = 0..5:
// n_x + n_y + n_z exponentials per Newton iteration instead of n_x n_y n_z. n[0] == 0: not a tensor grid (the sums
// run over the velocity points).
struct DeqTensor {
  int32_t n[3];
  const double* node;  // n[0] + n[1] + n[2] nodes, axis by axis
  const double* w;     // per-axis weights, same layout
};

template <class S, class M>
struct View {
  int32_t n_cells, nv, n_bfaces;
  int32_t max_entries;  // largest number of CSR entries of a cell
  const M* xi_x;
  const M* xi_y;
  const M* xi_z;
  const double* xid_x;  // FP64 velocities (moments, boundary / Newton sums)
  const double* xid_y;
  const double* xid_z;
  const double* wts;    // per-velocity weights, nullptr when uniform
  double weight;        // uniform weight
  const int32_t* csr_off;
  const CsrE<M>* csr;
  const M* eps2;
  const BFace<M>* bf;
  const Inflow<M>* inflow;
  const CellParams<M>* cp;
  S* f;
  const int32_t* mirror_map;  // [slot][nv]
  int32_t limiter_mode, positivity;
  M diag_scale, interface_damping;
  // partially accommodating walls
  const int64_t* mw_offset;  // per boundary face, -1 if not a Maxwell wall
  const double* mw_frac;
  M* specular;
  M* specular_first;
  const int32_t* grid_to_pos;
  int32_t grid_n[3];
  DeqGrid deq;
  // velocity grid of the discrete equilibrium: the stored velocities, or the full grid when this handle stores one
  // shard of it (any order: only sums over it are taken)
  const M* dq_x;
  const M* dq_y;
  const M* dq_z;
  const double* dq_xd;
  const double* dq_yd;
  const double* dq_zd;
  const double* dq_w;  // per-velocity weights, nullptr when uniform
  int32_t dq_nv;
  DeqTensor dq_tensor;  // the same grid factored per axis (n[0] == 0 when it is not a tensor grid)
};

// velocities per thread x resident CTAs per SM of the gradient, residual and LU-SGS tile kernels
struct KernelShape {
  int32_t res_u, res_occ, grad_u, grad_occ, tile_u, tile_blocks;
};

template <class S>
struct Chunk {
  int32_t k0, kc, stride;
  S* gx;
  S* gy;
  S* gz;
  S* r;
  // mixed precision, FP32 residual of the inner sweeps (kDefect*): defect [cell][nv] of the FP32 residual against
  // the FP64 one at the iteration's first sweep
  S* defect = nullptr;
  int32_t defect_mode = 0;
  KernelShape shape{};  // of the kernel the chunk is given to (gradient or residual)
};
enum : int32_t { kDefectNone = 0, kDefectStore = 1, kDefectApply = 2 };

// ---------------------------------------------------------------------------------------------------------
// boundary inflow and first-order boundary values
// ---------------------------------------------------------------------------------------------------------

template <class M>
__device__ __forceinline__ M inflow_value(const Inflow<M>& b, M x, M y, M z) {
  return b.scale * maxwellian(b.m, x, y, z);
}

template <class S, class M>
__device__ __forceinline__ M f_at(const View<S, M>& v, int cell, int q) {
  return static_cast<M>(v.f[static_cast<int64_t>(cell) * v.nv + q]);
}

// boundary_value_first_order (src/kinetic/kinetic_kernels.hpp:145-157)
template <class S, class M>
__device__ inline M boundary_value_first_order(const View<S, M>& v, const CsrE<M>& c, int cell, int q, M x, M y, M z,
                                               M fi) {
  const BFace<M>& b = v.bf[c.bface];
  if (b.kind == kPeriodic) return fi;
  if (b.kind == kSymmetry) return M(0.5) * (fi + f_at(v, cell, v.mirror_map[b.mirror * v.nv + q]));
  const M a = x * c.s[0] + y * c.s[1] + z * c.s[2];
  if (a >= M(0)) return fi;
  if (b.kind == kMaxwellWall) {
    return inflow_value(v.inflow[c.bface], x, y, z) +
           static_cast<M>(v.mw_frac[c.bface]) * v.specular_first[v.mw_offset[c.bface] + q];
  }
  return inflow_value(v.inflow[c.bface], x, y, z);
}

// limited LSQ gradient phi * grad f (limited_gradient, src/kinetic/kinetic_kernels.hpp:161-201)
template <class S, class M>
__device__ inline void limited_gradient(const View<S, M>& v, int cell, int q, M x, M y, M z, M fi, M& gx, M& gy,
                                        M& gz) {
  const int e0 = v.csr_off[cell];
  const int e1 = v.csr_off[cell + 1];
  M sx = M(0), sy = M(0), sz = M(0);
  M fmax = fi, fmin = fi;
  for (int e = e0; e < e1; ++e) {
    const CsrE<M>& c = v.csr[e];
    const M fk = c.other >= 0 ? f_at(v, c.other, q) : boundary_value_first_order(v, c, cell, q, x, y, z, fi);
    const M d = fk - fi;
    sx += c.c[0] * d;
    sy += c.c[1] * d;
    sz += c.c[2] * d;
    fmax = kmax(fmax, fk);
    fmin = kmin(fmin, fk);
  }
  if (v.limiter_mode == kLimNone && v.positivity == 0) {
    gx = sx;
    gy = sy;
    gz = sz;
    return;
  }
  if (v.positivity != 0 && !(fi > M(0))) {
    gx = gy = gz = M(0);
    return;
  }
  M eps2 = v.eps2[cell];
  if (v.limiter_mode == kLimRel) {
    const M s = kmax(kabs(fmax), kabs(fmin));
    eps2 *= s * s;
  }
  const M dmax = fmax - fi, dmin = fmin - fi;
  M phi = M(1);
  M proj_min = M(0);
  for (int e = e0; e < e1; ++e) {
    const CsrE<M>& c = v.csr[e];
    if (c.other < 0 && v.bf[c.bface].kind == kPeriodic) continue;
    const M proj = sx * c.ds[0] + sy * c.ds[1] + sz * c.ds[2];
    if (v.limiter_mode != kLimNone) phi = kmin(phi, venkat_face(proj, dmax, dmin, eps2));
    proj_min = kmin(proj_min, proj);
  }
  if (v.positivity != 0 && proj_min < M(0)) {
    phi = fi > M(0) ? kmin(phi, fi / (-proj_min)) : M(0);
  }
  gx = phi * sx;
  gy = phi * sy;
  gz = phi * sz;
}

// reconstruct_at_boundary (src/kinetic/kinetic_kernels.hpp:205-211)
template <class S, class M>
__device__ inline M reconstruct_at_boundary(const View<S, M>& v, const BFace<M>& b, int q) {
  const M fi = f_at(v, b.owner, q);
  if (b.kind == kPeriodic) return fi;
  const M x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
  M gx, gy, gz;
  limited_gradient(v, b.owner, q, x, y, z, fi, gx, gy, gz);
  return fi + gx * b.d[0] + gy * b.d[1] + gz * b.d[2];
}

// specular part of a Maxwell wall (maxwell_inflow, src/kinetic/kinetic_kernels.hpp:130-133)
template <class S, class M>
__device__ __forceinline__ M maxwell_inflow(const View<S, M>& v, int b, int q, M x, M y, M z) {
  return inflow_value(v.inflow[b], x, y, z) + static_cast<M>(v.mw_frac[b]) * v.specular[v.mw_offset[b] + q];
}

// ---------------------------------------------------------------------------------------------------------
// deterministic block reductions (fixed order; no atomics anywhere in the sums)
// ---------------------------------------------------------------------------------------------------------

// sums of N doubles over the block; result valid in thread 0. sh: N * (B/32) doubles.
template <int N, int B>
__device__ inline void block_sum(double (&vals)[N], double* sh) {
  constexpr int W = B / 32;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int k = 0; k < N; ++k) vals[k] += __shfl_down_sync(0xffffffffu, vals[k], off);
  }
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) sh[k * W + warp] = vals[k];
  }
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double s = 0.0;
      for (int w = 0; w < W; ++w) s += sh[k * W + w];
      vals[k] = s;
    }
  }
  __syncthreads();
}

template <int B, class T, class Op>
__device__ inline T block_reduce_op(T val, T* sh, Op op) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) val = op(val, __shfl_down_sync(0xffffffffu, val, off));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (lane == 0) sh[warp] = val;
  __syncthreads();
  if (tid == 0) {
    T r = sh[0];
    for (int w = 1; w < B / 32; ++w) r = op(r, sh[w]);
    sh[0] = r;
  }
  __syncthreads();
  const T r = sh[0];
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------------------------------------------------
// discrete Maxwellian of one cell computed by a whole CTA (block_discrete_maxwell semantics,
// src/kinetic/kinetic_cuda_kernels.cu:71-145 and discrete_maxwell_seq, kinetic_kernels.hpp:499-540).
// Terms in M, sums in double. Returns Newton iterations (0: resolved, -1: failed) in every thread.
// ---------------------------------------------------------------------------------------------------------
// per-axis sums X_a[k] = sum_i w_a[i] exp(-B (x_a[i] - u'_a)^2) c^k, c = x_a[i] - u_a, k = 0..5 (18 values, axis
// by axis), reduced over the CTA; the result is valid in thread 0
template <int B>
__device__ inline void deq_axis_sums(const DeqTensor& tn, const double (&up)[3], const double (&uc)[3], double Bd,
                                     double (&acc)[18], double* sh_red) {
#pragma unroll
  for (int k = 0; k < 18; ++k) acc[k] = 0.0;
  int base = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    for (int i = threadIdx.x; i < tn.n[a]; i += B) {
      const double x = tn.node[base + i];
      const double r = x - up[a];
      const double c = x - uc[a];
      double p = tn.w[base + i] * exp(-Bd * (r * r));
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        acc[6 * a + k] += p;
        p *= c;
      }
    }
    base += tn.n[a];
  }
  block_sum<18, B>(acc, sh_red);
}

// the 20 Newton sums (deq_terms order) from the per-axis sums: sum e c^(i,j,k) = A X[i] Y[j] Z[k], with
// h = |c|^2 / 2 and the Shakhov polynomial pm = coef (c . q) (|c|^2 / theta - 5) expanded into monomials
__device__ inline void deq_sums_from_axes(const double (&ax)[18], double A, bool with_poly, double coef,
                                          const double (&q)[3], double theta, double (&s)[kDeqSums]) {
  const double* X = ax;
  const double* Y = ax + 6;
  const double* Z = ax + 12;
  auto m3 = [&](int i, int j, int k) { return A * (X[i] * Y[j] * Z[k]); };
  auto hh = [&](int i, int j, int k) { return 0.5 * (m3(i + 2, j, k) + m3(i, j + 2, k) + m3(i, j, k + 2)); };
  auto pp = [&](int i, int j, int k) {
    double r = 0.0;
    for (int a = 0; a < 3; ++a) {
      const int i1 = i + (a == 0), j1 = j + (a == 1), k1 = k + (a == 2);
      const double q2 = m3(i1 + 2, j1, k1) + m3(i1, j1 + 2, k1) + m3(i1, j1, k1 + 2);
      r += q[a] * (q2 / theta - 5.0 * m3(i1, j1, k1));
    }
    return coef * r;
  };
  s[0] = m3(0, 0, 0);
  s[1] = m3(1, 0, 0);
  s[2] = m3(0, 1, 0);
  s[3] = m3(0, 0, 1);
  s[4] = hh(0, 0, 0);
  s[5] = m3(2, 0, 0);
  s[6] = m3(1, 1, 0);
  s[7] = m3(1, 0, 1);
  s[8] = hh(1, 0, 0);
  s[9] = m3(0, 2, 0);
  s[10] = m3(0, 1, 1);
  s[11] = hh(0, 1, 0);
  s[12] = m3(0, 0, 2);
  s[13] = hh(0, 0, 1);
  s[14] = 0.5 * (hh(2, 0, 0) + hh(0, 2, 0) + hh(0, 0, 2));
  if (with_poly) {
    s[15] = pp(0, 0, 0);
    s[16] = pp(1, 0, 0);
    s[17] = pp(0, 1, 0);
    s[18] = pp(0, 0, 1);
    s[19] = 0.5 * (pp(2, 0, 0) + pp(0, 2, 0) + pp(0, 0, 2));
  } else {
    s[15] = s[16] = s[17] = s[18] = s[19] = 0.0;
  }
}

template <class M, int B>
__device__ int block_discrete_maxwell_on(const M* __restrict__ vx, const M* __restrict__ vy, const M* __restrict__ vz,
                                         const double* __restrict__ wts, int nv, double weight, const DeqGrid& deq,
                                         const DeqTensor& tn, double rho, double ux, double uy, double uz, double T,
                                         const CellParams<M>* poly, Maxwell<M>& out, double (&gamma)[5],
                                         double* sh_red, double* sh_state) {
  for (double& x : gamma) x = 0.0;
  out = maxwell_from<M>(rho, ux, uy, uz, T);
  if (deq_resolved(deq, ux, uy, uz, T)) return 0;
  const int tid = threadIdx.x;
  if (tid == 0) {
    double beta[5];
    deq_initial_beta(rho, T, beta);
    for (int k = 0; k < 5; ++k) sh_state[k] = beta[k];
    sh_state[5] = 0.0;
    for (int k = 0; k < 5; ++k) sh_state[6 + k] = 0.0;
    sh_state[11] = 1e300;
  }
  __syncthreads();
  const M fux = static_cast<M>(ux), fuy = static_cast<M>(uy), fuz = static_cast<M>(uz);
  const bool uniform = wts == nullptr;
  const double w = uniform ? weight : 1.0;
  for (int it = 0;; ++it) {
    const double beta[5] = {sh_state[0], sh_state[1], sh_state[2], sh_state[3], sh_state[4]};
    const Maxwell<M> m = deq_params<M>(beta, ux, uy, uz);
    double acc[kDeqSums];
    if (tn.n[0] > 0) {
      // tensor grid: the same sums from per-axis sums (deq_params in FP64: B = -beta4 / 2, u' = u - beta_a / beta4,
      // A = exp(beta0 + B |u' - u|^2))
      const double Bd = -0.5 * beta[4];
      const double dd[3] = {-beta[1] / beta[4], -beta[2] / beta[4], -beta[3] / beta[4]};
      const double up[3] = {ux + dd[0], uy + dd[1], uz + dd[2]};
      const double uc[3] = {static_cast<double>(fux), static_cast<double>(fuy), static_cast<double>(fuz)};
      double ax[18];
      deq_axis_sums<B>(tn, up, uc, Bd, ax, sh_red);
      if (tid == 0) {
        const double A = exp(beta[0] + Bd * (dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]));
        double qv[3] = {0.0, 0.0, 0.0};
        double coef = 0.0, theta = 1.0;
        if (poly != nullptr) {
          qv[0] = static_cast<double>(poly->qx);
          qv[1] = static_cast<double>(poly->qy);
          qv[2] = static_cast<double>(poly->qz);
          coef = static_cast<double>(poly->coef);
          theta = static_cast<double>(poly->theta);
        }
        deq_sums_from_axes(ax, A, poly != nullptr, coef, qv, theta, acc);
      }
    } else {
#pragma unroll
      for (int k = 0; k < kDeqSums; ++k) acc[k] = 0.0;
      M t[kDeqSums];
      for (int q = tid; q < nv; q += B) {
        const M x = vx[q], y = vy[q], z = vz[q];
        const M cx = x - fux, cy = y - fuy, cz = z - fuz;
        M e = maxwellian(m, x, y, z);
        const M pm = poly != nullptr ? shakhov_poly(*poly, cx, cy, cz, cx * cx + cy * cy + cz * cz) : M(0);
        if (!uniform) e *= static_cast<M>(wts[q]);
        deq_terms<M>(e, pm, cx, cy, cz, t);
#pragma unroll
        for (int k = 0; k < kDeqSums; ++k) acc[k] += static_cast<double>(t[k]);
      }
      block_sum<kDeqSums, B>(acc, sh_red);
    }
    if (tid == 0) {
      double b[5] = {beta[0], beta[1], beta[2], beta[3], beta[4]};
      double rel = 0.0;
      const int r = deq_newton_step(acc, w, rho, T, deq.tolerance, b, rel);
      if (deq_accept(r, rel, sh_state[11], it + 1 == deq.max_iterations)) {
        sh_state[5] = 1.0;
        if (poly != nullptr) {
          double gm[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
          if (deq_shakhov_correction(acc, w, gm)) {
            for (int k = 0; k < 5; ++k) sh_state[6 + k] = gm[k];
          }
        }
      } else if (r < 0 || it + 1 >= deq.max_iterations) {
        sh_state[5] = -1.0;
      } else {
        for (int k = 0; k < 5; ++k) sh_state[k] = b[k];
        sh_state[11] = rel;
      }
    }
    __syncthreads();
    const double status = sh_state[5];
    if (status != 0.0) {
      int result = it + 1;
      if (status > 0.0) {
        out = m;
        for (int k = 0; k < 5; ++k) gamma[k] = sh_state[6 + k];
      } else {
        result = -1;
      }
      __syncthreads();
      return result;
    }
  }
}

// the same on the View's velocity grid (storage precision of the per-point terms)
template <class S, class M, int B>
__device__ inline int block_discrete_maxwell(const View<S, M>& v, double rho, double ux, double uy, double uz, double T,
                                             const CellParams<M>* poly, Maxwell<M>& out, double (&gamma)[5],
                                             double* sh_red, double* sh_state) {
  return block_discrete_maxwell_on<M, B>(v.dq_x, v.dq_y, v.dq_z, v.dq_w, v.dq_nv, v.weight, v.deq, v.dq_tensor, rho, ux,
                                         uy, uz, T, poly, out, gamma, sh_red, sh_state);
}

}  // namespace kin
