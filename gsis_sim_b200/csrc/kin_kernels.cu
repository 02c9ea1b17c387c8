// Kernels of the B200 kinetic backend. See kin_kernels.cuh for the data layout; every kernel names the
// reference routine whose semantics it reproduces.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <initializer_list>
#include <type_traits>
#include <utility>

#include "kin_kernels.cuh"
#include "kin_launch.h"

namespace kin {

constexpr int kCellThreads = 256;  // moments / Newton / correction: one CTA per cell
constexpr int kFaceThreads = 128;  // boundary sums / face fluxes: one CTA per face
constexpr int kTileThreads = 256;  // gradient / residual: one CTA per (cell, velocity tile)

// ---------------------------------------------------------------------------------------------------------
// f = f_eq(state), shift = u (k_set_equilibrium / CpuBackend::set_equilibrium,
// src/kinetic/kinetic_backend_cpu.cpp:64-80)
// ---------------------------------------------------------------------------------------------------------
template <class S, class M>
__global__ void __launch_bounds__(kCellThreads)
    k_set_equilibrium(View<S, M> v, const double* __restrict__ states, double* __restrict__ shift, int discrete) {
  __shared__ double sh_red[kDeqSums * (kCellThreads / 32)];
  __shared__ double sh_state[12];
  const int c = blockIdx.x;
  const double* st = states + 5 * static_cast<int64_t>(c);
  Maxwell<M> m = maxwell_from<M>(st[0], st[1], st[2], st[3], st[4]);
  if (discrete) {
    double gamma[5];
    block_discrete_maxwell<S, M, kCellThreads>(v, st[0], st[1], st[2], st[3], st[4], nullptr, m, gamma, sh_red,
                                               sh_state);
  }
  S* fc = v.f + static_cast<int64_t>(c) * v.nv;
  for (int q = threadIdx.x; q < v.nv; q += kCellThreads) {
    fc[q] = static_cast<S>(maxwellian(m, v.xi_x[q], v.xi_y[q], v.xi_z[q]));
  }
  if (threadIdx.x == 0) {
    shift[3 * static_cast<int64_t>(c) + 0] = st[1];
    shift[3 * static_cast<int64_t>(c) + 1] = st[2];
    shift[3 * static_cast<int64_t>(c) + 2] = st[3];
  }
}

// ---------------------------------------------------------------------------------------------------------
// 13 shifted sums in FP64 -> 15 moments (CpuBackend::compute_moments, kinetic_backend_cpu.cpp:92-120)
// One warp per cell, kMomentWarps cells per CTA: each lane sums velocities lane, lane + 32, ... (every load of f a
// 128- or 256-byte segment; four loads issued ahead of their sums), then a butterfly of warp shuffles combines the
// lanes in a fixed order (bitwise reproducible, no shared memory or barrier).
// ---------------------------------------------------------------------------------------------------------
constexpr int kMomentWarps = 8;

__device__ __forceinline__ void moment_terms(double f, double cx, double cy, double cz, double (&acc)[kMomentSums]) {
  const double t1 = f * cx, t2 = f * cy, t3 = f * cz;
  const double fc2 = f * (cx * cx + cy * cy + cz * cz);
  acc[0] += f;
  acc[1] += t1;
  acc[2] += t2;
  acc[3] += t3;
  acc[4] += t1 * cx;
  acc[5] += t2 * cy;
  acc[6] += t3 * cz;
  acc[7] += t1 * cy;
  acc[8] += t2 * cz;
  acc[9] += t1 * cz;
  acc[10] += fc2 * cx;
  acc[11] += fc2 * cy;
  acc[12] += fc2 * cz;
}

template <class S, class M, bool Finalize>
__global__ void __launch_bounds__(32 * kMomentWarps, 4)
    k_moments(View<S, M> v, double* __restrict__ shift, double* __restrict__ out) {
  constexpr int kAhead = 4;
  const int c = blockIdx.x * kMomentWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= v.n_cells) return;
  const double u0x = shift[3 * static_cast<int64_t>(c) + 0];
  const double u0y = shift[3 * static_cast<int64_t>(c) + 1];
  const double u0z = shift[3 * static_cast<int64_t>(c) + 2];
  const S* fc = v.f + static_cast<int64_t>(c) * v.nv;
  const bool uniform = v.wts == nullptr;
  double acc[kMomentSums];
#pragma unroll
  for (int k = 0; k < kMomentSums; ++k) acc[k] = 0.0;
  for (int q0 = 0; q0 < v.nv; q0 += 32 * kAhead) {
    S fs[kAhead];
#pragma unroll
    for (int j = 0; j < kAhead; ++j) {
      const int q = q0 + 32 * j + lane;
      fs[j] = q < v.nv ? __ldcs(fc + q) : S(0);
    }
#pragma unroll
    for (int j = 0; j < kAhead; ++j) {
      const int q = q0 + 32 * j + lane;
      if (q >= v.nv) break;
      double f = static_cast<double>(fs[j]);
      if (!uniform) f *= v.wts[q];
      moment_terms(f, v.xid_x[q] - u0x, v.xid_y[q] - u0y, v.xid_z[q] - u0z, acc);
    }
  }
#pragma unroll
  for (int k = 0; k < kMomentSums; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  }
  if (lane != 0) return;
  if (!Finalize) {  // raw sums of one velocity shard (kin_moment_sums); the shift stays
    for (int k = 0; k < kMomentSums; ++k) out[kMomentSums * static_cast<int64_t>(c) + k] = acc[k];
    return;
  }
  double* m = out + 15 * static_cast<int64_t>(c);
  finalize_moments(acc, uniform ? v.weight : 1.0, u0x, u0y, u0z, m);
  if (m[0] > 0.0) {
    shift[3 * static_cast<int64_t>(c) + 0] = m[1];
    shift[3 * static_cast<int64_t>(c) + 1] = m[2];
    shift[3 * static_cast<int64_t>(c) + 2] = m[3];
  }
}

// moments from moment sums already reduced over velocity shards in device memory (kin_finalize_moments): the
// finalisation and shift update of k_moments, one thread per cell
__global__ void k_finalize_sums(const double* __restrict__ sums, double weight, double* __restrict__ shift,
                                double* __restrict__ out, int n) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double* sh = shift + 3 * static_cast<int64_t>(c);
  double* m = out + 15 * static_cast<int64_t>(c);
  finalize_moments(sums + kMomentSums * static_cast<int64_t>(c), weight, sh[0], sh[1], sh[2], m);
  if (m[0] > 0.0) {
    sh[0] = m[1];
    sh[1] = m[2];
    sh[2] = m[3];
  }
}

// the shift of the next moment sums after moments were installed from outside (kin_set_moments)
__global__ void k_shift_from_moments(const double* __restrict__ m, double* __restrict__ shift, int n) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || !(m[15 * static_cast<int64_t>(c)] > 0.0)) return;
  for (int a = 0; a < 3; ++a) shift[3 * static_cast<int64_t>(c) + a] = m[15 * static_cast<int64_t>(c) + 1 + a];
}

// f *= s ; moments (rho, p, sigma, q) *= s   (k_scale / k_scale_moments, kinetic_cuda_kernels.cu:207-219)
template <class S>
__global__ void k_scale(S* __restrict__ f, int64_t n, double s) {
  const S sf = static_cast<S>(s);
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) f[i] *= sf;
}

__global__ void k_scale_moments(double* __restrict__ m, int n_cells, double s) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  double* mc = m + 15 * static_cast<int64_t>(c);
  mc[0] *= s;
  for (int k = 5; k < 15; ++k) mc[k] *= s;
}

// ---------------------------------------------------------------------------------------------------------
// cell parameters (k_cell_params / k_cell_params_deq, kinetic_cuda_kernels.cu:221-260;
// CpuBackend::update_cell_params, kinetic_backend_cpu.cpp:134-163)
// ---------------------------------------------------------------------------------------------------------
template <class M>
__global__ void k_cell_params(const double* __restrict__ moments, const double* __restrict__ volume,
                              const double* __restrict__ vdt, double mu0, double omega, double Pr,
                              CellParams<M>* __restrict__ out, int n_cells, double cold_bgk_T) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  out[c] = make_cell_params<M>(moments + 15 * static_cast<int64_t>(c), volume[c], vdt[c], mu0, omega, Pr, cold_bgk_T);
}

template <class S, class M>
__global__ void __launch_bounds__(kCellThreads)
    k_cell_params_deq(View<S, M> v, const double* __restrict__ moments, const double* __restrict__ volume,
                      const double* __restrict__ vdt, double mu0, double omega, double Pr, double cold_bgk_T,
                      int collisionless, CellParams<M>* __restrict__ out, int* __restrict__ flags) {
  __shared__ double sh_red[kDeqSums * (kCellThreads / 32)];
  __shared__ double sh_state[12];
  const int c = blockIdx.x;
  const double* m = moments + 15 * static_cast<int64_t>(c);
  CellParams<M> cp = make_cell_params<M>(m, volume[c], vdt[c], mu0, omega, Pr, cold_bgk_T);
  Maxwell<M> eq;
  double gamma[5];
  const int r = block_discrete_maxwell<S, M, kCellThreads>(v, m[0], m[1], m[2], m[3], m[4], &cp, eq, gamma, sh_red,
                                                           sh_state);
  if (threadIdx.x == 0) {
    if (r > 0) {
      cp.eq = eq;
      cp.g0 = static_cast<M>(gamma[0]);
      cp.gx = static_cast<M>(gamma[1]);
      cp.gy = static_cast<M>(gamma[2]);
      cp.gz = static_cast<M>(gamma[3]);
      cp.g4 = static_cast<M>(gamma[4]);
    } else if (r < 0 && collisionless) {
      cp.coll = M(0);
      cp.diag = static_cast<M>(vdt[c]);
    }
    out[c] = cp;
    flags[c] = r;
  }
}

// ---------------------------------------------------------------------------------------------------------
// specular cache of partially accommodating walls (k_maxwell_reflection / reflected_value,
// kinetic_cuda_kernels.cu:262-272, kinetic_kernels.hpp:86-127)
// ---------------------------------------------------------------------------------------------------------
template <bool Reconstruct, class S, class M>
__device__ inline M reflected_value(const View<S, M>& v, const BFace<M>& b, int q, M x, M y, M z) {
  if (b.mirror >= 0) {
    const int qm = v.mirror_map[b.mirror * v.nv + q];
    if (Reconstruct) return reconstruct_at_boundary(v, b, qm);
    return f_at(v, b.owner, qm);
  }
  const M un = x * b.n[0] + y * b.n[1] + z * b.n[2];
  const M r[3] = {x - M(2) * un * b.n[0], y - M(2) * un * b.n[1], z - M(2) * un * b.n[2]};
  int base[3];
  M t[3];
  for (int a = 0; a < 3; ++a) {
    const double zz = (static_cast<double>(r[a]) - v.deq.lo[a]) / v.deq.d[a] - 0.5;
    if (zz < -1e-5 || zz > v.grid_n[a] - 1.0 + 1e-5) return M(0);
    const double clipped = kmax(0.0, kmin(zz, v.grid_n[a] - 1.0));
    base[a] = static_cast<int>(clipped);
    if (base[a] >= v.grid_n[a] - 1) base[a] = v.grid_n[a] - 2;
    t[a] = static_cast<M>(clipped - base[a]);
  }
  M result = M(0);
  const CellParams<M> ref = v.cp[b.owner];
  for (int k = 0; k < 8; ++k) {
    const int ix = base[0] + (k & 1), iy = base[1] + ((k >> 1) & 1), iz = base[2] + ((k >> 2) & 1);
    const M w = ((k & 1) ? t[0] : M(1) - t[0]) * ((k & 2) ? t[1] : M(1) - t[1]) * ((k & 4) ? t[2] : M(1) - t[2]);
    if (w == M(0)) continue;
    const int qq = v.grid_to_pos[ix + v.grid_n[0] * (iy + v.grid_n[1] * iz)];
    M value;
    if (Reconstruct) value = reconstruct_at_boundary(v, b, qq);
    else value = f_at(v, b.owner, qq);
    const double drx = static_cast<double>(r[0]) - ref.eq.ux, dry = static_cast<double>(r[1]) - ref.eq.uy,
                 drz = static_cast<double>(r[2]) - ref.eq.uz;
    const double dqx = static_cast<double>(v.xi_x[qq]) - ref.eq.ux, dqy = static_cast<double>(v.xi_y[qq]) - ref.eq.uy,
                 dqz = static_cast<double>(v.xi_z[qq]) - ref.eq.uz;
    const double ratio =
        exp(-static_cast<double>(ref.eq.B) * (drx * drx + dry * dry + drz * drz - dqx * dqx - dqy * dqy - dqz * dqz));
    result += w * static_cast<M>(static_cast<double>(value) * ratio);
  }
  return result;
}

template <bool Reconstruct, class S, class M>
__global__ void k_maxwell_reflection(View<S, M> v) {
  const int b = blockIdx.y;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= v.nv || v.mw_offset[b] < 0) return;
  const BFace<M> bf = v.bf[b];
  const M x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
  M* buffer = Reconstruct ? v.specular : v.specular_first;
  buffer[v.mw_offset[b] + q] = (x * bf.n[0] + y * bf.n[1] + z * bf.n[2]) < M(0)
                                   ? reflected_value<Reconstruct>(v, bf, q, x, y, z)
                                   : M(0);
}

// ---------------------------------------------------------------------------------------------------------
// 20 half-space sums per boundary face (CpuBackend::boundary_sums, kinetic_backend_cpu.cpp:184-240;
// add_boundary_terms, kinetic_kernels.hpp:596-609). Terms in M, sums in FP64.
// ---------------------------------------------------------------------------------------------------------
template <class M>
__device__ __forceinline__ void add_boundary_terms(M wf, M x, M y, M z, M a_n, double* flux5, double* mom5) {
  const M e = M(0.5) * (x * x + y * y + z * z);
  const M af = a_n * wf;
  flux5[0] += static_cast<double>(af);
  flux5[1] += static_cast<double>(af * x);
  flux5[2] += static_cast<double>(af * y);
  flux5[3] += static_cast<double>(af * z);
  flux5[4] += static_cast<double>(af * e);
  mom5[0] += static_cast<double>(wf);
  mom5[1] += static_cast<double>(wf * x);
  mom5[2] += static_cast<double>(wf * y);
  mom5[3] += static_cast<double>(wf * z);
  mom5[4] += static_cast<double>(wf * e);
}

template <class S, class M>
__global__ void __launch_bounds__(kFaceThreads) k_boundary_sums(View<S, M> v, double* __restrict__ out) {
  __shared__ double sh[20 * (kFaceThreads / 32)];
  const int b = blockIdx.x;
  const BFace<M> bf = v.bf[b];
  const Maxwell<M> m_in = v.inflow[b].m;
  const M wu = static_cast<M>(v.weight);
  double acc[20];
#pragma unroll
  for (int k = 0; k < 20; ++k) acc[k] = 0.0;
  for (int q = threadIdx.x; q < v.nv; q += kFaceThreads) {
    const M x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
    const M w = v.wts == nullptr ? wu : static_cast<M>(v.wts[q]);
    const M a_n = x * bf.n[0] + y * bf.n[1] + z * bf.n[2];
    if (a_n >= M(0) || bf.kind == kPeriodic) {
      const M fb = reconstruct_at_boundary(v, bf, q);
      add_boundary_terms(w * fb, x, y, z, a_n, acc + 0, acc + 10);
    } else {
      M fb;
      if (bf.kind == kSymmetry) {
        fb = reconstruct_at_boundary(v, bf, v.mirror_map[bf.mirror * v.nv + q]);
      } else if (bf.kind == kMaxwellWall) {
        fb = maxwell_inflow(v, b, q, x, y, z);
      } else {
        fb = maxwellian(m_in, x, y, z);  // unit density, without scale
      }
      add_boundary_terms(w * fb, x, y, z, a_n, acc + 5, acc + 15);
    }
  }
  block_sum<20, kFaceThreads>(acc, sh);
  if (threadIdx.x == 0) {
    double* o = out + 20 * static_cast<int64_t>(b);
    for (int k = 0; k < 20; ++k) o[k] = acc[k];
  }
}

// ---------------------------------------------------------------------------------------------------------
// section mass flux through internal faces (internal_face_flux_term, kinetic_kernels.hpp:217-231;
// CpuBackend::internal_face_mass_flux, kinetic_backend_cpu.cpp:242-260)
// ---------------------------------------------------------------------------------------------------------
template <class S, class M>
__global__ void __launch_bounds__(kFaceThreads)
    k_internal_face_flux(View<S, M> v, const int32_t* __restrict__ cells, const int32_t* __restrict__ entries,
                         double* __restrict__ out) {
  __shared__ double sh[kFaceThreads / 32];
  const int i = blockIdx.x;
  const int c = cells[i];
  const CsrE<M> ce = v.csr[entries[i]];
  double acc[1] = {0.0};
  for (int q = threadIdx.x; q < v.nv; q += kFaceThreads) {
    const M x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
    const M a = x * ce.s[0] + y * ce.s[1] + z * ce.s[2];
    M ff, gx, gy, gz;
    if (a >= M(0)) {
      const M fi = f_at(v, c, q);
      limited_gradient(v, c, q, x, y, z, fi, gx, gy, gz);
      ff = fi + gx * ce.ds[0] + gy * ce.ds[1] + gz * ce.ds[2];
    } else {
      const M fj = f_at(v, ce.other, q);
      limited_gradient(v, ce.other, q, x, y, z, fj, gx, gy, gz);
      ff = fj + gx * ce.dn[0] + gy * ce.dn[1] + gz * ce.dn[2];
    }
    double term = static_cast<double>(a * ff);
    if (v.wts != nullptr) term *= v.wts[q];
    acc[0] += term;
  }
  block_sum<1, kFaceThreads>(acc, sh);
  if (threadIdx.x == 0) out[i] = (v.wts == nullptr ? static_cast<double>(static_cast<M>(v.weight)) : 1.0) * acc[0];
}

// ---------------------------------------------------------------------------------------------------------
// limited gradients and steady residual of one velocity chunk (k_gradient / k_residual,
// kinetic_cuda_kernels.cu:343-372; limited_gradient / residual_value, kinetic_kernels.hpp:161-201, 238-278).
// grid: (kCellsPerCta cells, velocity tile of 32 * U). The CTA stages its cells' CSR entries in shared memory
// once; every thread then carries its U velocities (the kernel shape) through each entry together, so an entry is
// read once per thread (not once per velocity) and the velocities give independent FP64 chains. The arithmetic
// of every velocity is that of the reference routines, entry by entry in CSR order.
// ---------------------------------------------------------------------------------------------------------
// stencil extrema: FP32 min / max instructions, FP64 compare and select (as kmax / kmin; measured faster on B200 than
// fmax / fmin of doubles in the gradient kernel)
__device__ __forceinline__ double ext_max(double a, double b) { return kmax(a, b); }
__device__ __forceinline__ float ext_max(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double ext_min(double a, double b) { return kmin(a, b); }
__device__ __forceinline__ float ext_min(float a, float b) { return fminf(a, b); }

constexpr int kCellsPerCta = 8;   // consecutive cells of one gradient / residual CTA
constexpr int kStageMulti = 96;   // CSR entries of those cells staged in shared memory

template <class M>
struct StagedEntry {
  CsrE<M> e;
  int32_t kind;          // -1 internal face, else the boundary kind
  float dsf[3], dnf[3];  // FP32 copies of ds, dn (mixed-precision face reconstruction)
};

// Stage the CSR entries of cells [c0, c1) (contiguous in CSR order) and their per-cell offsets in shared memory.
// Returns the number of entries; more than kStageMulti means nothing was staged (the caller reads global memory).
template <class S, class M>
__device__ __forceinline__ int stage_cells(const View<S, M>& v, int c0, int c1, StagedEntry<M>* sh, int* sh_off) {
  const int e0 = v.csr_off[c0], ne = v.csr_off[c1] - e0;
  if (static_cast<int>(threadIdx.x) <= c1 - c0) sh_off[threadIdx.x] = v.csr_off[c0 + threadIdx.x] - e0;
  if (ne <= kStageMulti) {
    for (int k = threadIdx.x; k < ne; k += blockDim.x) {
      StagedEntry<M> se;
      se.e = v.csr[e0 + k];
      se.kind = se.e.other >= 0 ? -1 : v.bf[se.e.bface].kind;
      for (int a = 0; a < 3; ++a) {
        se.dsf[a] = static_cast<float>(se.e.ds[a]);
        se.dnf[a] = static_cast<float>(se.e.dn[a]);
      }
      sh[k] = se;
    }
  }
  __syncthreads();
  return ne;
}

template <class S>
__device__ __forceinline__ S ldg_s(const S* p) { return __ldg(p); }

// Loop over the entries of one cell: unrolled with a compile-time bound NE (hexahedra, prisms, tetrahedra:
// NE = 6) so that loads of later entries can be issued before earlier ones are used, or a plain loop (NE = 0).
template <int NE, class F>
__device__ __forceinline__ void for_entries(int ne, F&& body) {
  if constexpr (NE > 0) {
#pragma unroll
    for (int j = 0; j < NE; ++j)
      if (j < ne) body(j);
  } else {
    for (int j = 0; j < ne; ++j) body(j);
  }
}

// venkat_face written with selects: the one division is taken only where its value can lower phi (0 <= num < den;
// otherwise the reference routine returns 1, 0, or a quotient that the clamp makes 1), so min(phi, .) is the same
template <class M>
__device__ __forceinline__ M venkat_face_sel(M d2, M dmax, M dmin, M eps2) {
  const bool pos = d2 > M(0), neg = d2 < M(0);
  const M d1 = pos ? dmax : dmin;
  const M num = (d1 * d1 + eps2) + M(2) * d1 * d2;
  const M den = d1 * d1 + M(2) * d2 * d2 + d1 * d2 + eps2;
  const bool sided = pos || neg;
  M r = (sided && !(den > M(0))) ? M(0) : M(1);
  if (sided && den > M(0) && num < den) r = kclamp(limiter_quotient(num, den), M(0), M(1));
  return r;
}

// Venkatakrishnan factor of one face kept as a fraction (FP64): phi = min over faces of clamp(num / den, 0, 1) is
// tracked as pn / pd, a candidate num / den in (0, 1) replacing it when num * pd < pn * den. The one division per
// velocity at the end divides the same num and den the reference divides for the minimising face, so phi is the
// reference's value (candidates closer than a rounding error may select the other face: phi then differs in the
// last bit). The cases that give exactly 0 or 1 follow venkat_face (src/physics/limiter.hpp via
// kinetic_kernels.hpp:161-201).
template <class M>
__device__ __forceinline__ void venkat_frac_update(M d2, M dmax, M dmin, M eps2, M& pn, M& pd) {
  const bool pos = d2 > M(0), neg = d2 < M(0);
  const M d1 = pos ? dmax : dmin;
  const M num = (d1 * d1 + eps2) + M(2) * d1 * d2;
  const M den = d1 * d1 + M(2) * d2 * d2 + d1 * d2 + eps2;
  const bool sided = pos || neg;
  const bool zero = sided && (!(den > M(0)) || (num < den && !(num > M(0))));
  const bool cand = sided && den > M(0) && num > M(0) && num < den && num * pd < pn * den;
  pn = zero ? M(0) : (cand ? num : pn);
  pd = zero ? M(1) : (cand ? den : pd);
}

// limited_gradient for U velocities of one cell at once (same arithmetic per velocity, entries in CSR order)
template <class S, class M, int U, int NE>
__device__ __forceinline__ void limited_gradient_tile(const View<S, M>& v, int cell, const StagedEntry<M>* E, int ne,
                                                      const int (&q)[U], const bool (&ok)[U], const M (&x)[U],
                                                      const M (&y)[U], const M (&z)[U], const M (&fi)[U],
                                                      M (&gx)[U], M (&gy)[U], M (&gz)[U]) {
  M sx[U], sy[U], sz[U], fmax[U], fmin[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    sx[u] = sy[u] = sz[u] = M(0);
    fmax[u] = fmin[u] = fi[u];
  }
  for_entries<NE>(ne, [&](int j) {
    const CsrE<M>& c = E[j].e;
    M fk[U];
    if (c.other >= 0) {
      const S* fo = v.f + static_cast<int64_t>(c.other) * v.nv;
#pragma unroll
      for (int u = 0; u < U; ++u) fk[u] = ok[u] ? static_cast<M>(ldg_s(fo + q[u])) : fi[u];
    } else {
#pragma unroll
      for (int u = 0; u < U; ++u)
        fk[u] = ok[u] ? boundary_value_first_order(v, c, cell, q[u], x[u], y[u], z[u], fi[u]) : fi[u];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const M d = fk[u] - fi[u];
      sx[u] += c.c[0] * d;
      sy[u] += c.c[1] * d;
      sz[u] += c.c[2] * d;
      fmax[u] = ext_max(fmax[u], fk[u]);
      fmin[u] = ext_min(fmin[u], fk[u]);
    }
  });
  if (v.limiter_mode == kLimNone && v.positivity == 0) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      gx[u] = sx[u];
      gy[u] = sy[u];
      gz[u] = sz[u];
    }
    return;
  }
  const M eps2c = v.eps2[cell];
  // FP64: the limiter as a fraction (one division per velocity); FP32 keeps the per-face division
  constexpr bool kFrac = sizeof(M) == 8;
  M eps2[U], phi[U], pden[U], pmin[U], dmx[U], dmn[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    eps2[u] = eps2c;
    if (v.limiter_mode == kLimRel) {
      const M sc = kmax(kabs(fmax[u]), kabs(fmin[u]));
      eps2[u] *= sc * sc;
    }
    phi[u] = M(1);
    pden[u] = M(1);
    pmin[u] = M(0);
    dmx[u] = fmax[u] - fi[u];
    dmn[u] = fmin[u] - fi[u];
  }
  const bool limit = v.limiter_mode != kLimNone;
  const bool posit = v.positivity != 0;
  for_entries<NE>(ne, [&](int j) {
    if (E[j].kind == kPeriodic) return;
    const CsrE<M>& c = E[j].e;
    const M ds0 = c.ds[0], ds1 = c.ds[1], ds2 = c.ds[2];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const M proj = sx[u] * ds0 + sy[u] * ds1 + sz[u] * ds2;
      if (limit) {
        if constexpr (kFrac) venkat_frac_update(proj, dmx[u], dmn[u], eps2[u], phi[u], pden[u]);
        else phi[u] = kmin(phi[u], venkat_face_sel(proj, dmx[u], dmn[u], eps2[u]));
      }
      if (posit) pmin[u] = kmin(pmin[u], proj);
    }
  });
#pragma unroll
  for (int u = 0; u < U; ++u) {
    M ph = phi[u];
    if constexpr (kFrac) {
      if (limit) ph = phi[u] / pden[u];
    }
    if (v.positivity != 0) {
      if (!(fi[u] > M(0))) ph = M(0);
      else if (pmin[u] < M(0)) ph = kmin(ph, fi[u] / (-pmin[u]));
    }
    gx[u] = ph * sx[u];
    gy[u] = ph * sy[u];
    gz[u] = ph * sz[u];
  }
}

template <class S, class M, int NE, int U, int OCC>
__global__ void __launch_bounds__(kTileThreads, OCC) k_gradient(View<S, M> v, Chunk<S> ch) {
  __shared__ StagedEntry<M> E[kStageMulti];
  __shared__ int off[kCellsPerCta + 1];
  const int c0 = blockIdx.x * kCellsPerCta, c1 = min(v.n_cells, c0 + kCellsPerCta);
  const int tb = blockIdx.y * (kTileThreads * U);
  const int te = min(ch.kc, tb + kTileThreads * U);
  const bool staged = stage_cells(v, c0, c1, E, off) <= kStageMulti;
  int q[U];
  bool ok[U];
  M x[U], y[U], z[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int t = tb + threadIdx.x + u * kTileThreads;
    ok[u] = t < te;
    q[u] = ch.k0 + t;  // affine in u: one address per neighbour serves all U velocities; used only where ok[u]
    x[u] = ok[u] ? v.xi_x[q[u]] : M(0);
    y[u] = ok[u] ? v.xi_y[q[u]] : M(0);
    z[u] = ok[u] ? v.xi_z[q[u]] : M(0);
  }
  for (int c = c0; c < c1; ++c) {
    const int64_t row = static_cast<int64_t>(c) * ch.stride - ch.k0;
    if (!staged) {  // many faces: one velocity at a time from global memory
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (!ok[u]) continue;
        M gx, gy, gz;
        limited_gradient(v, c, q[u], x[u], y[u], z[u], f_at(v, c, q[u]), gx, gy, gz);
        ch.gx[row + q[u]] = static_cast<S>(gx);
        ch.gy[row + q[u]] = static_cast<S>(gy);
        ch.gz[row + q[u]] = static_cast<S>(gz);
      }
      continue;
    }
    const S* fc = v.f + static_cast<int64_t>(c) * v.nv;
    M fi[U], gx[U], gy[U], gz[U];
#pragma unroll
    for (int u = 0; u < U; ++u) fi[u] = ok[u] ? static_cast<M>(ldg_s(fc + q[u])) : M(0);
    limited_gradient_tile<S, M, U, NE>(v, c, E + off[c - c0], off[c - c0 + 1] - off[c - c0], q, ok, x, y, z, fi,
                                       gx, gy, gz);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!ok[u]) continue;
      ch.gx[row + q[u]] = static_cast<S>(gx[u]);
      ch.gy[row + q[u]] = static_cast<S>(gy[u]);
      ch.gz[row + q[u]] = static_cast<S>(gz[u]);
    }
  }
}

// residual_value for one velocity (general path and the symmetry face term)
template <class S, class M>
__device__ inline M residual_value(const View<S, M>& v, const Chunk<S>& ch, int cell, int t) {
  const int q = ch.k0 + t;
  const M x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
  const M fi = f_at(v, cell, q);
  const int64_t wi = static_cast<int64_t>(cell) * ch.stride + t;
  const M gix = static_cast<M>(ch.gx[wi]), giy = static_cast<M>(ch.gy[wi]), giz = static_cast<M>(ch.gz[wi]);
  M R = M(0);
  const int e0 = v.csr_off[cell], e1 = v.csr_off[cell + 1];
  for (int e = e0; e < e1; ++e) {
    const CsrE<M>& c = v.csr[e];
    int kind = -1;
    if (c.other < 0) {
      kind = v.bf[c.bface].kind;
      if (kind == kPeriodic) continue;
    }
    const M a = x * c.s[0] + y * c.s[1] + z * c.s[2];
    M ff;
    if (a >= M(0)) {
      ff = fi + gix * c.ds[0] + giy * c.ds[1] + giz * c.ds[2];
    } else if (c.other >= 0) {
      const int64_t wj = static_cast<int64_t>(c.other) * ch.stride + t;
      ff = f_at(v, c.other, q) + static_cast<M>(ch.gx[wj]) * c.dn[0] + static_cast<M>(ch.gy[wj]) * c.dn[1] +
           static_cast<M>(ch.gz[wj]) * c.dn[2];
    } else if (kind == kSymmetry) {
      // outflow reconstruction of the mirrored velocity at the same cell (its gradient recomputed: the mirrored
      // velocity need not lie in this chunk)
      const int qm = v.mirror_map[v.bf[c.bface].mirror * v.nv + q];
      const M fm = f_at(v, cell, qm);
      M gx, gy, gz;
      limited_gradient(v, cell, qm, v.xi_x[qm], v.xi_y[qm], v.xi_z[qm], fm, gx, gy, gz);
      ff = fm + gx * c.ds[0] + gy * c.ds[1] + gz * c.ds[2];
    } else if (kind == kMaxwellWall) {
      ff = maxwell_inflow(v, c.bface, q, x, y, z);
    } else {
      ff = inflow_value(v.inflow[c.bface], x, y, z);
    }
    R += a * ff;
  }
  const CellParams<M>& cp = v.cp[cell];
  R -= cp.coll * (shakhov_target(cp, x, y, z) - fi);
  return R;
}

// residual of U velocities of one cell from staged entries (residual_value, kinetic_kernels.hpp:238-278). At an
// internal face the upwind value is chosen with a select between the two reconstructions (the neighbour's loads are
// predicated on a < 0), so the U velocities never branch apart; boundary faces follow the reference branches.
template <class S, class M, int U, int NE>
__device__ __forceinline__ void residual_tile(const View<S, M>& v, const Chunk<S>& ch, int c, const StagedEntry<M>* E,
                                              int ne, const int (&t)[U], const bool (&ok)[U], const M (&x)[U],
                                              const M (&y)[U], const M (&z)[U], M (&R)[U], M (&fi)[U]) {
  // mixed precision (FP32 storage, FP64 arithmetic): the face reconstructions f + g . d are formed in the storage
  // precision of their inputs; the flux balance and the collision term are summed in FP64
  constexpr bool kLowRecon = sizeof(S) < sizeof(M);
  const S* fc = v.f + static_cast<int64_t>(c) * v.nv + ch.k0;
  const int64_t row = static_cast<int64_t>(c) * ch.stride;
  S fs[U], gxs[U], gys[U], gzs[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    fs[u] = ok[u] ? ldg_s(fc + t[u]) : S(0);
    gxs[u] = ok[u] ? ldg_s(ch.gx + row + t[u]) : S(0);
    gys[u] = ok[u] ? ldg_s(ch.gy + row + t[u]) : S(0);
    gzs[u] = ok[u] ? ldg_s(ch.gz + row + t[u]) : S(0);
    fi[u] = static_cast<M>(fs[u]);
    R[u] = M(0);
  }
  M gix[U], giy[U], giz[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    gix[u] = static_cast<M>(gxs[u]);
    giy[u] = static_cast<M>(gys[u]);
    giz[u] = static_cast<M>(gzs[u]);
  }
  for_entries<NE>(ne, [&](int j) {
    const CsrE<M>& ce = E[j].e;
    const int kind = E[j].kind;
    if (kind == kPeriodic) return;
    const M s0 = ce.s[0], s1 = ce.s[1], s2 = ce.s[2];
    if (ce.other >= 0) {
      const S* fo = v.f + static_cast<int64_t>(ce.other) * v.nv + ch.k0;
      const int64_t wj = static_cast<int64_t>(ce.other) * ch.stride;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const M a = x[u] * s0 + y[u] * s1 + z[u] * s2;
        const bool up = a >= M(0);
        const bool ld = ok[u] && !up;
        if constexpr (kLowRecon) {
          const S fj = ld ? ldg_s(fo + t[u]) : S(0);
          const S gxj = ld ? ldg_s(ch.gx + wj + t[u]) : S(0);
          const S gyj = ld ? ldg_s(ch.gy + wj + t[u]) : S(0);
          const S gzj = ld ? ldg_s(ch.gz + wj + t[u]) : S(0);
          const S f_up = fs[u] + gxs[u] * E[j].dsf[0] + gys[u] * E[j].dsf[1] + gzs[u] * E[j].dsf[2];
          const S f_dn = fj + gxj * E[j].dnf[0] + gyj * E[j].dnf[1] + gzj * E[j].dnf[2];
          R[u] += a * static_cast<M>(up ? f_up : f_dn);
        } else {
          const M fj = ld ? static_cast<M>(ldg_s(fo + t[u])) : M(0);
          const M gxj = ld ? static_cast<M>(ldg_s(ch.gx + wj + t[u])) : M(0);
          const M gyj = ld ? static_cast<M>(ldg_s(ch.gy + wj + t[u])) : M(0);
          const M gzj = ld ? static_cast<M>(ldg_s(ch.gz + wj + t[u])) : M(0);
          const M f_up = fi[u] + gix[u] * ce.ds[0] + giy[u] * ce.ds[1] + giz[u] * ce.ds[2];
          const M f_dn = fj + gxj * ce.dn[0] + gyj * ce.dn[1] + gzj * ce.dn[2];
          R[u] += a * (up ? f_up : f_dn);
        }
      }
    } else {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const M a = x[u] * s0 + y[u] * s1 + z[u] * s2;
        M ff;
        if (a >= M(0)) {
          if constexpr (kLowRecon)
            ff = static_cast<M>(fs[u] + gxs[u] * E[j].dsf[0] + gys[u] * E[j].dsf[1] + gzs[u] * E[j].dsf[2]);
          else
            ff = fi[u] + gix[u] * ce.ds[0] + giy[u] * ce.ds[1] + giz[u] * ce.ds[2];
        } else if (!ok[u]) {
          ff = M(0);
        } else if (kind == kSymmetry) {
          // outflow reconstruction of the mirrored velocity at the same cell (its gradient recomputed: the
          // mirrored velocity need not lie in this chunk)
          const int q = ch.k0 + t[u];
          const int qm = v.mirror_map[v.bf[ce.bface].mirror * v.nv + q];
          const M fm = f_at(v, c, qm);
          M gx, gy, gz;
          limited_gradient(v, c, qm, v.xi_x[qm], v.xi_y[qm], v.xi_z[qm], fm, gx, gy, gz);
          ff = fm + gx * ce.ds[0] + gy * ce.ds[1] + gz * ce.ds[2];
        } else if (kind == kMaxwellWall) {
          ff = maxwell_inflow(v, ce.bface, ch.k0 + t[u], x[u], y[u], z[u]);
        } else {
          ff = inflow_value(v.inflow[ce.bface], x[u], y[u], z[u]);
        }
        R[u] += a * ff;
      }
    }
  });
  const CellParams<M> cp = v.cp[c];
#pragma unroll
  for (int u = 0; u < U; ++u) R[u] = R[u] - cp.coll * (shakhov_target(cp, x[u], y[u], z[u]) - fi[u]);
}

// residual of one chunk; partial[c * partial_stride + tile * warps + warp] = sum of R^2 over the warp's velocities
// (summed in a fixed order by k_residual_reduce: deterministic)
template <class S, class M, int NE, int U, int OCC>
__global__ void __launch_bounds__(kTileThreads, OCC)
    k_residual(View<S, M> v, Chunk<S> ch, double* __restrict__ partial, int partial_stride) {
  constexpr int kWarps = kTileThreads / 32;
  __shared__ StagedEntry<M> E[kStageMulti];
  __shared__ int off[kCellsPerCta + 1];
  const int c0 = blockIdx.x * kCellsPerCta, c1 = min(v.n_cells, c0 + kCellsPerCta);
  const int tb = blockIdx.y * (kTileThreads * U);
  const int te = min(ch.kc, tb + kTileThreads * U);
  const bool staged = stage_cells(v, c0, c1, E, off) <= kStageMulti;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int t[U];
  bool ok[U];
  M x[U], y[U], z[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    t[u] = tb + threadIdx.x + u * kTileThreads;  // affine in u; used only where ok[u]
    ok[u] = t[u] < te;
    const int q = ch.k0 + t[u];
    x[u] = ok[u] ? v.xi_x[q] : M(0);
    y[u] = ok[u] ? v.xi_y[q] : M(0);
    z[u] = ok[u] ? v.xi_z[q] : M(0);
  }
  // store R (or, in the defect modes of the mixed precision's FP32 residual, store the defect / R + defect)
  auto emit = [&](int c, int64_t row, int tt, M R, double& r2) {
    if (ch.defect_mode == kDefectNone) {
      ch.r[row + tt] = static_cast<S>(R);
      r2 += static_cast<double>(R) * static_cast<double>(R);
      return;
    }
    S* d = ch.defect + static_cast<int64_t>(c) * v.nv + ch.k0 + tt;
    if (ch.defect_mode == kDefectStore) {
      *d = static_cast<S>(ch.r[row + tt] - static_cast<S>(R));
    } else {
      const S Ru = static_cast<S>(static_cast<S>(R) + *d);
      ch.r[row + tt] = Ru;
      r2 += static_cast<double>(Ru) * static_cast<double>(Ru);
    }
  };
  for (int c = c0; c < c1; ++c) {
    const int64_t row = static_cast<int64_t>(c) * ch.stride;
    double r2 = 0.0;
    if (!staged) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (!ok[u]) continue;
        emit(c, row, t[u], residual_value(v, ch, c, t[u]), r2);
      }
    } else {
      M R[U], fi[U];
      residual_tile<S, M, U, NE>(v, ch, c, E + off[c - c0], off[c - c0 + 1] - off[c - c0], t, ok, x, y, z, R, fi);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (!ok[u]) continue;
        emit(c, row, t[u], R[u], r2);
      }
    }
    if (ch.defect_mode == kDefectStore) continue;  // the FP64 residual of the same f wrote the sums
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
    if (lane == 0) partial[static_cast<int64_t>(c) * partial_stride + blockIdx.y * kWarps + warp] = r2;
  }
}

__global__ void k_residual_reduce(const double* __restrict__ partial, int partial_stride, int n_tiles,
                                  double* __restrict__ residual_cell, int n_cells) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  double s = 0.0;
  for (int k = 0; k < n_tiles; ++k) s += partial[static_cast<int64_t>(c) * partial_stride + k];
  residual_cell[c] += s;
}

// ---------------------------------------------------------------------------------------------------------
// one LU-SGS block pass (sweep_forward_cell / sweep_backward_cell, kinetic_kernels.hpp:289-358):
// forward then backward sweep of one (direction group, block) chain for one tile of 32 velocities per CTA.
//   pass 1:  R = r,  dprev = nullptr (out-of-block coupling -> beta sum|a-| on the diagonal)
//   pass k:  R = r,  dprev = Delta f of pass k-1 (out-of-block upwind neighbours on the right-hand side)
// out receives Delta f* (forward) and then Delta f (backward); the last pass adds Delta f to f.
// The chain's cells are visited level by level; the 8 warps share the cells of a level (two cells in flight per
// warp, lane = velocity) and meet at a barrier before the next level, so every in-block upwind neighbour has
// been finished, exactly as in the reference's cell-by-cell order (same per-cell arithmetic, same entry order).
// ---------------------------------------------------------------------------------------------------------
template <class S, class M>
__device__ __forceinline__ M sweep_forward_value(const View<S, M>& v, const SweepArgs<S, M>& a, int4 p, int t, int cb,
                                                 int ce, M x, M y, M z) {
  M ap = M(0), am_out = M(0), L = M(0), Lout = M(0);
  const SweepE<M>* se = a.se + p.y;
  for (int j = 0; j < p.z; ++j) {
    const SweepE<M> e = se[j];
    if (e.other == -2) continue;
    const M af = x * e.s[0] + y * e.s[1] + z * e.s[2];
    if (af > M(0)) {
      ap += af;
    } else if (e.other >= 0) {
      if (e.other < cb || e.other >= ce) {
        if (a.dprev != nullptr) {
          Lout += af * static_cast<M>(a.dprev[static_cast<int64_t>(e.other) * a.stride + t]);
        } else {
          am_out -= af;
        }
      } else if ((p.w >> j) & 1) {
        L += af * static_cast<M>(a.out[static_cast<int64_t>(e.other) * a.stride + t]);
      }
    }
  }
  const M D = v.cp[p.x].diag + v.diag_scale * ap + v.interface_damping * am_out;
  const M Ri = static_cast<M>(a.R[static_cast<int64_t>(p.x) * a.stride + t]);
  return (-Ri - Lout - L) / D;
}

template <class S, class M>
__device__ __forceinline__ M sweep_backward_value(const View<S, M>& v, const SweepArgs<S, M>& a, int4 p, int t, int cb,
                                                  int ce, M x, M y, M z) {
  M ap = M(0), am_out = M(0), U = M(0);
  const SweepE<M>* se = a.se + p.y;
  for (int j = 0; j < p.z; ++j) {
    const SweepE<M> e = se[j];
    if (e.other == -2) continue;
    const M af = x * e.s[0] + y * e.s[1] + z * e.s[2];
    if (af > M(0)) {
      ap += af;
    } else if (e.other >= 0) {
      if (e.other < cb || e.other >= ce) {
        if (a.dprev == nullptr) am_out -= af;
      } else if (!((p.w >> j) & 1)) {
        U += af * static_cast<M>(a.out[static_cast<int64_t>(e.other) * a.stride + t]);
      }
    }
  }
  const M D = v.cp[p.x].diag + v.diag_scale * ap + v.interface_damping * am_out;
  return static_cast<M>(a.out[static_cast<int64_t>(p.x) * a.stride + t]) - U / D;
}

template <class S, class M>
__device__ __forceinline__ void sweep_backward_store(const View<S, M>& v, const SweepArgs<S, M>& a, int cell, int t,
                                                     int q, M df) {
  a.out[static_cast<int64_t>(cell) * a.stride + t] = static_cast<S>(df);
  if (a.update_f) {
    S* fp = v.f + static_cast<int64_t>(cell) * v.nv + q;
    *fp = static_cast<S>(static_cast<M>(*fp) + df);
  }
}

template <class S, class M>
__global__ void __launch_bounds__(kSweepThreads, 4) k_sweep_pass(View<S, M> v, SweepArgs<S, M> a) {
  constexpr int W = kSweepThreads / 32;
  const int4 it = a.items[blockIdx.x];  // (chain, t0, t1, -)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = it.y + lane;
  const bool active = t < it.z;
  const int q = a.k0 + t;
  const int chain = it.x;
  const int b = chain % a.n_blocks;
  const int cb = a.block_offsets[b], ce = a.block_offsets[b + 1];
  const int4* prog = a.prog + a.chain_start[chain];
  const int32_t* lb = a.lev_bounds + a.lev_start[chain];
  const int nlev = a.lev_count[chain];
  M x = M(0), y = M(0), z = M(0);
  if (active) {
    x = v.xi_x[q];
    y = v.xi_y[q];
    z = v.xi_z[q];
  }
  for (int L = 0; L < nlev; ++L) {
    const int i1 = lb[L + 1];
    if (active) {
      for (int i = lb[L] + warp; i < i1; i += 2 * W) {
        const int4 pa = prog[i];
        const bool two = i + W < i1;
        const int4 pb = two ? prog[i + W] : pa;
        const M va = sweep_forward_value(v, a, pa, t, cb, ce, x, y, z);
        const M vb = two ? sweep_forward_value(v, a, pb, t, cb, ce, x, y, z) : M(0);
        a.out[static_cast<int64_t>(pa.x) * a.stride + t] = static_cast<S>(va);
        if (two) a.out[static_cast<int64_t>(pb.x) * a.stride + t] = static_cast<S>(vb);
      }
    }
    __syncthreads();
  }
  for (int L = nlev - 1; L >= 0; --L) {
    const int i1 = lb[L + 1];
    if (active) {
      for (int i = lb[L] + warp; i < i1; i += 2 * W) {
        const int4 pa = prog[i];
        const bool two = i + W < i1;
        const int4 pb = two ? prog[i + W] : pa;
        const M da = sweep_backward_value(v, a, pa, t, cb, ce, x, y, z);
        const M db = two ? sweep_backward_value(v, a, pb, t, cb, ce, x, y, z) : M(0);
        sweep_backward_store(v, a, pa.x, t, q, da);
        if (two) sweep_backward_store(v, a, pb.x, t, q, db);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------------------
// staged LU-SGS block pass (k_sweep_tiles): the recurrence of k_sweep_pass, organised for instruction economy.
//  * One CTA of kTileThreadsSweep threads per (direction group, block, tile of 32 * KU velocities); a thread carries
//    KU velocities (lane, lane + 32, ...; KU is the kernel shape) through every stencil entry, so the per-entry work
//    that does not depend on the velocity (entry fetch, kind decode, addressing) is shared by KU velocities.
//  * The chain's levels are split on the host into sub-levels of at most kStageCells cells and kStageEntries
//    entries, stored contiguously with each entry's kind for this chain precomputed (periodic, boundary,
//    in-block lower, in-block upper, other block); the next sub-level is copied into shared memory with
//    cp.async while the current one computes (double buffer, one barrier per step).
//  * For each cell a warp first issues every load it needs (upwind Delta f, the previous pass at out-of-block
//    neighbours, R or Delta f*, f), then accumulates entry by entry in CSR order with the reference's arithmetic
//    (sweep_forward_cell / sweep_backward_cell, kinetic_kernels.hpp:289-358). The sign test of a = xi . S picks
//    between the two branches of the reference with selects: ap += (a > 0 ? a : 0) adds an exact zero where the
//    reference adds nothing, and the coupling terms use (a > 0 ? 0 : a), so every sum equals the reference's.
// ---------------------------------------------------------------------------------------------------------

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <class M>
struct StageBuf {
  int4 prog[kStageCells];
  StageE<M> se[kStageEntries];
};
static_assert(sizeof(StageE<float>) == 16 && sizeof(StageE<double>) == 32, "stage entries are whole 16-byte words");

// copy sub-level `l` (chain-relative) of the staged schedule into `dst` (every thread issues its share)
template <class S, class M>
__device__ __forceinline__ void stage_sublevel(const SweepArgs<S, M>& a, const int32_t* sh_sc, const int32_t* sh_se,
                                               int l, StageBuf<M>* dst) {
  constexpr int kWords = static_cast<int>(sizeof(StageE<M>) / 16);
  const int p0 = sh_sc[l], np = sh_sc[l + 1] - p0;
  const int e0 = sh_se[l], ne = sh_se[l + 1] - e0;
  const int n16 = np + ne * kWords;
  const char* src_e = reinterpret_cast<const char*>(a.sse + e0);
  char* dst_e = reinterpret_cast<char*>(dst->se);
  for (int k = threadIdx.x; k < n16; k += kTileThreadsSweep) {
    if (k < np) {
      cp_async16(&dst->prog[k], a.sprog + p0 + k);
    } else {
      const int w = k - np;
      cp_async16(dst_e + 16 * w, src_e + 16 * static_cast<int64_t>(w));
    }
  }
  cp_async_commit();
}

// the upwind split of a = xi . S: max(a, 0) and min(a, 0) (the reference's branch a > 0 adds a to the outflow sum
// and couples through a otherwise; the values are the same, zero's sign aside). FP32: one min / max instruction
// each; FP64: compare and select (measured faster on B200 than fmax / fmin of doubles in these kernels)
__device__ __forceinline__ double pos_part(double af) { return af > 0.0 ? af : 0.0; }
__device__ __forceinline__ float pos_part(float af) { return fmaxf(af, 0.0f); }
__device__ __forceinline__ double neg_part(double af) { return af > 0.0 ? 0.0 : af; }
__device__ __forceinline__ float neg_part(float af) { return fminf(af, 0.0f); }

// forward value of KU velocities of one cell; First: first block pass (no previous Delta f)
template <class S, class M, int NE, bool First, int KU>
__device__ __forceinline__ void tile_forward_cell(const View<S, M>& v, const SweepArgs<S, M>& a,
                                                  const StageE<M>* E, int4 p, const int (&t)[KU],
                                                  const bool (&ok)[KU], const M (&x)[KU],
                                                  const M (&y)[KU], const M (&z)[KU]) {
  M val[NE][KU];
#pragma unroll
  for (int j = 0; j < NE; ++j) {
    const uint32_t code = j < p.z ? E[p.y + j].code : 0u;
    const uint32_t kind = code >> kKindShift;
    const int64_t row = static_cast<int64_t>(code & kIndexMask) * a.stride;
    const bool load = kind == kKindLower || (!First && kind == kKindOther);
    const S* src = kind == kKindLower ? a.out : a.dprev;
#pragma unroll
    for (int u = 0; u < KU; ++u) val[j][u] = (load && ok[u]) ? static_cast<M>(src[row + t[u]]) : M(0);
  }
  const int64_t crow = static_cast<int64_t>(p.x) * a.stride;
  M own[KU];
#pragma unroll
  for (int u = 0; u < KU; ++u) own[u] = ok[u] ? static_cast<M>(__ldcs(a.R + crow + t[u])) : M(0);
  const M diag = v.cp[p.x].diag;
  M ap[KU], lo[KU], ext[KU];  // ext: am_out (first pass) or Lout (later passes)
#pragma unroll
  for (int u = 0; u < KU; ++u) ap[u] = lo[u] = ext[u] = M(0);
#pragma unroll
  for (int j = 0; j < NE; ++j) {
    if (j >= p.z) break;
    const StageE<M>& e = E[p.y + j];
    const uint32_t kind = e.code >> kKindShift;
    if (kind == kKindPeriodic) continue;
    const M s0 = e.s[0], s1 = e.s[1], s2 = e.s[2];
#pragma unroll
    for (int u = 0; u < KU; ++u) {
      const M af = x[u] * s0 + y[u] * s1 + z[u] * s2;
      ap[u] += pos_part(af);
      if (kind == kKindLower) lo[u] += neg_part(af) * val[j][u];
      else if (kind == kKindOther) {
        if (First) ext[u] -= neg_part(af);
        else ext[u] += neg_part(af) * val[j][u];
      }
    }
  }
#pragma unroll
  for (int u = 0; u < KU; ++u) {
    if (!ok[u]) continue;
    const M am_out = First ? ext[u] : M(0), Lout = First ? M(0) : ext[u];
    const M D = diag + v.diag_scale * ap[u] + v.interface_damping * am_out;
    a.out[crow + t[u]] = static_cast<S>((-own[u] - Lout - lo[u]) / D);
    // the block passes run with S = M (FP64, or FP32 storage and arithmetic in the fp32 and mixed precisions), so
    // the backward reads back exactly this D
    a.diag_store[crow + t[u]] = static_cast<S>(D);
  }
}

// backward value of KU velocities of one cell (and f += Delta f in the last pass); the diagonal is the forward
// sweep's, read back, so only the in-block upper entries are visited
template <class S, class M, int NE, bool First, int KU>
__device__ __forceinline__ void tile_backward_cell(const View<S, M>& v, const SweepArgs<S, M>& a,
                                                   const StageE<M>* E, int4 p, const int (&t)[KU],
                                                   const bool (&ok)[KU], const M (&x)[KU],
                                                   const M (&y)[KU], const M (&z)[KU]) {
  M val[NE][KU];
#pragma unroll
  for (int j = 0; j < NE; ++j) {
    const uint32_t code = j < p.z ? E[p.y + j].code : 0u;
    const bool load = (code >> kKindShift) == kKindUpper;
    const int64_t row = static_cast<int64_t>(code & kIndexMask) * a.stride;
#pragma unroll
    for (int u = 0; u < KU; ++u) val[j][u] = (load && ok[u]) ? static_cast<M>(a.out[row + t[u]]) : M(0);
  }
  const int64_t crow = static_cast<int64_t>(p.x) * a.stride;
  const int64_t frow = static_cast<int64_t>(p.x) * v.nv + a.k0;
  M own[KU], fv[KU], D[KU];
#pragma unroll
  for (int u = 0; u < KU; ++u) {
    own[u] = ok[u] ? static_cast<M>(a.out[crow + t[u]]) : M(0);
    D[u] = ok[u] ? static_cast<M>(a.diag_store[crow + t[u]]) : M(1);
    fv[u] = (ok[u] && a.update_f) ? static_cast<M>(__ldcs(v.f + frow + t[u])) : M(0);
  }
  M up[KU];
#pragma unroll
  for (int u = 0; u < KU; ++u) up[u] = M(0);
#pragma unroll
  for (int j = 0; j < NE; ++j) {
    if (j >= p.z) break;
    const StageE<M>& e = E[p.y + j];
    if ((e.code >> kKindShift) != kKindUpper) continue;
    const M s0 = e.s[0], s1 = e.s[1], s2 = e.s[2];
#pragma unroll
    for (int u = 0; u < KU; ++u) {
      const M af = x[u] * s0 + y[u] * s1 + z[u] * s2;
      up[u] += neg_part(af) * val[j][u];
    }
  }
#pragma unroll
  for (int u = 0; u < KU; ++u) {
    if (!ok[u]) continue;
    const M df = own[u] - up[u] / D[u];
    a.out[crow + t[u]] = static_cast<S>(df);
    if (a.update_f) __stcs(v.f + frow + t[u], static_cast<S>(fv[u] + df));
  }
}

template <class S, class M, int NE, bool First, int KU, int KB>
__global__ void __launch_bounds__(kTileThreadsSweep, KB) k_sweep_tiles(View<S, M> v, SweepArgs<S, M> a) {
  constexpr int W = kTileThreadsSweep / 32;
  __shared__ __align__(16) StageBuf<M> sh_buf[2];
  __shared__ int32_t sh_sc[kMaxSubLevels + 1], sh_se[kMaxSubLevels + 1];
  const int4 it = a.items[blockIdx.x];  // (chain, t0, t1, -)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int chain = it.x;
  const int nsub = a.sub_count[chain];
  if (nsub <= 0) return;
  const int s0 = a.sub_start[chain];
  for (int k = threadIdx.x; k <= nsub; k += kTileThreadsSweep) {
    sh_sc[k] = a.sub_cells[s0 + k];
    sh_se[k] = a.sub_entries[s0 + k];
  }
  int t[KU];
  bool ok[KU];
  M x[KU], y[KU], z[KU];
#pragma unroll
  for (int u = 0; u < KU; ++u) {
    t[u] = it.y + lane + 32 * u;
    ok[u] = t[u] < it.z;
    const int q = a.k0 + (ok[u] ? t[u] : it.y);
    x[u] = v.xi_x[q];
    y[u] = v.xi_y[q];
    z[u] = v.xi_z[q];
  }
  __syncthreads();
  stage_sublevel(a, sh_sc, sh_se, 0, &sh_buf[0]);
  cp_async_wait_all();
  __syncthreads();
  const int nsteps = 2 * nsub;  // forward over sub-levels 0..nsub-1, then backward over nsub-1..0
  for (int s = 0; s < nsteps; ++s) {
    const StageBuf<M>& cur = sh_buf[s & 1];
    if (s + 1 < nsteps) stage_sublevel(a, sh_sc, sh_se, s + 1 < nsub ? s + 1 : nsteps - 2 - s, &sh_buf[(s + 1) & 1]);
    const int l = s < nsub ? s : nsteps - 1 - s;
    const int ncl = sh_sc[l + 1] - sh_sc[l];
    if (s < nsub) {
      for (int k = warp; k < ncl; k += W) tile_forward_cell<S, M, NE, First, KU>(v, a, cur.se, cur.prog[k], t, ok, x, y, z);
    } else {
      for (int k = warp; k < ncl; k += W) tile_backward_cell<S, M, NE, First, KU>(v, a, cur.se, cur.prog[k], t, ok, x, y, z);
    }
    cp_async_wait_all();
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------------------
// GSIS correction f += f_eq(W_new) - f_eq(W_half) with the negativity rule (CpuBackend::gsis_correction,
// kinetic_backend_cpu.cpp:346-432; k_gsis_correction, kinetic_cuda_kernels.cu:427-518)
// ---------------------------------------------------------------------------------------------------------
template <class S, class M>
__global__ void __launch_bounds__(kCellThreads)
    k_gsis_correction(View<S, M> v, const double* __restrict__ w_half, const double* __restrict__ w_new,
                      int* __restrict__ flags, double* __restrict__ shift, int mode, int discrete,
                      int collisionless, int phase, double* __restrict__ ext) {
  // phase 0: the whole correction. Velocity shards split it: phase 1 writes this shard's part of the negativity
  // rule's reduction over the velocities into ext[c] (the minimum of the limit factor, the negated maximum of the
  // blend factor, or the minimum of the check value: the minimum over all shards is the whole grid's) and changes
  // nothing; phase 2 applies the correction with the reduced ext[c].
  __shared__ double sh_red[kDeqSums * (kCellThreads / 32)];
  __shared__ double sh_state[12];
  __shared__ M sh_m[kCellThreads / 32 + 1];
  const int c = blockIdx.x;
  const double* wh = w_half + 5 * static_cast<int64_t>(c);
  const double* wn = w_new + 5 * static_cast<int64_t>(c);
  Maxwell<M> mh = maxwell_from<M>(wh[0], wh[1], wh[2], wh[3], wh[4]);
  Maxwell<M> mn = maxwell_from<M>(wn[0], wn[1], wn[2], wn[3], wn[4]);
  if (discrete) {
    double gamma[5];
    const int rh = block_discrete_maxwell<S, M, kCellThreads>(v, wh[0], wh[1], wh[2], wh[3], wh[4], nullptr, mh,
                                                              gamma, sh_red, sh_state);
    const int rn = block_discrete_maxwell<S, M, kCellThreads>(v, wn[0], wn[1], wn[2], wn[3], wn[4], nullptr, mn,
                                                              gamma, sh_red, sh_state);
    if (collisionless && (rh < 0 || rn < 0)) {
      if (phase == 1) {
        if (threadIdx.x == 0) ext[c] = 1e300;
        return;
      }
      if (threadIdx.x == 0) {
        flags[c] = kCorrectionSkipped;
        shift[3 * static_cast<int64_t>(c) + 0] = wh[1];
        shift[3 * static_cast<int64_t>(c) + 1] = wh[2];
        shift[3 * static_cast<int64_t>(c) + 2] = wh[3];
      }
      return;
    }
  }
  S* fc = v.f + static_cast<int64_t>(c) * v.nv;
  const double threshold = -1e-8 * wn[0] / (wn[4] * sqrt(wn[4]));
  const M thr = static_cast<M>(threshold);
  bool replace;
  if (mode == kNegLimit) {
    M alpha = M(1);
    if (phase != 2) {
      for (int q = threadIdx.x; q < v.nv; q += kCellThreads) {
        const M x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
        alpha = kmin(alpha, correction_alpha_limit(static_cast<M>(fc[q]), maxwellian(mn, x, y, z) - maxwellian(mh, x, y, z), thr));
      }
      alpha = block_reduce_op<kCellThreads>(alpha, sh_m, [](M p, M r) { return kmin(p, r); });
    }
    if (phase == 1) {
      if (threadIdx.x == 0) ext[c] = static_cast<double>(alpha);
      return;
    }
    if (phase == 2) alpha = static_cast<M>(ext[c]);
    for (int q = threadIdx.x; q < v.nv; q += kCellThreads) {
      const M x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
      fc[q] = static_cast<S>(static_cast<M>(fc[q]) + alpha * (maxwellian(mn, x, y, z) - maxwellian(mh, x, y, z)));
    }
    replace = alpha < M(1);
  } else if (mode == kNegBlend) {
    M theta = M(0);
    if (phase != 2) {
      for (int q = threadIdx.x; q < v.nv; q += kCellThreads) {
        const M x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
        const M e = maxwellian(mn, x, y, z);
        theta = kmax(theta, blend_theta(static_cast<M>(fc[q]), e - maxwellian(mh, x, y, z), e, thr));
      }
      theta = block_reduce_op<kCellThreads>(theta, sh_m, [](M p, M r) { return kmax(p, r); });
    }
    if (phase == 1) {
      if (threadIdx.x == 0) ext[c] = -static_cast<double>(theta);
      return;
    }
    if (phase == 2) theta = static_cast<M>(-ext[c]);
    for (int q = threadIdx.x; q < v.nv; q += kCellThreads) {
      const M x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
      const M e = maxwellian(mn, x, y, z);
      const M g = static_cast<M>(fc[q]) + (e - maxwellian(mh, x, y, z));
      fc[q] = static_cast<S>((M(1) - theta) * g + theta * e);
    }
    replace = theta > M(0);
  } else {
    // minimum of the check value over all points (the first point seeds the minimum)
    M fmin = M(0);
    bool first = true;
    for (int q = threadIdx.x; q < v.nv; q += kCellThreads) {
      const M x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
      const M old = static_cast<M>(fc[q]);
      const M xnew = old + (maxwellian(mn, x, y, z) - maxwellian(mh, x, y, z));
      if (phase != 1) fc[q] = static_cast<S>(xnew);
      const M chk = negative_check_value(old, xnew, mode == kNegCreated);
      fmin = first ? chk : kmin(fmin, chk);
      first = false;
    }
    if (first) fmin = M(1e30);  // threads without points do not take part in the minimum
    fmin = block_reduce_op<kCellThreads>(fmin, sh_m, [](M p, M r) { return kmin(p, r); });
    if (phase == 1) {
      if (threadIdx.x == 0) ext[c] = static_cast<double>(fmin);
      return;
    }
    if (phase == 2) fmin = static_cast<M>(ext[c]);
    replace = static_cast<double>(fmin) < threshold;
    if (replace) {
      for (int q = threadIdx.x; q < v.nv; q += kCellThreads) {
        fc[q] = static_cast<S>(maxwellian(mn, v.xi_x[q], v.xi_y[q], v.xi_z[q]));
      }
    }
  }
  if (threadIdx.x == 0) {
    flags[c] = replace ? 1 : 0;
    shift[3 * static_cast<int64_t>(c) + 0] = wn[1];
    shift[3 * static_cast<int64_t>(c) + 1] = wn[2];
    shift[3 * static_cast<int64_t>(c) + 2] = wn[3];
  }
}


// ---------------------------------------------------------------------------------------------------------
// conservative discrete Maxwellian of given macroscopic states, FP64 on the FP64 velocity grid
// (correct_inflow, src/kinetic/kinetic_solver.cpp:103-114, and maxwell_params_to_state,
// src/kinetic/kinetic_kernels.hpp:544-552). out: corrected (rho, ux, uy, uz, T), result: Newton iterations
// (0: resolved, no correction; -1: failed)
// ---------------------------------------------------------------------------------------------------------
template <class S, class M>
__global__ void __launch_bounds__(kCellThreads)
    k_discrete_maxwell_states(View<S, M> v, DeqGrid deq, const double* __restrict__ states, double* __restrict__ out,
                              int* __restrict__ result) {
  __shared__ double sh_red[kDeqSums * (kCellThreads / 32)];
  __shared__ double sh_state[12];
  const int i = blockIdx.x;
  const double* st = states + 5 * static_cast<int64_t>(i);
  Maxwell<double> m;
  double gamma[5];
  const int r = block_discrete_maxwell_on<double, kCellThreads>(v.dq_xd, v.dq_yd, v.dq_zd, v.dq_w, v.dq_nv, v.weight, deq,
                                                               v.dq_tensor, st[0], st[1], st[2], st[3], st[4], nullptr,
                                                               m, gamma, sh_red, sh_state);
  if (threadIdx.x == 0) {
    double* o = out + 5 * static_cast<int64_t>(i);
    if (r > 0) {
      const double T = 1.0 / (2.0 * m.B);
      const double two_pi_T = 2.0 * kPi * T;
      o[0] = m.A * two_pi_T * sqrt(two_pi_T);
      o[1] = m.ux;
      o[2] = m.uy;
      o[3] = m.uz;
      o[4] = T;
    } else {
      for (int k = 0; k < 5; ++k) o[k] = st[k];
    }
    result[i] = r;
  }
}

// ---------------------------------------------------------------------------------------------------------
// f <-> host order (cells c0 .. c0 + n of a staging buffer in the reference storage order)
// ---------------------------------------------------------------------------------------------------------
template <class S>
__global__ void k_import(const double* __restrict__ src, S* __restrict__ f, const int32_t* __restrict__ perm, int64_t c0,
                         int n_cells, int nv) {
  const int64_t n = static_cast<int64_t>(n_cells) * nv;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int64_t c = i / nv;
    const int q = static_cast<int>(i - c * nv);
    f[(c0 + c) * nv + q] = static_cast<S>(src[c * nv + perm[q]]);
  }
}

template <class S>
__global__ void k_export(const S* __restrict__ f, double* __restrict__ dst, const int32_t* __restrict__ inv, int64_t c0,
                         int n_cells, int nv) {
  const int64_t n = static_cast<int64_t>(n_cells) * nv;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int64_t c = i / nv;
    const int p = static_cast<int>(i - c * nv);
    dst[c * nv + p] = static_cast<double>(f[(c0 + c) * nv + inv[p]]);
  }
}

// ---------------------------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------------------------
inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

template <class S, class M>
void Launch<S, M>::set_equilibrium(const View<S, M>& v, const double* states, double* shift, int discrete,
                                   cudaStream_t st) {
  if (v.n_cells > 0) k_set_equilibrium<S, M><<<v.n_cells, kCellThreads, 0, st>>>(v, states, shift, discrete);
}

template <class S, class M>
void Launch<S, M>::moments(const View<S, M>& v, double* shift, double* out, cudaStream_t st) {
  if (v.n_cells > 0)
    k_moments<S, M, true><<<ceil_div(v.n_cells, kMomentWarps), 32 * kMomentWarps, 0, st>>>(v, shift, out);
}

template <class S, class M>
void Launch<S, M>::moment_sums(const View<S, M>& v, double* shift, double* out, cudaStream_t st) {
  if (v.n_cells > 0)
    k_moments<S, M, false><<<ceil_div(v.n_cells, kMomentWarps), 32 * kMomentWarps, 0, st>>>(v, shift, out);
}

template <class S, class M>
void Launch<S, M>::finalize_sums(const double* sums, double weight, double* shift, double* moments, int n,
                                 cudaStream_t st) {
  if (n > 0) k_finalize_sums<<<ceil_div(n, 128), 128, 0, st>>>(sums, weight, shift, moments, n);
}

template <class S, class M>
void Launch<S, M>::shift_from_moments(const double* moments, double* shift, int n, cudaStream_t st) {
  if (n > 0) k_shift_from_moments<<<ceil_div(n, 256), 256, 0, st>>>(moments, shift, n);
}

template <class S, class M>
void Launch<S, M>::scale(S* f, int64_t n, double s, double* moments, int n_cells, cudaStream_t st) {
  if (n > 0) {
    const int64_t blocks = (n + 255) / 256;
    k_scale<S><<<static_cast<unsigned>(blocks < 148 * 64 ? blocks : 148 * 64), 256, 0, st>>>(f, n, s);
  }
  if (n_cells > 0) k_scale_moments<<<ceil_div(n_cells, 256), 256, 0, st>>>(moments, n_cells, s);
}

template <class S, class M>
void Launch<S, M>::cell_params(const View<S, M>& v, const double* moments, const double* volume, const double* vdt,
                               double mu0, double omega, double Pr, double cold_bgk_T, int discrete, int collisionless,
                               CellParams<M>* out, int* flags, cudaStream_t st) {
  if (v.n_cells <= 0) return;
  if (discrete) {
    k_cell_params_deq<S, M><<<v.n_cells, kCellThreads, 0, st>>>(v, moments, volume, vdt, mu0, omega, Pr, cold_bgk_T,
                                                                collisionless, out, flags);
  } else {
    k_cell_params<M><<<ceil_div(v.n_cells, 128), 128, 0, st>>>(moments, volume, vdt, mu0, omega, Pr, out, v.n_cells,
                                                               cold_bgk_T);
  }
}

template <class S, class M>
void Launch<S, M>::maxwell_reflection(const View<S, M>& v, cudaStream_t st) {
  if (v.n_bfaces <= 0) return;
  const dim3 grid(ceil_div(v.nv, 128), v.n_bfaces);
  k_maxwell_reflection<false, S, M><<<grid, 128, 0, st>>>(v);
  k_maxwell_reflection<true, S, M><<<grid, 128, 0, st>>>(v);
}

template <class S, class M>
void Launch<S, M>::boundary_sums(const View<S, M>& v, double* out, cudaStream_t st) {
  if (v.n_bfaces > 0) k_boundary_sums<S, M><<<v.n_bfaces, kFaceThreads, 0, st>>>(v, out);
}

template <class S, class M>
void Launch<S, M>::internal_face_flux(const View<S, M>& v, const int32_t* cells, const int32_t* entries, double* out,
                                      int n, cudaStream_t st) {
  if (n > 0) k_internal_face_flux<S, M><<<n, kFaceThreads, 0, st>>>(v, cells, entries, out);
}

// ---- kernel shapes: velocities per thread x CTAs per SM of the gradient, residual and LU-SGS tile kernels -------
// measured on the 134,528-cell tube, 32^3 (FP64 and the mixed precision's FP32 gradient / sweeps)
template <>
KernelShape default_shape<double>() {
  return {4, 2, 1, 6, 2, 6};
}
template <>
KernelShape default_shape<float>() {
  return {4, 3, 2, 6, 4, 6};
}

template <class M>
KernelShape read_shape() {
  KernelShape k = default_shape<M>();
  if (const char* e = std::getenv("KIN_SHAPE")) {
    const std::string str(e);
    auto pick = [&](const char* key, int32_t& uu, int32_t& bb) {
      const size_t pos = str.find(key);
      if (pos == std::string::npos) return;
      int a = 0, b2 = 0;
      if (std::sscanf(str.c_str() + pos + std::strlen(key), "%dx%d", &a, &b2) == 2) {
        uu = a;
        bb = b2;
      }
    };
    pick("res=", k.res_u, k.res_occ);
    pick("grad=", k.grad_u, k.grad_occ);
    pick("tile=", k.tile_u, k.tile_blocks);
  }
  // only the compiled shapes (the launchers' candidates); anything else falls back to the default
  const KernelShape d = default_shape<M>();
  const bool fp64 = std::is_same<M, double>::value;
  auto one_of = [](int32_t u, int32_t b, std::initializer_list<std::pair<int, int>> ok) {
    for (const auto& p : ok)
      if (p.first == u && p.second == b) return true;
    return false;
  };
  if (!one_of(k.res_u, k.res_occ, fp64 ? std::initializer_list<std::pair<int, int>>{{4, 2}, {2, 3}}
                                       : std::initializer_list<std::pair<int, int>>{{4, 3}, {4, 4}})) {
    k.res_u = d.res_u;
    k.res_occ = d.res_occ;
  }
  if (!one_of(k.grad_u, k.grad_occ, fp64 ? std::initializer_list<std::pair<int, int>>{{1, 6}, {2, 3}}
                                         : std::initializer_list<std::pair<int, int>>{{2, 6}, {2, 4}})) {
    k.grad_u = d.grad_u;
    k.grad_occ = d.grad_occ;
  }
  if (!one_of(k.tile_u, k.tile_blocks, fp64 ? std::initializer_list<std::pair<int, int>>{{2, 6}, {4, 4}}
                                            : std::initializer_list<std::pair<int, int>>{{4, 6}, {2, 8}})) {
    k.tile_u = d.tile_u;
    k.tile_blocks = d.tile_blocks;
  }
  return k;
}
template KernelShape read_shape<double>();
template KernelShape read_shape<float>();

template <class S, class M>
int Launch<S, M>::residual_tiles(int kc, int res_u) {
  return ceil_div(kc, kTileThreads * res_u) * (kTileThreads / 32);
}

template <class S, class M, int NE>
static void launch_gradient(const View<S, M>& v, const Chunk<S>& ch, cudaStream_t st) {
  const KernelShape& k = ch.shape;
#define KIN_GRAD(U, B)                                                                                           \
  if (k.grad_u == U && k.grad_occ == B) {                                                                        \
    const dim3 grid(ceil_div(v.n_cells, kCellsPerCta), ceil_div(ch.kc, kTileThreads * U));                       \
    k_gradient<S, M, NE, U, B><<<grid, kTileThreads, 0, st>>>(v, ch);                                            \
    return;                                                                                                      \
  }
  if constexpr (std::is_same<S, M>::value && std::is_same<M, double>::value) {
    KIN_GRAD(2, 3)
  }
  if constexpr (std::is_same<S, M>::value && std::is_same<M, float>::value) {
    KIN_GRAD(2, 4)
  }
#undef KIN_GRAD
  constexpr int U = std::is_same<M, double>::value ? 1 : 2, B = 6;
  const dim3 grid(ceil_div(v.n_cells, kCellsPerCta), ceil_div(ch.kc, kTileThreads * U));
  k_gradient<S, M, NE, U, B><<<grid, kTileThreads, 0, st>>>(v, ch);
}

template <class S, class M>
void Launch<S, M>::gradient(const View<S, M>& v, const Chunk<S>& ch, cudaStream_t st) {
  if (v.n_cells <= 0 || ch.kc <= 0) return;
  if (v.max_entries <= 6)
    launch_gradient<S, M, 6>(v, ch, st);
  else
    launch_gradient<S, M, 0>(v, ch, st);
}

template <class S, class M, int NE>
static void launch_residual(const View<S, M>& v, const Chunk<S>& ch, double* partial, int partial_stride,
                            cudaStream_t st) {
  const KernelShape& k = ch.shape;
#define KIN_RES(U, B)                                                                                            \
  if (k.res_u == U && k.res_occ == B) {                                                                          \
    const dim3 grid(ceil_div(v.n_cells, kCellsPerCta), ceil_div(ch.kc, kTileThreads * U));                       \
    k_residual<S, M, NE, U, B><<<grid, kTileThreads, 0, st>>>(v, ch, partial, partial_stride);                   \
    return;                                                                                                      \
  }
  if constexpr (std::is_same<M, double>::value) {
    KIN_RES(2, 3)
  } else {
    KIN_RES(4, 4)
  }
#undef KIN_RES
  constexpr int U = 4, B = std::is_same<M, double>::value ? 2 : 3;
  const dim3 grid(ceil_div(v.n_cells, kCellsPerCta), ceil_div(ch.kc, kTileThreads * U));
  k_residual<S, M, NE, U, B><<<grid, kTileThreads, 0, st>>>(v, ch, partial, partial_stride);
}

template <class S, class M>
void Launch<S, M>::residual(const View<S, M>& v, const Chunk<S>& ch, double* partial, int partial_stride,
                            double* residual_cell, cudaStream_t st) {
  if (v.n_cells <= 0 || ch.kc <= 0) return;
  if (v.max_entries <= 6)
    launch_residual<S, M, 6>(v, ch, partial, partial_stride, st);
  else
    launch_residual<S, M, 0>(v, ch, partial, partial_stride, st);
  if (ch.defect_mode == kDefectStore) return;  // no sums of its own: the FP64 residual's stand
  k_residual_reduce<<<ceil_div(v.n_cells, 256), 256, 0, st>>>(partial, partial_stride,
                                                             residual_tiles(ch.kc, ch.shape.res_u),
                                                             residual_cell, v.n_cells);
}

template <class S, class M, int NE, bool First>
static void launch_tiles(const View<S, M>& v, const SweepArgs<S, M>& a, cudaStream_t st) {
#define KIN_TILE(KU, KB)                                                                                         \
  if (a.tile_u == KU && a.tile_blocks == KB) {                                                                   \
    k_sweep_tiles<S, M, NE, First, KU, KB><<<a.n_items, kTileThreadsSweep, 0, st>>>(v, a);                       \
    return;                                                                                                      \
  }
  if constexpr (std::is_same<S, M>::value && std::is_same<M, double>::value) {
    KIN_TILE(4, 4)
  }
  if constexpr (std::is_same<S, M>::value && std::is_same<M, float>::value) {
    KIN_TILE(2, 8)
  }
#undef KIN_TILE
  constexpr int KU = std::is_same<M, double>::value ? 2 : 4;
  k_sweep_tiles<S, M, NE, First, KU, 6><<<a.n_items, kTileThreadsSweep, 0, st>>>(v, a);
}

template <class S, class M>
void Launch<S, M>::sweep_pass(const View<S, M>& v, const SweepArgs<S, M>& a, cudaStream_t st) {
  if (a.n_items <= 0) return;
  if (a.staged_ne == 6 && a.dprev == nullptr)
    launch_tiles<S, M, 6, true>(v, a, st);
  else if (a.staged_ne == 6)
    launch_tiles<S, M, 6, false>(v, a, st);
  else if (a.staged_ne == 8 && a.dprev == nullptr)
    launch_tiles<S, M, 8, true>(v, a, st);
  else if (a.staged_ne == 8)
    launch_tiles<S, M, 8, false>(v, a, st);
  else
    k_sweep_pass<S, M><<<a.n_items, kSweepThreads, 0, st>>>(v, a);
}

template <class S, class M>
void Launch<S, M>::gsis_correction(const View<S, M>& v, const double* wh, const double* wn, int* flags, double* shift,
                                   int mode, int discrete, int collisionless, int phase, double* ext,
                                   cudaStream_t st) {
  if (v.n_cells > 0)
    k_gsis_correction<S, M><<<v.n_cells, kCellThreads, 0, st>>>(v, wh, wn, flags, shift, mode, discrete,
                                                                 collisionless, phase, ext);
}

template <class S, class M>
void Launch<S, M>::import_f(const double* src, S* f, const int32_t* perm, int64_t c0, int n, int nv, cudaStream_t st) {
  if (n > 0) k_import<S><<<148 * 16, 256, 0, st>>>(src, f, perm, c0, n, nv);
}

template <class S, class M>
void Launch<S, M>::export_f(const S* f, double* dst, const int32_t* inv, int64_t c0, int n, int nv, cudaStream_t st) {
  if (n > 0) k_export<S><<<148 * 16, 256, 0, st>>>(f, dst, inv, c0, n, nv);
}

template <class S, class M>
void Launch<S, M>::discrete_maxwell_states(const View<S, M>& v, const DeqGrid& deq, const double* states, double* out,
                                           int* result, int n, cudaStream_t st) {
  if (n > 0) k_discrete_maxwell_states<S, M><<<n, kCellThreads, 0, st>>>(v, deq, states, out, result);
}

template <class M>
__global__ void k_cast_cell_params(const CellParams<M>* __restrict__ src, CellParams<float>* __restrict__ dst, int n) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) dst[c] = cast_cell_params<float>(src[c]);
}

template <class S, class M>
void Launch<S, M>::cast_cell_params(const CellParams<M>* src, CellParams<float>* dst, int n, cudaStream_t st) {
  if (n > 0) k_cast_cell_params<M><<<ceil_div(n, 256), 256, 0, st>>>(src, dst, n);
}

template struct Launch<float, float>;
template struct Launch<double, double>;
template struct Launch<float, double>;

}  // namespace kin
