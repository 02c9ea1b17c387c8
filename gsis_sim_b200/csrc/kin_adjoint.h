// Discrete adjoint of the converged CIS fixed point: launch interface of kin_adjoint.cu. Arithmetic is FP64; the
// stored arrays (f, lambda, the seeds and the operator output) are of the handle's storage type S: double for FP64
// handles, float for mixed-precision ones (lambda stored and swept in FP32, the operator O(y) evaluated in FP64
// arithmetic on the stored values: the adjoint counterpart of the forward's FP64 residual with FP32 sweeps).
//
// The steady discrete problem of the kinetic solver (residual_value with the limited LSQ gradient, the Shakhov target
// of the cell moments and the boundary inflow, src/kinetic/kinetic_kernels.hpp) together with the zero-net-flux
// equation of every diffuse-wall density rho_Gamma (process_boundary_sums, src/kinetic/kinetic_solver.cpp:280-335) is
// F(f, rho_Gamma; p) = 0. For the adjoint y = (lambda, nu) of the objective J (the tube mass flow M_dot) the kernels
// here evaluate the operator O(y) = y^T dF/dx - dJ/dx in pieces:
//   k_adj_cell       per cell: the velocity sums Lambda of lambda against the Shakhov target and its derivatives
//                    (moments -> cell parameters part, finished on the host)
//   k_adj_transport  per (cell, velocity): the transposed upwind flux and limited-gradient terms that land on the
//                    cell itself, plus the seeds the neighbours gather (gradient seed G_bar, limiter extremum seeds)
//   k_adj_faces      per boundary face: the seeds on the inflow values (wall density, pressure-face state) summed
//                    against the inflow Maxwellian and its derivatives
//   k_adj_gather     per (cell, velocity): the neighbour and mirror gathers, the collision diagonal and the moment
//                    expansion w (a0 + a.c + a2 c^2 + b.c c^2), written at the position of the reversed velocity
// The LU-SGS passes of the forward solver, run on velocity-reversed storage, are the transposed preconditioner.
#pragma once

#include <cuda_runtime.h>

#include "kin_kernels.cuh"

namespace kin {

// per cell: Lambda0 and the derivative sums with respect to (rho, u (3), T, q (3)); for a cell whose equilibrium is
// the discrete one also sum lambda E F psi (5) and sum lambda E psi (5), the derivative sums then at fixed
// (beta, gamma) (the host finishes the chain through the Newton solve)
constexpr int kAdjCellSums = 19;
// S0, S1 (3), S2, S5, S6, A1, A2, S_spec, S6 c (3), sum_in w psi f_spec (5) (k_adj_faces)
constexpr int kAdjFaceSums = 18;
constexpr int kAdjCoefs = 8;      // a0, a (3), a2, b (3)

template <class S>
struct AdjView {
  const S* lam;            // [cell][p]: the adjoint of velocity rev[p] (velocity-reversed storage)
  const int32_t* rev;      // position of -xi for every position
  const int32_t* rev_entry;  // for an internal CSR entry (cell j -> i): the entry of cell i that points back to j
  S* gbx;                  // gradient seeds G_bar [cell][q]
  S* gby;
  S* gbz;
  S* hmax;                 // seed on the stencil maximum / minimum of the limiter when it is a stencil entry
  S* hmin;
  int8_t* imax;            // that entry (offset within the cell's CSR row), -1 none
  int8_t* imin;
  S* lfb;                  // seeds that land on f[cell][q] itself
  const double* mu;        // per boundary face: seed weight of the outgoing face values (nu and objective terms)
  const double* mom_mu;    // per boundary face (5), nullptr if none: seed of the face moment sums
                           // sum_q w psi(xi_q) f_b(q), psi = (1, xi, |xi|^2 / 2) (the face states that the limited
                           // pressure-boundary reconstruction reads)
  const int32_t* flip;     // [axis][q]: position of xi with component `axis` negated (3 x nv)
  const int32_t* face_axis;  // per boundary face: the axis its normal is aligned with, -1 if none
  const double* coef;      // per cell: moment expansion coefficients (kAdjCoefs)
  const double* moments;   // per cell: the 15 moments of the forward state
  const int32_t* deq_flags;  // per cell: the discrete-equilibrium result of the forward state (> 0: discrete)
  S* out;                  // O_f(y) at the reversed position [cell][rev[q]]
};

template <class S>
void adj_cell_sums(const View<S, double>& v, const AdjView<S>& a, double* out, cudaStream_t st);
// cells != nullptr: only the n listed cells (the owners of wall and pressure faces, for the per-face sums)
template <class S>
void adj_transport(const View<S, double>& v, const AdjView<S>& a, const int32_t* cells, int n, cudaStream_t st);
template <class S>
void adj_face_sums(const View<S, double>& v, const AdjView<S>& a, double* out, cudaStream_t st);
template <class S>
void adj_gather(const View<S, double>& v, const AdjView<S>& a, double* res_cell, cudaStream_t st);

}  // namespace kin
