// Launch interface of the kinetic kernels (kin_kernels.cu). All launches go to the given stream and do not
// synchronise.
#pragma once

#include <cuda_runtime.h>

#include "kin_kernels.cuh"

namespace kin {

constexpr int kSweepThreads = 256;  // one CTA per (direction, block, velocity tile): 8 warps share every level
constexpr int kSweepTile = 32;      // velocities of one sweep CTA (one per lane)

// compact LU-SGS stencil entry: neighbour cell (>= 0), -1 boundary face, -2 periodic face (no coupling)
template <class M>
struct SweepE {
  int32_t other;
  M s[3];
};

// staged stencil entry of one chain: code = kind << 28 | neighbour cell (kinds: periodic, boundary, in-block lower,
// in-block upper, other block)
template <class M>
struct StageE {
  uint32_t code;
  M s[3];
};
enum : uint32_t { kKindPeriodic = 0, kKindBoundary = 1, kKindLower = 2, kKindUpper = 3, kKindOther = 4 };
constexpr uint32_t kKindShift = 28, kIndexMask = (1u << kKindShift) - 1;

constexpr int kTileThreadsSweep = 128;  // threads of one k_sweep_tiles CTA

// arguments of one LU-SGS block pass over a velocity chunk
template <class S, class M>
struct SweepArgs {
  const int4* items;  // per CTA: (chain, t0, t1, 0), chunk-local velocity range [t0, t1)
  int32_t n_items;
  int32_t n_blocks;
  const int32_t* block_offsets;
  const int4* prog;            // per chain, in level order: (cell, first CSR entry, entries, in-block-lower bitmask)
  const int32_t* chain_start;  // chain -> first index in prog
  const int32_t* lev_bounds;   // level boundaries relative to chain_start (n_levels + 1 per chain)
  const int32_t* lev_start;    // chain -> first index in lev_bounds
  const int32_t* lev_count;    // chain -> number of levels
  const SweepE<M>* se;         // compact stencil entries, CSR order
  const S* R;                  // steady residual of the chunk
  const S* dprev;              // Delta f of the previous pass (nullptr in the first pass)
  S* out;                      // Delta f* then Delta f
  // k_sweep_tiles: the diagonal D of every (cell, velocity), written by the forward sweep and read by the backward
  // one instead of being summed again (a chunk-sized work array that is free during the passes)
  S* diag_store;
  int32_t update_f;
  int32_t k0;
  int32_t stride;
  // staged schedule (k_sweep_tiles): every level split into sub-levels of at most kStageCells cells and
  // kStageEntries stencil entries, stored contiguously per chain so one sub-level is one copy into shared memory
  int32_t staged_ne;            // 0: use k_sweep_pass; else the entry bound of k_sweep_tiles (6 or 8)
  const int4* sprog;            // (cell, entry offset within the sub-level, entries, -)
  const StageE<M>* sse;         // stencil entries with their kind, in sub-level order (one copy per chain)
  const int32_t* sub_cells;     // absolute sub-level boundaries in sprog (n_sub + 1 per chain)
  const int32_t* sub_entries;   // absolute sub-level boundaries in sse (n_sub + 1 per chain)
  const int32_t* sub_start;     // chain -> first index in sub_cells / sub_entries
  const int32_t* sub_count;     // chain -> number of sub-levels
  // resident block pass (k_sweep_resident): one CTA per (chain, 64-byte velocity window) keeps the window of the
  // whole block in shared memory through the forward and backward sweeps
  const int4* ritems;           // per CTA: (chain, window start, first valid, end valid), chunk-local positions
  int32_t n_ritems;
  const uint32_t* scells;       // cell of every sprog slot | 1 << 31 when the cell has an out-of-block neighbour
  const S* Rs;                  // passes after the first: R + out-of-block coupling of the surface cells (k_lout)
  int32_t* err;                 // device status word (kSweepErrStaging: a staging wait gave up)
  int32_t tile_u, tile_blocks;  // shape of k_sweep_tiles (velocities per thread, CTAs per SM)
  int32_t resident_smem;        // dynamic shared memory of k_sweep_resident in bytes (0: not usable)
  int32_t max_block_cells;      // largest RCB block (rows of the resident window)
};

constexpr int32_t kSweepErrStaging = 1;

// out-of-block upwind coupling of a later block pass, folded into the residual of the cells that have an
// out-of-block neighbour (k_lout): Rs[c][t] = R[c][t] + sum over those entries of min(xi_t . S, 0) dprev[j][t]
template <class S, class P>
struct LoutArgs {
  const int4* surf;            // (cell, first entry in sent, number of entries, -)
  int32_t n_surf;
  const StageE<P>* sent;       // code = neighbour cell, s = S_out, CSR order
  const S* R;
  const S* dprev;
  S* Rs;
  int32_t k0, kc, stride;
};

// the resident block pass and its coupling kernel (kin_sweep.cu)
template <class S, class P>
struct SweepLaunch {
  static constexpr int kWidth = 64 / static_cast<int>(sizeof(S));  // velocities of a window: 64 bytes per cell row
  static int smem_bytes(int max_block_cells);                       // dynamic shared memory, 0 if too large
  static void resident(const View<S, P>& v, const SweepArgs<S, P>& a, bool first, bool last, cudaStream_t st);
  static void lout(const View<S, P>& v, const LoutArgs<S, P>& a, cudaStream_t st);
};

// the kernel shapes of an arithmetic type: the measured defaults, or another compiled shape named by the environment
// variable KIN_SHAPE ("res=UxB,grad=UxB,tile=UxB"; read when a handle is created)
template <class M>
KernelShape default_shape();
template <class M>
KernelShape read_shape();

constexpr int kStageCells = 64;     // cells of one staged sub-level
constexpr int kStageEntries = 384;  // stencil entries of one staged sub-level
constexpr int kMaxSubLevels = 512;  // sub-levels of one chain the staged kernel accepts

template <class S, class M>
struct Launch {
  static void set_equilibrium(const View<S, M>& v, const double* states, double* shift, int discrete, cudaStream_t st);
  static void moments(const View<S, M>& v, double* shift, double* out, cudaStream_t st);
  static void moment_sums(const View<S, M>& v, double* shift, double* out, cudaStream_t st);
  static void shift_from_moments(const double* moments, double* shift, int n, cudaStream_t st);
  static void finalize_sums(const double* sums, double weight, double* shift, double* moments, int n, cudaStream_t st);
  static void scale(S* f, int64_t n, double s, double* moments, int n_cells, cudaStream_t st);
  static void cell_params(const View<S, M>& v, const double* moments, const double* volume, const double* vdt,
                          double mu0, double omega, double Pr, double cold_bgk_T, int discrete, int collisionless,
                          CellParams<M>* out, int* flags, cudaStream_t st);
  static void maxwell_reflection(const View<S, M>& v, cudaStream_t st);
  static void cast_cell_params(const CellParams<M>* src, CellParams<float>* dst, int n, cudaStream_t st);
  static void boundary_sums(const View<S, M>& v, double* out, cudaStream_t st);
  static void internal_face_flux(const View<S, M>& v, const int32_t* cells, const int32_t* entries, double* out, int n,
                                 cudaStream_t st);
  static int residual_tiles(int kc, int res_u);
  static void gradient(const View<S, M>& v, const Chunk<S>& ch, cudaStream_t st);
  static void residual(const View<S, M>& v, const Chunk<S>& ch, double* partial, int partial_stride,
                       double* residual_cell, cudaStream_t st);
  static void sweep_pass(const View<S, M>& v, const SweepArgs<S, M>& a, cudaStream_t st);
  static void gsis_correction(const View<S, M>& v, const double* wh, const double* wn, int* flags, double* shift,
                              int mode, int discrete, int collisionless, int phase, double* ext, cudaStream_t st);
  static void discrete_maxwell_states(const View<S, M>& v, const DeqGrid& deq, const double* states, double* out,
                                      int* result, int n, cudaStream_t st);
  static void import_f(const double* src, S* f, const int32_t* perm, int64_t c0, int n, int nv, cudaStream_t st);
  static void export_f(const S* f, double* dst, const int32_t* inv, int64_t c0, int n, int nv, cudaStream_t st);
};

}  // namespace kin
