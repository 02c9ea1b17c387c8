// Resident LU-SGS block pass for sm_100a: the window of one (direction group, RCB block) chain stays in shared memory
// from the residual to the final correction.
//
// One CTA of kResThreads threads takes one chain and one 64-byte velocity window (8 FP64 or 16 FP32 velocities, the
// same window for every cell). The forward sweep writes Delta f* over R and the backward sweep writes Delta f over
// Delta f*, in place in shared memory, exactly as the reference overwrites its work array
// (sweep_forward_cell / sweep_backward_cell, src/kinetic/kinetic_kernels.hpp:289-358). So a pass reads R once and
// writes its result once (Delta f for the next pass, or f += Delta f in the last pass); nothing of the sweep spills
// to global memory in between.
//
// The chain's cells are visited in the host's level schedule (levels cut into sub-levels of at most kStageCells
// cells and kStageEntries stencil entries). Every step is staged one step ahead by the TMA engine: two 1-D bulk
// copies (cp.async.bulk) bring the next sub-level's program and stencil entries, and one 64-byte bulk copy per cell
// brings its R row straight into the window; an mbarrier per buffer counts the bytes. Per-cell scalars (the LU-SGS
// diagonal, and f in the last pass) are prefetched into registers one step ahead with ordinary loads. The compute of
// a step therefore only touches shared memory and registers, with one barrier per step.
//
// Passes after the first need Delta f of the previous pass at out-of-block upwind neighbours (the reference's Lout).
// k_lout adds that coupling to R of the cells that have such neighbours before the pass (R + Lout, the same sum in
// the same order), so the pass itself needs no scattered global loads.
#include "kin_kernels.cuh"
#include "kin_launch.h"

namespace kin {

constexpr int kResThreads = 512;                 // threads of a resident CTA (one CTA per SM)
constexpr long long kStagingWaitCycles = 2000000000LL;  // ~1 s: a staging wait that takes longer gives up

// ---------------------------------------------------------------------------------------------------------
// mbarrier and bulk-copy helpers (PTX ISA: mbarrier, cp.async.bulk)
// ---------------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// waits for the phase of the given parity to complete; false once about `limit` cycles have passed
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}
// global -> shared bulk copy completing on `bar` (both addresses 16-byte aligned, bytes a multiple of 16)
__device__ __forceinline__ void bulk_to_shared(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// the upwind split max(a, 0) / min(a, 0) of a = xi . S (FP32: min / max instructions; FP64: compare and select)
__device__ __forceinline__ double pos_part_r(double af) { return af > 0.0 ? af : 0.0; }
__device__ __forceinline__ float pos_part_r(float af) { return fmaxf(af, 0.0f); }
__device__ __forceinline__ double neg_part_r(double af) { return af > 0.0 ? 0.0 : af; }
__device__ __forceinline__ float neg_part_r(float af) { return fminf(af, 0.0f); }

template <class P>
struct ResidentStage {
  int4 prog[kStageCells];
  StageE<P> se[kStageEntries];
};

// dynamic shared memory layout of k_sweep_resident
template <class S, class P>
struct ResidentLayout {
  static constexpr size_t kBars = 0;                                       // 2 mbarriers + abort word
  static constexpr size_t kStage = 128;                                    // ResidentStage<P>[2]
  static constexpr size_t kSubCells = kStage + 2 * sizeof(ResidentStage<P>);  // sub-level cell bounds
  static constexpr size_t kSubEntries = kSubCells + 4 * (kMaxSubLevels + 1);
  static constexpr size_t kCells = kSubEntries + 4 * (kMaxSubLevels + 1);  // chain cells (uint32 each)
  __host__ __device__ static size_t window(int max_block) {                // X: max_block rows of 64 bytes
    return (kCells + 4 * static_cast<size_t>(max_block) + 127) / 128 * 128;
  }
  __host__ __device__ static size_t bytes(int max_block) { return window(max_block) + 64 * static_cast<size_t>(max_block); }
};
static_assert(sizeof(ResidentStage<double>) % 128 == 0 && sizeof(ResidentStage<float>) % 128 == 0,
              "stage buffers keep 128-byte alignment");

// ---------------------------------------------------------------------------------------------------------
// k_sweep_resident: one LU-SGS block pass of one chain for one velocity window
//   First: first pass (out-of-block coupling damped on the diagonal: beta sum |a-|, the reference's am_out)
//   Last:  last pass (f += Delta f); otherwise Delta f goes to a.out for the next pass
// ---------------------------------------------------------------------------------------------------------
template <class S, class P, int NE, bool First, bool Last>
__global__ void __launch_bounds__(kResThreads, 1) k_sweep_resident(View<S, P> v, SweepArgs<S, P> a) {
  constexpr int V = 64 / static_cast<int>(sizeof(S));
  constexpr int kRows = kResThreads / V;                     // cells covered by one round of the threads
  constexpr int MI = (kStageCells + kRows - 1) / kRows;      // cell slots per thread in one step
  using L = ResidentLayout<S, P>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::kBars);
  int* sh_abort = reinterpret_cast<int*>(smem + L::kBars + 16);
  ResidentStage<P>* stage_buf = reinterpret_cast<ResidentStage<P>*>(smem + L::kStage);
  int32_t* sh_sc = reinterpret_cast<int32_t*>(smem + L::kSubCells);
  int32_t* sh_se = reinterpret_cast<int32_t*>(smem + L::kSubEntries);
  uint32_t* sh_cells = reinterpret_cast<uint32_t*>(smem + L::kCells);
  S* X = reinterpret_cast<S*>(smem + L::window(a.max_block_cells));

  const int4 it = a.ritems[blockIdx.x];  // (chain, window start, first valid, end valid)
  const int chain = it.x, wb = it.y;
  const int nsub = a.sub_count[chain];
  if (nsub <= 0) return;
  const int cb = a.block_offsets[chain % a.n_blocks];
  const int s0 = a.sub_start[chain];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int u = tid % V;        // velocity of this thread within the window
  const int slot0 = tid / V;    // first cell slot of this thread in a step
  const bool act = wb + u >= it.z && wb + u < it.w;
  const int q = a.k0 + (act ? wb + u : it.z);
  const P x = v.xi_x[q], y = v.xi_y[q], z = v.xi_z[q];
  const int base = a.sub_cells[s0];
  const int nchain = a.sub_cells[s0 + nsub] - base;
  for (int k = tid; k <= nsub; k += kResThreads) {
    sh_sc[k] = a.sub_cells[s0 + k] - base;
    sh_se[k] = a.sub_entries[s0 + k];
  }
  for (int k = tid; k < nchain; k += kResThreads) sh_cells[k] = a.scells[base + k];
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    *sh_abort = 0;
    mbar_fence_init();
  }
  __syncthreads();

  const int nsteps = 2 * nsub;  // forward over sub-levels 0 .. nsub-1, then backward over nsub-1 .. 0
  auto level_of = [&](int s) { return s < nsub ? s : nsteps - 1 - s; };
  // warp 0 stages step s into buffer s & 1: program and entries of its sub-level, R rows in forward steps
  auto stage = [&](int s) {
    const int l = level_of(s);
    ResidentStage<P>& dst = stage_buf[s & 1];
    const int p0 = sh_sc[l], np = sh_sc[l + 1] - p0;
    const int e0 = sh_se[l], ne = sh_se[l + 1] - e0;
    const bool fwd = s < nsub;
    if (lane == 0) {
      const uint32_t bytes = static_cast<uint32_t>(np * sizeof(int4) + ne * sizeof(StageE<P>) + (fwd ? np * 64 : 0));
      mbar_arrive_expect_tx(&bar[s & 1], bytes);
      if (np > 0) bulk_to_shared(dst.prog, a.sprog + base + p0, static_cast<uint32_t>(np * sizeof(int4)), &bar[s & 1]);
      if (ne > 0) bulk_to_shared(dst.se, a.sse + e0, static_cast<uint32_t>(ne * sizeof(StageE<P>)), &bar[s & 1]);
    }
    if (fwd) {
      for (int k = lane; k < np; k += 32) {
        const uint32_t cw = sh_cells[p0 + k];
        const int cell = static_cast<int>(cw & 0x7fffffffu);
        const S* src = (!First && (cw >> 31)) ? a.Rs : a.R;
        bulk_to_shared(X + static_cast<int64_t>(cell - cb) * V, src + static_cast<int64_t>(cell) * a.stride + wb, 64,
                       &bar[s & 1]);
      }
    }
  };
  // per-cell scalars of step s for this thread's slots: the diagonal, and f in backward steps of the last pass
  P dg[MI], dgn[MI];
  S fv[MI], fvn[MI];
  auto prefetch = [&](int s, P (&d)[MI], S (&fo)[MI]) {
    const int l = level_of(s);
    const int p0 = sh_sc[l], np = sh_sc[l + 1] - p0;
#pragma unroll
    for (int m = 0; m < MI; ++m) {
      const int k = slot0 + m * kRows;
      d[m] = P(0);
      fo[m] = S(0);
      if (k < np) {
        const int cell = static_cast<int>(sh_cells[p0 + k] & 0x7fffffffu);
        d[m] = v.cp[cell].diag;
        if (Last && s >= nsub && act) fo[m] = v.f[static_cast<int64_t>(cell) * v.nv + a.k0 + wb + u];
      }
    }
  };

  if (warp == 0) stage(0);
  prefetch(0, dg, fv);
  for (int s = 0; s < nsteps; ++s) {
    const int b = s & 1;
    if (s + 1 < nsteps) {
      if (warp == 0) stage(s + 1);
      prefetch(s + 1, dgn, fvn);
    }
    const bool ready = mbar_wait_bounded(&bar[b], static_cast<uint32_t>((s >> 1) & 1), kStagingWaitCycles);
    if (!ready) {
      *sh_abort = 1;
    } else {
      const ResidentStage<P>& cur = stage_buf[b];
      const int l = level_of(s);
      const int np = sh_sc[l + 1] - sh_sc[l];
      const bool fwd = s < nsub;
#pragma unroll
      for (int m = 0; m < MI; ++m) {
        const int k = slot0 + m * kRows;
        if (k >= np || !act) continue;
        const int4 p = cur.prog[k];
        const int row = p.x - cb;
        const P own = static_cast<P>(X[row * V + u]);
        P ap = P(0), cpl = P(0), am = P(0);  // sum a+, in-block coupling (lower or upper), damped out-of-block a-
#pragma unroll
        for (int j = 0; j < NE; ++j) {
          if (j >= p.z) break;
          const StageE<P>& e = cur.se[p.y + j];
          const uint32_t kind = e.code >> kKindShift;
          if (kind == kKindPeriodic) continue;
          const P af = x * e.s[0] + y * e.s[1] + z * e.s[2];
          ap += pos_part_r(af);
          if (kind == (fwd ? kKindLower : kKindUpper)) {
            cpl += neg_part_r(af) * static_cast<P>(X[(static_cast<int>(e.code & kIndexMask) - cb) * V + u]);
          } else if (First && kind == kKindOther) {
            am -= neg_part_r(af);
          }
        }
        const P D = dg[m] + v.diag_scale * ap + v.interface_damping * am;
        if (fwd) {
          X[row * V + u] = static_cast<S>((-own - cpl) / D);
        } else {
          const P df = own - cpl / D;
          X[row * V + u] = static_cast<S>(df);
          if (Last) {
            v.f[static_cast<int64_t>(p.x) * v.nv + a.k0 + wb + u] = static_cast<S>(static_cast<P>(fv[m]) + df);
          } else {
            a.out[static_cast<int64_t>(p.x) * a.stride + wb + u] = static_cast<S>(df);
          }
        }
      }
    }
    __syncthreads();
    if (*sh_abort) {
      // a staging copy did not arrive in time: record it, let the copies in flight land (bounded) and stop
      if (tid == 0) {
        atomicExch(a.err, kSweepErrStaging);
        mbar_wait_bounded(&bar[b], static_cast<uint32_t>((s >> 1) & 1), kStagingWaitCycles);
        if (s + 1 < nsteps) mbar_wait_bounded(&bar[b ^ 1], static_cast<uint32_t>(((s + 1) >> 1) & 1), kStagingWaitCycles);
      }
      __syncthreads();
      return;
    }
#pragma unroll
    for (int m = 0; m < MI; ++m) {
      dg[m] = dgn[m];
      fv[m] = fvn[m];
    }
  }
}

// ---------------------------------------------------------------------------------------------------------
// k_lout: R + out-of-block upwind coupling of the previous pass for the cells that have out-of-block neighbours
// (the Lout of sweep_forward_cell, src/kinetic/kinetic_kernels.hpp:289-324, in CSR order)
// grid: (groups of kLoutCells surface cells, velocity tiles of kLoutThreads * kLoutU)
// ---------------------------------------------------------------------------------------------------------
constexpr int kLoutThreads = 256;
constexpr int kLoutU = 4;
constexpr int kLoutCells = 4;

template <class S, class P>
__global__ void __launch_bounds__(kLoutThreads) k_lout(View<S, P> v, LoutArgs<S, P> a) {
  const int i0 = blockIdx.x * kLoutCells, i1 = min(a.n_surf, i0 + kLoutCells);
  const int tb = blockIdx.y * (kLoutThreads * kLoutU);
  int t[kLoutU];
  bool ok[kLoutU];
  P x[kLoutU], y[kLoutU], z[kLoutU];
#pragma unroll
  for (int uu = 0; uu < kLoutU; ++uu) {
    t[uu] = tb + threadIdx.x + uu * kLoutThreads;
    ok[uu] = t[uu] < a.kc;
    const int q = a.k0 + (ok[uu] ? t[uu] : 0);
    x[uu] = v.xi_x[q];
    y[uu] = v.xi_y[q];
    z[uu] = v.xi_z[q];
  }
  for (int i = i0; i < i1; ++i) {
    const int4 sc = a.surf[i];
    const int64_t row = static_cast<int64_t>(sc.x) * a.stride;
    P ext[kLoutU], val[8][kLoutU];
#pragma unroll
    for (int uu = 0; uu < kLoutU; ++uu) ext[uu] = P(0);
    // issue every neighbour load of the cell first (at most 8 out-of-block entries per cell)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (j >= sc.z) break;
      const int64_t nrow = static_cast<int64_t>(a.sent[sc.y + j].code & kIndexMask) * a.stride;
#pragma unroll
      for (int uu = 0; uu < kLoutU; ++uu) val[j][uu] = ok[uu] ? static_cast<P>(a.dprev[nrow + t[uu]]) : P(0);
    }
    S r[kLoutU];
#pragma unroll
    for (int uu = 0; uu < kLoutU; ++uu) r[uu] = ok[uu] ? a.R[row + t[uu]] : S(0);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (j >= sc.z) break;
      const StageE<P>& e = a.sent[sc.y + j];
#pragma unroll
      for (int uu = 0; uu < kLoutU; ++uu) {
        const P af = x[uu] * e.s[0] + y[uu] * e.s[1] + z[uu] * e.s[2];
        ext[uu] += neg_part_r(af) * val[j][uu];
      }
    }
#pragma unroll
    for (int uu = 0; uu < kLoutU; ++uu)
      if (ok[uu]) a.Rs[row + t[uu]] = static_cast<S>(static_cast<P>(r[uu]) + ext[uu]);
  }
}

// ---------------------------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------------------------
template <class S, class P>
int SweepLaunch<S, P>::smem_bytes(int max_block_cells) {
  const size_t b = ResidentLayout<S, P>::bytes(max_block_cells);
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  return b <= static_cast<size_t>(optin) ? static_cast<int>(b) : 0;
}

template <class S, class P, int NE, bool First, bool Last>
static void launch_resident(const View<S, P>& v, const SweepArgs<S, P>& a, cudaStream_t st) {
  auto kern = k_sweep_resident<S, P, NE, First, Last>;
  // the attribute is per kernel and per device; setting it again is harmless
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, a.resident_smem);
  kern<<<a.n_ritems, kResThreads, a.resident_smem, st>>>(v, a);
}

template <class S, class P>
void SweepLaunch<S, P>::resident(const View<S, P>& v, const SweepArgs<S, P>& a, bool first, bool last,
                                 cudaStream_t st) {
  if (a.n_ritems <= 0) return;
#define KIN_RES(NE)                                                  \
  if (first && last) launch_resident<S, P, NE, true, true>(v, a, st);        \
  else if (first) launch_resident<S, P, NE, true, false>(v, a, st);          \
  else if (last) launch_resident<S, P, NE, false, true>(v, a, st);           \
  else launch_resident<S, P, NE, false, false>(v, a, st);
  if (a.staged_ne == 6) {
    KIN_RES(6)
  } else {
    KIN_RES(8)
  }
#undef KIN_RES
}

template <class S, class P>
void SweepLaunch<S, P>::lout(const View<S, P>& v, const LoutArgs<S, P>& a, cudaStream_t st) {
  if (a.n_surf <= 0 || a.kc <= 0) return;
  const dim3 grid((a.n_surf + kLoutCells - 1) / kLoutCells, (a.kc + kLoutThreads * kLoutU - 1) / (kLoutThreads * kLoutU));
  k_lout<S, P><<<grid, kLoutThreads, 0, st>>>(v, a);
}

template struct SweepLaunch<float, float>;
template struct SweepLaunch<double, double>;

}  // namespace kin
