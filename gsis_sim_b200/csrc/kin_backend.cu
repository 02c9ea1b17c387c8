// Host side of the B200 kinetic backend: device memory, level schedule, launch sequencing, timing, and the C ABI
// of include/gsis_b200.h. One KinHandle corresponds to one reference `CudaBackend<F>` object
// (src/kinetic/kinetic_backend_cuda.cpp:89-502).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "gsis_b200.h"
#include "kin_adjoint.h"
#include "kin_launch.h"

namespace {

thread_local std::string g_create_error;

struct KinError : std::runtime_error {
  int code;
  KinError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define KCHECK(cond, msg)                                     \
  do {                                                        \
    if (!(cond)) throw KinError(KIN_E_ARG, std::string(msg)); \
  } while (0)

#define KCUDA(call)                                                                                              \
  do {                                                                                                           \
    cudaError_t err_ = (call);                                                                                   \
    if (err_ != cudaSuccess)                                                                                     \
      throw KinError(KIN_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(err_) + " (" __FILE__ ":" +      \
                                     std::to_string(__LINE__) + ")");                                            \
  } while (0)

// RAII device array
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    release();
    n = count;
    if (count == 0) return;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      throw KinError(e == cudaErrorMemoryAllocation ? KIN_E_MEMORY : KIN_E_CUDA,
                     std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) + " bytes: " +
                         cudaGetErrorString(e));
    }
  }
  void upload(const T* host, size_t count, cudaStream_t st) {
    alloc(count);
    if (count) KCUDA(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  size_t bytes() const { return n * sizeof(T); }
};

// CUDA-event phase timer on the handle's stream (PhaseTimer, src/kinetic/kinetic_backend_cuda.cpp:29-87)
struct PhaseTimer {
  enum Phase { kMoments, kBoundary, kGradient, kResidual, kForward, kBackward, kOther };
  struct Pending {
    Phase phase;
    cudaEvent_t a, b;
  };
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<Pending> pending;
  Phase cur = kOther;
  cudaEvent_t start{};
  ~PhaseTimer() {
    for (auto e : pool) cudaEventDestroy(e);
  }
  cudaEvent_t take() {
    if (used == pool.size()) {
      cudaEvent_t e;
      KCUDA(cudaEventCreate(&e));
      pool.push_back(e);
    }
    return pool[used++];
  }
  void begin(Phase p, cudaStream_t st) {
    cur = p;
    start = take();
    KCUDA(cudaEventRecord(start, st));
  }
  void end(cudaStream_t st) {
    cudaEvent_t e = take();
    KCUDA(cudaEventRecord(e, st));
    pending.push_back({cur, start, e});
  }
  void flush(KinStepTimings& t) {
    if (pending.empty()) return;
    KCUDA(cudaEventSynchronize(pending.back().b));
    for (const auto& p : pending) {
      float ms = 0.f;
      KCUDA(cudaEventElapsedTime(&ms, p.a, p.b));
      const double s = 1e-3 * ms;
      switch (p.phase) {
        case kMoments: t.moments += s; break;
        case kBoundary: t.boundary += s; break;
        case kGradient: t.gradient += s; break;
        case kResidual: t.residual += s; break;
        case kForward: t.sweep_forward += s; break;
        case kBackward: t.sweep_backward += s; break;
        default: t.other += s; break;
      }
    }
    pending.clear();
    used = 0;
  }
};

// Factors a velocity set (m points, any order) as a tensor grid: per axis the distinct node values, every
// (i, j, k) combination present exactly once, and weights w(q) = w_x[i] w_y[j] w_z[k] (w == nullptr: uniform, all
// per-axis weights 1). Returns false when the set is not of that form; the caller then sums point by point.
bool factor_tensor_grid(const double* x, const double* y, const double* z, const double* w, int64_t m,
                        std::vector<double>& nodes, std::vector<double>& wax, int32_t (&n)[3]) {
  const double* xs[3] = {x, y, z};
  std::vector<double> ax[3];
  for (int a = 0; a < 3; ++a) {
    ax[a].assign(xs[a], xs[a] + m);
    std::sort(ax[a].begin(), ax[a].end());
    ax[a].erase(std::unique(ax[a].begin(), ax[a].end()), ax[a].end());
    n[a] = static_cast<int32_t>(ax[a].size());
  }
  if (m <= 0 || static_cast<int64_t>(n[0]) * n[1] * n[2] != m) return false;
  std::vector<int64_t> at(static_cast<size_t>(m), -1);  // grid index -> point
  for (int64_t q = 0; q < m; ++q) {
    int64_t g = 0;
    for (int a = 2; a >= 0; --a) {
      const auto it = std::lower_bound(ax[a].begin(), ax[a].end(), xs[a][q]);
      g = g * n[a] + (it - ax[a].begin());
    }
    if (at[g] >= 0) return false;
    at[g] = q;
  }
  nodes.clear();
  wax.assign(static_cast<size_t>(n[0] + n[1] + n[2]), 1.0);
  for (int a = 0; a < 3; ++a) nodes.insert(nodes.end(), ax[a].begin(), ax[a].end());
  if (w != nullptr) {
    auto wq = [&](int i, int j, int k) { return w[at[i + static_cast<int64_t>(n[0]) * (j + static_cast<int64_t>(n[1]) * k)]]; };
    const double w000 = wq(0, 0, 0);
    if (!(w000 > 0.0)) return false;
    for (int i = 0; i < n[0]; ++i) wax[i] = wq(i, 0, 0);
    for (int j = 0; j < n[1]; ++j) wax[n[0] + j] = wq(0, j, 0) / w000;
    for (int k = 0; k < n[2]; ++k) wax[n[0] + n[1] + k] = wq(0, 0, k) / w000;
    for (int k = 0; k < n[2]; ++k)
      for (int j = 0; j < n[1]; ++j)
        for (int i = 0; i < n[0]; ++i) {
          const double prod = wax[i] * wax[n[0] + j] * wax[n[0] + n[1] + k];
          const double ref = wq(i, j, k);
          if (!(std::abs(prod - ref) <= 1e-13 * std::abs(ref))) return false;
        }
  }
  return true;
}

}  // namespace

struct KinHandle {
  virtual ~KinHandle() = default;
  std::string err;
  cudaStream_t stream = nullptr;      // stream every kernel of the handle goes to
  cudaStream_t own_stream = nullptr;  // the stream the handle created (destroyed with it)
  int64_t launches = 0;
  int device = 0;
  virtual const char* name() const = 0;
  virtual int32_t chunk_width() const = 0;
  virtual uint64_t memory_bytes() const = 0;
  virtual void set_equilibrium(const double* s, int64_t n) = 0;
  virtual void set_distribution(const double* f, int64_t n) = 0;
  virtual void get_distribution(double* f, int64_t n) = 0;
  virtual void compute_moments(double* out, int64_t n) = 0;
  virtual void scale_distribution(double s) = 0;
  virtual void update_cell_params() = 0;
  virtual void set_inflow(const KinInflowState* in, int64_t n) = 0;
  virtual void boundary_sums(double* out, int64_t n) = 0;
  virtual void sweep(double* residual_cell, int64_t n) = 0;
  virtual void gsis_correction(const double* wh, const double* wn, int64_t n, int32_t* flags, int64_t* replaced) = 0;
  virtual void gsis_correction_extrema(const double* wh, const double* wn, int64_t n, double* ext, int64_t n_ext) = 0;
  virtual void gsis_correction_apply(const double* wh, const double* wn, int64_t n, const double* ext, int64_t n_ext,
                                     int32_t* flags, int64_t* replaced) = 0;
  virtual void internal_face_mass_flux(const int32_t* cells, const int32_t* entries, int64_t n, double* out) = 0;
  virtual void take_timings(KinStepTimings* out) = 0;
  virtual void deq_counts(KinDeqCounts* out) = 0;
  virtual void device_f(void** f, int32_t* es) = 0;
  virtual void velocity_permutation(int32_t* perm, int64_t n) const = 0;
  virtual void schedule_info(int32_t* max_levels, int32_t* n_chains) const = 0;
  virtual void discrete_maxwell(const double* states, int64_t n, double tol, double* out, int32_t* result) = 0;
  virtual void discrete_maxwell_noalloc(const double* states, int64_t n, double tol, double* out,
                                        int32_t* result) = 0;
  virtual void moment_sums(double* out, int64_t n) = 0;
  virtual void set_moments(const double* m, int64_t n) = 0;
  virtual void device_sums(int32_t which, double** ptr, int64_t* n) = 0;
  virtual void finalize_moments(double* out, int64_t n) = 0;
  virtual void read_sums(int32_t which, double* out, int64_t n) = 0;
  // discrete adjoint (FP64 handles with one velocity chunk)
  virtual void adjoint_begin(const int32_t* rev_velocity, const int32_t* rev_entry, int64_t n_entries,
                             const int32_t* flip_velocity, const int32_t* face_axis) = 0;
  virtual void adjoint_set(const double* lam, int64_t n) = 0;
  virtual void adjoint_get(double* lam, int64_t n) = 0;
  virtual void adjoint_reduce(const double* mu, int64_t n_mu, double* cell_sums, int64_t n_cell, double* face_sums,
                              int64_t n_face) = 0;
  virtual void adjoint_face_moment_seeds(const double* seeds, int64_t n) = 0;
  virtual void adjoint_update(const double* coef, int64_t n_coef, double* res_cell, int64_t n_res, int32_t run_passes,
                              double* op_out, int64_t n_op) = 0;
  virtual void adjoint_end() = 0;
};

// Scratch of kin_discrete_maxwell_noalloc: static device memory of this module (one copy per device), laid out as
// [input states: 5 doubles x KIN_NOALLOC_MAX_STATES][corrected states: same][Newton results: int32 x same].
static constexpr size_t kNoAllocStatesBytes = sizeof(double) * 5 * KIN_NOALLOC_MAX_STATES;
static constexpr size_t kNoAllocScratchBytes = 2 * kNoAllocStatesBytes + sizeof(int32_t) * KIN_NOALLOC_MAX_STATES;
static_assert(kNoAllocStatesBytes % 256 == 0, "each part of the scratch starts on a 256-byte boundary");
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_address[kNoAllocMaxDevices] = {};

// Device address of the scratch on `device`, looked up once per device (with that device current) and kept.
unsigned char* noalloc_scratch(int device) {
  KCHECK(device >= 0 && device < kNoAllocMaxDevices, "kin_discrete_maxwell_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_address[device] == nullptr) {
    KCUDA(cudaSetDevice(device));
    void* p = nullptr;
    KCUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_address[device] = p;
  }
  return static_cast<unsigned char*>(g_noalloc_address[device]);
}

}  // namespace

namespace {

using kin::BFace;
using kin::CellParams;
using kin::CsrE;
using kin::Inflow;

template <class S, class M>
struct Backend final : KinHandle {
  using L = kin::Launch<S, M>;
  // arithmetic of the gradient and the LU-SGS passes: FP32 in the mixed mode (f in FP32, residual and every sum in
  // FP64: the FP32 sweeps are a defect correction of the FP64 residual), M otherwise
  using P = typename std::conditional<std::is_same<S, float>::value && std::is_same<M, double>::value, float, M>::type;
  using LP = kin::Launch<S, P>;
  static constexpr bool kSplit = !std::is_same<P, M>::value;
  static constexpr size_t kMargin = size_t{1} << 30;  // device memory kept free (1 GiB)

  // sizes and parameters
  int32_t nc = 0, nv = 0, nb = 0, n_blocks = 0, n_groups = 1, precision = 0;
  int32_t block_passes = 1, discrete_eq = 0, collisionless = 0, negative_mode = 0, n_maxwell = 0;
  double mu0 = 0, omega = 0, Pr = 0, cold_bgk_T = 0;
  kin::View<S, M> view{};
  kin::View<S, P> pview{};  // mixed mode: the FP32 view of the gradient and the LU-SGS passes
  int32_t chunk = 0, partial_stride = 1, max_levels = 0, n_chains = 0, max_entries = 0;
  int32_t wstride = 0;  // row length of the chunk work arrays: the chunk rounded up to whole 64-byte windows
  // kernel shapes of the two arithmetic types (read when the handle is created)
  kin::KernelShape shape_m = kin::read_shape<M>(), shape_p = kin::read_shape<P>();

  // host copies
  std::vector<int32_t> perm, inv;
  struct GroupRange {
    int32_t g, begin, end;  // velocities [begin, end) of the handle's order belong to sweep direction g
  };
  std::vector<GroupRange> group_ranges;
  int32_t orbit_size = 1;
  std::vector<int32_t> h_block_offsets;
  // per chunk: sweep items
  struct ChunkPlan {
    int32_t k0, kc;
    DevBuf<int4> items;
    int32_t n_items;
    DevBuf<int4> ritems;  // resident block pass: (chain, window start, first valid, end valid)
    int32_t n_ritems;
  };
  std::vector<std::unique_ptr<ChunkPlan>> chunks;

  // device arrays
  DevBuf<M> xi_x, xi_y, xi_z;
  // full velocity grid of the discrete equilibrium when this handle stores one shard (else unused)
  DevBuf<M> dq_x, dq_y, dq_z;
  DevBuf<double> dq_xd, dq_yd, dq_zd, dq_w;
  int32_t dq_nv = 0;
  // the equilibrium's velocity grid factored per axis (kin::DeqTensor; tn_n[0] == 0: not a tensor grid)
  DevBuf<double> tn_nodes, tn_w;
  int32_t tn_n[3] = {0, 0, 0};
  DevBuf<double> xid_x, xid_y, xid_z, wts;
  DevBuf<int32_t> csr_off;
  DevBuf<CsrE<M>> csr;
  DevBuf<M> eps2;
  DevBuf<BFace<M>> bfaces;
  DevBuf<Inflow<M>> inflow;
  DevBuf<CellParams<M>> cells;
  DevBuf<int32_t> mirror_map;
  DevBuf<int64_t> mw_offset;
  DevBuf<double> mw_frac;
  DevBuf<M> specular, specular_first;
  DevBuf<int32_t> grid_to_pos;
  DevBuf<double> volume, vdt;
  DevBuf<int32_t> block_offsets, chain_start, lev_bounds, lev_start, lev_count;
  DevBuf<int4> prog;
  DevBuf<kin::SweepE<P>> sweep_entries;
  // staged schedule of k_sweep_staged (staged_ne == 0: not usable for this mesh, k_sweep_pass runs instead)
  int32_t staged_ne = 0;
  DevBuf<int4> sprog;
  DevBuf<kin::StageE<P>> sse;
  // mixed mode: FP32 copies of the tables the FP32 kernels read
  DevBuf<P> pxi_x, pxi_y, pxi_z, peps2, pspecular, pspecular_first;
  DevBuf<CsrE<P>> pcsr;
  DevBuf<BFace<P>> pbfaces;
  DevBuf<Inflow<P>> pinflow;
  DevBuf<CellParams<P>> pcells;
  DevBuf<int32_t> sub_cells, sub_entries, sub_start, sub_count;
  // resident block pass (k_sweep_resident): cell of every staged slot with its surface bit, the cells that have
  // out-of-block neighbours with those entries (k_lout), the kernel's shared memory and the device status word
  enum SweepMode { kSweepResident, kSweepTiles, kSweepLegacy };
  SweepMode sweep_mode = kSweepTiles;
  int32_t resident_smem = 0, max_block_cells = 0, n_surf = 0;
  std::vector<uint8_t> h_surface;
  DevBuf<uint32_t> scells;
  DevBuf<int4> surf;
  DevBuf<kin::StageE<P>> sent;
  DevBuf<int32_t> err_word;
  DevBuf<int32_t> d_perm, d_inv;
  DevBuf<double> moments, shift, residual_cell, bsums, partial, w_half, w_new, staging;
  DevBuf<int32_t> flags, face_cells, face_entries;
  DevBuf<double> face_out;
  DevBuf<double> corr_ext;  // per-cell extrema of a velocity-sharded GSIS correction
  DevBuf<S> f, gx, gy, gz, r;

  // discrete adjoint: lambda in velocity-reversed storage, seeds of the transposed gradient
  bool adj_on = false;
  DevBuf<S> adj_lam, adj_lfb, adj_hmax, adj_hmin;  // of the storage type (FP32 in mixed precision)
  DevBuf<double> adj_mu, adj_coef, adj_cell, adj_face, adj_res;
  DevBuf<double> adj_mom;  // per boundary face (5): seeds of the face moment sums (limited pressure reconstruction)
  bool adj_mom_on = false;
  DevBuf<int8_t> adj_imax, adj_imin;
  DevBuf<int32_t> adj_rev, adj_rev_entry, adj_perm2, adj_inv2, adj_flip, adj_face_axis;
  DevBuf<int32_t> adj_face_cells;  // owners of wall and pressure faces (the transport the per-face sums need)
  int n_adj_face_cells = 0;

  bool inflow_set = false;
  bool deq_valid = false;
  // mixed precision: the defect of the FP32 residual against the FP64 one, [cell][nv] in FP32, taken at the first
  // sweep after the cell parameters or f changed (defect_valid false); the inner sweeps after it run the FP32
  // residual plus this defect, so the iteration's fixed point is the FP64 residual's zero
  DevBuf<S> defect;
  bool defect_valid = false;
  // KIN_MIXED_RESIDUAL=defect selects the defect scheme; by default every sweep evaluates the FP64 residual (faster
  // on B200: the FP32 residual is latency-bound like the FP64 one and the defect adds a read per sweep)
  bool defect_scheme = std::getenv("KIN_MIXED_RESIDUAL") != nullptr &&
                       std::strcmp(std::getenv("KIN_MIXED_RESIDUAL"), "defect") == 0;
  PhaseTimer timer;
  KinStepTimings timings{};

  const kin::View<S, P>& sweep_view() const {
    if constexpr (kSplit) return pview;
    else return view;
  }

  const char* name() const override { return "b200"; }
  int32_t chunk_width() const override { return chunk; }

  explicit Backend(const KinSetupDesc& d) {
    device = d.device;
    KCUDA(cudaSetDevice(device));
    // the static scratch of kin_discrete_maxwell_noalloc becomes resident when its address is first taken (lazy
    // module loading): take it now, before f and the velocity chunk are sized to the free memory, so that later
    // calls of the allocation-free entry point reserve nothing
    noalloc_scratch(device);
    nc = d.n_cells;
    nv = d.nv;
    nb = d.n_bfaces;
    n_blocks = d.n_blocks;
    precision = d.precision;
    KCHECK(nc > 0 && nv > 0 && nb >= 0 && n_blocks >= 1, "invalid sizes in KinSetupDesc");
    KCHECK(d.xi_x && d.xi_y && d.xi_z && d.csr_offsets && d.csr_other && d.csr_bface && d.csr_geom && d.eps2 &&
               d.volume && d.vdt && d.block_offsets,
           "missing array in KinSetupDesc");
    KCHECK(nb == 0 || (d.bface_owner && d.bface_kind && d.bface_mirror_xor && d.bface_geom),
           "missing boundary-face array in KinSetupDesc");
    KCHECK(d.block_offsets[0] == 0 && d.block_offsets[n_blocks] == nc, "block_offsets do not cover the cells");
    block_passes = std::max(1, d.block_passes);
    discrete_eq = d.discrete_eq;
    collisionless = d.deq_fallback_collisionless;
    negative_mode = d.negative_check_mode;
    mu0 = d.mu0;
    omega = d.omega;
    Pr = d.Pr;
    cold_bgk_T = d.cold_bgk_temperature;
    n_maxwell = d.n_maxwell_faces;

    // free device memory check for f (kinetic_backend_cuda.cpp:102-106)
    size_t free_b = 0, total_b = 0;
    KCUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t f_bytes = (kSplit && defect_scheme ? 2 : 1) * sizeof(S) * static_cast<size_t>(nc) * static_cast<size_t>(nv);
    if (f_bytes + kMargin >= free_b)
      throw KinError(KIN_E_MEMORY, "distribution function of " + std::to_string(f_bytes / 1e9) +
                                       " GB does not fit in the free device memory of " +
                                       std::to_string(free_b / 1e9) + " GB");
    KCUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
    stream = own_stream;

    // velocity chunk: given (rounded up to whole mirror orbits, kinetic_backend_cuda.cpp:151-152) or from the
    // memory left after f (kinetic_backend_cuda.cpp:147-161). Mirror orbits never straddle a chunk, so a chunk
    // only reads f of its own velocities before updating them and the result does not depend on the chunking.
    int32_t xor_all = 0;
    for (int b = 0; b < nb; ++b) xor_all |= d.bface_mirror_xor[b];
    orbit_size = xor_all + 1;
    KCHECK((orbit_size & (orbit_size - 1)) == 0 && nv % orbit_size == 0, "mirror orbits do not tile the velocity grid");
    {
      const double per_velocity = static_cast<double>(nc) * (4.0 * sizeof(S) + 8.0 / (256.0 * 2));
      int64_t k;
      if (d.velocity_chunk > 0) {
        k = (d.velocity_chunk + orbit_size - 1) / orbit_size * orbit_size;
      } else {
        const double avail = static_cast<double>(free_b) - static_cast<double>(f_bytes) - 2.0 * kMargin;
        k = static_cast<int64_t>(avail / per_velocity);
        k = k / 256 * 256;
        if (k < 256 && k < nv) throw KinError(KIN_E_MEMORY, "not enough device memory for the velocity-chunk work arrays");
      }
      chunk = static_cast<int32_t>(std::min<int64_t>(k, nv));
    }

    build_velocity_layout(d);
    build_mesh(d);
    build_schedule(d);

    const size_t ncs = static_cast<size_t>(nc);
    moments.alloc(ncs * 15);
    shift.alloc(ncs * 3);
    KCUDA(cudaMemsetAsync(shift.p, 0, shift.bytes(), stream));
    residual_cell.alloc(ncs);
    bsums.alloc(static_cast<size_t>(std::max(nb, 1)) * 20);
    w_half.alloc(ncs * 5);
    w_new.alloc(ncs * 5);
    flags.alloc(ncs);
    inflow.alloc(static_cast<size_t>(std::max(nb, 1)));
    KCUDA(cudaMemsetAsync(inflow.p, 0, inflow.bytes(), stream));
    cells.alloc(ncs);
    KCUDA(cudaMemsetAsync(cells.p, 0, cells.bytes(), stream));
    if constexpr (kSplit) {
      pinflow.alloc(static_cast<size_t>(std::max(nb, 1)));
      KCUDA(cudaMemsetAsync(pinflow.p, 0, pinflow.bytes(), stream));
      pcells.alloc(ncs);
      KCUDA(cudaMemsetAsync(pcells.p, 0, pcells.bytes(), stream));
    }
    f.alloc(ncs * static_cast<size_t>(nv));
    KCUDA(cudaMemsetAsync(f.p, 0, f.bytes(), stream));
    if (kSplit && defect_scheme) defect.alloc(ncs * static_cast<size_t>(nv));

    constexpr int32_t kWindow = kin::SweepLaunch<S, P>::kWidth;
    wstride = (chunk + kWindow - 1) / kWindow * kWindow;
    const size_t work = ncs * static_cast<size_t>(wstride);
    err_word.alloc(1);
    KCUDA(cudaMemsetAsync(err_word.p, 0, err_word.bytes(), stream));
    gx.alloc(work);
    gy.alloc(work);
    gz.alloc(work);
    r.alloc(work);
    partial_stride = std::max(L::residual_tiles(chunk, shape_m.res_u), LP::residual_tiles(chunk, shape_p.res_u));
    partial.alloc(ncs * static_cast<size_t>(partial_stride));
    build_chunks();
    staging_alloc();
    update_view();
    KCUDA(cudaStreamSynchronize(stream));
  }

  ~Backend() override {
    if (stream) cudaStreamSynchronize(stream);
    if (own_stream) {
      cudaStreamSynchronize(own_stream);
      cudaStreamDestroy(own_stream);
    }
  }

  // ---- set-up ----------------------------------------------------------------------------------------------
  void build_velocity_layout(const KinSetupDesc& d) {
    // velocities grouped by LU-SGS sweep direction (stable: reference storage order inside a group)
    n_groups = d.n_sweep_dirs > 0 ? d.n_sweep_dirs : 1;
    std::vector<int32_t> grp(static_cast<size_t>(nv), 0);
    if (d.n_sweep_dirs > 0) {
      KCHECK(d.sweep_dir_of && d.sweep_order && d.sweep_pos, "sweep order arrays missing");
      for (int p = 0; p < nv; ++p) {
        grp[p] = d.sweep_dir_of[p];
        KCHECK(grp[p] < n_groups, "sweep_dir_of out of range");
      }
    }
    // order: velocity chunk of the reference storage position first, then sweep direction (stable)
    perm.resize(nv);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) {
      const int ca = a / chunk, cb = b / chunk;
      return ca != cb ? ca < cb : grp[a] < grp[b];
    });
    inv.assign(nv, -1);
    for (int q = 0; q < nv; ++q) inv[perm[q]] = q;
    // contiguous (chunk, group) ranges
    group_ranges.clear();
    for (int q = 0; q < nv;) {
      const int g = grp[perm[q]], ck = perm[q] / chunk;
      int e = q;
      while (e < nv && grp[perm[e]] == g && perm[e] / chunk == ck) ++e;
      group_ranges.push_back({g, q, e});
      q = e;
    }
    std::vector<M> hx(nv), hy(nv), hz(nv);
    std::vector<double> dx(nv), dy(nv), dz(nv), hw;
    for (int q = 0; q < nv; ++q) {
      const int p = perm[q];
      dx[q] = d.xi_x[p];
      dy[q] = d.xi_y[p];
      dz[q] = d.xi_z[p];
      hx[q] = static_cast<M>(dx[q]);
      hy[q] = static_cast<M>(dy[q]);
      hz[q] = static_cast<M>(dz[q]);
    }
    xi_x.upload(hx.data(), nv, stream);
    xi_y.upload(hy.data(), nv, stream);
    xi_z.upload(hz.data(), nv, stream);
    if constexpr (kSplit) {
      std::vector<P> px(dx.begin(), dx.end()), py(dy.begin(), dy.end()), pz(dz.begin(), dz.end());
      pxi_x.upload(px.data(), nv, stream);
      pxi_y.upload(py.data(), nv, stream);
      pxi_z.upload(pz.data(), nv, stream);
      KCUDA(cudaStreamSynchronize(stream));
    }
    xid_x.upload(dx.data(), nv, stream);
    xid_y.upload(dy.data(), nv, stream);
    xid_z.upload(dz.data(), nv, stream);
    if (d.weights) {
      hw.resize(nv);
      for (int q = 0; q < nv; ++q) hw[q] = d.weights[perm[q]];
      wts.upload(hw.data(), nv, stream);
    }
    dq_nv = 0;
    if (d.deq_nv > 0) {
      KCHECK(d.deq_xi_x && d.deq_xi_y && d.deq_xi_z, "deq_nv > 0 needs deq_xi_x / y / z");
      dq_nv = d.deq_nv;
      const size_t m = static_cast<size_t>(dq_nv);
      std::vector<M> tx(d.deq_xi_x, d.deq_xi_x + m), ty(d.deq_xi_y, d.deq_xi_y + m), tz(d.deq_xi_z, d.deq_xi_z + m);
      dq_x.upload(tx.data(), m, stream);
      dq_y.upload(ty.data(), m, stream);
      dq_z.upload(tz.data(), m, stream);
      dq_xd.upload(d.deq_xi_x, m, stream);
      dq_yd.upload(d.deq_xi_y, m, stream);
      dq_zd.upload(d.deq_xi_z, m, stream);
      if (d.deq_weights) dq_w.upload(d.deq_weights, m, stream);
      KCUDA(cudaStreamSynchronize(stream));
    }
    // KIN_VELOCITY_SUMS=pointwise keeps the per-velocity Newton sums of the discrete equilibrium on a tensor grid too
    // (both give the same results to rounding; the tests use this to cover both paths)
    const char* sums_env = std::getenv("KIN_VELOCITY_SUMS");
    const bool pointwise = sums_env != nullptr && std::strcmp(sums_env, "pointwise") == 0;
    if (!pointwise) {
      const bool shard = dq_nv > 0;
      std::vector<double> nodes, wax;
      int32_t n[3];
      const bool tensor =
          shard ? factor_tensor_grid(d.deq_xi_x, d.deq_xi_y, d.deq_xi_z, d.deq_weights, dq_nv, nodes, wax, n)
                : factor_tensor_grid(dx.data(), dy.data(), dz.data(), d.weights ? hw.data() : nullptr, nv, nodes, wax,
                                     n);
      for (int a = 0; a < 3; ++a) tn_n[a] = tensor ? n[a] : 0;
      if (tensor) {
        tn_nodes.upload(nodes.data(), nodes.size(), stream);
        tn_w.upload(wax.data(), wax.size(), stream);
        KCUDA(cudaStreamSynchronize(stream));
      }
    }
    d_perm.upload(perm.data(), nv, stream);
    d_inv.upload(inv.data(), nv, stream);
    KCUDA(cudaStreamSynchronize(stream));
  }

  void build_mesh(const KinSetupDesc& d) {
    const int64_t n_csr = d.csr_offsets[nc];
    csr_off.upload(d.csr_offsets, static_cast<size_t>(nc) + 1, stream);
    for (int c = 0; c < nc; ++c) max_entries = std::max(max_entries, d.csr_offsets[c + 1] - d.csr_offsets[c]);
    std::vector<CsrE<M>> hc(static_cast<size_t>(n_csr));
    for (int64_t k = 0; k < n_csr; ++k) {
      CsrE<M>& e = hc[k];
      e.other = d.csr_other[k];
      e.bface = d.csr_bface[k];
      KCHECK(e.other < nc && e.bface < nb && (e.other >= 0) != (e.bface >= 0), "invalid CSR entry");
      const double* g = d.csr_geom + 12 * k;
      for (int a = 0; a < 3; ++a) {
        e.s[a] = static_cast<M>(g[a]);
        e.ds[a] = static_cast<M>(g[3 + a]);
        e.dn[a] = static_cast<M>(g[6 + a]);
        e.c[a] = static_cast<M>(g[9 + a]);
      }
    }
    csr.upload(hc.data(), hc.size(), stream);
    std::vector<M> he(nc);
    for (int c = 0; c < nc; ++c) he[c] = static_cast<M>(d.eps2[c]);
    eps2.upload(he.data(), nc, stream);
    if constexpr (kSplit) {
      std::vector<CsrE<P>> pc(hc.size());
      for (size_t k = 0; k < hc.size(); ++k) {
        pc[k].other = hc[k].other;
        pc[k].bface = hc[k].bface;
        const double* g = d.csr_geom + 12 * k;
        for (int a = 0; a < 3; ++a) {
          pc[k].s[a] = static_cast<P>(g[a]);
          pc[k].ds[a] = static_cast<P>(g[3 + a]);
          pc[k].dn[a] = static_cast<P>(g[6 + a]);
          pc[k].c[a] = static_cast<P>(g[9 + a]);
        }
      }
      pcsr.upload(pc.data(), pc.size(), stream);
      std::vector<P> pe(nc);
      for (int c = 0; c < nc; ++c) pe[c] = static_cast<P>(d.eps2[c]);
      peps2.upload(pe.data(), nc, stream);
      KCUDA(cudaStreamSynchronize(stream));
    }
    volume.upload(d.volume, nc, stream);
    vdt.upload(d.vdt, nc, stream);
    h_block_offsets.assign(d.block_offsets, d.block_offsets + n_blocks + 1);
    block_offsets.upload(h_block_offsets.data(), h_block_offsets.size(), stream);

    // mirror maps: one per distinct mirror xor of symmetry / Maxwell faces
    std::vector<int32_t> xors;
    std::vector<BFace<M>> hb(static_cast<size_t>(std::max(nb, 1)));
    for (int b = 0; b < nb; ++b) {
      BFace<M>& o = hb[b];
      o.owner = d.bface_owner[b];
      o.kind = d.bface_kind[b];
      o.patch = d.bface_patch ? d.bface_patch[b] : 0;
      KCHECK(o.owner >= 0 && o.owner < nc, "invalid boundary face owner");
      const int x = d.bface_mirror_xor[b];
      o.mirror = -1;
      if (x != 0) {
        auto it = std::find(xors.begin(), xors.end(), x);
        if (it == xors.end()) {
          xors.push_back(x);
          it = xors.end() - 1;
        }
        o.mirror = static_cast<int32_t>(it - xors.begin());
      }
      KCHECK(o.kind != kin::kSymmetry || o.mirror >= 0, "symmetry face without a mirror map");
      const double* g = d.bface_geom + 7 * b;
      for (int a = 0; a < 3; ++a) {
        o.n[a] = static_cast<M>(g[a]);
        o.d[a] = static_cast<M>(g[4 + a]);
      }
      o.area = static_cast<M>(g[3]);
    }
    bfaces.upload(hb.data(), hb.size(), stream);
    if constexpr (kSplit) {
      std::vector<BFace<P>> pb(hb.size());
      for (size_t b = 0; b < hb.size(); ++b) {
        pb[b].owner = hb[b].owner;
        pb[b].kind = hb[b].kind;
        pb[b].mirror = hb[b].mirror;
        pb[b].patch = hb[b].patch;
        const double* g = b < static_cast<size_t>(nb) ? d.bface_geom + 7 * b : nullptr;
        for (int a = 0; a < 3; ++a) {
          pb[b].n[a] = g ? static_cast<P>(g[a]) : P(0);
          pb[b].d[a] = g ? static_cast<P>(g[4 + a]) : P(0);
        }
        pb[b].area = g ? static_cast<P>(g[3]) : P(0);
      }
      pbfaces.upload(pb.data(), pb.size(), stream);
      KCUDA(cudaStreamSynchronize(stream));
    }
    std::vector<int32_t> mm(std::max<size_t>(xors.size(), 1) * nv, 0);
    for (size_t s = 0; s < xors.size(); ++s) {
      for (int q = 0; q < nv; ++q) {
        const int pm = perm[q] ^ xors[s];
        KCHECK(pm >= 0 && pm < nv, "mirror xor out of range");
        mm[s * nv + q] = inv[pm];
      }
    }
    mirror_map.upload(mm.data(), mm.size(), stream);

    if (n_maxwell > 0) {
      KCHECK(d.maxwell_offset && d.maxwell_specular_fraction && d.grid_to_storage, "Maxwell-wall arrays missing");
      mw_offset.upload(d.maxwell_offset, nb, stream);
      mw_frac.upload(d.maxwell_specular_fraction, nb, stream);
      specular.alloc(static_cast<size_t>(n_maxwell) * nv);
      specular_first.alloc(static_cast<size_t>(n_maxwell) * nv);
      KCUDA(cudaMemsetAsync(specular.p, 0, specular.bytes(), stream));
      KCUDA(cudaMemsetAsync(specular_first.p, 0, specular_first.bytes(), stream));
      if constexpr (kSplit) {
        pspecular.alloc(static_cast<size_t>(n_maxwell) * nv);
        pspecular_first.alloc(static_cast<size_t>(n_maxwell) * nv);
        KCUDA(cudaMemsetAsync(pspecular.p, 0, pspecular.bytes(), stream));
        KCUDA(cudaMemsetAsync(pspecular_first.p, 0, pspecular_first.bytes(), stream));
      }
      std::vector<int32_t> g2p(nv);
      for (int k = 0; k < nv; ++k) g2p[k] = inv[d.grid_to_storage[k]];
      grid_to_pos.upload(g2p.data(), nv, stream);
    }
    KCUDA(cudaStreamSynchronize(stream));
  }

  // level schedule of every (direction group, block) chain: level(c) = 1 + max level of the in-block neighbours
  // that precede c in the group's sweep order (sweep_order / sweep_pos, kinetic_setup.cpp:474-506)
  void build_schedule(const KinSetupDesc& d) {
    const size_t ncs = static_cast<size_t>(nc);
    std::vector<int32_t> hpos(static_cast<size_t>(n_groups) * ncs);
    for (int g = 0; g < n_groups; ++g) {
      for (int c = 0; c < nc; ++c) hpos[g * ncs + c] = d.n_sweep_dirs > 0 ? d.sweep_pos[g * ncs + c] : c;
    }
    n_chains = n_groups * n_blocks;
    std::vector<int32_t> hcells(static_cast<size_t>(n_groups) * ncs), hstart(n_chains), hlev_start(n_chains),
        hlev_count(n_chains);
    std::vector<int32_t> hbounds;
    std::vector<int32_t> level(ncs, 0);
    max_levels = 0;
    for (int g = 0; g < n_groups; ++g) {
      const int32_t* order = d.n_sweep_dirs > 0 ? d.sweep_order + g * ncs : nullptr;
      const int32_t* pg = hpos.data() + g * ncs;
      for (int b = 0; b < n_blocks; ++b) {
        const int cb = h_block_offsets[b], ce = h_block_offsets[b + 1];
        int nlev = 0;
        for (int k = cb; k < ce; ++k) {
          const int c = order ? order[k] : k;
          KCHECK(c >= cb && c < ce && pg[c] == k, "sweep_order / sweep_pos inconsistent with the blocks");
          int lv = 0;
          for (int e = d.csr_offsets[c]; e < d.csr_offsets[c + 1]; ++e) {
            const int o = d.csr_other[e];
            if (o >= cb && o < ce && pg[o] < pg[c]) lv = std::max(lv, level[o] + 1);
          }
          level[c] = lv;
          nlev = std::max(nlev, lv + 1);
        }
        // bucket the block's cells by level (stable in sweep order)
        const int chain = g * n_blocks + b;
        hstart[chain] = static_cast<int32_t>(static_cast<size_t>(g) * ncs + cb);
        hlev_start[chain] = static_cast<int32_t>(hbounds.size());
        hlev_count[chain] = nlev;
        std::vector<int32_t> count(nlev + 1, 0);
        for (int k = cb; k < ce; ++k) ++count[level[order ? order[k] : k] + 1];
        for (int l = 0; l < nlev; ++l) count[l + 1] += count[l];
        for (int l = 0; l <= nlev; ++l) hbounds.push_back(count[l]);
        std::vector<int32_t> fill(count.begin(), count.end() - 1);
        for (int k = cb; k < ce; ++k) {
          const int c = order ? order[k] : k;
          hcells[static_cast<size_t>(g) * ncs + cb + fill[level[c]]++] = c;
        }
        max_levels = std::max(max_levels, nlev);
      }
    }
    // per-chain program: (cell, first CSR entry, number of entries, bitmask of the in-block neighbours that precede
    // the cell in the group's sweep order); the stencil entries keep only what the sweep reads
    std::vector<int4> hprog(hcells.size());
    for (int g = 0; g < n_groups; ++g) {
      const int32_t* pg = hpos.data() + g * ncs;
      for (int b = 0; b < n_blocks; ++b) {
        const int cb = h_block_offsets[b], ce = h_block_offsets[b + 1];
        for (int k = cb; k < ce; ++k) {
          const size_t i = static_cast<size_t>(g) * ncs + k;
          const int c = hcells[i];
          const int e0 = d.csr_offsets[c], ne = d.csr_offsets[c + 1] - e0;
          KCHECK(ne <= 32, "a cell with more than 32 faces is not supported by the LU-SGS sweep kernel");
          uint32_t mask = 0;
          for (int j = 0; j < ne; ++j) {
            const int o = d.csr_other[e0 + j];
            if (o >= cb && o < ce && pg[o] < pg[c]) mask |= 1u << j;
          }
          hprog[i] = make_int4(c, e0, ne, static_cast<int>(mask));
        }
      }
    }
    const int64_t n_csr = d.csr_offsets[nc];
    std::vector<kin::SweepE<P>> hse(static_cast<size_t>(std::max<int64_t>(n_csr, 1)));
    for (int64_t e = 0; e < n_csr; ++e) {
      const int o = d.csr_other[e];
      hse[e].other = o >= 0 ? o : (d.bface_kind[d.csr_bface[e]] == kin::kPeriodic ? -2 : -1);
      for (int a = 0; a < 3; ++a) hse[e].s[a] = static_cast<P>(d.csr_geom[12 * e + a]);
    }
    // cells with a neighbour in another block ("surface" cells) and those entries in CSR order: the later block
    // passes couple them to the previous pass (k_lout)
    h_surface.assign(ncs, 0);
    {
      std::vector<int4> hsurf;
      std::vector<kin::StageE<P>> hsent;
      for (int b = 0; b < n_blocks; ++b) {
        const int cb = h_block_offsets[b], ce = h_block_offsets[b + 1];
        max_block_cells = std::max(max_block_cells, ce - cb);
        for (int c = cb; c < ce; ++c) {
          const int first = static_cast<int>(hsent.size());
          for (int e = d.csr_offsets[c]; e < d.csr_offsets[c + 1]; ++e) {
            const int o = d.csr_other[e];
            if (o < 0 || (o >= cb && o < ce)) continue;
            kin::StageE<P> st{};
            st.code = static_cast<uint32_t>(o);
            for (int a3 = 0; a3 < 3; ++a3) st.s[a3] = hse[e].s[a3];
            hsent.push_back(st);
          }
          const int cnt = static_cast<int>(hsent.size()) - first;
          if (cnt > 0) {
            h_surface[c] = 1;
            hsurf.push_back(make_int4(c, first, cnt, 0));
          }
        }
      }
      n_surf = static_cast<int32_t>(hsurf.size());
      if (n_surf > 0) {
        surf.upload(hsurf.data(), hsurf.size(), stream);
        sent.upload(hsent.data(), hsent.size(), stream);
        KCUDA(cudaStreamSynchronize(stream));
      }
    }
    build_staged_schedule(hprog, hse, hstart, hlev_start, hlev_count, hbounds);
    prog.upload(hprog.data(), hprog.size(), stream);
    sweep_entries.upload(hse.data(), hse.size(), stream);
    chain_start.upload(hstart.data(), hstart.size(), stream);
    lev_bounds.upload(hbounds.data(), hbounds.size(), stream);
    lev_start.upload(hlev_start.data(), hlev_start.size(), stream);
    lev_count.upload(hlev_count.data(), hlev_count.size(), stream);
    KCUDA(cudaStreamSynchronize(stream));
  }

  // Sub-levels of the staged sweep: each level of a chain cut (in its order) into pieces of at most kStageCells
  // cells and kStageEntries entries; the program refers to entries relative to its sub-level, and the entries are
  // stored again in program order so that a sub-level is one contiguous range of each.
  void build_staged_schedule(const std::vector<int4>& hprog, const std::vector<kin::SweepE<P>>& hse,
                             const std::vector<int32_t>& hstart, const std::vector<int32_t>& hlev_start,
                             const std::vector<int32_t>& hlev_count, const std::vector<int32_t>& hbounds) {
    // entry kinds of the staged stencil (k_sweep_tiles): code = kind << 28 | neighbour cell
    constexpr uint32_t kKindPeriodic = 0, kKindBoundary = 1, kKindLower = 2, kKindUpper = 3, kKindOther = 4;
    constexpr uint32_t kKindShift = 28;
    staged_ne = 0;
    sweep_mode = kSweepLegacy;
    if (nc >= (1 << kKindShift)) return;
    int max_ne = 0;
    for (const int4& p : hprog) max_ne = std::max(max_ne, p.z);
    const int ne_bound = max_ne <= 6 ? 6 : (max_ne <= 8 ? 8 : 0);
    if (ne_bound == 0) return;
    std::vector<int4> sp;
    std::vector<kin::StageE<P>> se;
    std::vector<int32_t> sc, sen, sst(n_chains), scnt(n_chains);
    sp.reserve(hprog.size());
    se.reserve(hprog.size() * static_cast<size_t>(max_ne));
    for (int ch = 0; ch < n_chains; ++ch) {
      sst[ch] = static_cast<int32_t>(sc.size());
      int nsub = 0;
      const int blk = ch % n_blocks;
      const int cb = h_block_offsets[blk], ce = h_block_offsets[blk + 1];
      for (int l = 0; l < hlev_count[ch]; ++l) {
        const size_t pb = static_cast<size_t>(hstart[ch]) + hbounds[hlev_start[ch] + l];
        const size_t pe = static_cast<size_t>(hstart[ch]) + hbounds[hlev_start[ch] + l + 1];
        size_t k = pb;
        while (k < pe) {
          sc.push_back(static_cast<int32_t>(sp.size()));
          sen.push_back(static_cast<int32_t>(se.size()));
          int ncell = 0, nent = 0;
          while (k < pe && ncell < kin::kStageCells && nent + hprog[k].z <= kin::kStageEntries) {
            const int4 p = hprog[k];
            sp.push_back(make_int4(p.x, nent, p.z, 0));
            for (int j = 0; j < p.z; ++j) {
              const kin::SweepE<P>& e = hse[static_cast<size_t>(p.y) + j];
              uint32_t kind;
              if (e.other == -2) kind = kKindPeriodic;
              else if (e.other < 0) kind = kKindBoundary;
              else if (e.other < cb || e.other >= ce) kind = kKindOther;
              else kind = ((p.w >> j) & 1) ? kKindLower : kKindUpper;
              kin::StageE<P> st{};
              st.code = (kind << kKindShift) | static_cast<uint32_t>(e.other >= 0 ? e.other : 0);
              for (int a3 = 0; a3 < 3; ++a3) st.s[a3] = e.s[a3];
              se.push_back(st);
            }
            nent += p.z;
            ++ncell;
            ++k;
          }
          ++nsub;
        }
      }
      sc.push_back(static_cast<int32_t>(sp.size()));
      sen.push_back(static_cast<int32_t>(se.size()));
      scnt[ch] = nsub;
      if (nsub > kin::kMaxSubLevels) return;  // too many sub-levels for the kernel's table: k_sweep_pass
    }
    if (sp.empty() || se.empty()) return;
    KCHECK(se.size() < static_cast<size_t>(INT32_MAX), "staged LU-SGS schedule too large");
    sprog.upload(sp.data(), sp.size(), stream);
    sse.upload(se.data(), se.size(), stream);
    {
      std::vector<uint32_t> sc_cells(sp.size());
      for (size_t k = 0; k < sp.size(); ++k)
        sc_cells[k] = static_cast<uint32_t>(sp[k].x) | (h_surface[static_cast<size_t>(sp[k].x)] ? 0x80000000u : 0u);
      scells.upload(sc_cells.data(), sc_cells.size(), stream);
      KCUDA(cudaStreamSynchronize(stream));
    }
    sub_cells.upload(sc.data(), sc.size(), stream);
    sub_entries.upload(sen.data(), sen.size(), stream);
    sub_start.upload(sst.data(), sst.size(), stream);
    sub_count.upload(scnt.data(), scnt.size(), stream);
    staged_ne = ne_bound;
    resident_smem = n_surf < (1 << 30) ? kin::SweepLaunch<S, P>::smem_bytes(max_block_cells) : 0;
    sweep_mode = kSweepTiles;
    // KIN_SWEEP_KERNEL selects another LU-SGS kernel: legacy (k_sweep_pass), tiles / staged8 (k_sweep_tiles with 6-
    // or 8-entry bounds), resident8 (k_sweep_resident with the 8-entry bound). All give the same results; the tests
    // use this to cover every sweep kernel on the available meshes.
    if (const char* e = std::getenv("KIN_SWEEP_KERNEL")) {
      if (std::strcmp(e, "legacy") == 0) {
        staged_ne = 0;
        sweep_mode = kSweepLegacy;
      }
      if (std::strcmp(e, "tiles") == 0) sweep_mode = kSweepTiles;
      if (std::strcmp(e, "staged8") == 0) {
        staged_ne = 8;
        sweep_mode = kSweepTiles;
      }
      if (std::strcmp(e, "resident") == 0 && resident_smem > 0) sweep_mode = kSweepResident;
      if (std::strcmp(e, "resident8") == 0 && resident_smem > 0) {
        sweep_mode = kSweepResident;
        staged_ne = 8;
      }

    }
  }

  void build_chunks() {
    chunks.clear();
    for (int k0 = 0; k0 < nv; k0 += chunk) {
      auto cp = std::make_unique<ChunkPlan>();
      cp->k0 = k0;
      cp->kc = std::min(chunk, nv - k0);
      std::vector<int4> items;
      for (const GroupRange& gr : group_ranges) {
        const int s = std::max(gr.begin, k0), e = std::min(gr.end, k0 + cp->kc);
        if (s >= e) continue;
        for (int b = 0; b < n_blocks; ++b) {
          if (h_block_offsets[b + 1] == h_block_offsets[b]) continue;
          const int tile = staged_ne != 0 ? 32 * shape_p.tile_u : kin::kSweepTile;
          for (int t = s; t < e; t += tile)
            items.push_back(make_int4(gr.g * n_blocks + b, t - k0, std::min(t + tile, e) - k0, 0));
        }
      }
      cp->n_items = static_cast<int32_t>(items.size());
      cp->items.upload(items.data(), items.size(), stream);
      // resident block pass: 64-byte windows aligned in the chunk's work-array rows, clipped to each direction
      // group; a window that straddles two groups becomes two items with disjoint valid ranges
      std::vector<int4> ritems;
      constexpr int kW = kin::SweepLaunch<S, P>::kWidth;
      for (const GroupRange& gr : group_ranges) {
        const int s = std::max(gr.begin, k0) - k0, e = std::min(gr.end, k0 + cp->kc) - k0;
        if (s >= e) continue;
        for (int b = 0; b < n_blocks; ++b) {
          if (h_block_offsets[b + 1] == h_block_offsets[b]) continue;
          for (int w = s / kW * kW; w < e; w += kW)
            ritems.push_back(make_int4(gr.g * n_blocks + b, w, std::max(s, w), std::min(e, w + kW)));
        }
      }
      cp->n_ritems = static_cast<int32_t>(ritems.size());
      if (!ritems.empty()) cp->ritems.upload(ritems.data(), ritems.size(), stream);
      chunks.push_back(std::move(cp));
    }
    KCUDA(cudaStreamSynchronize(stream));
  }

  // staging buffer for set/get_distribution (bounded: at most 256 MB of doubles)
  int32_t staging_cells = 1;
  void staging_alloc() {
    staging_cells = static_cast<int32_t>(std::max<int64_t>(1, std::min<int64_t>(nc, (int64_t{32} << 20) / nv)));
    staging.alloc(static_cast<size_t>(staging_cells) * nv);
  }

  void update_view() {
    kin::View<S, M>& v = view;
    v.n_cells = nc;
    v.nv = nv;
    v.n_bfaces = nb;
    v.max_entries = max_entries;
    v.xi_x = xi_x.p;
    v.xi_y = xi_y.p;
    v.xi_z = xi_z.p;
    v.xid_x = xid_x.p;
    v.xid_y = xid_y.p;
    v.xid_z = xid_z.p;
    v.wts = wts.p;
    v.csr_off = csr_off.p;
    v.csr = csr.p;
    v.eps2 = eps2.p;
    v.bf = bfaces.p;
    v.inflow = inflow.p;
    v.cp = cells.p;
    v.f = f.p;
    v.mirror_map = mirror_map.p;
    v.mw_offset = mw_offset.p;
    v.mw_frac = mw_frac.p;
    v.specular = specular.p;
    v.specular_first = specular_first.p;
    v.grid_to_pos = grid_to_pos.p;
    const bool shard = dq_nv > 0;
    v.dq_x = shard ? dq_x.p : xi_x.p;
    v.dq_y = shard ? dq_y.p : xi_y.p;
    v.dq_z = shard ? dq_z.p : xi_z.p;
    v.dq_xd = shard ? dq_xd.p : xid_x.p;
    v.dq_yd = shard ? dq_yd.p : xid_y.p;
    v.dq_zd = shard ? dq_zd.p : xid_z.p;
    v.dq_w = shard ? dq_w.p : wts.p;
    v.dq_nv = shard ? dq_nv : nv;
    for (int a = 0; a < 3; ++a) v.dq_tensor.n[a] = tn_n[a];
    v.dq_tensor.node = tn_nodes.p;
    v.dq_tensor.w = tn_w.p;
    if constexpr (kSplit) {
      kin::View<S, P>& w = pview;
      w.n_cells = nc;
      w.nv = nv;
      w.n_bfaces = nb;
      w.max_entries = max_entries;
      w.xi_x = pxi_x.p;
      w.xi_y = pxi_y.p;
      w.xi_z = pxi_z.p;
      w.xid_x = xid_x.p;
      w.xid_y = xid_y.p;
      w.xid_z = xid_z.p;
      w.wts = wts.p;
      w.csr_off = csr_off.p;
      w.csr = pcsr.p;
      w.eps2 = peps2.p;
      w.bf = pbfaces.p;
      w.inflow = pinflow.p;
      w.cp = pcells.p;
      w.f = f.p;
      w.mirror_map = mirror_map.p;
      w.mw_offset = mw_offset.p;
      w.mw_frac = mw_frac.p;
      w.specular = pspecular.p;
      w.specular_first = pspecular_first.p;
      w.grid_to_pos = grid_to_pos.p;
      // the FP32 kernels never solve the discrete equilibrium: only the FP64 grid is shared
      w.dq_xd = v.dq_xd;
      w.dq_yd = v.dq_yd;
      w.dq_zd = v.dq_zd;
      w.dq_w = v.dq_w;
      w.dq_nv = v.dq_nv;
      w.dq_tensor = v.dq_tensor;
    }
  }

  void set_params(const KinSetupDesc& d) {
    view.weight = d.weight;
    view.limiter_mode = d.limiter_mode;
    view.positivity = d.positivity;
    view.diag_scale = static_cast<M>(d.diag_scale);
    view.interface_damping = static_cast<M>(d.interface_damping);
    for (int a = 0; a < 3; ++a) {
      view.grid_n[a] = d.grid_n[a];
      view.deq.lo[a] = d.deq_lo[a];
      view.deq.hi[a] = d.deq_hi[a];
      view.deq.d[a] = d.deq_d[a];
    }
    view.deq.criterion = d.deq_criterion;
    view.deq.tolerance = d.deq_tolerance;
    view.deq.max_iterations = d.deq_max_iterations;
    if constexpr (kSplit) {
      pview.weight = view.weight;
      pview.limiter_mode = view.limiter_mode;
      pview.positivity = view.positivity;
      pview.diag_scale = static_cast<P>(d.diag_scale);
      pview.interface_damping = static_cast<P>(d.interface_damping);
      for (int a = 0; a < 3; ++a) pview.grid_n[a] = view.grid_n[a];
      pview.deq = view.deq;
    }
  }

  void launched(int n = 1) {
    launches += n;
    KCUDA(cudaGetLastError());
  }

  uint64_t memory_bytes() const override {
    return xi_x.bytes() * 3 + xid_x.bytes() * 3 + wts.bytes() + csr_off.bytes() + csr.bytes() + eps2.bytes() +
           bfaces.bytes() + inflow.bytes() + cells.bytes() + mirror_map.bytes() + mw_offset.bytes() + mw_frac.bytes() +
           specular.bytes() * 2 + grid_to_pos.bytes() + volume.bytes() + vdt.bytes() + block_offsets.bytes() +
           prog.bytes() + sweep_entries.bytes() + chain_start.bytes() + lev_bounds.bytes() + lev_start.bytes() +
           lev_count.bytes() + sprog.bytes() + sse.bytes() + sub_cells.bytes() + sub_entries.bytes() +
           sub_start.bytes() + sub_count.bytes() + d_perm.bytes() * 2 + moments.bytes() + shift.bytes() + residual_cell.bytes() + bsums.bytes() +
           partial.bytes() + w_half.bytes() * 2 + staging.bytes() + flags.bytes() + f.bytes() + gx.bytes() * 4 +
           pxi_x.bytes() * 3 + peps2.bytes() + pspecular.bytes() * 2 + pcsr.bytes() + pbfaces.bytes() +
           pinflow.bytes() + pcells.bytes();
  }

  // ---- KineticBackend methods ------------------------------------------------------------------------------
  void set_equilibrium(const double* states, int64_t n) override {
    KCHECK(n == 5LL * nc, "length of the initial states does not match the number of cells");
    DevBuf<double> d_states;
    d_states.upload(states, static_cast<size_t>(n), stream);
    timer.begin(PhaseTimer::kOther, stream);
    L::set_equilibrium(view, d_states.p, shift.p, discrete_eq, stream);
    launched();
    defect_valid = false;
    timer.end(stream);
    timer.flush(timings);
  }

  void set_distribution(const double* h, int64_t n) override {
    KCHECK(n == static_cast<int64_t>(nc) * nv, "length of the distribution function does not match");
    for (int64_t c0 = 0; c0 < nc; c0 += staging_cells) {
      const int cnt = static_cast<int>(std::min<int64_t>(staging_cells, nc - c0));
      KCUDA(cudaMemcpyAsync(staging.p, h + c0 * nv, sizeof(double) * cnt * nv, cudaMemcpyHostToDevice, stream));
      L::import_f(staging.p, f.p, d_perm.p, c0, cnt, nv, stream);
      launched();
    }
    defect_valid = false;
    KCUDA(cudaStreamSynchronize(stream));
  }

  void get_distribution(double* h, int64_t n) override {
    KCHECK(n == static_cast<int64_t>(nc) * nv, "length of the distribution function does not match");
    for (int64_t c0 = 0; c0 < nc; c0 += staging_cells) {
      const int cnt = static_cast<int>(std::min<int64_t>(staging_cells, nc - c0));
      L::export_f(f.p, staging.p, d_inv.p, c0, cnt, nv, stream);
      launched();
      KCUDA(cudaMemcpyAsync(h + c0 * nv, staging.p, sizeof(double) * cnt * nv, cudaMemcpyDeviceToHost, stream));
    }
    KCUDA(cudaStreamSynchronize(stream));
  }

  void compute_moments(double* out, int64_t n) override {
    KCHECK(n == 15LL * nc, "length of the moment output does not match");
    timer.begin(PhaseTimer::kMoments, stream);
    L::moments(view, shift.p, moments.p, stream);
    launched();
    timer.end(stream);
    KCUDA(cudaMemcpyAsync(out, moments.p, moments.bytes(), cudaMemcpyDeviceToHost, stream));
    timer.flush(timings);
    KCUDA(cudaStreamSynchronize(stream));
  }

  void moment_sums(double* out, int64_t n) override {
    KCHECK(out == nullptr || n == 13LL * nc, "length of the moment-sum output does not match");
    timer.begin(PhaseTimer::kMoments, stream);
    L::moment_sums(view, shift.p, staging_sums(), stream);
    launched();
    timer.end(stream);
    if (out != nullptr)  // NULL: the sums stay in the device buffer (KIN_SUMS_MOMENTS) for a device reduction
      KCUDA(cudaMemcpyAsync(out, sums.p, sizeof(double) * 13 * nc, cudaMemcpyDeviceToHost, stream));
    timer.flush(timings);
    KCUDA(cudaStreamSynchronize(stream));
  }

  // device buffer of one kind of velocity sum, for an in-place reduction across velocity shards
  void device_sums(int32_t which, double** ptr, int64_t* n) override {
    switch (which) {
      case KIN_SUMS_MOMENTS:
        *ptr = staging_sums();
        *n = 13LL * nc;
        break;
      case KIN_SUMS_BOUNDARY:
        *ptr = bsums.p;
        *n = 20LL * nb;
        break;
      case KIN_SUMS_RESIDUAL:
        *ptr = residual_cell.p;
        *n = nc;
        break;
      default:
        throw KinError(KIN_E_ARG, "kin_device_sums: unknown buffer " + std::to_string(which));
    }
  }

  // the moments from the (reduced) moment sums in device memory: finalised, installed, shift moved
  void finalize_moments(double* out, int64_t n) override {
    KCHECK(out == nullptr || n == 15LL * nc, "length of the moment output does not match");
    timer.begin(PhaseTimer::kMoments, stream);
    L::finalize_sums(staging_sums(), view.wts == nullptr ? view.weight : 1.0, shift.p, moments.p, nc, stream);
    launched();
    timer.end(stream);
    defect_valid = false;
    if (out != nullptr) KCUDA(cudaMemcpyAsync(out, moments.p, moments.bytes(), cudaMemcpyDeviceToHost, stream));
    timer.flush(timings);
    KCUDA(cudaStreamSynchronize(stream));
  }

  void read_sums(int32_t which, double* out, int64_t n) override {
    double* p = nullptr;
    int64_t m = 0;
    device_sums(which, &p, &m);
    KCHECK(n == m, "length of the sums output does not match");
    if (m > 0) KCUDA(cudaMemcpyAsync(out, p, sizeof(double) * m, cudaMemcpyDeviceToHost, stream));
    KCUDA(cudaStreamSynchronize(stream));
  }

  void set_moments(const double* m, int64_t n) override {
    KCHECK(n == 15LL * nc, "length of the moments does not match");
    KCUDA(cudaMemcpyAsync(moments.p, m, moments.bytes(), cudaMemcpyHostToDevice, stream));
    L::shift_from_moments(moments.p, shift.p, nc, stream);
    launched();
    defect_valid = false;
    KCUDA(cudaStreamSynchronize(stream));
  }

  DevBuf<double> sums;
  double* staging_sums() {
    if (sums.n != static_cast<size_t>(13) * nc) sums.alloc(static_cast<size_t>(13) * nc);
    return sums.p;
  }

  void scale_distribution(double s) override {
    timer.begin(PhaseTimer::kOther, stream);
    L::scale(f.p, static_cast<int64_t>(f.n), s, moments.p, nc, stream);
    launched(2);
    defect_valid = false;
    timer.end(stream);
    timer.flush(timings);
  }

  void update_cell_params() override {
    timer.begin(PhaseTimer::kOther, stream);
    L::cell_params(view, moments.p, volume.p, vdt.p, mu0, omega, Pr, cold_bgk_T, discrete_eq, collisionless, cells.p,
                   flags.p, stream);
    launched();
    if constexpr (kSplit) {
      L::cast_cell_params(cells.p, pcells.p, nc, stream);
      launched();
    }
    deq_valid = discrete_eq != 0;
    defect_valid = false;
    timer.end(stream);
    timer.flush(timings);
  }

  void deq_counts(KinDeqCounts* out) override {
    out->corrected = 0;
    out->failed = 0;
    out->max_iterations = 0;
    if (!deq_valid) return;
    std::vector<int32_t> h(nc);
    KCUDA(cudaMemcpyAsync(h.data(), flags.p, flags.bytes(), cudaMemcpyDeviceToHost, stream));
    KCUDA(cudaStreamSynchronize(stream));
    for (int x : h) {
      if (x > 0) ++out->corrected;
      if (x < 0) ++out->failed;
      out->max_iterations = std::max(out->max_iterations, x);
    }
  }

  void set_inflow(const KinInflowState* in, int64_t n) override {
    KCHECK(n == nb, "length of the inflow states does not match the number of boundary faces");
    inflow_set = true;
    if (nb == 0) return;
    std::vector<Inflow<M>> h(nb);
    for (int b = 0; b < nb; ++b) {
      h[b].m = kin::maxwell_from<M>(in[b].rho, in[b].ux, in[b].uy, in[b].uz, in[b].T);
      h[b].scale = static_cast<M>(in[b].scale);
    }
    KCUDA(cudaMemcpyAsync(inflow.p, h.data(), sizeof(Inflow<M>) * nb, cudaMemcpyHostToDevice, stream));
    if constexpr (kSplit) {
      std::vector<Inflow<P>> hp(nb);
      for (int b = 0; b < nb; ++b) {
        hp[b].m = kin::maxwell_from<P>(in[b].rho, in[b].ux, in[b].uy, in[b].uz, in[b].T);
        hp[b].scale = static_cast<P>(in[b].scale);
      }
      KCUDA(cudaMemcpyAsync(pinflow.p, hp.data(), sizeof(Inflow<P>) * nb, cudaMemcpyHostToDevice, stream));
      KCUDA(cudaStreamSynchronize(stream));
    }
    KCUDA(cudaStreamSynchronize(stream));
  }

  void boundary_sums(double* out, int64_t n) override {
    KCHECK(out == nullptr || n == 20LL * nb, "length of the boundary-sum output does not match");
    if (nb == 0) return;
    timer.begin(PhaseTimer::kBoundary, stream);
    if (n_maxwell > 0) {
      L::maxwell_reflection(view, stream);
      launched(2);
      if constexpr (kSplit) {
        LP::maxwell_reflection(pview, stream);
        launched(2);
      }
    }
    L::boundary_sums(view, bsums.p, stream);
    launched();
    timer.end(stream);
    if (out != nullptr)  // NULL: the sums stay in the device buffer (KIN_SUMS_BOUNDARY)
      KCUDA(cudaMemcpyAsync(out, bsums.p, sizeof(double) * 20 * nb, cudaMemcpyDeviceToHost, stream));
    timer.flush(timings);
    KCUDA(cudaStreamSynchronize(stream));
  }

  void internal_face_mass_flux(const int32_t* hc, const int32_t* he, int64_t n, double* out) override {
    if (n == 0) return;
    for (int64_t i = 0; i < n; ++i) {
      KCHECK(hc[i] >= 0 && hc[i] < nc && he[i] >= 0 && he[i] < static_cast<int64_t>(csr.n),
             "internal-face cell / entry index out of range");
    }
    face_cells.upload(hc, static_cast<size_t>(n), stream);
    face_entries.upload(he, static_cast<size_t>(n), stream);
    face_out.alloc(static_cast<size_t>(n));
    timer.begin(PhaseTimer::kOther, stream);
    L::internal_face_flux(view, face_cells.p, face_entries.p, face_out.p, static_cast<int>(n), stream);
    launched();
    timer.end(stream);
    KCUDA(cudaMemcpyAsync(out, face_out.p, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
    timer.flush(timings);
    KCUDA(cudaStreamSynchronize(stream));
  }

  // arguments of one LU-SGS block pass of a chunk (the schedule tables; R / dprev / out / update_f set by the caller)
  kin::SweepArgs<S, P> sweep_args(const ChunkPlan& cp, int32_t stride) const {
    kin::SweepArgs<S, P> a{};
    a.items = cp.items.p;
    a.n_items = cp.n_items;
    a.n_blocks = n_blocks;
    a.block_offsets = block_offsets.p;
    a.prog = prog.p;
    a.chain_start = chain_start.p;
    a.lev_bounds = lev_bounds.p;
    a.lev_start = lev_start.p;
    a.lev_count = lev_count.p;
    a.se = sweep_entries.p;
    a.staged_ne = sweep_mode == kSweepLegacy ? 0 : staged_ne;
    a.sprog = sprog.p;
    a.sse = sse.p;
    a.sub_cells = sub_cells.p;
    a.sub_entries = sub_entries.p;
    a.sub_start = sub_start.p;
    a.sub_count = sub_count.p;
    a.ritems = cp.ritems.p;
    a.n_ritems = cp.n_ritems;
    a.scells = scells.p;
    a.err = err_word.p;
    a.tile_u = shape_p.tile_u;
    a.tile_blocks = shape_p.tile_blocks;
    a.resident_smem = resident_smem;
    a.max_block_cells = max_block_cells;
    a.k0 = cp.k0;
    a.stride = stride;
    return a;
  }

  // block_passes x (forward + backward) on the residual in r for one chunk, correcting sv.f in the last pass.
  // Resident kernel: pass k > 1 first folds the out-of-block coupling to pass k - 1 into R (k_lout -> gx); the
  // kernels then read R, and Delta f goes to gz / gy alternately. Other kernels: pass k writes Delta f into gz / gy
  // and reads pass k - 1 from the other one.
  void run_block_passes(const kin::View<S, P>& sv, const ChunkPlan& cp, int32_t stride, bool timed) {
    const bool resident = sweep_mode == kSweepResident && stride % kin::SweepLaunch<S, P>::kWidth == 0;
    S* prev = nullptr;
    for (int pass = 0; pass < block_passes; ++pass) {
      const bool first = pass == 0, last = pass + 1 == block_passes;
      S* out = (pass % 2 == 0) ? gz.p : gy.p;
      kin::SweepArgs<S, P> a = sweep_args(cp, stride);
      a.R = r.p;
      a.dprev = prev;
      a.out = out;
      a.diag_store = gx.p;  // free during the passes (the gradient is dead after the residual)
      a.update_f = last ? 1 : 0;
      if (resident) {
        a.Rs = gx.p;
        if (!first && n_surf > 0) {
          const kin::LoutArgs<S, P> la{surf.p, n_surf, sent.p, r.p, prev, gx.p, cp.k0, cp.kc, stride};
          if (timed) timer.begin(PhaseTimer::kBackward, stream);
          kin::SweepLaunch<S, P>::lout(sv, la, stream);
          launched();
          if (timed) timer.end(stream);
        }
        if (timed) timer.begin(PhaseTimer::kForward, stream);
        kin::SweepLaunch<S, P>::resident(sv, a, first, last, stream);
      } else {
        if (timed) timer.begin(PhaseTimer::kForward, stream);
        LP::sweep_pass(sv, a, stream);
      }
      launched();
      if (timed) timer.end(stream);
      prev = out;
    }
  }

  // the device status word: nonzero when a bounded wait of a kernel gave up (read after the stream is synchronised)
  void check_status(const int32_t& h_err) {
    if (h_err != 0) {
      KCUDA(cudaMemsetAsync(err_word.p, 0, err_word.bytes(), stream));
      KCUDA(cudaStreamSynchronize(stream));
      throw KinError(KIN_E_TIMEOUT, "an LU-SGS block pass gave up waiting for its staged data (status " +
                                        std::to_string(h_err) + "); the results of this sweep are not valid");
    }
  }

  // gradient, residual and block_passes x (forward + backward) per velocity chunk
  // (CudaBackend::sweep, kinetic_backend_cuda.cpp:317-372)
  void sweep(double* residual_out, int64_t n) override {
    KCHECK(residual_out == nullptr || n == nc, "length of the residual output does not match the number of cells");
    KCUDA(cudaMemsetAsync(residual_cell.p, 0, residual_cell.bytes(), stream));
    for (const auto& cp : chunks) {
      kin::Chunk<S> ch{cp->k0, cp->kc, wstride, gx.p, gy.p, gz.p, r.p};
      ch.shape = shape_p;
      timer.begin(PhaseTimer::kGradient, stream);
      LP::gradient(sweep_view(), ch, stream);
      launched();
      timer.end(stream);
      ch.shape = shape_m;
      timer.begin(PhaseTimer::kResidual, stream);
      if (kSplit && !defect_scheme) {
        L::residual(view, ch, partial.p, partial_stride, residual_cell.p, stream);
        launched(2);
      } else if constexpr (kSplit) {
        // mixed precision: FP64 residual and the FP32 one's defect at the iteration's first sweep, FP32 residual +
        // defect at the inner sweeps after it
        kin::Chunk<S> cd = ch;
        cd.shape = shape_p;
        cd.defect = defect.p;
        if (!defect_valid) {
          L::residual(view, ch, partial.p, partial_stride, residual_cell.p, stream);
          launched(2);
          cd.defect_mode = kin::kDefectStore;
          LP::residual(sweep_view(), cd, partial.p, partial_stride, residual_cell.p, stream);
          launched();
        } else {
          cd.defect_mode = kin::kDefectApply;
          LP::residual(sweep_view(), cd, partial.p, partial_stride, residual_cell.p, stream);
          launched(2);
        }
      } else {
        L::residual(view, ch, partial.p, partial_stride, residual_cell.p, stream);
        launched(2);
      }
      timer.end(stream);
      // gradients are dead after the residual
      run_block_passes(sweep_view(), *cp, wstride, true);
    }
    if constexpr (kSplit) defect_valid = true;
    int32_t h_err = 0;
    if (residual_out != nullptr)  // NULL: the per-cell sums stay in the device buffer (KIN_SUMS_RESIDUAL)
      KCUDA(cudaMemcpyAsync(residual_out, residual_cell.p, residual_cell.bytes(), cudaMemcpyDeviceToHost, stream));
    KCUDA(cudaMemcpyAsync(&h_err, err_word.p, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    timer.flush(timings);
    KCUDA(cudaStreamSynchronize(stream));
    check_status(h_err);
  }

  // the GSIS correction in one pass (phase 0), or one of the two phases of a velocity-sharded correction
  void gsis_correction_phase(const double* wh, const double* wn, int64_t n, int phase, const double* ext_in,
                             double* ext_out, int32_t* out_flags, int64_t* replaced) {
    KCHECK(n == 5LL * nc, "length of the GSIS macroscopic states does not match the number of cells");
    KCUDA(cudaMemcpyAsync(w_half.p, wh, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
    KCUDA(cudaMemcpyAsync(w_new.p, wn, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
    if (phase != 0) {
      if (corr_ext.n != static_cast<size_t>(nc)) corr_ext.alloc(static_cast<size_t>(nc));
      if (phase == 2)
        KCUDA(cudaMemcpyAsync(corr_ext.p, ext_in, sizeof(double) * nc, cudaMemcpyHostToDevice, stream));
    }
    timer.begin(PhaseTimer::kOther, stream);
    L::gsis_correction(view, w_half.p, w_new.p, flags.p, shift.p, negative_mode, discrete_eq, collisionless, phase,
                       phase != 0 ? corr_ext.p : nullptr, stream);
    launched();
    timer.end(stream);
    if (phase == 1) {
      KCUDA(cudaMemcpyAsync(ext_out, corr_ext.p, sizeof(double) * nc, cudaMemcpyDeviceToHost, stream));
      timer.flush(timings);
      KCUDA(cudaStreamSynchronize(stream));
      return;
    }
    std::vector<int32_t> h(nc);
    KCUDA(cudaMemcpyAsync(h.data(), flags.p, flags.bytes(), cudaMemcpyDeviceToHost, stream));
    timer.flush(timings);
    KCUDA(cudaStreamSynchronize(stream));
    int64_t cnt = 0;
    for (int x : h) cnt += x != 0 ? 1 : 0;
    if (out_flags) std::copy(h.begin(), h.end(), out_flags);
    *replaced = cnt;
    deq_valid = false;
    defect_valid = false;
  }

  void gsis_correction(const double* wh, const double* wn, int64_t n, int32_t* out_flags,
                       int64_t* replaced) override {
    gsis_correction_phase(wh, wn, n, 0, nullptr, nullptr, out_flags, replaced);
  }

  void gsis_correction_extrema(const double* wh, const double* wn, int64_t n, double* ext, int64_t n_ext) override {
    KCHECK(n_ext == nc, "length of the per-cell extrema does not match the number of cells");
    gsis_correction_phase(wh, wn, n, 1, nullptr, ext, nullptr, nullptr);
  }

  void gsis_correction_apply(const double* wh, const double* wn, int64_t n, const double* ext, int64_t n_ext,
                             int32_t* out_flags, int64_t* replaced) override {
    KCHECK(n_ext == nc, "length of the per-cell extrema does not match the number of cells");
    gsis_correction_phase(wh, wn, n, 2, ext, nullptr, out_flags, replaced);
  }

  void discrete_maxwell(const double* states, int64_t n, double tol, double* out, int32_t* result) override {
    if (n <= 0) return;
    DevBuf<double> d_states, d_out;
    DevBuf<int32_t> d_res;
    d_states.upload(states, static_cast<size_t>(5 * n), stream);
    d_out.alloc(static_cast<size_t>(5 * n));
    d_res.alloc(static_cast<size_t>(n));
    kin::DeqGrid g = view.deq;
    g.tolerance = tol;
    timer.begin(PhaseTimer::kOther, stream);
    L::discrete_maxwell_states(view, g, d_states.p, d_out.p, d_res.p, static_cast<int>(n), stream);
    launched();
    timer.end(stream);
    KCUDA(cudaMemcpyAsync(out, d_out.p, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, stream));
    KCUDA(cudaMemcpyAsync(result, d_res.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, stream));
    timer.flush(timings);
    KCUDA(cudaStreamSynchronize(stream));
  }

  // discrete_maxwell in the static scratch: no device or host allocation, no phase timer (its events may grow a
  // pool). Nothing in the scratch has to start at zero: the kernel writes all five values and the result of each
  // of the n states before they are copied back.
  void discrete_maxwell_noalloc(const double* states, int64_t n, double tol, double* out, int32_t* result) override {
    KCHECK(n >= 0, "kin_discrete_maxwell_noalloc: negative number of states");
    KCHECK(n <= KIN_NOALLOC_MAX_STATES, "kin_discrete_maxwell_noalloc: " + std::to_string(n) +
                                            " states exceed the static scratch of " +
                                            std::to_string(KIN_NOALLOC_MAX_STATES) + " states; split the batch");
    if (n == 0) return;
    KCHECK(states != nullptr && out != nullptr && result != nullptr, "kin_discrete_maxwell_noalloc: null pointer");
    unsigned char* base = noalloc_scratch(device);
    double* d_states = reinterpret_cast<double*>(base);
    double* d_out = reinterpret_cast<double*>(base + kNoAllocStatesBytes);
    int32_t* d_res = reinterpret_cast<int32_t*>(base + 2 * kNoAllocStatesBytes);
    KCUDA(cudaMemcpyAsync(d_states, states, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, stream));
    kin::DeqGrid g = view.deq;
    g.tolerance = tol;
    L::discrete_maxwell_states(view, g, d_states, d_out, d_res, static_cast<int>(n), stream);
    launched();
    KCUDA(cudaMemcpyAsync(out, d_out, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, stream));
    KCUDA(cudaMemcpyAsync(result, d_res, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, stream));
    KCUDA(cudaStreamSynchronize(stream));
  }

  void take_timings(KinStepTimings* out) override {
    timer.flush(timings);
    *out = timings;
    timings = KinStepTimings{};
  }

  void device_f(void** p, int32_t* es) override {
    *p = f.p;
    *es = static_cast<int32_t>(sizeof(S));
  }

  void velocity_permutation(int32_t* out, int64_t n) const override {
    KCHECK(n == nv, "length of the permutation output does not match nv");
    std::copy(perm.begin(), perm.end(), out);
  }

  void schedule_info(int32_t* ml, int32_t* nch) const override {
    *ml = max_levels;
    *nch = n_chains;
  }

  // ---- discrete adjoint ------------------------------------------------------------------------------------
  // lambda is stored at the position of the reversed velocity, so that the forward LU-SGS passes (which at
  // position p use xi_p and the sweep direction of p) act on the adjoint of -xi_p as the transposed preconditioner:
  // the in-block lower / upper couplings of velocity -xi are the transposes of the upper / lower ones of xi.
  void adjoint_begin(const int32_t* rev_velocity, const int32_t* rev_entry, int64_t n_entries,
                     const int32_t* flip_velocity, const int32_t* face_axis) override {
    if constexpr (!std::is_same<M, double>::value) {
      throw KinError(KIN_E_ARG, "the adjoint needs an FP64 or mixed-precision handle");
    } else {
      KCHECK(chunk == nv, "the adjoint needs one velocity chunk (velocity_chunk = 0 with enough device memory)");
      KCHECK(n_maxwell == 0, "the adjoint does not cover Maxwell walls");
      KCHECK(max_entries <= 127, "the adjoint stores stencil entry offsets in 8 bits (at most 127 faces per cell)");
      KCHECK(rev_velocity != nullptr && rev_entry != nullptr, "missing adjoint maps");
      std::vector<int32_t> hcsr(static_cast<size_t>(nc) + 1);
      KCUDA(cudaMemcpy(hcsr.data(), csr_off.p, hcsr.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
      KCHECK(n_entries == hcsr[nc], "length of the reverse CSR entry map does not match");
      std::vector<int32_t> rev(nv), perm2(nv), inv2(nv);
      for (int q = 0; q < nv; ++q) {
        const int s = rev_velocity[perm[q]];
        KCHECK(s >= 0 && s < nv, "reversed velocity out of range");
        rev[q] = inv[s];
      }
      for (int q = 0; q < nv; ++q) KCHECK(rev[rev[q]] == q, "the velocity reversal is not an involution");
      for (int p = 0; p < nv; ++p) perm2[p] = perm[rev[p]];
      for (int s = 0; s < nv; ++s) inv2[s] = rev[inv[s]];
      for (int64_t e = 0; e < n_entries; ++e) KCHECK(rev_entry[e] >= -1 && rev_entry[e] < n_entries, "reverse entry out of range");
      const size_t nf = static_cast<size_t>(nc) * nv;
      adj_rev.upload(rev.data(), nv, stream);
      adj_perm2.upload(perm2.data(), nv, stream);
      adj_inv2.upload(inv2.data(), nv, stream);
      adj_rev_entry.upload(rev_entry, static_cast<size_t>(n_entries), stream);
      adj_flip.release();
      adj_face_axis.release();
      if (flip_velocity != nullptr && face_axis != nullptr && nb > 0) {
        std::vector<int32_t> flip(3 * static_cast<size_t>(nv));
        for (int ax = 0; ax < 3; ++ax)
          for (int q = 0; q < nv; ++q) {
            const int s2 = flip_velocity[ax * nv + perm[q]];
            KCHECK(s2 >= 0 && s2 < nv, "flipped velocity out of range");
            flip[static_cast<size_t>(ax) * nv + q] = inv[s2];
          }
        for (int b = 0; b < nb; ++b) KCHECK(face_axis[b] >= -1 && face_axis[b] <= 2, "face axis out of range");
        adj_flip.upload(flip.data(), flip.size(), stream);
        adj_face_axis.upload(face_axis, static_cast<size_t>(nb), stream);
      }
      {
        std::vector<kin::BFace<M>> hb(static_cast<size_t>(nb));
        if (nb > 0)
          KCUDA(cudaMemcpy(hb.data(), bfaces.p, sizeof(kin::BFace<M>) * static_cast<size_t>(nb),
                           cudaMemcpyDeviceToHost));
        std::vector<int32_t> owners;
        for (const auto& b : hb)
          if (b.kind == kin::kDiffuseWall || b.kind == kin::kPressure) owners.push_back(b.owner);
        std::sort(owners.begin(), owners.end());
        owners.erase(std::unique(owners.begin(), owners.end()), owners.end());
        n_adj_face_cells = static_cast<int>(owners.size());
        adj_face_cells.release();
        if (!owners.empty()) adj_face_cells.upload(owners.data(), owners.size(), stream);
      }
      adj_lam.alloc(nf);
      KCUDA(cudaMemsetAsync(adj_lam.p, 0, adj_lam.bytes(), stream));
      adj_lfb.alloc(nf);
      adj_hmax.alloc(nf);
      adj_hmin.alloc(nf);
      adj_imax.alloc(nf);
      adj_imin.alloc(nf);
      adj_mu.alloc(static_cast<size_t>(std::max(nb, 1)));
      KCUDA(cudaMemsetAsync(adj_mu.p, 0, adj_mu.bytes(), stream));
      adj_coef.alloc(static_cast<size_t>(nc) * kin::kAdjCoefs);
      KCUDA(cudaMemsetAsync(adj_coef.p, 0, adj_coef.bytes(), stream));
      adj_cell.alloc(static_cast<size_t>(nc) * kin::kAdjCellSums);
      adj_face.alloc(static_cast<size_t>(std::max(nb, 1)) * kin::kAdjFaceSums);
      adj_res.alloc(static_cast<size_t>(nc));
      KCUDA(cudaStreamSynchronize(stream));
      adj_on = true;
    }
  }

  kin::AdjView<S> adj_view() {
    kin::AdjView<S> a{};
    a.lam = adj_lam.p;
    a.rev = adj_rev.p;
    a.rev_entry = adj_rev_entry.p;
    a.gbx = gx.p;
    a.gby = gy.p;
    a.gbz = gz.p;
    a.hmax = adj_hmax.p;
    a.hmin = adj_hmin.p;
    a.imax = adj_imax.p;
    a.imin = adj_imin.p;
    a.lfb = adj_lfb.p;
    a.mu = adj_mu.p;
    a.mom_mu = adj_mom_on ? adj_mom.p : nullptr;
    a.flip = adj_flip.p;
    a.face_axis = adj_face_axis.p;
    a.coef = adj_coef.p;
    a.moments = moments.p;
    a.deq_flags = deq_valid ? flags.p : nullptr;
    a.out = r.p;
    return a;
  }

  void adjoint_set(const double* h, int64_t n) override {
    KCHECK(adj_on, "adjoint_begin first");
    KCHECK(n == static_cast<int64_t>(nc) * nv, "length of lambda does not match");
    for (int64_t c0 = 0; c0 < nc; c0 += staging_cells) {
      const int cnt = static_cast<int>(std::min<int64_t>(staging_cells, nc - c0));
      KCUDA(cudaMemcpyAsync(staging.p, h + c0 * nv, sizeof(double) * cnt * nv, cudaMemcpyHostToDevice, stream));
      kin::Launch<S, M>::import_f(staging.p, adj_lam.p, adj_perm2.p, c0, cnt, nv, stream);
      launched();
    }
    KCUDA(cudaStreamSynchronize(stream));
  }

  void adjoint_get(double* h, int64_t n) override {
    KCHECK(adj_on, "adjoint_begin first");
    KCHECK(n == static_cast<int64_t>(nc) * nv, "length of lambda does not match");
    for (int64_t c0 = 0; c0 < nc; c0 += staging_cells) {
      const int cnt = static_cast<int>(std::min<int64_t>(staging_cells, nc - c0));
      kin::Launch<S, M>::export_f(adj_lam.p, staging.p, adj_inv2.p, c0, cnt, nv, stream);
      launched();
      KCUDA(cudaMemcpyAsync(h + c0 * nv, staging.p, sizeof(double) * cnt * nv, cudaMemcpyDeviceToHost, stream));
    }
    KCUDA(cudaStreamSynchronize(stream));
  }

  void adjoint_reduce(const double* mu, int64_t n_mu, double* cell_sums, int64_t n_cell, double* face_sums,
                      int64_t n_face) override {
    if constexpr (std::is_same<M, double>::value) {
      KCHECK(adj_on, "adjoint_begin first");
      // a NULL output with length 0 skips that sum (the transport always runs)
      const bool want_cells = cell_sums != nullptr;
      const bool want_faces = face_sums != nullptr && nb > 0;
      KCHECK(n_mu == nb && n_cell == (cell_sums != nullptr ? static_cast<int64_t>(nc) * kin::kAdjCellSums : 0) &&
                 n_face == (face_sums != nullptr ? static_cast<int64_t>(nb) * kin::kAdjFaceSums : 0),
             "adjoint_reduce: array lengths do not match");
      if (nb > 0) KCUDA(cudaMemcpyAsync(adj_mu.p, mu, sizeof(double) * nb, cudaMemcpyHostToDevice, stream));
      const kin::AdjView<S> a = adj_view();
      if (want_cells) kin::adj_cell_sums(view, a, adj_cell.p, stream);
      // per-face sums alone read the seeds of the face owners only: the transport runs on those cells (the other
      // cells' seeds are stale until the next full reduce)
      if (!want_cells && want_faces)
        kin::adj_transport(view, a, adj_face_cells.p, n_adj_face_cells, stream);
      else
        kin::adj_transport(view, a, nullptr, 0, stream);
      if (want_faces) kin::adj_face_sums(view, a, adj_face.p, stream);
      launched(1 + (want_cells ? 1 : 0) + (want_faces ? 1 : 0));
      KCUDA(cudaGetLastError());
      if (want_cells)
        KCUDA(cudaMemcpyAsync(cell_sums, adj_cell.p, sizeof(double) * n_cell, cudaMemcpyDeviceToHost, stream));
      if (want_faces)
        KCUDA(cudaMemcpyAsync(face_sums, adj_face.p, sizeof(double) * n_face, cudaMemcpyDeviceToHost, stream));
      KCUDA(cudaStreamSynchronize(stream));
    } else {
      throw KinError(KIN_E_ARG, "the adjoint needs an FP64 or mixed-precision handle");
    }
  }

  void adjoint_face_moment_seeds(const double* seeds, int64_t n) override {
    if constexpr (std::is_same<M, double>::value) {
      KCHECK(adj_on, "adjoint_begin first");
      if (seeds == nullptr || n == 0) {
        adj_mom_on = false;
        return;
      }
      KCHECK(n == 5 * static_cast<int64_t>(nb), "adjoint_face_moment_seeds: length must be 5 * n_bfaces");
      if (adj_mom.n < static_cast<size_t>(n)) adj_mom.alloc(static_cast<size_t>(n));
      KCUDA(cudaMemcpyAsync(adj_mom.p, seeds, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
      KCUDA(cudaStreamSynchronize(stream));
      adj_mom_on = true;
    } else {
      throw KinError(KIN_E_ARG, "the adjoint needs an FP64 or mixed-precision handle");
    }
  }

  void adjoint_update(const double* coef, int64_t n_coef, double* res_cell, int64_t n_res, int32_t run_passes,
                      double* op_out, int64_t n_op) override {
    if constexpr (std::is_same<M, double>::value) {
      KCHECK(adj_on, "adjoint_begin first");
      KCHECK(n_coef == static_cast<int64_t>(nc) * kin::kAdjCoefs && n_res == nc, "adjoint_update: array lengths");
      KCHECK(op_out == nullptr || n_op == static_cast<int64_t>(nc) * nv, "adjoint_update: operator output length");
      KCUDA(cudaMemcpyAsync(adj_coef.p, coef, sizeof(double) * n_coef, cudaMemcpyHostToDevice, stream));
      kin::adj_gather(view, adj_view(), adj_res.p, stream);
      launched();
      KCUDA(cudaGetLastError());
      if (op_out != nullptr) {
        for (int64_t c0 = 0; c0 < nc; c0 += staging_cells) {
          const int cnt = static_cast<int>(std::min<int64_t>(staging_cells, nc - c0));
          kin::Launch<S, M>::export_f(r.p, staging.p, adj_inv2.p, c0, cnt, nv, stream);
          launched();
          KCUDA(cudaMemcpyAsync(op_out + c0 * nv, staging.p, sizeof(double) * cnt * nv, cudaMemcpyDeviceToHost,
                                stream));
        }
      }
      if (run_passes) {
        // the forward block passes on lambda (reversed storage) with R = O_f(y): lambda += -P^-T O_f(y). The
        // adjoint keeps its arrays with rows of nv (= chunk) values, so the passes get that row stride.
        kin::View<S, P> av = sweep_view();
        av.f = adj_lam.p;
        run_block_passes(av, *chunks.front(), chunk, false);
        KCUDA(cudaGetLastError());
      }
      int32_t h_err = 0;
      KCUDA(cudaMemcpyAsync(res_cell, adj_res.p, sizeof(double) * nc, cudaMemcpyDeviceToHost, stream));
      KCUDA(cudaMemcpyAsync(&h_err, err_word.p, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
      KCUDA(cudaStreamSynchronize(stream));
      check_status(h_err);
    } else {
      throw KinError(KIN_E_ARG, "the adjoint needs an FP64 or mixed-precision handle");
    }
  }

  void adjoint_end() override {
    for (auto* b : {&adj_lam, &adj_lfb, &adj_hmax, &adj_hmin}) b->release();
    for (auto* b : {&adj_mu, &adj_coef, &adj_cell, &adj_face, &adj_res, &adj_mom}) b->release();
    adj_mom_on = false;
    adj_imax.release();
    adj_imin.release();
    adj_rev.release();
    adj_rev_entry.release();
    adj_perm2.release();
    adj_inv2.release();
    adj_flip.release();
    adj_face_axis.release();
    adj_face_cells.release();
    n_adj_face_cells = 0;
    adj_on = false;
  }
};

template <class Fn>
int guard(KinHandle* h, Fn&& fn) {
  if (h == nullptr) return KIN_E_ARG;
  try {
    cudaSetDevice(h->device);
    fn();
    return KIN_OK;
  } catch (const KinError& e) {
    h->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    h->err = e.what();
    return KIN_E_ARG;
  }
}

}  // namespace

extern "C" {

int kin_create(const KinSetupDesc* d, KinHandle** out) {
  if (out == nullptr || d == nullptr) {
    g_create_error = "kin_create: null argument";
    return KIN_E_ARG;
  }
  *out = nullptr;
  try {
    if (d->abi_version != KIN_ABI_VERSION) throw KinError(KIN_E_ARG, "KinSetupDesc ABI version mismatch");
    KinHandle* h = nullptr;
    switch (d->precision) {
      case KIN_PREC_FP32: {
        auto* b = new Backend<float, float>(*d);
        b->set_params(*d);
        h = b;
        break;
      }
      case KIN_PREC_FP64: {
        auto* b = new Backend<double, double>(*d);
        b->set_params(*d);
        h = b;
        break;
      }
      case KIN_PREC_MIXED: {
        auto* b = new Backend<float, double>(*d);
        b->set_params(*d);
        h = b;
        break;
      }
      default:
        throw KinError(KIN_E_ARG, "unknown precision");
    }
    *out = h;
    return KIN_OK;
  } catch (const KinError& e) {
    g_create_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    return KIN_E_ARG;
  }
}

void kin_destroy(KinHandle* h) { delete h; }

const char* kin_last_error(const KinHandle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }
const char* kin_name(const KinHandle* h) { return h ? h->name() : "b200"; }

int kin_chunk_width(const KinHandle* h, int32_t* out) {
  return guard(const_cast<KinHandle*>(h), [&] { *out = h->chunk_width(); });
}
int kin_memory_bytes(const KinHandle* h, uint64_t* out) {
  return guard(const_cast<KinHandle*>(h), [&] { *out = h->memory_bytes(); });
}
int kin_set_equilibrium(KinHandle* h, const double* s, int64_t n) { return guard(h, [&] { h->set_equilibrium(s, n); }); }
int kin_set_distribution(KinHandle* h, const double* f, int64_t n) {
  return guard(h, [&] { h->set_distribution(f, n); });
}
int kin_get_distribution(KinHandle* h, double* f, int64_t n) { return guard(h, [&] { h->get_distribution(f, n); }); }
int kin_compute_moments(KinHandle* h, double* out, int64_t n) { return guard(h, [&] { h->compute_moments(out, n); }); }
int kin_scale_distribution(KinHandle* h, double s) { return guard(h, [&] { h->scale_distribution(s); }); }
int kin_update_cell_params(KinHandle* h) { return guard(h, [&] { h->update_cell_params(); }); }
int kin_set_inflow(KinHandle* h, const KinInflowState* in, int64_t n) { return guard(h, [&] { h->set_inflow(in, n); }); }
int kin_boundary_sums(KinHandle* h, double* out, int64_t n) { return guard(h, [&] { h->boundary_sums(out, n); }); }
int kin_sweep(KinHandle* h, double* res, int64_t n) { return guard(h, [&] { h->sweep(res, n); }); }
int kin_gsis_correction(KinHandle* h, const double* wh, const double* wn, int64_t n, int32_t* flags,
                        int64_t* replaced) {
  return guard(h, [&] { h->gsis_correction(wh, wn, n, flags, replaced); });
}
int kin_gsis_correction_extrema(KinHandle* h, const double* wh, const double* wn, int64_t n, double* ext,
                                int64_t n_ext) {
  return guard(h, [&] { h->gsis_correction_extrema(wh, wn, n, ext, n_ext); });
}
int kin_gsis_correction_apply(KinHandle* h, const double* wh, const double* wn, int64_t n, const double* ext,
                              int64_t n_ext, int32_t* flags, int64_t* replaced) {
  return guard(h, [&] { h->gsis_correction_apply(wh, wn, n, ext, n_ext, flags, replaced); });
}
int kin_internal_face_mass_flux(KinHandle* h, const int32_t* cells, const int32_t* entries, int64_t n, double* out) {
  return guard(h, [&] { h->internal_face_mass_flux(cells, entries, n, out); });
}
int kin_take_timings(KinHandle* h, KinStepTimings* out) { return guard(h, [&] { h->take_timings(out); }); }
int kin_deq_counts(KinHandle* h, KinDeqCounts* out) { return guard(h, [&] { h->deq_counts(out); }); }

int kin_set_stream(KinHandle* h, void* stream) {
  return guard(h, [&] {
    KCUDA(cudaStreamSynchronize(h->stream));
    h->stream = stream != nullptr ? static_cast<cudaStream_t>(stream) : h->own_stream;
  });
}
int kin_launch_count(const KinHandle* h, int64_t* out) {
  return guard(const_cast<KinHandle*>(h), [&] { *out = h->launches; });
}
int kin_device_f(KinHandle* h, void** f, int32_t* es) { return guard(h, [&] { h->device_f(f, es); }); }
int kin_velocity_permutation(const KinHandle* h, int32_t* perm, int64_t n) {
  return guard(const_cast<KinHandle*>(h), [&] { h->velocity_permutation(perm, n); });
}
int kin_discrete_maxwell(KinHandle* h, const double* states, int64_t n, double tolerance, double* out,
                         int32_t* result) {
  return guard(h, [&] { h->discrete_maxwell(states, n, tolerance, out, result); });
}
int kin_discrete_maxwell_noalloc(KinHandle* h, const double* states, int64_t n, double tolerance, double* out,
                                 int32_t* result) {
  return guard(h, [&] { h->discrete_maxwell_noalloc(states, n, tolerance, out, result); });
}
int kin_moment_sums(KinHandle* h, double* out, int64_t n) { return guard(h, [&] { h->moment_sums(out, n); }); }
int kin_adjoint_begin(KinHandle* h, const int32_t* rev_velocity, const int32_t* rev_entry, int64_t n_entries,
                      const int32_t* flip_velocity, const int32_t* face_axis) {
  return guard(h, [&] { h->adjoint_begin(rev_velocity, rev_entry, n_entries, flip_velocity, face_axis); });
}
int kin_adjoint_set(KinHandle* h, const double* lam, int64_t n) { return guard(h, [&] { h->adjoint_set(lam, n); }); }
int kin_adjoint_get(KinHandle* h, double* lam, int64_t n) { return guard(h, [&] { h->adjoint_get(lam, n); }); }
int kin_adjoint_reduce(KinHandle* h, const double* mu, int64_t n_mu, double* cell_sums, int64_t n_cell,
                       double* face_sums, int64_t n_face) {
  return guard(h, [&] { h->adjoint_reduce(mu, n_mu, cell_sums, n_cell, face_sums, n_face); });
}
int kin_adjoint_face_moment_seeds(KinHandle* h, const double* seeds, int64_t n) {
  return guard(h, [&] { h->adjoint_face_moment_seeds(seeds, n); });
}
int kin_adjoint_update(KinHandle* h, const double* coef, int64_t n_coef, double* res_cell, int64_t n_res,
                       int32_t run_passes, double* op_out, int64_t n_op) {
  return guard(h, [&] { h->adjoint_update(coef, n_coef, res_cell, n_res, run_passes, op_out, n_op); });
}
int kin_adjoint_end(KinHandle* h) { return guard(h, [&] { h->adjoint_end(); }); }
int kin_set_moments(KinHandle* h, const double* m, int64_t n) { return guard(h, [&] { h->set_moments(m, n); }); }
int kin_device_sums(KinHandle* h, int32_t which, double** ptr, int64_t* n) {
  return guard(h, [&] { h->device_sums(which, ptr, n); });
}
int kin_finalize_moments(KinHandle* h, double* out, int64_t n) { return guard(h, [&] { h->finalize_moments(out, n); }); }
int kin_read_sums(KinHandle* h, int32_t which, double* out, int64_t n) {
  return guard(h, [&] { h->read_sums(which, out, n); });
}
int kin_schedule_info(const KinHandle* h, int32_t* max_levels, int32_t* n_chains) {
  return guard(const_cast<KinHandle*>(h), [&] { h->schedule_info(max_levels, n_chains); });
}

}  // extern "C"
