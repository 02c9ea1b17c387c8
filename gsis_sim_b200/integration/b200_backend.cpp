// Drop-in KineticBackend of GSIS-Sim over the B200 C ABI (include/gsis_b200.h).
//
// Build the reference host code WITHOUT src/kinetic/kinetic_backend_cuda.cpp and kinetic_cuda_kernels.cu, with
// GSIS_WITH_CUDA=1 (so src/kinetic/kinetic_backend_factory.cpp defines nothing), add this file and link
// libgsis_b200.so: `KineticSolver` (src/kinetic/kinetic_solver.cpp:83-87) then obtains this backend from
// `make_cuda_backend` for every case with kinetic.backend = "cuda". Nothing else in the reference changes.
//
// Each method forwards to one C entry point; failures come back as gsis::Error with the library's message, like
// the GSIS_CHECK / GSIS_CUDA_CHECK failures of the CUDA backend it replaces (src/kinetic/kinetic_backend_cuda.cpp).
#include <cstring>
#include <memory>
#include <span>
#include <string>
#include <vector>

#include "core/error.hpp"
#include "gsis_b200.h"
#include "kinetic/kinetic_backend.hpp"
#include "kinetic/kinetic_setup.hpp"

namespace gsis::kinetic {
namespace {

static_assert(sizeof(InflowState) == sizeof(KinInflowState), "InflowState and KinInflowState must match");

class B200Backend final : public KineticBackend {
 public:
  explicit B200Backend(const KineticSetup& s) {
    // the setup tables in FP64, as make_csr_entries / make_bface_infos / make_eps2 produce them
    csr_offsets_ = make_csr_offsets(s);
    for (const auto& e : make_csr_entries<double>(s)) {
      csr_other_.push_back(e.other);
      csr_bface_.push_back(e.bface);
      const double g[KIN_CSR_GEOM] = {e.sx, e.sy, e.sz, e.dsx, e.dsy, e.dsz, e.dox, e.doy, e.doz, e.cx, e.cy, e.cz};
      csr_geom_.insert(csr_geom_.end(), g, g + KIN_CSR_GEOM);
    }
    eps2_ = make_eps2<double>(s);
    for (const auto& b : make_bface_infos<double>(s)) {
      bface_owner_.push_back(b.owner);
      bface_kind_.push_back(b.kind);
      bface_mirror_.push_back(b.mirror_xor);
      bface_patch_.push_back(b.patch);
      const double g[KIN_BFACE_GEOM] = {b.nx, b.ny, b.nz, b.area, b.dx, b.dy, b.dz};
      bface_geom_.insert(bface_geom_.end(), g, g + KIN_BFACE_GEOM);
    }
    block_offsets_.assign(s.block_offsets.begin(), s.block_offsets.end());
    for (const auto& m : s.maxwell) {
      maxwell_offset_.push_back(m.offset);
      maxwell_frac_.push_back(m.specular_fraction);
    }
    KinSetupDesc d;
    std::memset(&d, 0, sizeof(d));
    d.abi_version = KIN_ABI_VERSION;
    d.precision = s.params.precision == "fp64" ? KIN_PREC_FP64 : KIN_PREC_FP32;
    d.device = 0;
    d.n_cells = s.n_cells();
    d.nv = s.nv();
    d.n_bfaces = s.n_bfaces();
    d.n_blocks = s.n_blocks();
    d.xi_x = s.velocity.xi_x.data();
    d.xi_y = s.velocity.xi_y.data();
    d.xi_z = s.velocity.xi_z.data();
    d.weights = nullptr;
    d.weight = s.velocity.weight;
    d.csr_offsets = csr_offsets_.data();
    d.csr_other = csr_other_.data();
    d.csr_bface = csr_bface_.data();
    d.csr_geom = csr_geom_.data();
    d.eps2 = eps2_.data();
    d.bface_owner = bface_owner_.data();
    d.bface_kind = bface_kind_.data();
    d.bface_mirror_xor = bface_mirror_.data();
    d.bface_patch = bface_patch_.data();
    d.bface_geom = bface_geom_.data();
    d.volume = s.volume.data();
    d.vdt = s.vdt.data();
    d.block_offsets = block_offsets_.data();
    d.n_sweep_dirs = s.n_sweep_dirs;
    d.sweep_order = s.n_sweep_dirs > 0 ? s.sweep_order.data() : nullptr;
    d.sweep_pos = s.n_sweep_dirs > 0 ? s.sweep_pos.data() : nullptr;
    d.sweep_dir_of = s.n_sweep_dirs > 0 ? s.sweep_dir_of.data() : nullptr;
    d.limiter_mode = s.limiter_mode;
    d.positivity = s.params.positivity_limiter ? 1 : 0;
    d.diag_scale = s.diag_scale;
    d.interface_damping = s.params.interface_damping;
    d.block_passes = static_cast<int32_t>(s.params.block_passes);
    const std::string& rule = s.params.gsis_negative_check;
    d.negative_check_mode = rule == "created" ? KIN_NEGATIVE_CREATED
                            : rule == "limit" ? KIN_NEGATIVE_LIMIT
                            : rule == "blend" ? KIN_NEGATIVE_BLEND
                                              : KIN_NEGATIVE_ALL;
    d.velocity_chunk = s.params.velocity_chunk;
    d.mu0 = s.mu0;
    d.omega = s.omega;
    d.Pr = s.Pr;
    d.cold_bgk_temperature = s.params.cold_bgk_temperature;
    d.discrete_eq = s.discrete_eq ? 1 : 0;
    d.deq_fallback_collisionless = s.params.deq_fallback == "collisionless" ? 1 : 0;
    for (int a = 0; a < 3; ++a) {
      d.deq_lo[a] = s.deq_grid.lo[a];
      d.deq_hi[a] = s.deq_grid.hi[a];
      d.deq_d[a] = s.deq_grid.d[a];
      d.grid_n[a] = s.grid_n[a];
    }
    d.deq_criterion = s.deq_grid.criterion;
    d.deq_tolerance = s.deq_grid.tolerance;
    d.deq_max_iterations = s.deq_grid.max_iterations;
    d.n_maxwell_faces = s.n_maxwell_faces;
    d.maxwell_offset = s.n_maxwell_faces > 0 ? maxwell_offset_.data() : nullptr;
    d.maxwell_specular_fraction = s.n_maxwell_faces > 0 ? maxwell_frac_.data() : nullptr;
    d.grid_to_storage = s.n_maxwell_faces > 0 ? s.velocity.grid_to_storage.data() : nullptr;
    if (kin_create(&d, &h_) != KIN_OK) throw Error(std::string("B200 kinetic backend: ") + kin_last_error(nullptr));
  }

  ~B200Backend() override { kin_destroy(h_); }

  const char* name() const override { return "b200"; }
  int chunk_width() const override {
    int32_t c = 0;
    check(kin_chunk_width(h_, &c));
    return c;
  }
  std::size_t memory_bytes() const override {
    uint64_t b = 0;
    check(kin_memory_bytes(h_, &b));
    return static_cast<std::size_t>(b);
  }
  void set_equilibrium(std::span<const double> st) override {
    check(kin_set_equilibrium(h_, st.data(), static_cast<int64_t>(st.size())));
  }
  void set_distribution(std::span<const double> f) override {
    check(kin_set_distribution(h_, f.data(), static_cast<int64_t>(f.size())));
  }
  void get_distribution(std::span<double> f) override {
    check(kin_get_distribution(h_, f.data(), static_cast<int64_t>(f.size())));
  }
  void compute_moments(std::span<double> out) override {
    check(kin_compute_moments(h_, out.data(), static_cast<int64_t>(out.size())));
  }
  void scale_distribution(double s) override { check(kin_scale_distribution(h_, s)); }
  void update_cell_params() override { check(kin_update_cell_params(h_)); }
  void set_inflow(std::span<const InflowState> in) override {
    check(kin_set_inflow(h_, reinterpret_cast<const KinInflowState*>(in.data()), static_cast<int64_t>(in.size())));
  }
  void boundary_sums(std::span<double> out) override {
    check(kin_boundary_sums(h_, out.data(), static_cast<int64_t>(out.size())));
  }
  void sweep(std::span<double> residual_cell) override {
    check(kin_sweep(h_, residual_cell.data(), static_cast<int64_t>(residual_cell.size())));
  }
  long long gsis_correction(std::span<const double> w_half, std::span<const double> w_new,
                            std::span<int> replaced) override {
    GSIS_CHECK(w_half.size() == w_new.size(), "GSIS correction: W_half and W_new differ in length");
    std::vector<int32_t> flags(w_half.size() / 5, 0);
    int64_t n = 0;
    check(kin_gsis_correction(h_, w_half.data(), w_new.data(), static_cast<int64_t>(w_half.size()), flags.data(), &n));
    if (!replaced.empty()) std::copy(flags.begin(), flags.end(), replaced.begin());
    return static_cast<long long>(n);
  }
  void internal_face_mass_flux(std::span<const std::int32_t> cells, std::span<const std::int32_t> entries,
                               std::span<double> out) override {
    GSIS_CHECK(cells.size() == entries.size() && out.size() == cells.size(),
               "internal face mass flux: argument lengths differ");
    check(kin_internal_face_mass_flux(h_, cells.data(), entries.data(), static_cast<int64_t>(cells.size()),
                                      out.data()));
  }
  StepTimings take_timings() override {
    KinStepTimings t{};
    check(kin_take_timings(h_, &t));
    StepTimings o;
    o.moments = t.moments;
    o.boundary = t.boundary;
    o.gradient = t.gradient;
    o.residual = t.residual;
    o.sweep_forward = t.sweep_forward;
    o.sweep_backward = t.sweep_backward;
    o.other = t.other;
    return o;
  }
  DeqCounts deq_counts() override {
    KinDeqCounts c{};
    check(kin_deq_counts(h_, &c));
    DeqCounts o;
    o.corrected = c.corrected;
    o.failed = c.failed;
    o.max_iterations = c.max_iterations;
    return o;
  }

 private:
  void check(int rc) const {
    if (rc != KIN_OK) throw Error(std::string("B200 kinetic backend: ") + kin_last_error(h_));
  }

  KinHandle* h_ = nullptr;
  std::vector<std::int32_t> csr_offsets_, csr_other_, csr_bface_, bface_owner_, bface_kind_, bface_mirror_,
      bface_patch_, block_offsets_;
  std::vector<double> csr_geom_, eps2_, bface_geom_, maxwell_frac_;
  std::vector<std::int64_t> maxwell_offset_;
};

}  // namespace

std::unique_ptr<KineticBackend> make_cuda_backend(const KineticSetup& setup) {
  return std::make_unique<B200Backend>(setup);
}

}  // namespace gsis::kinetic
