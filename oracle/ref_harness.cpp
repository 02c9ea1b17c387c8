// Test harness over the reference's own CPU kinetic path. TEST INFRASTRUCTURE ONLY: it is compiled from the
// reference sources (oracle/Makefile) into oracle/_ref/libgsisref.so and is used by tests/, the golden-fixture
// generator and the CPU baseline of bench.py, never by the product path.
//
// It drives the reference's `KineticSolver` (src/kinetic/kinetic_solver.hpp:61-115) with backend = "cpu" and a
// separate `CpuBackend` (src/kinetic/kinetic_backend_cpu.cpp) for operation-level checks, and exports the
// reference `KineticSetup` (src/kinetic/kinetic_setup.hpp:56-115) as a KinSetupDesc (include/gsis_b200.h).
// The case is filled programmatically, as the reference tests do (tests/kinetic/kinetic_test_cases.cpp:36-60),
// because the TOML parser of the reference (toml++) is not available here.

#include <cstdint>
#include <cstring>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "config/case_config.hpp"
#include "core/error.hpp"
#include "gsis_b200.h"
#include "kinetic/kinetic_backend.hpp"
#include "kinetic/kinetic_params.hpp"
#include "kinetic/kinetic_setup.hpp"
#include "kinetic/kinetic_solver.hpp"
#include "mesh/pmesh_io.hpp"
#include "support/box_mesh.hpp"

using namespace gsis;

namespace {

thread_local std::string g_error;

std::vector<std::string> split_ws(const std::string& s) {
  std::istringstream is(s);
  std::vector<std::string> out;
  std::string w;
  while (is >> w) out.push_back(w);
  return out;
}

std::string trim(const std::string& s) {
  const auto b = s.find_first_not_of(" \t\r");
  if (b == std::string::npos) return {};
  const auto e = s.find_last_not_of(" \t\r");
  return s.substr(b, e - b + 1);
}

// "key = value" lines; '#' starts a comment
std::vector<std::pair<std::string, std::string>> parse_lines(const char* text) {
  std::vector<std::pair<std::string, std::string>> out;
  std::istringstream is(text ? text : "");
  std::string line;
  while (std::getline(is, line)) {
    const auto hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    const auto eq = line.find('=');
    if (eq == std::string::npos) continue;
    out.emplace_back(trim(line.substr(0, eq)), trim(line.substr(eq + 1)));
  }
  return out;
}

ParamValue param_value(const std::string& v) {
  if (v == "true") return true;
  if (v == "false") return false;
  if (v.size() >= 2 && v.front() == '"' && v.back() == '"') return v.substr(1, v.size() - 2);
  if (v.find_first_of(".eE") == std::string::npos) return static_cast<long long>(std::stoll(v));
  return std::stod(v);
}

BoundaryType boundary_type(const std::string& s) {
  if (s == "diffuse_wall") return BoundaryType::DiffuseWall;
  if (s == "maxwell_wall") return BoundaryType::MaxwellWall;
  if (s == "pressure_inlet") return BoundaryType::PressureInlet;
  if (s == "pressure_outlet") return BoundaryType::PressureOutlet;
  if (s == "vacuum") return BoundaryType::Vacuum;
  if (s == "symmetry") return BoundaryType::Symmetry;
  if (s == "periodic_slab") return BoundaryType::PeriodicSlab;
  if (s == "mass_flow_inlet") return BoundaryType::MassFlowInlet;
  throw Error("unknown boundary type " + s);
}

struct NondimBc {
  std::string patch, type;
  double T = 1.0, p = 1.0, alpha = 1.0, mdot = 0.0;
  Vec3 u{};
};

CaseConfig make_config(const char* spec) {
  CaseConfig cfg;
  cfg.case_info.name = "ref_harness";
  cfg.case_info.mode = SolverMode::Cis;
  std::vector<NondimBc> bcs;
  ModuleSection kin("kinetic");
  for (const auto& [k, v] : parse_lines(spec)) {
    const auto w = split_ws(v);
    if (k == "gas.molecular_mass") cfg.gas.molecular_mass = std::stod(v);
    else if (k == "gas.mu_ref") cfg.gas.mu_ref = std::stod(v);
    else if (k == "gas.T_ref") cfg.gas.T_ref = std::stod(v);
    else if (k == "gas.omega") cfg.gas.omega = std::stod(v);
    else if (k == "conditions.L_ref") cfg.conditions.L_ref = std::stod(v);
    else if (k == "conditions.T0") cfg.conditions.T0 = std::stod(v);
    else if (k == "conditions.Kn") cfg.conditions.Kn = std::stod(v);
    else if (k == "conditions.delta_rp") cfg.conditions.delta_rp = std::stod(v);
    else if (k == "conditions.p_ref") cfg.conditions.p_ref = std::stod(v);
    else if (k == "velocity_grid.n") for (int a = 0; a < 3; ++a) cfg.velocity_grid.n[a] = std::stoi(w.at(a));
    else if (k == "velocity_grid.lo") for (int a = 0; a < 3; ++a) cfg.velocity_grid.lo[a] = std::stod(w.at(a));
    else if (k == "velocity_grid.hi") for (int a = 0; a < 3; ++a) cfg.velocity_grid.hi[a] = std::stod(w.at(a));
    else if (k == "boundary") {
      NondimBc b;
      b.patch = w.at(0);
      b.type = w.at(1);
      for (std::size_t i = 2; i < w.size(); ++i) {
        const auto eq = w[i].find('=');
        const std::string key = w[i].substr(0, eq), val = w[i].substr(eq + 1);
        if (key == "T") b.T = std::stod(val);
        else if (key == "p") b.p = std::stod(val);
        else if (key == "alpha") b.alpha = std::stod(val);
        else if (key == "mdot") b.mdot = std::stod(val);
        else if (key == "u") {
          std::string t = val;
          for (char& ch : t) if (ch == ',') ch = ' ';
          const auto uw = split_ws(t);
          b.u = Vec3{std::stod(uw.at(0)), std::stod(uw.at(1)), std::stod(uw.at(2))};
        }
      }
      bcs.push_back(b);
    } else if (k.rfind("kinetic.", 0) == 0) {
      kin.values[k.substr(8)] = param_value(v);
    }
  }
  cfg.module_sections["kinetic"] = kin;
  // SI boundary values from nondimensional ones, as tests/kinetic/kinetic_test_cases.cpp:36-60 does
  const DerivedQuantities d = derive_quantities(cfg);
  for (const NondimBc& b : bcs) {
    BoundarySpec s;
    s.patch = b.patch;
    s.type = boundary_type(b.type);
    s.accommodation = b.alpha;
    if (b.type == "diffuse_wall" || b.type == "maxwell_wall") {
      s.temperature = b.T * d.ref.temperature;
      if (norm(b.u) > 0.0) s.velocity = b.u * d.ref.velocity;
    } else if (b.type == "pressure_inlet") {
      s.temperature = b.T * d.ref.temperature;
      s.pressure = b.p * d.ref.pressure;
    } else if (b.type == "mass_flow_inlet") {
      // nondimensional target (inflow positive) -> kg/s, the inverse of kinetic_setup.cpp:372
      s.temperature = b.T * d.ref.temperature;
      s.pressure = b.p * d.ref.pressure;
      s.mass_flow = b.mdot * d.ref.mass_flux * d.ref.length * d.ref.length;
    } else if (b.type == "pressure_outlet") {
      s.pressure = b.p * d.ref.pressure;
    }
    cfg.boundaries.push_back(s);
  }
  return cfg;
}

struct RefCase {
  kinetic::StepTimings last_timings;  // backend times of the last CIS iteration
  CaseConfig cfg;
  KineticParams params;
  std::unique_ptr<KineticSolver> solver;
  std::unique_ptr<kinetic::KineticBackend> backend;  // separate CpuBackend on the solver's setup
  // flattened setup (FP64) for KinSetupDesc
  std::vector<double> xi_x, xi_y, xi_z;
  std::vector<int32_t> csr_offsets, csr_other, csr_bface, bface_owner, bface_kind, bface_mirror, bface_patch;
  std::vector<double> csr_geom, eps2, bface_geom;
  std::vector<int32_t> block_offsets;
  std::vector<int64_t> maxwell_offset;
  std::vector<double> maxwell_frac;
  std::vector<int32_t> grid_to_storage;
};

kinetic::InflowState to_inflow(const KinInflowState& s) {
  kinetic::InflowState o;
  o.scale = s.scale;
  o.rho = s.rho;
  o.u = Vec3{s.ux, s.uy, s.uz};
  o.T = s.T;
  return o;
}

#define GUARD_BEGIN try {
#define GUARD_END                     \
  }                                   \
  catch (const std::exception& e) {   \
    g_error = e.what();               \
    return -1;                        \
  }                                   \
  return 0;

}  // namespace

extern "C" {

const char* ref_error(void) { return g_error.c_str(); }

// --- meshes -----------------------------------------------------------------------------------------------

// Box mesh of the reference tests (tests/support/box_mesh.cpp:45-148): keys mesh.n, mesh.lo, mesh.hi,
// mesh.patches (6 names: x-, x+, y-, y+, z-, z+), mesh.distortion, mesh.tetrahedra, mesh.seed
void* ref_mesh_box(const char* spec) {
  try {
    test::BoxMeshOptions o;
    for (const auto& [k, v] : parse_lines(spec)) {
      const auto w = split_ws(v);
      if (k == "mesh.n") for (int a = 0; a < 3; ++a) o.n[a] = std::stoi(w.at(a));
      else if (k == "mesh.lo") o.lo = Vec3{std::stod(w.at(0)), std::stod(w.at(1)), std::stod(w.at(2))};
      else if (k == "mesh.hi") o.hi = Vec3{std::stod(w.at(0)), std::stod(w.at(1)), std::stod(w.at(2))};
      else if (k == "mesh.patches") for (int s = 0; s < 6; ++s) o.patch_names[s] = w.at(s);
      else if (k == "mesh.distortion") o.distortion = std::stod(v);
      else if (k == "mesh.tetrahedra") o.tetrahedra = std::stoi(v) != 0;
      else if (k == "mesh.seed") o.seed = static_cast<unsigned>(std::stoul(v));
    }
    return new LoadedMesh(validate_mesh(test::make_box_mesh(o)));
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

// Mesh from face-based arrays (.pmesh content, docs/pmesh_format.md); patch names separated by '\n'
void* ref_mesh_arrays(int32_t n_points, const double* points, int32_t n_faces, const int64_t* face_offsets,
                      const int32_t* face_nodes, const int32_t* owner, int32_t n_internal, const int32_t* neighbour,
                      int32_t n_cells, int32_t n_patches, const char* names, const int32_t* patch_start,
                      const int32_t* patch_count) {
  try {
    PolyMesh m;
    m.points.resize(static_cast<std::size_t>(n_points));
    for (int32_t i = 0; i < n_points; ++i) m.points[i] = Vec3{points[3 * i], points[3 * i + 1], points[3 * i + 2]};
    m.face_offsets.assign(face_offsets, face_offsets + n_faces + 1);
    m.face_nodes.assign(face_nodes, face_nodes + face_offsets[n_faces]);
    m.owner.assign(owner, owner + n_faces);
    m.neighbour.assign(neighbour, neighbour + n_internal);
    m.n_cells = n_cells;
    std::istringstream is(names);
    for (int32_t p = 0; p < n_patches; ++p) {
      Patch patch;
      std::getline(is, patch.name);
      patch.start = patch_start[p];
      patch.count = patch_count[p];
      m.patches.push_back(patch);
    }
    return new LoadedMesh(validate_mesh(std::move(m)));
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

void ref_mesh_free(void* m) { delete static_cast<LoadedMesh*>(m); }

// out: n_points, n_faces, n_internal, n_face_nodes, n_cells, n_patches
int ref_mesh_sizes(void* mp, int64_t* out) {
  const LoadedMesh& lm = *static_cast<LoadedMesh*>(mp);
  out[0] = lm.mesh.n_points();
  out[1] = lm.mesh.n_faces();
  out[2] = lm.mesh.n_internal_faces();
  out[3] = static_cast<int64_t>(lm.mesh.face_nodes.size());
  out[4] = lm.mesh.n_cells;
  out[5] = static_cast<int64_t>(lm.mesh.patches.size());
  return 0;
}

// Topology plus the reference geometry (compute_geometry, src/mesh/geometry.cpp:188-252)
int ref_mesh_export(void* mp, double* points, int64_t* face_offsets, int32_t* face_nodes, int32_t* owner,
                    int32_t* neighbour, int32_t* patch_start, int32_t* patch_count, char* names, int32_t names_cap,
                    double* cell_volume, double* cell_center, double* face_area_vector, double* face_center) {
  const LoadedMesh& lm = *static_cast<LoadedMesh*>(mp);
  const PolyMesh& m = lm.mesh;
  for (int32_t i = 0; i < m.n_points(); ++i) {
    points[3 * i] = m.points[i].x;
    points[3 * i + 1] = m.points[i].y;
    points[3 * i + 2] = m.points[i].z;
  }
  std::copy(m.face_offsets.begin(), m.face_offsets.end(), face_offsets);
  std::copy(m.face_nodes.begin(), m.face_nodes.end(), face_nodes);
  std::copy(m.owner.begin(), m.owner.end(), owner);
  std::copy(m.neighbour.begin(), m.neighbour.end(), neighbour);
  std::string all;
  for (std::size_t p = 0; p < m.patches.size(); ++p) {
    patch_start[p] = m.patches[p].start;
    patch_count[p] = m.patches[p].count;
    all += m.patches[p].name + "\n";
  }
  std::strncpy(names, all.c_str(), static_cast<std::size_t>(names_cap));
  const MeshGeometry& g = lm.geometry;
  for (int32_t c = 0; c < m.n_cells; ++c) {
    cell_volume[c] = g.cell_volume[c];
    for (int a = 0; a < 3; ++a) cell_center[3 * c + a] = g.cell_center[c][a];
  }
  for (int32_t f = 0; f < m.n_faces(); ++f) {
    for (int a = 0; a < 3; ++a) {
      face_area_vector[3 * f + a] = g.face_area_vector[f][a];
      face_center[3 * f + a] = g.face_center[f][a];
    }
  }
  return 0;
}

// --- cases ------------------------------------------------------------------------------------------------

void* ref_case_create(void* mp, const char* spec) {
  try {
    const LoadedMesh& lm = *static_cast<LoadedMesh*>(mp);
    auto rc = std::make_unique<RefCase>();
    rc->cfg = make_config(spec);
#if defined(REF_HARNESS_DROPIN) || defined(REF_HARNESS_REFCUDA)
    // drop-in build: the reference KineticSolver on the B200 backend (gsis_sim_b200/integration/b200_backend.cpp);
    // reference-CUDA build: the reference KineticSolver on the reference's own CudaBackend
    rc->cfg.module_sections["kinetic"].values["backend"] = std::string("cuda");
#else
    rc->cfg.module_sections["kinetic"].values["backend"] = std::string("cpu");
#endif
    rc->params = parse_kinetic_params(rc->cfg);
    rc->solver = std::make_unique<KineticSolver>(rc->cfg, lm.mesh, lm.geometry, rc->params);
    const kinetic::KineticSetup& s = rc->solver->setup();
    // flatten the setup
    rc->xi_x = s.velocity.xi_x;
    rc->xi_y = s.velocity.xi_y;
    rc->xi_z = s.velocity.xi_z;
    rc->csr_offsets = kinetic::make_csr_offsets(s);
    const auto csr = kinetic::make_csr_entries<double>(s);
    for (const auto& e : csr) {
      rc->csr_other.push_back(e.other);
      rc->csr_bface.push_back(e.bface);
      const double g[12] = {e.sx, e.sy, e.sz, e.dsx, e.dsy, e.dsz, e.dox, e.doy, e.doz, e.cx, e.cy, e.cz};
      rc->csr_geom.insert(rc->csr_geom.end(), g, g + 12);
    }
    rc->eps2 = kinetic::make_eps2<double>(s);
    for (const auto& b : kinetic::make_bface_infos<double>(s)) {
      rc->bface_owner.push_back(b.owner);
      rc->bface_kind.push_back(b.kind);
      rc->bface_mirror.push_back(b.mirror_xor);
      rc->bface_patch.push_back(b.patch);
      const double g[7] = {b.nx, b.ny, b.nz, b.area, b.dx, b.dy, b.dz};
      rc->bface_geom.insert(rc->bface_geom.end(), g, g + 7);
    }
    rc->block_offsets.assign(s.block_offsets.begin(), s.block_offsets.end());
    if (s.n_maxwell_faces > 0) {
      for (const auto& m : s.maxwell) {
        rc->maxwell_offset.push_back(m.offset);
        rc->maxwell_frac.push_back(m.specular_fraction);
      }
      rc->grid_to_storage.assign(s.velocity.grid_to_storage.begin(), s.velocity.grid_to_storage.end());
    }
    return rc.release();
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

void ref_case_free(void* c) { delete static_cast<RefCase*>(c); }

// KinSetupDesc with pointers into the case (valid while the case lives)
int ref_case_desc(void* cp, KinSetupDesc* d) {
  GUARD_BEGIN
  RefCase& rc = *static_cast<RefCase*>(cp);
  const kinetic::KineticSetup& s = rc.solver->setup();
  std::memset(d, 0, sizeof(*d));
  d->abi_version = KIN_ABI_VERSION;
  d->precision = s.params.precision == "fp64" ? KIN_PREC_FP64 : KIN_PREC_FP32;
  d->n_cells = s.n_cells();
  d->nv = s.nv();
  d->n_bfaces = s.n_bfaces();
  d->n_blocks = s.n_blocks();
  d->xi_x = rc.xi_x.data();
  d->xi_y = rc.xi_y.data();
  d->xi_z = rc.xi_z.data();
  d->weights = nullptr;
  d->weight = s.velocity.weight;
  d->csr_offsets = rc.csr_offsets.data();
  d->csr_other = rc.csr_other.data();
  d->csr_bface = rc.csr_bface.data();
  d->csr_geom = rc.csr_geom.data();
  d->eps2 = rc.eps2.data();
  d->bface_owner = rc.bface_owner.data();
  d->bface_kind = rc.bface_kind.data();
  d->bface_mirror_xor = rc.bface_mirror.data();
  d->bface_patch = rc.bface_patch.data();
  d->bface_geom = rc.bface_geom.data();
  d->volume = s.volume.data();
  d->vdt = s.vdt.data();
  d->block_offsets = rc.block_offsets.data();
  d->n_sweep_dirs = s.n_sweep_dirs;
  d->sweep_order = s.n_sweep_dirs > 0 ? s.sweep_order.data() : nullptr;
  d->sweep_pos = s.n_sweep_dirs > 0 ? s.sweep_pos.data() : nullptr;
  d->sweep_dir_of = s.n_sweep_dirs > 0 ? s.sweep_dir_of.data() : nullptr;
  d->limiter_mode = s.limiter_mode;
  d->positivity = s.params.positivity_limiter ? 1 : 0;
  d->diag_scale = s.diag_scale;
  d->interface_damping = s.params.interface_damping;
  d->block_passes = static_cast<int32_t>(s.params.block_passes);
  const std::string& rule = s.params.gsis_negative_check;
  d->negative_check_mode = rule == "created" ? KIN_NEGATIVE_CREATED
                           : rule == "limit" ? KIN_NEGATIVE_LIMIT
                           : rule == "blend" ? KIN_NEGATIVE_BLEND
                                             : KIN_NEGATIVE_ALL;
  d->velocity_chunk = s.params.velocity_chunk;
  d->mu0 = s.mu0;
  d->omega = s.omega;
  d->Pr = s.Pr;
  d->cold_bgk_temperature = s.params.cold_bgk_temperature;
  d->discrete_eq = s.discrete_eq ? 1 : 0;
  d->deq_fallback_collisionless = s.params.deq_fallback == "collisionless" ? 1 : 0;
  for (int a = 0; a < 3; ++a) {
    d->deq_lo[a] = s.deq_grid.lo[a];
    d->deq_hi[a] = s.deq_grid.hi[a];
    d->deq_d[a] = s.deq_grid.d[a];
    d->grid_n[a] = s.grid_n[a];
  }
  d->deq_criterion = s.deq_grid.criterion;
  d->deq_tolerance = s.deq_grid.tolerance;
  d->deq_max_iterations = s.deq_grid.max_iterations;
  d->n_maxwell_faces = s.n_maxwell_faces;
  d->maxwell_offset = s.n_maxwell_faces > 0 ? rc.maxwell_offset.data() : nullptr;
  d->maxwell_specular_fraction = s.n_maxwell_faces > 0 ? rc.maxwell_frac.data() : nullptr;
  d->grid_to_storage = s.n_maxwell_faces > 0 ? rc.grid_to_storage.data() : nullptr;
  d->device = 0;
  GUARD_END
}

// n_csr, closed_domain, n_patches, length_scale... (out: int64[8]); doubles (out: [8])
int ref_case_info(void* cp, int64_t* iout, double* dout) {
  GUARD_BEGIN
  RefCase& rc = *static_cast<RefCase*>(cp);
  const kinetic::KineticSetup& s = rc.solver->setup();
  iout[0] = static_cast<int64_t>(rc.csr_other.size());
  iout[1] = s.closed_domain ? 1 : 0;
  iout[2] = static_cast<int64_t>(s.patches.size());
  iout[3] = s.mesh.n_internal_faces();
  iout[4] = s.params.inner_sweeps;
  iout[5] = s.params.inner_wall_update ? 1 : 0;
  iout[6] = s.params.boundary_iterations;
  iout[7] = s.velocity.orbit_size;
  dout[0] = s.length_scale;
  dout[1] = s.gamma;
  dout[2] = s.params.limiter_k;
  dout[3] = s.params.wall_relaxation;
  dout[4] = s.params.convergence_u_floor;
  dout[5] = s.derived.mass_flow_scale;
  dout[6] = s.derived.mu_hat0;
  dout[7] = s.velocity.xi_max;
  GUARD_END
}

// Numbering maps and per-patch conditions:
//   cell_new_to_old[n_cells], bface_new_to_old[n_bfaces], storage_to_grid[nv],
//   patch_int[n_patches*4] = (kind, first_bface, n_faces, type), patch_dbl[n_patches*7] = (T, p, ux, uy, uz,
//   accommodation, zero_tangential)
int ref_case_maps(void* cp, int32_t* cell_new_to_old, int32_t* bface_new_to_old, int32_t* storage_to_grid,
                  int32_t* patch_int, double* patch_dbl) {
  GUARD_BEGIN
  RefCase& rc = *static_cast<RefCase*>(cp);
  const kinetic::KineticSetup& s = rc.solver->setup();
  std::copy(s.cell_new_to_old.begin(), s.cell_new_to_old.end(), cell_new_to_old);
  std::copy(s.bface_new_to_old.begin(), s.bface_new_to_old.end(), bface_new_to_old);
  std::copy(s.velocity.storage_to_grid.begin(), s.velocity.storage_to_grid.end(), storage_to_grid);
  for (std::size_t p = 0; p < s.patches.size(); ++p) {
    const auto& pc = s.patches[p];
    patch_int[4 * p + 0] = pc.kind;
    patch_int[4 * p + 1] = pc.first_bface;
    patch_int[4 * p + 2] = pc.n_faces;
    patch_int[4 * p + 3] = static_cast<int32_t>(pc.type);
    const double v[7] = {pc.T, pc.p, pc.u_wall.x, pc.u_wall.y, pc.u_wall.z, pc.accommodation,
                         pc.zero_tangential ? 1.0 : 0.0};
    std::copy(v, v + 7, patch_dbl + 7 * p);
  }
  GUARD_END
}

// Internal-numbering geometry of the renumbered mesh: cell_center[3 nc], face_center[3 nf], face_normal[3 nf],
// face_area[nf], owner[nf]; LSQ coefficients (unscaled, m^-1) lsq[3 n_csr]; csr face index [n_csr]
int ref_case_geometry(void* cp, double* cell_center, double* face_center, double* face_normal, double* face_area,
                      int32_t* owner, double* lsq, int32_t* csr_faces) {
  GUARD_BEGIN
  RefCase& rc = *static_cast<RefCase*>(cp);
  const kinetic::KineticSetup& s = rc.solver->setup();
  for (int32_t c = 0; c < s.n_cells(); ++c)
    for (int a = 0; a < 3; ++a) cell_center[3 * c + a] = s.geometry.cell_center[c][a];
  for (int32_t f = 0; f < s.mesh.n_faces(); ++f) {
    for (int a = 0; a < 3; ++a) {
      face_center[3 * f + a] = s.geometry.face_center[f][a];
      face_normal[3 * f + a] = s.geometry.face_normal[f][a];
    }
    face_area[f] = s.geometry.face_area[f];
    owner[f] = s.mesh.owner[f];
  }
  for (std::size_t k = 0; k < s.lsq.coeff.size(); ++k) {
    for (int a = 0; a < 3; ++a) lsq[3 * k + a] = s.lsq.coeff[k][a];
    csr_faces[k] = s.csr.faces[k];
  }
  GUARD_END
}

// --- reference KineticSolver (host loop + CpuBackend) -------------------------------------------------------

// info[12]: iteration, epsilon, eps_rho, eps_u, eps_T, has_epsilon, residual, has_residual, total_mass,
//           mass_scale, deq_corrected, deq_failed
static void fill_info(const KineticIterationInfo& i, double* info) {
  if (info == nullptr) return;
  info[0] = static_cast<double>(i.iteration);
  info[1] = i.epsilon;
  info[2] = i.eps_rho;
  info[3] = i.eps_u;
  info[4] = i.eps_T;
  info[5] = i.has_epsilon ? 1.0 : 0.0;
  info[6] = i.residual;
  info[7] = i.has_residual ? 1.0 : 0.0;
  info[8] = i.total_mass;
  info[9] = i.mass_scale;
  info[10] = static_cast<double>(i.deq_corrected);
  info[11] = static_cast<double>(i.deq_failed);
}

int ref_solver_init_uniform(void* cp, double rho, double ux, double uy, double uz, double T) {
  GUARD_BEGIN
  static_cast<RefCase*>(cp)->solver->initialize_uniform(rho, Vec3{ux, uy, uz}, T);
  GUARD_END
}

// states: 5 per cell, ORIGINAL cell numbering
int ref_solver_init_states(void* cp, const double* states) {
  GUARD_BEGIN
  RefCase& rc = *static_cast<RefCase*>(cp);
  const std::size_t nc = static_cast<std::size_t>(rc.solver->setup().n_cells());
  CellMacroState st;
  st.resize(nc);
  for (std::size_t c = 0; c < nc; ++c) {
    st.rho[c] = states[5 * c];
    st.ux[c] = states[5 * c + 1];
    st.uy[c] = states[5 * c + 2];
    st.uz[c] = states[5 * c + 3];
    st.T[c] = states[5 * c + 4];
  }
  rc.solver->initialize_equilibrium(st);
  GUARD_END
}

int ref_solver_prepare(void* cp, double* info) {
  GUARD_BEGIN
  fill_info(static_cast<RefCase*>(cp)->solver->prepare(), info);
  GUARD_END
}

int ref_solver_sweep(void* cp, int update_pressure, double* info) {
  GUARD_BEGIN
  RefCase* rc = static_cast<RefCase*>(cp);
  const KineticIterationInfo& i = rc->solver->sweep(update_pressure != 0);
  rc->last_timings = i.timings;
  fill_info(i, info);
  GUARD_END
}

// per-phase backend times of the last CIS iteration (StepTimings, src/kinetic/kinetic_backend.hpp:18-40): moments,
// boundary, gradient, residual, sweep_forward, sweep_backward, other [s]
int ref_solver_last_timings(void* cp, double* out) {
  GUARD_BEGIN
  const auto& t = static_cast<RefCase*>(cp)->last_timings;
  out[0] = t.moments;
  out[1] = t.boundary;
  out[2] = t.gradient;
  out[3] = t.residual;
  out[4] = t.sweep_forward;
  out[5] = t.sweep_backward;
  out[6] = t.other;
  GUARD_END
}

// patch mass flows of the last prepare (n_patches)
int ref_solver_patch_mass_flow(void* cp, double* out) {
  GUARD_BEGIN
  const auto& pm = static_cast<RefCase*>(cp)->solver->prepare().patch_mass_flow;
  std::copy(pm.begin(), pm.end(), out);
  GUARD_END
}

// moments in ORIGINAL numbering: 15 per cell in the backend order
int ref_solver_moments(void* cp, double* out) {
  GUARD_BEGIN
  const KineticMoments m = static_cast<RefCase*>(cp)->solver->moments();
  for (std::size_t c = 0; c < m.state.size(); ++c) {
    double* o = out + 15 * c;
    o[0] = m.state.rho[c];
    o[1] = m.state.ux[c];
    o[2] = m.state.uy[c];
    o[3] = m.state.uz[c];
    o[4] = m.state.T[c];
    o[5] = m.state.p[c];
    for (int k = 0; k < 6; ++k) o[6 + k] = m.sigma[c][k];
    for (int k = 0; k < 3; ++k) o[12 + k] = m.q[c][k];
  }
  GUARD_END
}

// boundary fluxes in ORIGINAL boundary-face numbering: F_plus[5 nb], F_minus[5 nb], face_state[5 nb]
int ref_solver_boundary_fluxes(void* cp, double* fp, double* fm, double* fs) {
  GUARD_BEGIN
  const BoundaryKineticFluxes b = static_cast<RefCase*>(cp)->solver->boundary_fluxes();
  for (std::size_t i = 0; i < b.F_plus.size(); ++i) {
    for (int k = 0; k < 5; ++k) {
      fp[5 * i + k] = b.F_plus[i][k];
      fm[5 * i + k] = b.F_minus[i][k];
      fs[5 * i + k] = b.face_state[i][k];
    }
  }
  GUARD_END
}

// f in ORIGINAL cell numbering x velocity-GRID order
int ref_solver_distribution(void* cp, double* f) {
  GUARD_BEGIN
  const std::vector<double> d = static_cast<RefCase*>(cp)->solver->distribution();
  std::copy(d.begin(), d.end(), f);
  GUARD_END
}

int ref_solver_set_distribution(void* cp, const double* f, int64_t n) {
  GUARD_BEGIN
  static_cast<RefCase*>(cp)->solver->set_distribution(std::span<const double>(f, static_cast<std::size_t>(n)));
  GUARD_END
}

// GSIS correction with W in ORIGINAL numbering (5 per cell); replaced cells count in *replaced
int ref_solver_gsis_correction(void* cp, const double* w_half, const double* w_new, int64_t* replaced) {
  GUARD_BEGIN
  RefCase& rc = *static_cast<RefCase*>(cp);
  const std::size_t nc = static_cast<std::size_t>(rc.solver->setup().n_cells());
  CellMacroState a, b;
  a.resize(nc);
  b.resize(nc);
  for (std::size_t c = 0; c < nc; ++c) {
    a.rho[c] = w_half[5 * c]; a.ux[c] = w_half[5 * c + 1]; a.uy[c] = w_half[5 * c + 2];
    a.uz[c] = w_half[5 * c + 3]; a.T[c] = w_half[5 * c + 4];
    b.rho[c] = w_new[5 * c]; b.ux[c] = w_new[5 * c + 1]; b.uy[c] = w_new[5 * c + 2];
    b.uz[c] = w_new[5 * c + 3]; b.T[c] = w_new[5 * c + 4];
  }
  *replaced = rc.solver->apply_gsis_correction(a, b);
  GUARD_END
}

// section mass flows at x positions (SectionSpec, src/mesh/section_cut.hpp)
int ref_solver_section_mass_flow(void* cp, int32_t axis, const double* positions, int32_t n, double* out) {
  GUARD_BEGIN
  SectionSpec spec;
  spec.axis = axis;
  spec.positions.assign(positions, positions + n);
  const std::vector<double> r = static_cast<RefCase*>(cp)->solver->section_mass_flow(spec);
  std::copy(r.begin(), r.end(), out);
  GUARD_END
}

// --- reference CpuBackend, operation by operation (same signatures as the kin_* entry points) --------------

// the separate backend of the operation-level checks, created on first use (a solver-only run allocates no second f)
static kinetic::KineticBackend& backend_of(void* cp) {
  RefCase* rc = static_cast<RefCase*>(cp);
  if (!rc->backend) {
#if defined(REF_HARNESS_DROPIN) || defined(REF_HARNESS_REFCUDA)
    rc->backend = kinetic::make_cuda_backend(rc->solver->setup());
#else
    rc->backend = kinetic::make_cpu_backend(rc->solver->setup());
#endif
  }
  return *rc->backend;
}
#define BK(cp) backend_of(cp)

int ref_kin_set_equilibrium(void* cp, const double* states, int64_t n) {
  GUARD_BEGIN BK(cp).set_equilibrium(std::span<const double>(states, static_cast<std::size_t>(n))); GUARD_END
}
int ref_kin_set_distribution(void* cp, const double* f, int64_t n) {
  GUARD_BEGIN BK(cp).set_distribution(std::span<const double>(f, static_cast<std::size_t>(n))); GUARD_END
}
int ref_kin_get_distribution(void* cp, double* f, int64_t n) {
  GUARD_BEGIN BK(cp).get_distribution(std::span<double>(f, static_cast<std::size_t>(n))); GUARD_END
}
int ref_kin_compute_moments(void* cp, double* out, int64_t n) {
  GUARD_BEGIN BK(cp).compute_moments(std::span<double>(out, static_cast<std::size_t>(n))); GUARD_END
}
int ref_kin_scale_distribution(void* cp, double s) { GUARD_BEGIN BK(cp).scale_distribution(s); GUARD_END }
int ref_kin_update_cell_params(void* cp) { GUARD_BEGIN BK(cp).update_cell_params(); GUARD_END }
int ref_kin_set_inflow(void* cp, const KinInflowState* in, int64_t n) {
  GUARD_BEGIN
  std::vector<kinetic::InflowState> v(static_cast<std::size_t>(n));
  for (int64_t i = 0; i < n; ++i) v[static_cast<std::size_t>(i)] = to_inflow(in[i]);
  BK(cp).set_inflow(v);
  GUARD_END
}
int ref_kin_boundary_sums(void* cp, double* out, int64_t n) {
  GUARD_BEGIN BK(cp).boundary_sums(std::span<double>(out, static_cast<std::size_t>(n))); GUARD_END
}
int ref_kin_sweep(void* cp, double* residual_cell, int64_t n) {
  GUARD_BEGIN BK(cp).sweep(std::span<double>(residual_cell, static_cast<std::size_t>(n))); GUARD_END
}
int ref_kin_gsis_correction(void* cp, const double* w_half, const double* w_new, int64_t n, int32_t* flags,
                            int64_t* replaced) {
  GUARD_BEGIN
  const std::size_t nc = static_cast<std::size_t>(n / 5);
  std::vector<int> fl(nc, 0);
  *replaced = BK(cp).gsis_correction(std::span<const double>(w_half, static_cast<std::size_t>(n)),
                                     std::span<const double>(w_new, static_cast<std::size_t>(n)), std::span<int>(fl));
  if (flags != nullptr) std::copy(fl.begin(), fl.end(), flags);
  GUARD_END
}
int ref_kin_internal_face_mass_flux(void* cp, const int32_t* cells, const int32_t* entries, int64_t n, double* out) {
  GUARD_BEGIN
  BK(cp).internal_face_mass_flux(std::span<const int32_t>(cells, static_cast<std::size_t>(n)),
                                 std::span<const int32_t>(entries, static_cast<std::size_t>(n)),
                                 std::span<double>(out, static_cast<std::size_t>(n)));
  GUARD_END
}
int ref_kin_deq_counts(void* cp, KinDeqCounts* out) {
  GUARD_BEGIN
  const kinetic::DeqCounts d = BK(cp).deq_counts();
  out->corrected = d.corrected;
  out->failed = d.failed;
  out->max_iterations = d.max_iterations;
  GUARD_END
}
int ref_kin_chunk_width(void* cp, int32_t* out) { GUARD_BEGIN *out = BK(cp).chunk_width(); GUARD_END }

}  // extern "C"
