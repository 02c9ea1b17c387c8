"""Generates the golden fixtures of tests/golden/*.npz from the reference's OWN CPU kinetic path.

Run in a container that has the reference sources (it builds oracle/_ref/libgsisref.so from them):
    python tests/golden/make_golden.py
Each fixture holds
  * the reference `KineticSetup` of the case as flat arrays (`setup.*`, the KinSetupDesc content), plus the
    host-side data the kinetic host loop needs (`host.*`: patches, geometry, numbering maps);
  * `op.*`: outputs of the reference CpuBackend (src/kinetic/kinetic_backend_cpu.cpp) for a fixed operation
    sequence (set_equilibrium, compute_moments, update_cell_params, set_inflow, boundary_sums, 2 x sweep,
    gsis_correction, internal_face_mass_flux);
  * `solver.*`: the reference KineticSolver (src/kinetic/kinetic_solver.cpp) after a few CIS iterations from a
    uniform state: residual history, moments, boundary fluxes, f (original numbering) and section mass flows
    (KineticSolver::section_mass_flow, src/kinetic/kinetic_solver.cpp:669-685) at fixed x and y positions.
The cases are the reference GPU tests' cases (tests/kinetic/test_kinetic_gpu.cpp:50-91, 160-173, 261-273) with a
smaller velocity grid so that every fixture stays small.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402

MIXED_PATCHES = ["inlet", "outlet", "wall", "wall", "sym", "sym"]
MIXED_BCS = [("inlet", "pressure_inlet", dict(T=1.0, p=1.1)), ("outlet", "pressure_outlet", dict(p=0.3)),
             ("wall", "diffuse_wall", dict(T=1.0, u=(0.1, 0.0, 0.05))), ("sym", "symmetry", {})]
SECTION_X = [0.0, 0.13, 0.5, 0.5, 0.71, 0.99, 3.0]
SECTION_Y = [0.3, 0.45]
OLD_CIS = dict(sweep_order="block", inner_sweeps=1, inner_wall_update=False, block_passes=1, equilibrium="continuous")

# name -> (mesh kwargs, bcs, Kn, nv, kinetic, init (rho, u, T), iterations)
CASES = {
    "mixed_strong_fp64": (dict(n=(5, 3, 2), lo=(0, 0, 0), hi=(1, 0.6, 0.4), patches=MIXED_PATCHES, distortion=0.15),
                          MIXED_BCS, 0.1, (8, 8, 8), dict(sweep_blocks=3, precision="fp64"), (0.7, (0.1, 0, 0), 1.0), 3),
    "mixed_strong_fp32": (dict(n=(5, 3, 2), lo=(0, 0, 0), hi=(1, 0.6, 0.4), patches=MIXED_PATCHES, distortion=0.15),
                          MIXED_BCS, 0.1, (8, 8, 8), dict(sweep_blocks=3, precision="fp32"), (0.7, (0.1, 0, 0), 1.0), 3),
    "mixed_old_fp64": (dict(n=(5, 3, 2), lo=(0, 0, 0), hi=(1, 0.6, 0.4), patches=MIXED_PATCHES, distortion=0.15),
                       MIXED_BCS, 0.1, (8, 8, 8),
                       dict(sweep_blocks=4, precision="fp64", limiter_eps="relative", **OLD_CIS),
                       (0.7, (0.1, 0, 0), 1.0), 4),
    "couette_fp64": (dict(n=(6, 1, 1), lo=(0, 0, 0), hi=(1, 1 / 6, 1 / 6),
                          patches=["wall_left", "wall_right", "sym_y", "sym_y", "sym_z", "sym_z"]),
                     [("wall_left", "diffuse_wall", dict(T=0.95, u=(0, -0.4, 0))),
                      ("wall_right", "diffuse_wall", dict(T=1.05, u=(0, 0.4, 0))),
                      ("sym_y", "periodic_slab", {}), ("sym_z", "symmetry", {})],
                     0.5, (8, 8, 8), dict(sweep_blocks=2, precision="fp64"), (1.0, (0, 0, 0), 1.0), 4),
    "dir13_fp32": (dict(n=(5, 3, 2), lo=(0, 0, 0), hi=(1, 0.6, 0.4), patches=MIXED_PATCHES, distortion=0.15),
                   MIXED_BCS, 0.1, (8, 8, 8), dict(sweep_blocks=2, sweep_order="dir13", precision="fp32"),
                   (0.7, (0.1, 0, 0), 1.0), 3),
    "tet_positivity_fp32": (dict(n=(4, 2, 2), lo=(0, 0, 0), hi=(1, 0.6, 0.4), patches=MIXED_PATCHES, distortion=0.2,
                                 tetrahedra=True),
                            MIXED_BCS, 0.1, (8, 8, 8),
                            dict(sweep_blocks=3, positivity_limiter=True, boundary_iterations=4, precision="fp32"),
                            (0.7, (0.1, 0, 0), 1.0), 3),
    "maxwell_wall_fp64": (dict(n=(4, 3, 2), lo=(0, 0, 0), hi=(1, 0.6, 0.4),
                               patches=["inlet", "outlet", "wall", "wall", "wall", "wall"], distortion=0.0),
                          [("inlet", "pressure_inlet", dict(T=1.0, p=1.1)), ("outlet", "pressure_outlet", dict(p=0.5)),
                           ("wall", "diffuse_wall", dict(T=1.0, alpha=0.8))],
                          0.2, (8, 8, 8), dict(sweep_blocks=2, precision="fp64"), (0.8, (0.05, 0, 0), 1.0), 3),
    "mass_flow_inlet_fp64": (dict(n=(6, 2, 2), lo=(0, 0, 0), hi=(1.5, 0.5, 0.5),
                                  patches=["inlet", "outlet", "wall", "wall", "wall", "wall"], distortion=0.1),
                             [("inlet", "mass_flow_inlet", dict(T=1.0, p=1.0, mdot=0.05)),
                              ("outlet", "pressure_outlet", dict(p=0.4)), ("wall", "diffuse_wall", dict(T=1.0))],
                             0.3, (8, 8, 8), dict(sweep_blocks=2, precision="fp64"), (0.8, (0.1, 0, 0), 1.0), 4),
    "vacuum_tube_fp64": (dict(n=(6, 2, 2), lo=(0, 0, 0), hi=(1.5, 0.5, 0.5),
                              patches=["inlet", "outlet", "wall", "wall", "wall", "wall"], distortion=0.1),
                         [("inlet", "pressure_inlet", dict(T=1.0, p=1.0)), ("outlet", "vacuum", {}),
                          ("wall", "diffuse_wall", dict(T=1.0))],
                         0.3, (8, 8, 8), dict(sweep_blocks=2, precision="fp64", velocity_chunk=128),
                         (0.6, (0.1, 0, 0), 1.0), 3),
}


def host_arrays(case: ref.RefCase) -> dict:
    """Host-side data of the kinetic host loop (kinetic_solver.cpp) in internal numbering."""
    return dict(ref.host_arrays(case))


def inflow_for(case: ref.RefCase) -> np.ndarray:
    """A fixed, physically plausible inflow table per boundary face (scale, rho, ux, uy, uz, T)."""
    s = case.setup
    out = np.zeros((s.n_bfaces, 6))
    out[:, 5] = 1.0  # InflowState{} default (src/kinetic/kinetic_backend.hpp:45-50): scale 0, rho 0, T 1
    for b in range(s.n_bfaces):
        pi = s["bface_patch"][b]
        kind = case.patch_int[pi, 0]
        T, p, ux, uy, uz = case.patch_dbl[pi, :5]
        if kind in (0, 5):  # walls: unit density, rho_Gamma as scale
            out[b] = (0.9, 1.0, ux, uy, uz, T)
        elif kind == 1:  # pressure boundary: W_b
            Tb = T if T > 0 else 1.0
            out[b] = (1.0, p / Tb, 0.05, 0.0, 0.0, Tb)
    return out


def run_case(name, mesh_kw, bcs, Kn, nv, kinetic, init, iterations) -> dict:
    mesh = ref.RefMesh.box(**mesh_kw)
    spec = ref.case_spec(bcs, Kn=Kn, nv=nv, kinetic=kinetic)
    case = ref.RefCase(mesh, spec)
    s = case.setup
    out = {}
    out.update(s.to_npz_dict())
    out.update(host_arrays(case))
    # target mass flow per patch (nondimensional, inflow positive; PatchCondition::target_mass_flow,
    # src/kinetic/kinetic_setup.cpp:372): the mass_flow_inlet's given value, patches in order of first appearance
    names = list(dict.fromkeys(mesh_kw["patches"]))
    targets = {patch: o.get("mdot", 0.0) for patch, typ, o in bcs if typ == "mass_flow_inlet"}
    out["host.patch_target"] = np.array([targets.get(n, 0.0) for n in names])
    nc, nb = s.n_cells, s.n_bfaces
    # --- operation sequence on the reference CpuBackend -------------------------------------------------------
    rng = np.random.default_rng(2026)
    st = np.column_stack([init[0] * (1 + 0.1 * rng.random(nc)), init[1][0] + 0.05 * rng.random(nc),
                          0.02 * rng.standard_normal(nc), 0.02 * rng.standard_normal(nc),
                          init[2] * (1 + 0.05 * rng.random(nc))])
    be = case.backend
    be.set_equilibrium(st)
    out["op.states"] = st
    out["op.moments0"] = be.compute_moments().copy()
    be.update_cell_params()
    out["op.deq0"] = np.array(be.deq_counts())
    inflow = inflow_for(case)
    out["op.inflow"] = inflow
    be.set_inflow(inflow)
    out["op.bsums0"] = be.boundary_sums().copy()
    out["op.res1"] = be.sweep().copy()
    out["op.f1"] = be.get_distribution().copy()
    out["op.res2"] = be.sweep().copy()
    m2 = be.compute_moments().copy()
    out["op.moments2"] = m2
    wh = m2[:, [0, 1, 2, 3, 4]].copy()
    wn = wh.copy()
    wn[:, 0] *= 1.02
    wn[:, 4] *= 1.01
    wn[:, 1] += 0.01
    wn[min(4, nc - 1), 1] = 2.5  # one strongly shifted cell so the negativity rule triggers
    replaced, flags = be.gsis_correction(wh, wn)
    out["op.w_half"], out["op.w_new"] = wh, wn
    out["op.replaced"] = np.array([replaced])
    out["op.flags"] = flags
    out["op.f3"] = be.get_distribution().copy()
    offs, oth = s["csr_offsets"], s["csr_other"]
    cells, ents = [], []
    for c in range(nc):
        for e in range(offs[c], offs[c + 1]):
            if oth[e] >= 0:
                cells.append(c)
                ents.append(e)
    out["op.face_cells"] = np.array(cells, np.int32)
    out["op.face_entries"] = np.array(ents, np.int32)
    out["op.face_flux"] = be.internal_face_mass_flux(cells, ents)
    # --- reference KineticSolver --------------------------------------------------------------------------------
    case.init_uniform(init[0], init[1], init[2])
    infos = [case.sweep() for _ in range(iterations)]
    out["solver.init"] = np.array([init[0], *init[1], init[2]])
    out["solver.infos"] = np.array(infos)
    out["solver.patch_mass_flow"] = case.patch_mass_flow()
    out["solver.moments"] = case.moments()
    fp, fm, fs = case.boundary_fluxes()
    out["solver.F_plus"], out["solver.F_minus"], out["solver.face_state"] = fp, fm, fs
    out["solver.f"] = case.distribution()
    # section mass flows (KineticSolver::section_mass_flow): x cuts across the box, one outside it, one y cut
    out["solver.section_x"] = np.array(SECTION_X)
    out["solver.section_flow_x"] = case.section_mass_flow(SECTION_X, axis=0)
    out["solver.section_y"] = np.array(SECTION_Y)
    out["solver.section_flow_y"] = case.section_mass_flow(SECTION_Y, axis=1)
    out["meta.name"] = np.array(name)
    return out


# Converged runs (tests/golden/converged/<name>.npz): the reference KineticSolver iterated from a uniform state
# until its residual falls below `tol`. Only the setup, the per-iteration history and the converged macroscopic
# fields are stored (f alone would be 22 MB for the slab).
# The planar Couette slab: x in [0, 1] in 200 cells, one cell thick with periodic y sides (the wall motion
# direction) and symmetry z sides; diffuse walls at T = 1 moving along y at -+0.1 most-probable speeds
# (u = -+0.1 sqrt(2) in units of sqrt(R T0)); delta_rp = 1, omega = 0.81, the reference's uniform midpoint 24^3
# grid on [-5, 5]^3, FP64, default CIS settings, residual 1e-8.
_U_WALL = float(0.1 * np.sqrt(2.0))
CONVERGED = {
    "couette_slab_200": (dict(n=(200, 1, 1), lo=(0, 0, 0), hi=(1, 1 / 200, 1 / 200),
                              patches=["wall_left", "wall_right", "sym_y", "sym_y", "sym_z", "sym_z"]),
                         [("wall_left", "diffuse_wall", dict(T=1.0, u=(0.0, -_U_WALL, 0.0))),
                          ("wall_right", "diffuse_wall", dict(T=1.0, u=(0.0, _U_WALL, 0.0))),
                          ("sym_y", "periodic_slab", {}), ("sym_z", "symmetry", {})],
                         dict(delta_rp=1.0, omega=0.81, nv=(24, 24, 24)), dict(precision="fp64"),
                         (1.0, (0.0, 0.0, 0.0), 1.0), 1e-8, 3000),
}


def run_converged(name, mesh_kw, bcs, conditions, kinetic, init, tol, max_iterations) -> dict:
    mesh = ref.RefMesh.box(**mesh_kw)
    spec = ref.case_spec(bcs, kinetic=kinetic, **conditions)
    case = ref.RefCase(mesh, spec)
    out = {}
    out.update(case.setup.to_npz_dict())
    out.update(host_arrays(case))
    case.init_uniform(init[0], init[1], init[2])
    infos = []
    while len(infos) < max_iterations:
        infos.append(case.sweep())
        if len(infos) > 1 and infos[-1][6] < tol:
            break
    out["solver.init"] = np.array([init[0], *init[1], init[2]])
    out["solver.tol"] = np.array(tol)
    out["solver.infos"] = np.array(infos)
    out["solver.patch_mass_flow"] = case.patch_mass_flow()
    out["solver.moments"] = case.moments()
    fp, fm, fs = case.boundary_fluxes()
    out["solver.F_plus"], out["solver.F_minus"], out["solver.face_state"] = fp, fm, fs
    out["meta.name"] = np.array(name)
    return out


def main(names=None):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    for name, args in CASES.items():
        if names and name not in names:
            continue
        data = run_case(name, *args)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB")
    for name, args in CONVERGED.items():
        if names and name not in names:
            continue
        data = run_converged(name, *args)
        os.makedirs(os.path.join(HERE, "converged"), exist_ok=True)
        path = os.path.join(HERE, "converged", f"{name}.npz")
        np.savez_compressed(path, **data)
        print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB, {len(data['solver.infos'])} iterations")


if __name__ == "__main__":
    main(sys.argv[1:])
