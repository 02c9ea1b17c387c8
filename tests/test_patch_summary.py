"""Per-patch SI flows (summarize_patches / KineticSolver.patch_summary) against the reference's own known answer
(tests/kinetic/test_kinetic_phase5c.cpp, "SI patch output separates central heat and transported energy"): with the
fluxes of a uniform state at unit density and temperature moving with u and carrying a heat flux q, a one-face patch
reports the mass, heat and total-energy flows into the domain and the force, each from its own part of the flux."""
import numpy as np

from gsis_sim_b200 import kinetic_setup as ks
from gsis_sim_b200.mesh import box_mesh, compute_geometry
from gsis_sim_b200.solver import KineticSolver, summarize_patches


def _case():
    mesh = box_mesh((1, 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), ("wall",) * 6)
    cond = ks.Conditions(L_ref=1.0, T0=273.15, Kn=0.5)
    setup, host = ks.build_kinetic_setup(mesh, ks.Gas(omega=0.66), cond, [ks.BC("wall", "diffuse_wall")],
                                         ks.VelocityGrid(n=(6, 6, 6)), ks.KineticParams(precision="fp64"))
    return mesh, setup, host, ks.derive_quantities(ks.Gas(omega=0.66), cond)


def test_si_patch_output_separates_central_heat_and_transported_energy():
    mesh, setup, host, d = _case()
    g = compute_geometry(mesh)
    ni = host.n_internal_faces
    nb = len(g.face_area) - ni
    L2 = host.length_scale ** 2
    u = np.array([0.3, -0.2, 0.1])
    q = np.array([0.07, -0.04, 0.02])
    area = g.face_area[ni:] / L2
    normal = g.face_normal[ni:]
    F_plus = np.zeros((nb, 5))
    for b in range(nb):
        un = u @ normal[b]
        mom = u * un + normal[b]
        F_plus[b] = np.array([un, *mom, (2.5 + 0.5 * u @ u) * un + q @ normal[b]]) * area[b]
    face_state = np.tile([1.0, *u, 1.0], (nb, 1))
    mass_flux = d["ref_density"] * d["ref_velocity"]
    heat_flux = d["ref_pressure"] * d["ref_velocity"]
    for b in range(nb):
        p = summarize_patches(["wall"], ["diffuse_wall"], [[b]], area, normal, F_plus, np.zeros((nb, 5)), face_state,
                              length=host.length_scale, ref_pressure=host.ref_pressure,
                              ref_velocity=host.ref_velocity)[0]
        un = u @ normal[b]
        assert np.isclose(p["mass_flow_kg_s"], -un * area[b] * mass_flux * L2, rtol=1e-12)
        assert np.isclose(p["heat_flow_W"], -(q @ normal[b]) * area[b] * heat_flux * L2, rtol=1e-12, atol=1e-300)
        assert np.isclose(p["energy_flow_W"], -F_plus[b, 4] * heat_flux * L2, rtol=1e-12)
        mom = u * un + normal[b]
        assert np.allclose(p["force_N"], mom * area[b] * d["ref_pressure"] * L2, rtol=1e-12, atol=0)
        assert p["faces"] == 1 and np.isclose(p["face_T_nd"], 1.0) and np.allclose(p["face_u_nd"], u)


def test_patch_summary_of_a_closed_box_at_rest():
    from oracle.kinetic_oracle import OracleBackend

    _, setup, host, _ = _case()
    s = KineticSolver(setup, host, OracleBackend(setup))
    s.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
    (p,) = s.patch_summary()
    assert p["name"] == "wall" and p["type"] == "diffuse_wall" and p["faces"] == 6
    assert np.isclose(p["area_nd"], 6.0) and np.isclose(p["area_m2"], 6.0)
    # equilibrium at rest in a closed box: no net mass, heat or energy through the walls; the pressure forces cancel
    assert abs(p["mdot_nd"]) < 1e-12 and abs(p["heat_flow_W"]) < 1e-9 * host.ref_pressure * host.ref_velocity
    assert np.max(np.abs(p["force_N"])) < 1e-9 * host.ref_pressure
    assert np.isclose(p["face_rho_nd"], 1.0, rtol=1e-6) and np.isclose(p["face_T_nd"], 1.0, rtol=1e-6)
