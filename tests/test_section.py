"""Section cuts and the flow diagnostics around them (src/mesh/section_cut.cpp, src/kinetic/kinetic_output.cpp:39-76,
KineticSolver::section_mass_flow, src/kinetic/kinetic_solver.cpp:669-690), on the CPU oracle backend.

The analytic pins follow the reference's own section tests (tests/kinetic/test_kinetic_phase5c.cpp:88-186): a uniform
flowing equilibrium carries rho u_x times the cross-section through every cut to 1e-12; at a converged steady state
the section flows equal the inlet and outlet flows to 1e-7. The golden section flows of the reference solver are
checked in tests/test_solver_host.py."""
import math
import os

import numpy as np
import pytest

from gsis_sim_b200 import case, kinetic_setup as ks
from gsis_sim_b200 import section as sec
from gsis_sim_b200.mesh import box_mesh, compute_geometry
from gsis_sim_b200.solver import KineticSolver


def _solver(mesh, bcs, Kn, nv, **kp):
    from oracle.kinetic_oracle import OracleBackend

    setup, host = ks.build_kinetic_setup(mesh, ks.Gas(omega=0.81), ks.Conditions(L_ref=1.0, T0=273.15, Kn=Kn), bcs,
                                         ks.VelocityGrid(n=nv), ks.KineticParams(**kp))
    return KineticSolver(setup, host, OracleBackend(setup))


def test_parse_section_spec():
    s = sec.parse_section_spec("0, 2.5;5\t-1e-1  7.", "Z")
    assert s.axis == 2 and s.positions == [0.0, 2.5, 5.0, -0.1, 7.0]
    assert sec.parse_section_spec("", "y").empty() and sec.parse_section_spec(" ,; ").empty()
    assert sec.parse_section_spec("1, 1").positions == [1.0, 1.0]  # order and repeats kept
    for bad in ("1, x", "inf", "nan", "+1", "1e", "1.2.3"):
        with pytest.raises(sec.SectionError):
            sec.parse_section_spec(bad)
    with pytest.raises(sec.SectionError):
        sec.parse_section_spec("1", "w")
    assert [sec.section_axis_name(a) for a in range(3)] == ["x", "y", "z"]


def test_output_sections_from_case():
    with open(os.path.join(os.path.dirname(__file__), "golden", "case_channel", "channel.toml")) as fh:
        base = fh.read()
    try:
        cfg = case.parse_case_toml(base + '[output]\nmass_flow_sections = "0, 2.5, 5"\nmass_flow_section_axis = "z"\n')
    except case.CaseError as e:  # the minimal case above must satisfy the case rules
        pytest.fail(str(e))
    s = case.output_sections(cfg)
    assert s.axis == 2 and s.positions == [0.0, 2.5, 5.0]
    assert case.output_sections(case.parse_case_toml(base)).empty()
    with pytest.raises(case.CaseError, match="mass_flow_sectoins"):
        case.output_sections(case.parse_case_toml(base + '[output]\nmass_flow_sectoins = "1"\n'))
    with pytest.raises(case.CaseError):
        case.output_sections(case.parse_case_toml(base + '[output]\nmass_flow_sections = "1, x"\n'))


def test_mass_balance_and_flow_spread():
    b = sec.mass_balance([-2.0, 1.9, 0.0, 0.05])
    assert b.valid and b.inflow == 2.0 and math.isclose(b.outflow, 1.95) and math.isclose(b.imbalance, -0.025)
    assert not sec.mass_balance([0.0, 0.0]).valid and not sec.mass_balance([]).valid
    assert not sec.mass_balance([-1.0, math.nan]).valid
    assert math.isclose(sec.flow_spread([1.0, 1.1, 0.9]), 0.2)
    assert math.isnan(sec.flow_spread([1.0])) and math.isnan(sec.flow_spread([1.0, math.nan]))
    assert math.isnan(sec.flow_spread([1.0, -1.0]))


def test_cuts_of_an_aligned_box():
    m = box_mesh((8, 3, 2), (0, 0, 0), (1, 0.6, 0.4))
    g = compute_geometry(m)
    ni = m.n_internal
    cuts = sec.build_section_cuts(m.owner, m.neighbour, g.cell_center, g.face_center, g.face_normal, g.face_area,
                                  1.0, sec.SectionSpec(0, [0.37, 0.5, 0.0, 1.5]))
    for c in cuts[:2]:  # a plane of 3 x 2 faces between two cell layers
        assert len(c.faces) == 6 and np.all(c.sign == 1) and np.all(c.faces < ni)
        assert abs(c.area - 0.24) < 1e-12 and abs(c.projected_area - 0.24) < 1e-12
    assert abs(cuts[0].face_position - 0.375) < 1e-12 and abs(cuts[1].face_position - 0.5) < 1e-12
    for c in cuts[2:]:  # before / behind every cell centre: no faces
        assert len(c.faces) == 0 and c.area == 0.0 and c.face_position == c.position
    # the length scale divides positions and areas
    c2 = sec.build_section_cuts(m.owner, m.neighbour, g.cell_center * 2, g.face_center * 2, g.face_normal,
                                g.face_area * 4, 2.0, sec.SectionSpec(0, [0.37]))[0]
    assert np.array_equal(c2.faces, cuts[0].faces) and abs(c2.area - 0.24) < 1e-12
    with pytest.raises(sec.SectionError):
        sec.build_section_cuts(m.owner, m.neighbour, g.cell_center, g.face_center, g.face_normal, g.face_area,
                               0.0, sec.SectionSpec(0, [0.5]))
    with pytest.raises(sec.SectionError):
        sec.section_flow(cuts[0], np.zeros(3))


def test_uniform_flowing_equilibrium_section_flow():
    """tests/kinetic/test_kinetic_phase5c.cpp:88-121 (on an undistorted box)."""
    m = box_mesh((8, 3, 2), (0, 0, 0), (1, 0.6, 0.4), ("inlet", "outlet", "sym_y", "sym_y", "sym_z", "sym_z"))
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("outlet", "pressure_outlet", T=1.0, p=0.5),
           ks.BC("sym_y", "symmetry"), ks.BC("sym_z", "symmetry")]
    sol = _solver(m, bcs, 0.1, (8, 8, 8), precision="fp64", sweep_blocks=2)
    sol.initialize_uniform(0.8, (0.3, 0.0, 0.0), 1.1)
    spec = sec.SectionSpec(0, [0.37, 0.5, 0.63])
    flow = sol.section_mass_flow(spec)
    mom = sol.moments()
    rhou = mom[0, 0] * mom[0, 1]
    assert len(flow) == 3 and abs(rhou - 0.24) < 1e-6 * 0.24
    assert np.all(np.abs(flow - rhou * 0.24) <= 1e-12 * rhou * 0.24)
    g = compute_geometry(m)
    ref = sec.build_section_cuts(m.owner, m.neighbour, g.cell_center, g.face_center, g.face_normal, g.face_area,
                                 1.0, spec)
    for a, b in zip(sol.section_cuts(spec), ref):  # cuts on the internal numbering = cuts on the original mesh
        assert len(a.faces) == len(b.faces) and abs(a.area - b.area) < 1e-12 and abs(a.projected_area - 0.24) < 1e-12
    assert len(sol.section_mass_flow(sec.SectionSpec())) == 0


@pytest.mark.timeout(600)
def test_converged_section_flows_equal_boundary_flows():
    """tests/kinetic/test_kinetic_phase5c.cpp:123-159 (on an undistorted box): mid-way the boundary flows disagree;
    converged, inlet, outlet and section flows agree to 1e-7."""
    m = box_mesh((8, 2, 2), (0, 0, 0), (1, 0.25, 0.25), ("inlet", "outlet", "wall", "wall", "wall", "wall"))
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("outlet", "vacuum"), ks.BC("wall", "diffuse_wall")]
    sol = _solver(m, bcs, 0.2, (8, 8, 8), precision="fp64", sweep_blocks=1)
    sol.initialize_uniform(0.5, (0.0, 0.0, 0.0), 1.0)
    spec = sec.SectionSpec(0, [0.2, 0.5, 0.8])
    for _ in range(3):
        sol.sweep()
    mb = sec.mass_balance(sol.prepare().patch_mass_flow)
    assert mb.valid and abs(mb.imbalance) > 1e-3
    residual = 1.0
    for _ in range(1500):
        if residual <= 1e-12:
            break
        residual = sol.sweep().residual
    assert residual < 1e-10
    mb = sec.mass_balance(sol.prepare().patch_mass_flow)
    flow = sol.section_mass_flow(spec)
    assert mb.valid and mb.inflow > 0 and abs(mb.imbalance) < 1e-7
    assert np.all(np.abs(flow - mb.inflow) <= 1e-7 * mb.inflow)
    assert sec.flow_spread([mb.inflow, mb.outflow, *flow]) < 1e-7
