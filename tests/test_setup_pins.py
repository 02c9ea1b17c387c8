"""Set-up and solver known answers of the reference's own kinetic tests on this repository's builder and host loop:

* the velocity layout groups mirror orbits (tests/kinetic/test_kinetic_cpu.cpp:49-69);
* octant sweep directions group the velocity points (tests/kinetic/test_kinetic_phase5.cpp:241-262);
* a uniform equilibrium between pressure boundaries and walls at the same state is a fixed point of the CIS
  iteration (tests/kinetic/test_kinetic_cpu.cpp:71-97), with the C oracle as the backend (the B200 version on the
  full-size tube is tests/test_gpu_fullsize.py);
* the equilibrium initialisation reproduces the given macroscopic states (tests/kinetic/test_kinetic_cpu.cpp:
  275-306)."""
import numpy as np
import pytest

from gsis_sim_b200 import kinetic_setup as ks
from gsis_sim_b200.mesh import box_mesh
from gsis_sim_b200.solver import KineticSolver


def test_velocity_layout_groups_mirror_orbits():
    grid = ks.VelocityGrid(n=(6, 4, 8), lo=(-3.0, -2.0, -4.0), hi=(3.0, 2.0, 4.0))
    L = ks.velocity_layout(grid, [2, 0], np.zeros((0, 3)))
    assert L["orbit_size"] == 4 and L["axis_xor"] == [1, 0, 2]
    xi = L["xi"]
    p = np.arange(len(xi))
    q = p ^ L["axis_xor"][0]
    assert np.array_equal(xi[q, 0], -xi[p, 0]) and np.array_equal(xi[q, 1], xi[p, 1])
    r = p ^ L["axis_xor"][2]
    assert np.array_equal(xi[r, 2], -xi[p, 2])
    # without mirror axes (and no sweep directions) the storage order is the grid order
    L0 = ks.velocity_layout(grid, [], np.zeros((0, 3)))
    assert np.array_equal(L0["storage_to_grid"], p)
    # an axis whose range is not symmetric cannot mirror
    skew = ks.VelocityGrid(n=(4, 4, 4), lo=(-1.0, -2.0, -2.0), hi=(3.0, 2.0, 2.0))
    with pytest.raises(ValueError):
        ks.velocity_layout(skew, [0], np.zeros((0, 3)))


def test_octant_sweep_directions_group_the_velocity_points():
    d4 = ks.sweep_directions("octant")
    assert len(d4) == 4 and len(ks.sweep_directions("dir13")) == 13 and len(ks.sweep_directions("block")) == 0
    g = ks.sweep_direction_of(d4, np.array([[1.0, 0.2, 3.0], [-1.0, -0.2, -3.0], [1.0, -0.2, 3.0]]))
    assert g[0] == g[1] and g[0] != g[2]  # xi and -xi share a direction; the sign pattern decides it
    grid = ks.VelocityGrid(n=(6, 4, 4), lo=(-3.0, -2.0, -2.0), hi=(3.0, 2.0, 2.0))
    L = ks.velocity_layout(grid, [], d4)
    groups = ks.sweep_direction_of(d4, L["xi"])
    assert np.all(np.diff(groups) >= 0)
    assert len(np.unique(groups)) == 4 and np.count_nonzero(np.diff(groups)) == 3


def test_equilibrium_is_preserved():
    from oracle.kinetic_oracle import OracleBackend

    mesh = box_mesh((4, 3, 3), (0.0, 0.0, 0.0), (1.0, 0.8, 0.6), ("inlet", "outlet", "wall", "wall", "wall", "wall"))
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("outlet", "pressure_outlet", p=1.0),
           ks.BC("wall", "diffuse_wall", T=1.0)]
    # +-6: the truncation error of the discrete Maxwellian's moments is about 1e-8
    grid = ks.VelocityGrid(n=(12, 12, 12), lo=(-6.0,) * 3, hi=(6.0,) * 3)
    setup, host = ks.build_kinetic_setup(mesh, ks.Gas(omega=0.66), ks.Conditions(L_ref=1.0, T0=273.15, Kn=0.5), bcs,
                                         grid, ks.KineticParams(precision="fp64", sweep_blocks=2))
    s = KineticSolver(setup, host, OracleBackend(setup))
    s.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
    f0 = s.distribution()
    for _ in range(5):
        info = s.sweep()
    f1 = s.distribution()
    assert np.max(np.abs(f1 - f0)) < 2e-6 * f0.max()
    assert info.residual < 1e-8  # the reference asks < 1e-6 of its default FP32 run
    m = s.moments()
    assert np.max(np.abs(m[:, 0] - 1.0)) < 1e-5 and np.max(np.abs(m[:, 4] - 1.0)) < 1e-5
    assert np.max(np.abs(m[:, 1])) < 1e-5


def test_equilibrium_initialization_reproduces_the_macroscopic_state():
    """tests/kinetic/test_kinetic_cpu.cpp:275-306, with the C oracle as the backend."""
    from oracle.kinetic_oracle import OracleBackend

    mesh = box_mesh((3, 2, 2), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), ("inlet", "outlet", "wall", "wall", "wall", "wall"))
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("outlet", "vacuum"), ks.BC("wall", "diffuse_wall")]
    grid = ks.VelocityGrid(n=(16, 16, 16), lo=(-8.0,) * 3, hi=(8.0,) * 3)
    setup, host = ks.build_kinetic_setup(mesh, ks.Gas(omega=0.66), ks.Conditions(L_ref=1.0, T0=273.15, Kn=0.5), bcs,
                                         grid, ks.KineticParams(precision="fp64"))
    s = KineticSolver(setup, host, OracleBackend(setup))
    c = np.arange(12, dtype=float)
    w = np.column_stack([0.5 + 0.1 * c, 0.3 - 0.05 * c, np.full(12, 0.1), np.full(12, -0.2), 0.8 + 0.03 * c])
    s.initialize_equilibrium(w)
    m = s.moments()
    np.testing.assert_allclose(m[:, 0], w[:, 0], rtol=1e-6, atol=0)
    np.testing.assert_allclose(m[:, 1], w[:, 1], rtol=0, atol=1e-6)
    np.testing.assert_allclose(m[:, 3], w[:, 3], rtol=0, atol=1e-6)
    np.testing.assert_allclose(m[:, 4], w[:, 4], rtol=1e-5, atol=0)
    assert np.max(np.abs(m[:, 12])) < 1e-5 and np.max(np.abs(m[:, 9])) < 1e-5  # q_x, P_xy
