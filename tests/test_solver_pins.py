"""Solver-level known answers of the reference's own kinetic tests, on this repository's set-up builder and host loop
(gsis_sim_b200.kinetic_setup, gsis_sim_b200.solver) with the CPU oracle as the backend:

* sweep orderings and inner-sweep settings converge to the same solution (tests/kinetic/test_kinetic_phase5.cpp:
  200-239): block / octant / 13-direction orders, 1-3 inner sweeps with and without wall refresh, 1-3 block passes;
* symmetry and periodic slab sides give the same heat conduction (tests/kinetic/test_kinetic_cpu.cpp:142-176);
* Couette flow between walls moving at -+0.3 is antisymmetric, with a slip at the walls
  (tests/kinetic/test_kinetic_cpu.cpp:178-199).

The reference runs them with its test gas (omega = 0.66, tests/kinetic/kinetic_test_cases.cpp:9-32), 10^3
velocities on [-5, 5]^3 and its default FP32 precision; here FP64. Its tolerances are kept. The distorted box of the
ordering test is an undistorted one here (this repository's box mesher has no distortion)."""
import numpy as np
import pytest

from gsis_sim_b200 import kinetic_setup as ks
from gsis_sim_b200.mesh import box_mesh
from gsis_sim_b200.solver import KineticSolver

SLAB = ("wall_left", "wall_right", "sym_y", "sym_y", "sym_z", "sym_z")
RHO, UX, UY, UZ, T = 0, 1, 2, 3, 4
QX = 12
SXY = 9


def solve(mesh, bcs, Kn, iterations, **kinetic):
    from oracle.kinetic_oracle import OracleBackend

    params = ks.KineticParams(precision="fp64", **kinetic)
    setup, host = ks.build_kinetic_setup(mesh, ks.Gas(omega=0.66), ks.Conditions(L_ref=1.0, T0=273.15, Kn=Kn), bcs,
                                         ks.VelocityGrid(n=(10, 10, 10)), params)
    sol = KineticSolver(setup, host, OracleBackend(setup))
    sol.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
    eps = 1.0
    for _ in range(iterations):
        eps = sol.prepare().epsilon
        sol.sweep()
    return sol.moments(), eps  # original cell numbering


def cis(order, inner, wall, passes):
    return dict(sweep_order=order, inner_sweeps=inner, inner_wall_update=wall, block_passes=passes)


def test_sweep_orderings_and_inner_sweeps_converge_to_the_same_solution():
    mesh = box_mesh((6, 3, 3), (0.0, 0.0, 0.0), (1.2, 0.6, 0.6), ("inlet", "outlet", "wall", "wall", "wall", "wall"))
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("outlet", "vacuum"), ks.BC("wall", "diffuse_wall")]
    a, eps = solve(mesh, bcs, 0.3, 400, sweep_blocks=2, **cis("block", 1, False, 1))
    assert eps < 1e-6
    variants = [cis("octant", 1, False, 1), cis("dir13", 1, False, 1), cis("block", 3, True, 1),
                cis("octant", 2, False, 1), cis("octant", 1, False, 3), {}]  # {}: the default (strong) settings
    for v in variants:
        b, eps = solve(mesh, bcs, 0.3, 300, sweep_blocks=2, **v)
        assert eps < 1e-6, v
        np.testing.assert_allclose(b[:, RHO], a[:, RHO], rtol=2e-5, atol=0, err_msg=str(v))
        np.testing.assert_allclose(b[:, T], a[:, T], rtol=2e-5, atol=0, err_msg=str(v))
        np.testing.assert_allclose(b[:, UX], a[:, UX], rtol=0, atol=2e-5, err_msg=str(v))


def test_symmetry_and_periodic_slab_give_the_same_heat_conduction():
    mesh = box_mesh((8, 1, 1), (0.0, 0.0, 0.0), (1.0, 0.125, 0.125), SLAB)

    def run(side):
        bcs = [ks.BC("wall_left", "diffuse_wall", T=0.9), ks.BC("wall_right", "diffuse_wall", T=1.1),
               ks.BC("sym_y", side), ks.BC("sym_z", side)]
        return solve(mesh, bcs, 0.2, 150, sweep_blocks=1)[0]

    a, b = run("symmetry"), run("periodic_slab")
    x = np.argsort(mesh_x(mesh))
    np.testing.assert_allclose(a[:, T], b[:, T], rtol=2e-5, atol=0)
    np.testing.assert_allclose(a[:, RHO], b[:, RHO], rtol=2e-5, atol=0)
    np.testing.assert_allclose(a[:, QX], b[:, QX], rtol=2e-3, atol=0)
    assert np.max(np.abs(a[:, UY])) < 1e-6 and np.max(np.abs(b[:, UZ])) < 1e-6
    # heat flows from the hot right wall to the cold left one (q_x < 0), nearly uniform over 8 cells
    q = a[x, QX]
    assert q.max() < 0.0 and q.max() - q.min() < 0.1 * abs(q.min())


def test_couette_flow_with_periodic_sides_is_antisymmetric():
    mesh = box_mesh((8, 1, 1), (0.0, 0.0, 0.0), (1.0, 0.125, 0.125), SLAB)
    bcs = [ks.BC("wall_left", "diffuse_wall", u=(0.0, -0.3, 0.0)), ks.BC("wall_right", "diffuse_wall", u=(0.0, 0.3, 0.0)),
           ks.BC("sym_y", "periodic_slab"), ks.BC("sym_z", "symmetry")]
    m = solve(mesh, bcs, 0.2, 150, sweep_blocks=1)[0][np.argsort(mesh_x(mesh))]
    np.testing.assert_allclose(m[:, UY], -m[::-1, UY], rtol=0, atol=2e-5)
    np.testing.assert_allclose(m[:, T], m[::-1, T], rtol=0, atol=2e-5)
    assert np.all(m[:, SXY] < 0.0)  # P_xy < 0: the left wall moves to -y, the right one to +y
    assert 0.0 < m[-1, UY] < 0.3  # slip at the wall


def mesh_x(mesh):
    """x of the cell centres of an axis-aligned box mesh in original cell order."""
    from gsis_sim_b200.mesh import compute_geometry

    return compute_geometry(mesh).cell_center[:, 0]


@pytest.mark.parametrize("side", ["symmetry", "periodic_slab"])
def test_slab_sides_build(side):
    mesh = box_mesh((8, 1, 1), (0.0, 0.0, 0.0), (1.0, 0.125, 0.125), SLAB)
    bcs = [ks.BC("wall_left", "diffuse_wall"), ks.BC("wall_right", "diffuse_wall"), ks.BC("sym_y", side),
           ks.BC("sym_z", side)]
    setup, host = ks.build_kinetic_setup(mesh, ks.Gas(omega=0.66), ks.Conditions(Kn=0.2), bcs,
                                         ks.VelocityGrid(n=(10, 10, 10)), ks.KineticParams(precision="fp64"))
    assert setup.n_cells == 8 and setup.nv == 1000


def _solver(mesh, bcs, grid, Kn=0.5, **kinetic):
    from oracle.kinetic_oracle import OracleBackend

    params = ks.KineticParams(precision="fp64", **kinetic)
    setup, host = ks.build_kinetic_setup(mesh, ks.Gas(omega=0.66), ks.Conditions(L_ref=1.0, T0=273.15, Kn=Kn), bcs,
                                         grid, params)
    return KineticSolver(setup, host, OracleBackend(setup))


@pytest.mark.parametrize("fallback", ["collisionless", "continuous"])
def test_cells_the_grid_cannot_hold_become_collisionless_and_skip_the_correction(fallback):
    """tests/kinetic/test_kinetic_phase5.cpp:264-321: on a grid with unit spacing (points +-0.5, +-1.5, ...) cell 0
    holds a distribution on a few points, with negative values, whose temperature 0.05 is below the lowest one a
    non-negative distribution on the grid can have at its velocity, so the discrete equilibrium does not exist."""
    mesh = box_mesh((2, 1, 1), (0.0, 0.0, 0.0), (1.0, 0.5, 0.5), ("inlet", "outlet", "wall", "wall", "wall", "wall"))
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("outlet", "vacuum"), ks.BC("wall", "diffuse_wall")]
    grid = ks.VelocityGrid(n=(12, 12, 12), lo=(-6.0,) * 3, hi=(6.0,) * 3)
    s = _solver(mesh, bcs, grid, deq_fallback=fallback)
    xs = [grid.axis(a) for a in range(3)]
    # grid order: x fastest
    X, Y, Z = (np.meshgrid(*xs, indexing="ij")[a].transpose(2, 1, 0).ravel() for a in range(3))
    nv = X.size
    f = np.zeros((2, nv))
    f[1] = (2 * np.pi) ** -1.5 * np.exp(-0.5 * (X * X + Y * Y + Z * Z))
    ax = np.where(np.abs(X - 1.5) < 1e-9, 1.1, np.where((np.abs(X - 0.5) < 1e-9) | (np.abs(X - 2.5) < 1e-9), -0.05, 0.0))
    by = np.where((np.abs(Y - 0.5) < 1e-9) | (np.abs(Y - 1.5) < 1e-9), 0.5, 0.0)
    cz = np.where(np.abs(Z - 0.5) < 1e-9, 1.0, 0.0)
    f[0] = ax * by * cz  # the uniform weight is 1
    s.set_distribution(f)
    info = s.prepare()
    assert info.deq_failed == 1
    m = s.moments()
    wh = m[:, :5].copy()
    wn = wh.copy()
    wn[:, 0] *= 1.02
    replaced = s.apply_gsis_correction(wh, wn)
    m2 = s.moments()
    assert abs(m2[1, 0] / wn[1, 0] - 1.0) < 1e-6  # the equilibrium cell is corrected either way
    d0 = np.max(np.abs(s.distribution()[0] - f[0]))
    if fallback == "collisionless":
        assert replaced == 1 and s.replaced[0] == 1
        assert d0 == 0.0  # f of the collisionless cell is left as it is
        s.sweep()
        assert np.all(np.isfinite(s.distribution()))
    else:
        assert d0 > 0.0  # corrected with the continuous Maxwellian


def test_cell_pressure_reconstruction_changes_the_inflow():
    """tests/kinetic/test_kinetic_phase5.cpp:323-371: with a density gradient along x, the inlet's incoming mass flux
    F- differs between the limited reconstruction of W_b and the cell state."""
    mesh = box_mesh((4, 1, 1), (0.0, 0.0, 0.0), (1.0, 0.25, 0.25), ("inlet", "outlet", "side", "side", "side", "side"))
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("outlet", "vacuum"), ks.BC("side", "periodic_slab")]
    grid = ks.VelocityGrid(n=(16, 16, 16), lo=(-8.0,) * 3, hi=(8.0,) * 3)
    x = mesh_x(mesh)
    w = np.column_stack([1.0 - 0.6 * x, 0.2 + 0.3 * x, np.zeros_like(x), np.zeros_like(x), np.ones_like(x)])
    fm = []
    for mode in ("limited", "cell"):
        s = _solver(mesh, bcs, grid, equilibrium="continuous", pressure_boundary_reconstruction=mode)
        s.initialize_equilibrium(w)
        s.prepare()
        _, F_minus, _ = s.boundary_fluxes()
        fm.append(F_minus[0, 0])  # boundary face 0: the inlet, the first patch
    assert abs(fm[0] - fm[1]) > 1e-4 * abs(fm[1])


def test_closed_domain_keeps_total_mass_and_walls_have_zero_net_mass_flux():
    """tests/kinetic/test_kinetic_cpu.cpp:99-139: a box closed by a hot, a cold and moving diffuse walls."""
    mesh = box_mesh((5, 3, 2), (0.0, 0.0, 0.0), (1.0, 0.6, 0.4), ("hot", "cold", "wall", "wall", "wall", "wall"))
    bcs = [ks.BC("hot", "diffuse_wall", T=1.3), ks.BC("cold", "diffuse_wall", T=0.8),
           ks.BC("wall", "diffuse_wall", T=1.0, u=(0.2, 0.0, 0.0))]
    s = _solver(mesh, bcs, ks.VelocityGrid(n=(10, 10, 10)), Kn=0.3, sweep_blocks=3)
    assert s.h.closed_domain
    s.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
    total0 = float(np.sum(s.volume))
    max_scale_dev = 0.0
    for _ in range(15):
        max_scale_dev = max(max_scale_dev, abs(s.prepare().mass_scale - 1.0))
        s.sweep()
    s.prepare()
    total = float(np.sum(s.moments_[:, 0] * s.volume))
    assert abs(total / s.mass_target - 1.0) < 1e-12
    assert abs(s.mass_target / total0 - 1.0) < 1e-4
    assert max_scale_dev < 1e-2
    F_plus, F_minus, _ = s.boundary_fluxes()
    assert np.max(np.abs(F_plus[:, 0] + F_minus[:, 0])) < 1e-6 * np.max(np.abs(F_plus[:, 0]))


def test_discrete_equilibrium_keeps_cold_states_conservative():
    """tests/kinetic/test_kinetic_phase5.cpp:135-198: on a grid with unit spacing the moments of a T = 0.3 Maxwellian
    are 0.3% off; the discrete equilibrium initialises and corrects to the given states to 2e-6."""
    mesh = box_mesh((3, 2, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 0.5), ("inlet", "outlet", "wall", "wall", "wall", "wall"))
    bcs = [ks.BC("inlet", "pressure_inlet", T=0.3, p=0.3), ks.BC("outlet", "vacuum"),
           ks.BC("wall", "diffuse_wall", T=0.3)]
    grid = ks.VelocityGrid(n=(12, 12, 12), lo=(-6.0,) * 3, hi=(6.0,) * 3)
    c = np.arange(6, dtype=float)
    w = np.column_stack([0.8 + 0.1 * c, 0.4 - 0.1 * c, np.full(6, 0.15), np.full(6, -0.05), 0.25 + 0.02 * c])
    wn = np.column_stack([w[:, 0] * 1.03, w[:, 1] + 0.05, np.full(6, 0.1), np.zeros(6), w[:, 4] * 0.97])

    def error(m, ref):
        return max(np.max(np.abs(m[:, 0] / ref[:, 0] - 1.0)), np.max(np.abs(m[:, 4] / ref[:, 4] - 1.0)),
                   np.max(np.abs(m[:, 1] - ref[:, 1]) / np.sqrt(ref[:, 4])))

    cont = _solver(mesh, bcs, grid, equilibrium="continuous")
    cont.initialize_equilibrium(w)
    assert error(cont.moments(), w) > 1e-3
    disc = _solver(mesh, bcs, grid, equilibrium="discrete")
    assert disc.discrete_eq
    disc.initialize_equilibrium(w)
    assert error(disc.moments(), w) < 2e-6
    disc.sweep()
    half = disc.moments()
    disc.apply_gsis_correction(half[:, :5], wn)
    assert error(disc.moments(), wn) < 2e-6
    info = disc.prepare()
    assert info.deq_corrected == 6 and info.deq_failed == 0


def test_boundary_iterations_solve_the_lag_without_changing_the_distribution():
    """tests/kinetic/test_kinetic_cpu.cpp:511-560: boundary_iterations = 8 in one prepare equals eight prepares
    (each invalidated by a zero GSIS correction, which leaves f as it is) of boundary_iterations = 1, and the repeated
    boundary update changes the inflow. (The reference runs it on distorted tetrahedra; this box is hexahedral.)"""
    mesh = box_mesh((3, 2, 2), (0.0, 0.0, 0.0), (3.0, 2.0, 2.0), ("inlet", "outlet", "wall", "wall", "wall", "wall"))
    bcs = [ks.BC("inlet", "pressure_inlet"), ks.BC("outlet", "vacuum"), ks.BC("wall", "diffuse_wall")]
    grid = ks.VelocityGrid(n=(10, 10, 10))
    a = _solver(mesh, bcs, grid, sweep_blocks=1, positivity_limiter=True, boundary_iterations=1)
    b = _solver(mesh, bcs, grid, sweep_blocks=1, positivity_limiter=True, boundary_iterations=8)
    from gsis_sim_b200.mesh import compute_geometry

    xc = compute_geometry(mesh).cell_center
    w = np.column_stack([0.8 + 0.15 * xc[:, 0], 0.05 + 0.03 * xc[:, 1], 0.02 * xc[:, 2], np.zeros(len(xc)),
                         0.9 + 0.04 * xc[:, 2]])
    a.initialize_equilibrium(w)
    b.initialize_equilibrium(w)
    f = a.distribution()
    first = a.boundary_fluxes()
    m = a.moments()
    repeated = first
    for _ in range(1, 8):
        a.apply_gsis_correction(m[:, :5], m[:, :5])
        repeated = a.boundary_fluxes()
    batched = b.boundary_fluxes()
    assert np.array_equal(a.distribution(), f) and np.array_equal(b.distribution(), f)
    np.testing.assert_allclose(batched[0], repeated[0], rtol=0, atol=1e-12)
    np.testing.assert_allclose(batched[1], repeated[1], rtol=0, atol=1e-12)
    assert np.max(np.abs(first[1] - repeated[1])) > 1e-6
    # the fixed-f boundary update converges: 64 updates as the reference, 8 are much closer to it than 1
    reference = repeated
    for _ in range(8, 64):
        a.apply_gsis_correction(m[:, :5], m[:, :5])
        reference = a.boundary_fluxes()
    error1 = np.max(np.abs(first[1] - reference[1]))
    error8 = np.max(np.abs(batched[1] - reference[1]))
    assert error8 < 0.1 * error1
    assert np.array_equal(a.distribution(), f)
