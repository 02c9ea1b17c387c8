"""The planar Couette slab at full size: 200 cells across x in [0, 1], diffuse walls at T = 1 moving along y at
-+0.1 most-probable speeds, delta_rp = 1, omega = 0.81, the uniform 24^3 grid on [-5, 5]^3 (13,824 velocities),
FP64, the reference's default CIS settings, iterated from rest to residual 1e-8.

Golden values: the reference KineticSolver (src/kinetic/kinetic_solver.cpp) run to convergence
(tests/golden/converged/couette_slab_200.npz, made by tests/golden/make_golden.py). The CPU tests pin the fixture
by the physics of a steady planar Couette flow and check the first CIS iteration of the host loop on the CPU oracle
against the reference's; tests/test_gpu_couette_slab.py runs the whole solve on the B200 backend.

Independent check: the reference's 1-D solver ref1d on the same problem (tests/golden/converged/
couette_slab_ref1d.npz, made by tests/golden/make_ref1d.py), with the same 24-point x velocity grid (the solvers then
differ only in their discretisation in x) and with its velocity-converged Gauss-Legendre grid (the physical answer;
the 24^3 grid's velocity error is 0.2% on the shear stress and 2% on the flow velocity)."""
import os

import numpy as np
import pytest

from gsis_sim_b200 import abi
from gsis_sim_b200.kinetic_setup import HostSetup
from gsis_sim_b200.solver import KineticSolver
from tests import common

FIXTURE = os.path.join(common.GOLDEN, "converged", "couette_slab_200.npz")
REF1D = os.path.join(common.GOLDEN, "converged", "couette_slab_ref1d.npz")
# moments order of the backend (src/kinetic/kinetic_types.hpp:107-109)
RHO, UX, UY, UZ, T, P, SXX, SYY, SZZ, SXY, SYZ, SXZ, QX, QY, QZ = range(15)


def load():
    z = np.load(FIXTURE, allow_pickle=False)
    return z, abi.SetupArrays.from_npz(z), HostSetup.from_npz(z)


def x_original(z):
    """x of the cell centres in the original cell numbering (the solver's moments are in that numbering, the host
    arrays of the fixture in the internal one)."""
    x = np.empty(len(z["host.cell_center"]))
    x[z["host.cell_new_to_old"]] = z["host.cell_center"][:, 0]
    return x


def x_order(z):
    """Original cell numbers sorted by the cell centre's x."""
    return np.argsort(x_original(z), kind="stable")


def test_fixture_is_a_converged_couette_flow():
    z, setup, _ = load()
    infos = z["solver.infos"]
    assert setup.n_cells == 200 and setup.nv == 24 ** 3
    assert infos[-1][6] < float(z["solver.tol"]) <= infos[-2][6]
    m = z["solver.moments"][x_order(z)]
    # steady planar flow: no mass flux across the slab, uniform shear stress, the walls drag the gas along y
    assert np.max(np.abs(m[:, RHO] * m[:, UX])) < 1e-6
    # (the cell-centred P_xy of the wall cells differs from the interior by a few 1e-4: the one-sided
    # reconstruction at the wall; away from the walls it is uniform to the discretisation's rounding)
    sxy = m[:, SXY]
    assert np.all(sxy < 0) and np.ptp(sxy) < 1e-3 * abs(sxy.mean())
    assert np.ptp(sxy[5:-5]) < 1e-5 * abs(sxy.mean())
    assert np.all(np.diff(m[:, UY]) > 0) and abs(m[:, UY]).max() < 0.1 * np.sqrt(2.0)
    # mirror symmetry about the mid-plane x = 1/2: rho, T even; u_y odd
    for k, sign in ((RHO, 1), (T, 1), (P, 1), (UY, -1), (SXY, 1)):
        assert common.max_rel(m[:, k], sign * m[::-1, k]) < 1e-6, k
    # closed domain: the walls carry no net mass
    assert np.max(np.abs(z["solver.patch_mass_flow"])) < 1e-8


def test_first_iterations_of_the_host_loop_on_the_oracle():
    from oracle.kinetic_oracle import OracleBackend

    z, setup, host = load()
    sol = KineticSolver(setup, host, OracleBackend(setup))
    init = z["solver.init"]
    sol.initialize_uniform(init[0], init[1:4], init[4])
    for ref in z["solver.infos"][:4]:
        info = sol.sweep()
        assert info.iteration == ref[0]
        assert abs(info.residual - ref[6]) <= 1e-9 * ref[6]
        assert abs(info.total_mass - ref[8]) <= 1e-12 * ref[8]


# field -> (moment column, tolerance against ref1d on the 24-point grid, against ref1d velocity-converged), both
# relative to the field's largest magnitude over the slab
REF1D_FIELDS = {"rho": (RHO, 1e-5, 1e-4), "uy": (UY, 5e-4, 3e-2), "T": (T, 2e-5, 1e-4), "qx": (QX, 3e-3, 5e-2),
                "qy": (QY, 3e-3, 1e-1), "Pxy": (SXY, 1e-3, 5e-3)}


def check_against_ref1d(z, moments):
    """Fields of a converged slab (moments in the original cell numbering) against ref1d, interpolated to the cell
    centres."""
    r = np.load(REF1D, allow_pickle=False)
    order = x_order(z)
    xc = x_original(z)[order]
    m = moments[order]
    for name, (k, tol_mid, tol_gl) in REF1D_FIELDS.items():
        for grid, tol in (("mid24", tol_mid), ("gl", tol_gl)):
            ref = np.interp(xc, r[f"{grid}.x"], r[f"{grid}.{name}"])
            err = np.max(np.abs(m[:, k] - ref)) / np.max(np.abs(ref))
            assert err < tol, (name, grid, err)
    # away from the wall cells the shear stress agrees with ref1d's on the same velocity grid to 1e-4
    sxy = m[5:-5, SXY]
    assert np.max(np.abs(sxy - r["mid24.Pxy"].mean())) < 1e-4 * abs(r["mid24.Pxy"].mean())


def test_fixture_agrees_with_the_independent_1d_solver():
    z, _, _ = load()
    check_against_ref1d(z, z["solver.moments"])


@pytest.mark.parametrize("key", ["solver.moments", "solver.F_plus", "solver.F_minus"])
def test_fixture_fields_are_finite(key):
    z, _, _ = load()
    assert np.all(np.isfinite(z[key]))
