"""The GSIS coupling loop (gsis_sim_b200/gsis.py, GsisSolver::iterate of src/gsis/gsis_solver.cpp:168-277) on the CPU
oracle with stand-in macroscopic stages (the reference's PBC stage needs AMGCL, which is absent):
* eq. (59) against the reference's cell loop;
* a stage that returns W^{n+1/2} unchanged: the correction f - f^eq(W) + f^eq(W) changes f by rounding only, so a
  GSIS iteration is N_CIS CIS iterations;
* a stage that moves W: with the discrete equilibrium (the Newton solve active on this grid) the corrected f carries
  exactly the new conserved moments, so its (rho, u, T) equal the stage's output;
* the Kn damping of the correction."""
import math

import numpy as np
import pytest

from gsis_sim_b200 import gsis
from gsis_sim_b200.solver import KineticSolver, KineticSolverError
from tests.test_adjoint import channel_case


def _solver(**kw):
    from oracle.kinetic_oracle import OracleBackend

    setup, host = channel_case(**kw)
    return KineticSolver(setup, host, OracleBackend(setup))


class Identity:
    def solve_gsis_stage(self, stage):
        return stage.state


class Shift:
    """Moves every cell's state by a smooth field (a stand-in for the PBC stage's W^{n+1})."""

    def __init__(self, eps):
        self.eps = eps
        self.calls = 0

    def solve_gsis_stage(self, stage):
        self.calls += 1
        w = stage.state
        assert stage.moments.shape == (len(w), 15) and stage.F_plus.shape == stage.F_minus.shape
        assert stage.face_state.shape == stage.F_plus.shape
        k = np.arange(len(w))
        w[:, 0] *= 1.0 + self.eps * np.cos(k)
        w[:, 1] += self.eps * np.sin(k)
        w[:, 4] *= 1.0 - self.eps * np.cos(2 * k)
        return w


def test_relative_change_matches_the_cell_loop():
    rng = np.random.default_rng(1)
    n = 40
    a, b = rng.random((n, 5)) + 0.5, rng.random((n, 5)) + 0.5
    b[:, 1:4] *= 1e-3  # small velocities: the floor decides the velocity denominator
    V = rng.random(n) + 0.1
    num, den = [0.0] * 3, [0.0] * 3
    for c in range(n):
        num[0] += (a[c, 0] - b[c, 0]) ** 2 * V[c]
        den[0] += b[c, 0] ** 2 * V[c]
        num[1] += np.sum((a[c, 1:4] - b[c, 1:4]) ** 2) * V[c]
        den[1] += np.sum(b[c, 1:4] ** 2) * V[c]
        num[2] += (a[c, 4] - b[c, 4]) ** 2 * V[c]
        den[2] += b[c, 4] ** 2 * V[c]
    den[1] = max(den[1], 0.01 ** 2 * V.sum())
    r = gsis.relative_change(a, b, V, 0.01)
    ref = [math.sqrt(x / y) for x, y in zip(num, den)]
    assert abs(r.rho - ref[0]) <= 1e-14 * ref[0] and abs(r.u - ref[1]) <= 1e-14 * ref[1]
    assert abs(r.T - ref[2]) <= 1e-14 * ref[2] and r.epsilon == max(r.rho, r.u, r.T)
    assert gsis.relative_change(b, b, V, 0.01).epsilon == 0.0
    with pytest.raises(KineticSolverError):
        gsis.relative_change(a[:5], b, V, 0.01)


@pytest.mark.timeout(300)
def test_identity_stage_is_plain_cis():
    init = (0.75, 0.0, 0.0, 0.0, 1.0)
    plain = _solver()
    plain.initialize_uniform(0.75, (0.0, 0.0, 0.0), 1.0)
    for _ in range(6):
        plain.sweep()
    g = gsis.GsisSolver(_solver(), Identity(), gsis.GsisOptions(n_cis=3)).initialize(init)
    infos = [g.iterate() for _ in range(2)]
    assert [i.iteration for i in infos] == [1, 2] and infos[-1].cis_iterations == 6
    assert all(i.replaced_cells == 0 for i in infos)
    f, f0 = g.kinetic.distribution(), plain.distribution()
    assert np.max(np.abs(f - f0)) <= 1e-13 * np.max(np.abs(f0))
    # W^{n+1} = W^{n+1/2}: no change by the stage, and the change of W is that of the CIS moments
    assert infos[-1].pbc_change.epsilon == 0.0
    assert infos[-1].change.epsilon == infos[-1].change_half.epsilon > 0.0
    assert math.isnan(infos[0].change_half.epsilon)
    assert abs(infos[-1].kinetic.residual - plain.info.residual) <= 1e-10 * plain.info.residual


@pytest.mark.timeout(300)
def test_correction_installs_the_stage_state():
    st = Shift(2e-3)
    g = gsis.GsisSolver(_solver(equilibrium="discrete"), st, gsis.GsisOptions(n_cis=2))
    g.initialize((0.75, 0.0, 0.0, 0.0, 1.0))
    info = g.iterate()
    assert st.calls == 1 and info.replaced_cells == 0 and info.pbc_change.epsilon > 1e-4
    kin = g.kinetic
    m = kin.moments()  # of the corrected f
    assert kin.backend.deq_counts()[0] == kin.nc  # the discrete equilibrium is active in every cell
    assert np.max(np.abs(m[:, 0:5] - g.w) / np.maximum(np.abs(g.w), 1.0)) < 1e-9
    with pytest.raises(KineticSolverError):
        gsis.GsisSolver(kin, st, gsis.GsisOptions(n_cis=0))


def test_kn_damping():
    kin = _solver()
    g = gsis.GsisSolver(kin, Identity(), gsis.GsisOptions(damp_kn=0.5))
    rng = np.random.default_rng(2)
    w_half = np.column_stack([0.5 + rng.random(kin.nc), 0.1 * rng.standard_normal((kin.nc, 3)),
                              0.8 + 0.4 * rng.random(kin.nc)])
    w_new = w_half * (1.0 + 0.05 * rng.standard_normal(w_half.shape))
    out = g._damp(w_half, w_new)
    mu0, om = float(kin.s["mu0"]), float(kin.s["omega"])
    for c in range(0, kin.nc, 3):
        rho, T = w_half[c, 0], w_half[c, 4]
        kn = mu0 * T ** om / (rho * T) * math.sqrt(math.pi * T / 2.0)
        wgt = 1.0 / (1.0 + (kn / 0.5) ** 2)
        assert abs(out[c, 0] - rho * (w_new[c, 0] / rho) ** wgt) <= 1e-14
        assert np.allclose(out[c, 1:4], w_half[c, 1:4] + wgt * (w_new[c, 1:4] - w_half[c, 1:4]), rtol=0, atol=1e-15)
        assert abs(out[c, 4] - T * (w_new[c, 4] / T) ** wgt) <= 1e-14
