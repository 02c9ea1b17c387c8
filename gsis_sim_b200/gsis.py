"""The GSIS coupling loop of the kinetic solver with a macroscopic stage (GsisSolver::iterate,
src/gsis/gsis_solver.cpp:168-277; paper Fig. 1, eqs. (12)-(14), (59)).

One iteration: N_CIS CIS iterations f^n -> f^{n+1/2} on the kinetic backend; the moments W^{n+1/2}, sigma, q and the
boundary faces' F^{+-} and face states of f^{n+1/2}; the macroscopic stage (the reference's pressure-based coupled
solver, PBC) turns them into W^{n+1}; the correction f^{n+1} = f^{n+1/2} - f^eq(W^{n+1/2}) + f^eq(W^{n+1}) with the
negativity rule runs on the backend (kin_gsis_correction); eq. (59) measures the change of W.

The macroscopic stage is any object with `solve_gsis_stage(stage: GsisStageInput) -> W^{n+1}`; the reference's PBC
solver (src/macro/pbc_solver.cpp) needs AMGCL, which is not part of this package, so none is bundled. With a C++
host, the reference's own GsisSolver runs unchanged on this backend through the drop-in library
(integration/b200_backend.cpp). Everything here is host logic over the KineticSolver calls; arrays are in the
original cell / boundary-face numbering, nondimensional (R = 1, p = rho T), states W as (rho, u_x, u_y, u_z, T).
The reference's low-pass filter of the correction (PbcSolver::filter_correction) belongs to the PBC solver and is not
restated.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from .solver import KineticSolver, KineticSolverError


@dataclass
class RelativeChange:
    epsilon: float = 0.0
    rho: float = 0.0
    u: float = 0.0
    T: float = 0.0


def relative_change(a, b, volume, u_floor: float) -> RelativeChange:
    """Eq. (59): the volume-weighted relative change of (rho, u, T) from b to a (relative_change,
    src/gsis/gsis_solver.cpp:37-66); the velocity denominator is at least u_floor^2 sum V. a, b: (n_cells, 5)."""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    V = np.asarray(volume, float)
    if a.shape != b.shape or a.shape != (len(V), 5):
        raise KineticSolverError(f"relative_change: states of shape {a.shape} / {b.shape} for {len(V)} cells")
    d = a - b
    num = (d * d).T @ V
    den = (b * b).T @ V
    n = [num[0], num[1] + num[2] + num[3], num[4]]
    m = [den[0], den[1] + den[2] + den[3], den[4]]
    m[1] = max(m[1], u_floor * u_floor * float(np.sum(V)))
    ratio = lambda x, y: math.sqrt(x / y) if y > 0 else (1.0 if x > 0 else 0.0)  # noqa: E731
    r = RelativeChange(rho=ratio(n[0], m[0]), u=ratio(n[1], m[1]), T=ratio(n[2], m[2]))
    r.epsilon = max(r.rho, r.u, r.T)
    return r


@dataclass
class GsisStageInput:
    """What the macroscopic stage receives (interfaces.hpp: KineticMoments, BoundaryKineticFluxes): the 15 moments
    per cell of f^{n+1/2} (rho, u (3), T, p, sigma (6: xx yy zz xy yz xz), q (3)), the area-weighted outgoing and
    incoming half-space fluxes per boundary face (mass, momentum (3), energy), the face states (rho, u, T) of the
    boundary faces' distributions, and the current pressure of every patch (a mass-flow inlet's is adjusted by the
    kinetic host loop)."""
    moments: np.ndarray
    F_plus: np.ndarray
    F_minus: np.ndarray
    face_state: np.ndarray
    patch_pressure: np.ndarray

    @property
    def state(self) -> np.ndarray:
        """W^{n+1/2} = (rho, u, T) per cell."""
        return self.moments[:, 0:5].copy()


@dataclass
class GsisOptions:
    n_cis: int = 5           # CIS iterations per GSIS iteration ([gsis].n_cis)
    u_floor: float = 1e-2    # velocity floor of eq. (59) ([kinetic].convergence_u_floor)
    damp_kn: float = 0.0     # damping of the correction by the local Kn, w = 1 / (1 + (Kn / damp_kn)^2); 0: off
    sections: object = None  # gsis_sim_b200.section spec of cuts whose mass flow is reported; None: none


@dataclass
class GsisIterationInfo:
    iteration: int = 0
    cis_iterations: int = 0
    change: RelativeChange = field(default_factory=RelativeChange)       # W^{n+1} against W^n (eq. (59))
    change_half: RelativeChange = field(default_factory=lambda: RelativeChange(*(4 * [math.nan])))
    pbc_change: RelativeChange = field(default_factory=RelativeChange)   # W^{n+1} against W^{n+1/2}
    kinetic: object = None            # the KineticSolver's IterationInfo of f^{n+1/2} (last CIS residual)
    replaced_cells: int = 0
    patch_mass_flow_kinetic: np.ndarray = field(default_factory=lambda: np.zeros(0))
    section_flow_kinetic: np.ndarray = field(default_factory=lambda: np.zeros(0))
    t_cis: float = 0.0
    t_moments: float = 0.0
    t_macro: float = 0.0
    t_correction: float = 0.0
    t_total: float = 0.0


class GsisSolver:
    """GsisSolver (src/gsis/gsis_solver.hpp) over a KineticSolver and a macroscopic stage."""

    def __init__(self, kinetic: KineticSolver, macro, options: GsisOptions | None = None):
        self.kinetic = kinetic
        self.macro = macro
        self.options = options or GsisOptions()
        if self.options.n_cis < 1:
            raise KineticSolverError(f"GSIS needs n_cis >= 1 (got {self.options.n_cis})")
        if not self.options.damp_kn >= 0.0:
            raise KineticSolverError("damp_kn must be >= 0")
        self.volume = np.empty(kinetic.nc)
        self.volume[kinetic.h.cell_new_to_old] = kinetic.volume
        self.iteration = 0
        self.cis_iterations = 0
        self.w = None
        self.w_half_prev = None
        self.last = GsisIterationInfo()

    def initialize(self, initial):
        """f = f^eq(W) of the given state: (n_cells, 5) per cell, or one (rho, u (3), T) for every cell. A macroscopic
        stage with `solve_standalone(W) -> W` (the reference's NSF-only PBC initialisation) refines W first."""
        w = np.asarray(initial, float)
        if w.shape == (5,):
            w = np.tile(w, (self.kinetic.nc, 1))
        if w.shape != (self.kinetic.nc, 5):
            raise KineticSolverError(f"initial state of shape {w.shape} for {self.kinetic.nc} cells")
        if hasattr(self.macro, "solve_standalone"):
            w = np.asarray(self.macro.solve_standalone(w.copy()), float)
        if not np.all((w[:, 0] > 0) & (w[:, 4] > 0) & np.isfinite(w).all(axis=1)):
            raise KineticSolverError("initial density and temperature must be positive and finite")
        self.kinetic.initialize_equilibrium(w)
        self.w = w.copy()
        self.iteration = 0
        self.cis_iterations = 0
        self.w_half_prev = None
        return self

    def _damp(self, w_half, w_new):
        """The correction's damping by the local Knudsen number (gsis_solver.cpp:237-256):
        Kn = mu(T) / (rho T) sqrt(pi T / 2), mu = mu0 T^omega of the kinetic set-up."""
        s = self.kinetic.s
        rho, T = w_half[:, 0], w_half[:, 4]
        kn = float(s["mu0"]) * T ** float(s["omega"]) / (rho * T) * np.sqrt(math.pi * T / 2.0)
        x = kn / self.options.damp_kn
        wgt = 1.0 / (1.0 + x * x)
        d = wgt < 1.0
        out = w_new.copy()
        out[d, 0] = rho[d] * np.exp(wgt[d] * np.log(w_new[d, 0] / rho[d]))
        out[d, 1:4] = w_half[d, 1:4] + wgt[d, None] * (w_new[d, 1:4] - w_half[d, 1:4])
        out[d, 4] = T[d] * np.exp(wgt[d] * np.log(w_new[d, 4] / T[d]))
        return out

    def iterate(self) -> GsisIterationInfo:
        if self.w is None:
            raise KineticSolverError("initialize the GSIS solver before iterating")
        kin, opt = self.kinetic, self.options
        t_all = time.perf_counter()
        info = GsisIterationInfo()
        kin.update_mass_flow_pressure()
        # 1. CIS: f^n -> f^{n+1/2}
        t = time.perf_counter()
        for _ in range(opt.n_cis):
            kin.sweep(update_pressure=False)
        self.cis_iterations += opt.n_cis
        info.t_cis = time.perf_counter() - t
        residual = kin.info.residual
        # 2. moments and boundary fluxes of f^{n+1/2}
        t = time.perf_counter()
        info.kinetic = kin.prepare()
        info.kinetic.residual, info.kinetic.has_residual = residual, True
        m = kin.moments()
        fp, fm, fs = kin.boundary_fluxes()
        info.patch_mass_flow_kinetic = np.asarray(info.kinetic.patch_mass_flow, float).copy()
        if opt.sections is not None and not opt.sections.empty():
            info.section_flow_kinetic = kin.section_mass_flow(opt.sections)
        info.t_moments = time.perf_counter() - t
        # 3. the macroscopic stage
        t = time.perf_counter()
        stage = GsisStageInput(moments=m, F_plus=fp, F_minus=fm, face_state=fs,
                               patch_pressure=np.asarray(kin.h.patch_dbl[:, 1], float).copy())
        w_half = stage.state
        w_new = np.asarray(self.macro.solve_gsis_stage(stage), float)
        if w_new.shape != w_half.shape:
            raise KineticSolverError(f"the macroscopic stage returned a state of shape {w_new.shape}, "
                                     f"expected {w_half.shape}")
        info.t_macro = time.perf_counter() - t
        if opt.damp_kn > 0.0:
            w_new = self._damp(w_half, w_new)
        # 4. correction (eq. (14)) with the negativity rule
        t = time.perf_counter()
        info.replaced_cells = kin.apply_gsis_correction(w_half, w_new)
        info.t_correction = time.perf_counter() - t
        # 5. convergence measures (eq. (59))
        info.change = relative_change(w_new, self.w, self.volume, opt.u_floor)
        info.pbc_change = relative_change(w_new, w_half, self.volume, opt.u_floor)
        if self.w_half_prev is not None:
            info.change_half = relative_change(w_half, self.w_half_prev, self.volume, opt.u_floor)
        self.w_half_prev = w_half
        self.w = w_new
        self.iteration += 1
        info.iteration = self.iteration
        info.cis_iterations = self.cis_iterations
        info.t_total = time.perf_counter() - t_all
        self.last = info
        return info
