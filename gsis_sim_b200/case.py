"""Case files of the reference (TOML, parse_case_toml / derive_quantities, src/config/case_config.cpp:130-665; kinetic
parameters, src/kinetic/kinetic_params.cpp:8-92) and the kinetic set-up they describe.

`load_case(path)` reads a case file with the reference's rules: required sections [case], [gas], [conditions],
[[boundary]], [velocity_grid]; optional [gsis], [kinetic], [macro], [output]; unknown keys in the typed sections and
wrong value types are errors; exactly one of conditions.delta_rp / Kn / p_ref; SI units (K, m/s, Pa, kg/s) in the
boundary conditions; the velocity range in units of sqrt(R T0). `case_setup(cfg)` reads the case's `.pmesh` and
builds the nondimensional kinetic set-up (the reference's build_kinetic_setup, src/kinetic/kinetic_setup.cpp:293-514)
for the B200 backend. Only the kinetic path is built: [gsis], [macro] and [output] are read and kept, not used.
"""
from __future__ import annotations

import math
import os
import tomllib
from dataclasses import dataclass, field

from . import kinetic_setup as ks
from .pmesh import read_pmesh

BOUNDARY_TYPES = ("maxwell_wall", "mass_flow_inlet", "diffuse_wall", "pressure_inlet", "pressure_outlet", "vacuum",
                  "symmetry", "periodic_slab")


class CaseError(ValueError):
    """The case file breaks one of the reference's rules (it raises gsis::Error in the same places)."""


def _check(cond, msg):
    if not cond:
        raise CaseError(msg)


class _Table:
    """One TOML table read key by key; keys never asked for are errors at finish() (TableReader,
    case_config.cpp:153-280)."""

    def __init__(self, table, name):
        _check(isinstance(table, dict), f"[{name}] must be a table")
        self.t, self.name, self.known = table, name, set()

    def find(self, key):
        self.known.add(key)
        return self.t.get(key)

    def require(self, key):
        v = self.find(key)
        _check(v is not None, f"[{self.name}] has no {key}")
        return v

    def _number(self, key, v):
        _check(isinstance(v, (int, float)) and not isinstance(v, bool), f"{self.name}.{key} must be a number")
        _check(math.isfinite(float(v)), f"{self.name}.{key} is not finite")
        return float(v)

    def number(self, key):
        return self._number(key, self.require(key))

    def opt_number(self, key):
        v = self.find(key)
        return None if v is None else self._number(key, v)

    def string(self, key):
        v = self.require(key)
        _check(isinstance(v, str), f"{self.name}.{key} must be a string")
        return v

    def opt_string(self, key):
        v = self.find(key)
        _check(v is None or isinstance(v, str), f"{self.name}.{key} must be a string")
        return v

    def opt_integer(self, key):
        v = self.find(key)
        _check(v is None or (isinstance(v, int) and not isinstance(v, bool)), f"{self.name}.{key} must be an integer")
        return v

    def opt_boolean(self, key):
        v = self.find(key)
        _check(v is None or isinstance(v, bool), f"{self.name}.{key} must be a boolean")
        return v

    def opt_vec3(self, key):
        v = self.find(key)
        if v is None:
            return None
        _check(isinstance(v, list) and len(v) == 3, f"{self.name}.{key} must be an array of 3 numbers")
        return tuple(self._number(key, x) for x in v)

    def int3(self, key):
        v = self.require(key)
        _check(isinstance(v, list) and len(v) == 3 and all(isinstance(x, int) and not isinstance(x, bool) for x in v),
               f"{self.name}.{key} must be an array of 3 integers")
        for x in v:
            _check(1 <= x <= 100000, f"{self.name}.{key} element {x} out of range")
        return tuple(v)

    def range3(self, key):
        v = self.require(key)
        ok = isinstance(v, list) and len(v) == 3 and all(isinstance(p, list) and len(p) == 2 for p in v)
        _check(ok, f"{self.name}.{key} must be [[lo, hi], [lo, hi], [lo, hi]]")
        return [[self._number(key, x) for x in p] for p in v]

    def finish(self):
        unknown = [k for k in self.t if k not in self.known]
        _check(not unknown, f"[{self.name}] has unknown key(s) {', '.join(unknown)}; allowed: "
                            f"{', '.join(sorted(self.known))}")


@dataclass
class BoundarySpec:
    patch: str
    type: str
    temperature: float | None = None  # K
    velocity: tuple | None = None     # m/s
    pressure: float | None = None     # Pa
    mass_flow: float | None = None    # kg/s
    accommodation: float = 1.0
    inlet_zero_tangential: bool = False


@dataclass
class CaseConfig:
    name: str
    mesh: str  # absolute path of the .pmesh file
    mode: str
    gas: ks.Gas
    conditions: ks.Conditions
    boundaries: list
    velocity_grid: dict           # n, lo, hi (nondimensional) or automatic
    gsis: dict = field(default_factory=dict)
    kinetic: dict = field(default_factory=dict)
    macro: dict = field(default_factory=dict)
    output: dict = field(default_factory=dict)
    ignored_sections: list = field(default_factory=list)
    source: str = ""

    def boundary(self, patch):
        for b in self.boundaries:
            if b.patch == patch:
                return b
        return None


def _positive(x, name):
    _check(x > 0.0, f"{name} must be positive (value {x})")


def _parse_boundaries(arr, cfg_bcs):
    _check(isinstance(arr, list) and all(isinstance(t, dict) for t in arr), "boundary must be an array of tables")
    for i, t in enumerate(arr):
        name = f"boundary[{i}]"
        r = _Table(t, name)
        b = BoundarySpec(patch=r.string("patch"), type=r.string("type"))
        _check(b.patch != "", f"{name}.patch is empty")
        _check(b.type in BOUNDARY_TYPES, f'{name}.type = "{b.type}" is not a known boundary condition')
        if b.type in ("maxwell_wall", "diffuse_wall"):
            if b.type == "maxwell_wall":
                b.accommodation = r.number("accommodation")
                _check(0.0 < b.accommodation <= 1.0, f"{name}.accommodation must be in (0, 1]")
            b.temperature = r.number("temperature")
            b.velocity = r.opt_vec3("velocity")
        elif b.type in ("mass_flow_inlet", "pressure_inlet"):
            b.temperature = r.number("temperature")
            if b.type == "mass_flow_inlet":
                b.mass_flow = r.number("mass_flow")
                _positive(b.mass_flow, f"{name}.mass_flow")
            else:
                b.pressure = r.opt_number("pressure")
            tv = r.opt_string("tangential_velocity") or "extrapolate"
            _check(tv in ("extrapolate", "zero"), f'{name}.tangential_velocity is "extrapolate" or "zero"')
            b.inlet_zero_tangential = tv == "zero"
        elif b.type == "pressure_outlet":
            b.pressure = r.number("pressure")
        r.finish()
        if b.temperature is not None:
            _positive(b.temperature, f"{name}.temperature")
        if b.pressure is not None:
            if b.type == "pressure_outlet":
                _check(b.pressure >= 0.0, f"{name}.pressure must be >= 0")
            else:
                _positive(b.pressure, f"{name}.pressure")
        _check(all(x.patch != b.patch for x in cfg_bcs), f'boundary condition of patch "{b.patch}" given twice')
        cfg_bcs.append(b)
    _check(cfg_bcs, "no [[boundary]] given")


def _module(t, name):
    _check(isinstance(t, dict), f"[{name}] must be a table")
    for k, v in t.items():
        _check(isinstance(v, (bool, int, float, str)), f"[{name}].{k} must be a scalar")
    return dict(t)


def parse_case_toml(text: str, source: str = "<string>") -> CaseConfig:
    try:
        root = tomllib.loads(text)
    except tomllib.TOMLDecodeError as e:
        raise CaseError(f"TOML parse error in {source}: {e}") from e
    for sec in ("case", "gas", "conditions", "boundary", "velocity_grid"):
        _check(sec in root, f"{source}: required section [{sec}] missing")
    known = {"case", "gas", "conditions", "boundary", "velocity_grid", "gsis", "kinetic", "macro", "output"}
    ignored = [k for k in root if k not in known]

    r = _Table(root["case"], "case")
    name, mesh = r.string("name"), r.string("mesh")
    mode = r.opt_string("mode") or "gsis"
    r.finish()
    _check(name != "" and mesh != "", "case.name and case.mesh must not be empty")
    _check(mode in ("gsis", "cis", "nsf"), f'case.mode is "gsis", "cis" or "nsf" (value "{mode}")')
    base = os.path.dirname(os.path.abspath(source)) if source != "<string>" else os.getcwd()
    mesh_path = mesh if os.path.isabs(mesh) else os.path.normpath(os.path.join(base, mesh))

    r = _Table(root["gas"], "gas")
    gas = ks.Gas(molecular_mass=r.number("molecular_mass"), mu_ref=r.number("mu_ref"), T_ref=r.number("T_ref"),
                 omega=r.number("omega"))
    r.finish()
    for k in ("molecular_mass", "mu_ref", "T_ref", "omega"):
        _positive(getattr(gas, k), f"gas.{k}")
    _check(gas.molecular_mass < 1e-20, f"gas.molecular_mass = {gas.molecular_mass} kg is too large for a molecule")

    r = _Table(root["conditions"], "conditions")
    cond = ks.Conditions(L_ref=r.number("L_ref"), T0=r.number("T0"), delta_rp=r.opt_number("delta_rp"),
                         Kn=r.opt_number("Kn"), p_ref=r.opt_number("p_ref"))
    r.finish()
    _positive(cond.L_ref, "conditions.L_ref")
    _positive(cond.T0, "conditions.T0")
    given = [x for x in (cond.delta_rp, cond.Kn, cond.p_ref) if x is not None]
    _check(len(given) == 1, "conditions needs exactly one of delta_rp, Kn, p_ref")
    _positive(given[0], "conditions.delta_rp / Kn / p_ref")

    bcs = []
    _parse_boundaries(root["boundary"], bcs)

    r = _Table(root["velocity_grid"], "velocity_grid")
    vg = {"automatic": bool(r.opt_boolean("auto") or False)}
    if vg["automatic"]:
        _check(r.find("n") is None and r.find("range") is None, "velocity_grid.auto = true excludes n and range")
        r.finish()
    else:
        vg["n"] = r.int3("n")
        rng = r.range3("range")
        r.finish()
        vg["lo"] = tuple(p[0] for p in rng)
        vg["hi"] = tuple(p[1] for p in rng)
        for a in range(3):
            _check(vg["lo"][a] < vg["hi"][a], f"velocity_grid.range axis {a}: lo < hi required")
        _check(vg["n"][0] * vg["n"][1] * vg["n"][2] <= 100_000_000, "too many velocity points")

    cfg = CaseConfig(name=name, mesh=mesh_path, mode=mode, gas=gas, conditions=cond, boundaries=bcs,
                     velocity_grid=vg, ignored_sections=ignored, source=source)
    for sec in ("gsis", "kinetic", "macro", "output"):
        if sec in root:
            setattr(cfg, sec, _module(root[sec], sec))
    if vg["automatic"]:
        _auto_velocity_grid(cfg)
    for b in bcs:
        _check(b.type != "pressure_inlet" or b.pressure is not None or cond.delta_rp is not None,
               f'pressure inlet "{b.patch}" may omit pressure only when conditions.delta_rp is given')
    return cfg


def _auto_velocity_grid(cfg: CaseConfig) -> None:
    """velocity_grid.auto (case_config.cpp:600-618): range u_max + 5 sqrt(R T_max), spacing 0.7 sqrt(R T_min)."""
    temps = [b.temperature for b in cfg.boundaries if b.temperature is not None]
    t_min, t_max = (min(temps), max(temps)) if temps else (cfg.conditions.T0, cfg.conditions.T0)
    u_max = max([math.sqrt(sum(x * x for x in b.velocity)) for b in cfg.boundaries if b.velocity] or [0.0])
    R = ks.K_BOLTZMANN / cfg.gas.molecular_mass
    limit = u_max + 5.0 * math.sqrt(R * t_max)
    n = max(2.0, 2.0 * math.ceil(limit / (0.7 * math.sqrt(R * t_min))))
    _check(math.isfinite(n) and n ** 3 <= 100_000_000, "automatic velocity grid has too many points")
    lim = limit / math.sqrt(R * cfg.conditions.T0)
    cfg.velocity_grid.update(n=(int(n),) * 3, lo=(-lim,) * 3, hi=(lim,) * 3)


def load_case(path: str) -> CaseConfig:
    with open(path, "rb") as fh:
        text = fh.read().decode("utf-8")
    return parse_case_toml(text, source=os.path.abspath(path))


_KINETIC_KEYS = {  # key: (type, check) of parse_kinetic_params (kinetic_params.cpp:8-92)
    "pseudo_cfl": float, "pseudo_time": str, "limiter_k": float, "limiter": str, "limiter_eps": str,
    "lsq_weight_power": float, "positivity_limiter": bool, "velocity_chunk": int, "sweep_blocks": int,
    "cell_ordering": str, "precision": str, "backend": str, "max_iterations": int, "initial_pressure": float,
    "initial_temperature": float, "convergence_u_floor": float, "wall_relaxation": float,
    "boundary_iterations": int, "interface_damping": float, "gsis_negative_check": str, "launch_cells": int,
    "sweep_cells_per_launch": int, "inner_sweeps": int, "inner_wall_update": bool, "block_passes": int,
    "sweep_order": str, "equilibrium": str, "deq_fallback": str, "pressure_boundary_reconstruction": str,
    "cold_bgk_temperature": float,
}
_CHOICES = {"pseudo_time": ("global", "velocity"), "limiter": ("venkatakrishnan", "none"),
            "limiter_eps": ("absolute", "relative"), "cell_ordering": ("rcb", "rcm", "none"),
            "precision": ("fp32", "fp64", "mixed"), "backend": ("cuda", "cpu"),
            "gsis_negative_check": ("all", "created", "limit", "blend"), "sweep_order": ("block", "octant", "dir13"),
            "equilibrium": ("continuous", "discrete"), "deq_fallback": ("collisionless", "continuous"),
            "pressure_boundary_reconstruction": ("limited", "cell")}


def kinetic_params(cfg: CaseConfig, precision: str | None = None) -> ks.KineticParams:
    """[kinetic] -> KineticParams with the reference's types, choices and ranges. `backend`, `launch_cells` and
    `sweep_cells_per_launch` are accepted and not used (the B200 backend needs no launch splitting); `precision`
    also accepts "mixed" (FP32 storage and sweeps over an FP64 residual)."""
    kp = ks.KineticParams()
    for k, v in cfg.kinetic.items():
        _check(k in _KINETIC_KEYS, f"[kinetic] has unknown key {k}")
        typ = _KINETIC_KEYS[k]
        if typ is float:
            _check(isinstance(v, (int, float)) and not isinstance(v, bool), f"kinetic.{k} must be a number")
            v = float(v)
        elif typ is int:
            _check(isinstance(v, int) and not isinstance(v, bool), f"kinetic.{k} must be an integer")
        elif typ is bool:
            _check(isinstance(v, bool), f"kinetic.{k} must be a boolean")
        else:
            _check(isinstance(v, str), f"kinetic.{k} must be a string")
        if k in _CHOICES:
            _check(v in _CHOICES[k], f'kinetic.{k} is one of {", ".join(_CHOICES[k])} (value "{v}")')
        if hasattr(kp, k):
            setattr(kp, k, v)
    if precision is not None:
        kp.precision = precision
    _check(kp.pseudo_cfl >= 0 and kp.limiter_k >= 0 and kp.lsq_weight_power >= 0, "kinetic parameter < 0")
    _check(kp.velocity_chunk >= 0 and kp.sweep_blocks >= 0, "kinetic.velocity_chunk / sweep_blocks must be >= 0")
    _check(kp.max_iterations >= 1, "kinetic.max_iterations must be >= 1")
    _check(kp.initial_pressure > 0 and kp.initial_temperature > 0, "kinetic initial state must be positive")
    _check(kp.convergence_u_floor >= 0, "kinetic.convergence_u_floor must be >= 0")
    _check(0 < kp.wall_relaxation <= 1, "kinetic.wall_relaxation is in (0, 1]")
    _check(1 <= kp.boundary_iterations <= 1000, "kinetic.boundary_iterations is 1..1000")
    _check(kp.interface_damping >= 0, "kinetic.interface_damping must be >= 0")
    _check(1 <= kp.inner_sweeps <= 1000, "kinetic.inner_sweeps is 1..1000")
    _check(1 <= kp.block_passes <= 100, "kinetic.block_passes is 1..100")
    _check(kp.cold_bgk_temperature >= 0, "kinetic.cold_bgk_temperature must be >= 0")
    return kp


def boundary_conditions(cfg: CaseConfig, patch_names) -> list:
    """Nondimensional boundary conditions of the mesh's patches (PatchCondition, kinetic_setup.cpp:353-398):
    T / T0, u / sqrt(R T0), p / p_ref (a pressure inlet without pressure takes p_in = p_ref), mass flow /
    (rho_ref sqrt(R T0) L_ref^2)."""
    d = ks.derive_quantities(cfg.gas, cfg.conditions)
    out = []
    for name in patch_names:
        b = cfg.boundary(name)
        _check(b is not None, f'mesh patch "{name}" has no [[boundary]]')
        bc = ks.BC(patch=name, type=b.type)
        if b.temperature is not None:
            bc.T = b.temperature / d["ref_temperature"]
        if b.velocity is not None:
            bc.u = tuple(x / d["ref_velocity"] for x in b.velocity)
        if b.type in ("pressure_inlet", "mass_flow_inlet"):
            bc.p = (b.pressure if b.pressure is not None else d["p_in"]) / d["ref_pressure"]
            bc.zero_tangential = b.inlet_zero_tangential
        if b.type == "pressure_outlet":
            bc.p = b.pressure / d["ref_pressure"]
        if b.mass_flow is not None:
            ref_mass_flux = d["ref_density"] * d["ref_velocity"]
            bc.mass_flow = b.mass_flow / (ref_mass_flux * cfg.conditions.L_ref ** 2)
        bc.alpha = b.accommodation
        out.append(bc)
    for b in cfg.boundaries:
        _check(b.patch in patch_names, f'[[boundary]] patch "{b.patch}" is not a patch of the mesh')
    return out


def case_setup(cfg: CaseConfig, precision: str | None = None, mesh=None):
    """The kinetic set-up of a case: reads its .pmesh (unless `mesh` is given) and returns (SetupArrays, HostSetup)
    for `gsis_sim_b200.backend.B200Backend` and `gsis_sim_b200.solver.KineticSolver`."""
    if mesh is None:
        mesh = read_pmesh(cfg.mesh)
    bcs = boundary_conditions(cfg, mesh.patch_names)
    vg = cfg.velocity_grid
    grid = ks.VelocityGrid(n=tuple(vg["n"]), lo=tuple(vg["lo"]), hi=tuple(vg["hi"]))
    return ks.build_kinetic_setup(mesh, cfg.gas, cfg.conditions, bcs, grid, kinetic_params(cfg, precision))


def output_sections(cfg: CaseConfig):
    """parse_output_sections (src/kinetic/kinetic_output.cpp:70-76): the section cuts of [output]
    (`mass_flow_sections`, a string of positions in L_ref units; `mass_flow_section_axis`, "x" by default). Any other
    key of [output] is an error, as the reference's ModuleSection::finish makes it; an empty or missing string gives
    no sections."""
    from . import section as sec

    out = cfg.output or {}
    for k, v in out.items():
        _check(k in ("mass_flow_sections", "mass_flow_section_axis"), f"[output] has unknown key {k}")
        _check(isinstance(v, str), f"output.{k} must be a string")
    try:
        return sec.parse_section_spec(out.get("mass_flow_sections", ""), out.get("mass_flow_section_axis", "x"))
    except sec.SectionError as e:
        raise CaseError(str(e)) from e
