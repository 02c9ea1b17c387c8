"""Kinetic set-up on the host: case description + mesh -> the flat arrays of a KinSetupDesc and the host-side data
of the kinetic host loop.

Follows the reference's `build_kinetic_setup` (src/kinetic/kinetic_setup.cpp:293-514) and the derived scales of
`derive_quantities` (src/config/case_config.cpp:626-665): RCB blocks with block RCM, renumbered mesh and
geometry, cell-face CSR, LSQ coefficients, patch conditions, velocity storage layout (mirror orbits or sweep
direction groups), pseudo time step, per-direction sweep orders, nondimensional geometry.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .mesh import PolyMesh, build_cell_faces, build_lsq, compute_geometry, rcb_ordering, renumber_cells

K_BOLTZMANN = 1.380649e-23
SQRT_PI = 1.77245385090551602730

# BoundaryType (src/config/case_config.hpp:26-35), in declaration order
BOUNDARY_TYPES = ["maxwell_wall", "mass_flow_inlet", "diffuse_wall", "pressure_inlet", "pressure_outlet", "vacuum",
                  "symmetry", "periodic_slab"]


@dataclass
class Gas:
    molecular_mass: float = 6.65e-27
    mu_ref: float = 1.916e-5
    T_ref: float = 273.15
    omega: float = 0.66
    Pr: float = 2.0 / 3.0
    gamma: float = 5.0 / 3.0


@dataclass
class Conditions:
    L_ref: float = 1.0
    T0: float = 273.15
    Kn: float | None = None
    delta_rp: float | None = None
    p_ref: float | None = None


@dataclass
class BC:
    """Boundary condition of one patch; T, p and u are nondimensional (ratios to T0, p_ref, sqrt(R T0))."""
    patch: str
    type: str
    T: float = 1.0
    p: float = 1.0
    u: tuple = (0.0, 0.0, 0.0)
    alpha: float = 1.0
    zero_tangential: bool = False
    mass_flow: float = 0.0  # nondimensional target mass flow (mass_flow_inlet)


@dataclass
class VelocityGrid:
    """Tensor velocity grid: uniform midpoint rule on [lo, hi] (src/velocity/velocity_grid.hpp:1-72), or given
    per-axis nodes and weights (nonuniform / Newton-Cotes grids; per-velocity weights on the device)."""
    n: tuple = (10, 10, 10)
    lo: tuple = (-5.0, -5.0, -5.0)
    hi: tuple = (5.0, 5.0, 5.0)
    nodes: tuple | None = None     # per axis 1-D node arrays (nonuniform grids)
    weights: tuple | None = None   # per axis 1-D quadrature weights

    def axis(self, a):
        if self.nodes is not None:
            return np.asarray(self.nodes[a], float)
        n = self.n[a]
        center = 0.5 * (self.lo[a] + self.hi[a])
        half = (self.hi[a] - self.lo[a]) / (2.0 * n)
        return center + (2 * np.arange(n) + 1 - n) * half

    def axis_weights(self, a):
        if self.weights is not None:
            return np.asarray(self.weights[a], float)
        return np.full(self.n[a], (self.hi[a] - self.lo[a]) / self.n[a])

    @property
    def uniform(self) -> bool:
        return self.nodes is None and self.weights is None

    @classmethod
    def clustered(cls, n, vmax: float, stretch: float = 2.0) -> "VelocityGrid":
        """Nonuniform tensor grid clustered near zero: the midpoint rule in s on (-1, 1) mapped by
        xi = vmax sinh(c s) / sinh(c) (c = stretch), weights d xi / d s * (2 / n) per axis. Symmetric about zero, so
        symmetry planes keep exact mirror pairs; an extension of the reference's uniform grids."""
        nodes, weights = [], []
        for m in n:
            sk = -1.0 + (2.0 * np.arange(m) + 1.0) / m
            nodes.append(vmax * np.sinh(stretch * sk) / np.sinh(stretch))
            weights.append(vmax * stretch * np.cosh(stretch * sk) / np.sinh(stretch) * (2.0 / m))
        return cls(n=tuple(n), lo=(-vmax,) * 3, hi=(vmax,) * 3, nodes=tuple(nodes), weights=tuple(weights))

    def delta(self, a):
        return (self.hi[a] - self.lo[a]) / self.n[a]

    def symmetric(self, a):
        return abs(self.lo[a] + self.hi[a]) <= 1e-12 * (self.hi[a] - self.lo[a])


@dataclass
class KineticParams:
    """[kinetic] parameters with the reference defaults (src/kinetic/kinetic_params.hpp:11-117)."""
    pseudo_cfl: float = 0.0
    pseudo_time: str = "global"
    limiter_k: float = 3.0
    limiter: str = "venkatakrishnan"
    limiter_eps: str = "relative"
    lsq_weight_power: float = 0.0
    positivity_limiter: bool = False
    velocity_chunk: int = 0
    sweep_blocks: int = 0
    cell_ordering: str = "rcb"
    precision: str = "fp32"
    max_iterations: int = 100000
    initial_pressure: float = 1.0
    initial_temperature: float = 1.0
    convergence_u_floor: float = 1.0e-2
    wall_relaxation: float = 1.0
    boundary_iterations: int = 1
    interface_damping: float = 0.5
    gsis_negative_check: str = "blend"
    inner_sweeps: int = 4
    inner_wall_update: bool = True
    block_passes: int = 2
    sweep_order: str = "octant"
    equilibrium: str = "discrete"
    deq_fallback: str = "collisionless"
    pressure_boundary_reconstruction: str = "limited"
    cold_bgk_temperature: float = 0.0


def derive_quantities(gas: Gas, c: Conditions) -> dict:
    """derive_quantities (src/config/case_config.cpp:626-665)."""
    R = K_BOLTZMANN / gas.molecular_mass
    mu0 = gas.mu_ref * (c.T0 / gas.T_ref) ** gas.omega
    mps = math.sqrt(2.0 * R * c.T0)
    kn_factor = mu0 / c.L_ref * math.sqrt(math.pi * R * c.T0 / 2.0)
    if c.delta_rp is not None:
        p_ref = c.delta_rp * mu0 * mps / c.L_ref
    elif c.Kn is not None:
        p_ref = kn_factor / c.Kn
    else:
        p_ref = c.p_ref
    ref_velocity = math.sqrt(R * c.T0)
    ref_viscosity = p_ref * c.L_ref / ref_velocity
    return dict(R=R, mu0=mu0, p_ref=p_ref, p_in=p_ref, Kn=kn_factor / p_ref, mu_hat0=mu0 / ref_viscosity,
                mass_flow_scale=SQRT_PI * c.L_ref * c.L_ref * p_ref / mps, ref_velocity=ref_velocity,
                ref_temperature=c.T0, ref_pressure=p_ref, ref_density=p_ref / (R * c.T0))


def sweep_directions(order: str) -> np.ndarray:
    """make_sweep_directions (src/kinetic/kinetic_setup.cpp:182-205)."""
    d = []
    if order in ("octant", "dir13"):
        if order == "dir13":
            d += [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1), (0, 1, 1), (0, 1, -1)]
        d += [(1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1)]
    elif order != "block":
        raise ValueError(f"unknown sweep_order {order!r}")
    d = np.array(d, float).reshape(-1, 3)
    if len(d):
        d = d / np.sqrt(np.sum(d * d, axis=1))[:, None]
    return d


def sweep_direction_of(dirs: np.ndarray, xi: np.ndarray) -> np.ndarray:
    """sweep_direction_of (src/kinetic/kinetic_setup.cpp:207-218) for many velocities: first g with the largest
    |d_g . xi| (ties within 1e-12 keep the smaller g)."""
    best = np.zeros(len(xi), np.int64)
    best_v = np.full(len(xi), -1.0)
    for g in range(len(dirs)):
        v = np.abs(xi[:, 0] * dirs[g, 0] + xi[:, 1] * dirs[g, 1] + xi[:, 2] * dirs[g, 2])
        upd = v > best_v + 1e-12
        best = np.where(upd, g, best)
        best_v = np.where(upd, v, best_v)
    return best


def velocity_layout(grid: VelocityGrid, mirror_axes, dirs: np.ndarray):
    """make_velocity_layout (src/kinetic/kinetic_setup.cpp:220-291)."""
    n = grid.n
    nv = n[0] * n[1] * n[2]
    axes = sorted(set(mirror_axes))
    for a in axes:
        if not grid.symmetric(a) or n[a] % 2:
            raise ValueError(f"mirror axis {a} needs a symmetric range with an even number of points")
    axis_xor = [0, 0, 0]
    for r, a in enumerate(axes):
        axis_xor[a] = 1 << r
    orbit = 1 << len(axes)
    k = np.arange(nv)
    ijk = np.stack([k % n[0], (k // n[0]) % n[1], k // (n[0] * n[1])], 1)
    rep = np.ones(nv, bool)
    for a in axes:
        rep &= ijk[:, a] < n[a] // 2
    s2g = []
    for kk in np.flatnonzero(rep):
        for m in range(orbit):
            mm = ijk[kk].copy()
            for r, a in enumerate(axes):
                if m & (1 << r):
                    mm[a] = n[a] - 1 - mm[a]
            s2g.append(mm[0] + n[0] * (mm[1] + n[1] * mm[2]))
    s2g = np.array(s2g, np.int64)
    xs = [grid.axis(a) for a in range(3)]
    xi_grid = np.stack([xs[0][ijk[:, 0]], xs[1][ijk[:, 1]], xs[2][ijk[:, 2]]], 1)
    if not axes and len(dirs):
        grp = sweep_direction_of(dirs, xi_grid)
        s2g = s2g[np.argsort(grp[s2g], kind="stable")]
    g2s = np.empty(nv, np.int64)
    g2s[s2g] = np.arange(nv)
    xi = xi_grid[s2g]
    ws = [grid.axis_weights(a) for a in range(3)]
    w_grid = ws[0][ijk[:, 0]] * ws[1][ijk[:, 1]] * ws[2][ijk[:, 2]]
    return dict(storage_to_grid=s2g, grid_to_storage=g2s, xi=xi, weights=None if grid.uniform else w_grid[s2g],
                weight=grid.delta(0) * grid.delta(1) * grid.delta(2), xi_max=float(np.max(np.sqrt(np.sum(xi * xi, 1)))),
                axis_xor=axis_xor, orbit_size=orbit)


@dataclass
class HostSetup:
    """Host-side data of the kinetic host loop (internal numbering), as kept by the reference KineticSolver."""
    n_internal_faces: int
    owner: np.ndarray
    cell_center: np.ndarray
    face_center: np.ndarray
    face_normal: np.ndarray
    face_area: np.ndarray
    lsq: np.ndarray
    csr_faces: np.ndarray
    patch_int: np.ndarray   # (n_patches, 4): kind, first_bface, n_faces, BoundaryType index
    patch_dbl: np.ndarray   # (n_patches, 7): T, p, ux, uy, uz, accommodation, zero_tangential
    patch_target: np.ndarray  # target mass flow per patch (nondimensional, inflow positive)
    cell_new_to_old: np.ndarray
    bface_new_to_old: np.ndarray
    storage_to_grid: np.ndarray
    length_scale: float
    gamma: float
    limiter_k: float
    wall_relaxation: float
    convergence_u_floor: float
    mass_flow_scale: float
    closed_domain: bool
    inner_sweeps: int
    inner_wall_update: bool
    boundary_iterations: int
    pressure_boundary_reconstruction: str = "limited"
    patch_names: list = field(default_factory=list)
    # reference scales for SI output (ReferenceScales, src/config/case_config.hpp): p_ref and sqrt(R T0); 0 = unknown
    ref_pressure: float = 0.0
    ref_velocity: float = 0.0

    @classmethod
    def from_npz(cls, z) -> "HostSetup":
        sc, isc = z["host.scalars"], z["host.iscalars"]
        n_patches = len(z["host.patch_int"])
        return cls(n_internal_faces=int(isc[0]), owner=z["host.owner"], cell_center=z["host.cell_center"],
                   face_center=z["host.face_center"], face_normal=z["host.face_normal"],
                   face_area=z["host.face_area"], lsq=z["host.lsq"], csr_faces=z["host.csr_faces"],
                   patch_int=z["host.patch_int"], patch_dbl=z["host.patch_dbl"],
                   patch_target=(np.asarray(z["host.patch_target"], float) if "host.patch_target" in z.files
                                 else np.zeros(n_patches)),
                   cell_new_to_old=z["host.cell_new_to_old"], bface_new_to_old=z["host.bface_new_to_old"],
                   storage_to_grid=z["host.storage_to_grid"], length_scale=float(sc[0]), gamma=float(sc[1]),
                   limiter_k=float(sc[2]), wall_relaxation=float(sc[3]), convergence_u_floor=float(sc[4]),
                   mass_flow_scale=float(sc[5]), closed_domain=bool(isc[1]), inner_sweeps=int(isc[2]),
                   inner_wall_update=bool(isc[3]), boundary_iterations=int(isc[4]))


KIND_OF_TYPE = {"diffuse_wall": abi.BC_DIFFUSE_WALL, "maxwell_wall": abi.BC_DIFFUSE_WALL,
                "pressure_inlet": abi.BC_PRESSURE, "mass_flow_inlet": abi.BC_PRESSURE, "vacuum": abi.BC_VACUUM,
                "symmetry": abi.BC_SYMMETRY, "periodic_slab": abi.BC_PERIODIC}


def build_kinetic_setup(mesh: PolyMesh, gas: Gas, cond: Conditions, bcs: list, grid: VelocityGrid,
                        params: KineticParams):
    """build_kinetic_setup (src/kinetic/kinetic_setup.cpp:293-514). Returns (SetupArrays, HostSetup)."""
    d = derive_quantities(gas, cond)
    geometry = compute_geometry(mesh)
    nc = mesh.n_cells
    P = params.sweep_blocks if params.sweep_blocks > 0 else min(max(nc // 2048, 1), 64)
    P = min(P, nc)
    if params.cell_ordering == "rcb":
        new_to_old, block_offsets = rcb_ordering(mesh, geometry, P)
        m, bface_new_to_old = renumber_cells(mesh, new_to_old)
        g = compute_geometry(m)
    elif params.cell_ordering == "none":
        new_to_old = np.arange(nc, dtype=np.int32)
        m, g = mesh, geometry
        bface_new_to_old = np.arange(mesh.n_boundary, dtype=np.int32)
        base, rem = divmod(nc, P)
        block_offsets = np.concatenate([[0], np.cumsum([base + (b < rem) for b in range(P)])]).astype(np.int32)
    else:
        raise ValueError(f"cell_ordering {params.cell_ordering!r} is not supported by this set-up builder")
    csr = build_cell_faces(m)
    lsq = build_lsq(m, g, csr, params.lsq_weight_power)
    L = cond.L_ref
    ni = m.n_internal
    nb = m.n_boundary
    by_patch = {b.patch: b for b in bcs}
    patch_int = np.zeros((len(m.patch_names), 4), np.int32)
    patch_dbl = np.zeros((len(m.patch_names), 7))
    patch_target = np.zeros(len(m.patch_names))
    mirror_axes = []
    closed = True
    maxwell_axes = []
    for pi, name in enumerate(m.patch_names):
        b = by_patch[name]
        start, count = int(m.patch_start[pi]), int(m.patch_count[pi])
        kind = KIND_OF_TYPE.get(b.type)
        T, p = 1.0, 0.0  # PatchCondition defaults (src/kinetic/kinetic_setup.hpp:41-54)
        u = (0.0, 0.0, 0.0)
        acc = 1.0
        if b.type in ("diffuse_wall", "maxwell_wall"):
            acc = b.alpha
            T = b.T
            u = tuple(b.u)
        elif b.type in ("pressure_inlet", "mass_flow_inlet"):
            T = b.T
            p = b.p
            patch_target[pi] = b.mass_flow
            closed = False
        elif b.type == "pressure_outlet":
            p = b.p
            kind = abi.BC_PRESSURE if p > 0.0 else abi.BC_VACUUM
            closed = False
        elif b.type == "vacuum":
            closed = False
        elif b.type == "symmetry" and count > 0:
            nrm = g.face_normal[start:start + count]
            axis = -1
            for a in range(3):
                if np.all(np.abs(np.abs(nrm[:, a]) - 1.0) <= 1e-8):
                    axis = a
            if axis < 0:
                raise ValueError(f"symmetry patch {name!r} is not aligned with a velocity axis")
            mirror_axes.append(axis)
        if acc < 1.0:
            kind = abi.BC_MAXWELL_WALL
            nrm = g.face_normal[start:start + count]
            for a in range(3):
                if np.any(np.abs(np.abs(nrm[:, a]) - 1.0) < 1e-10):
                    mirror_axes.append(a)
                    maxwell_axes.append(a)
        patch_int[pi] = (kind, start - ni, count, BOUNDARY_TYPES.index(b.type))
        patch_dbl[pi] = (T, p, u[0], u[1], u[2], acc, 1.0 if b.zero_tangential else 0.0)
    sym_axes = {}
    for pi, name in enumerate(m.patch_names):
        if by_patch[name].type == "symmetry" and m.patch_count[pi] > 0:
            s0 = int(m.patch_start[pi])
            nrm = g.face_normal[s0:s0 + int(m.patch_count[pi])]
            for a in range(3):
                if np.all(np.abs(np.abs(nrm[:, a]) - 1.0) <= 1e-8):
                    sym_axes[pi] = a
    dirs = sweep_directions(params.sweep_order)
    lay = velocity_layout(grid, mirror_axes, dirs)
    nv = len(lay["xi"])

    s = abi.SetupArrays()
    s["precision"] = abi.PRECISIONS[params.precision]
    s["device"] = 0
    s["n_cells"], s["nv"], s["n_bfaces"], s["n_blocks"] = nc, nv, nb, len(block_offsets) - 1
    s["xi_x"], s["xi_y"], s["xi_z"] = lay["xi"][:, 0], lay["xi"][:, 1], lay["xi"][:, 2]
    s["weights"] = lay["weights"]
    s["weight"] = lay["weight"]
    # CSR entries (make_csr_entries, src/kinetic/kinetic_setup.cpp:523-559)
    cell = np.repeat(np.arange(nc), np.diff(csr.offsets))
    S = csr.sign[:, None].astype(float) * g.face_area_vector[csr.faces] / (L * L)
    ds = (g.face_center[csr.faces] - g.cell_center[cell]) / L
    dn = np.where((csr.other >= 0)[:, None], (g.face_center[csr.faces] - g.cell_center[np.maximum(csr.other, 0)]) / L,
                  0.0)
    s["csr_offsets"] = csr.offsets
    s["csr_other"] = csr.other
    s["csr_bface"] = np.where(csr.other < 0, csr.faces - ni, -1)
    s["csr_geom"] = np.concatenate([S, ds, dn, lsq * L], 1).ravel()
    volume = g.cell_volume / L ** 3
    s["eps2"] = params.limiter_k ** 3 * volume
    # boundary faces (make_bface_infos, :562-591)
    bpatch = m.boundary_face_patches()
    fb = np.arange(ni, ni + nb)
    owner_b = m.owner[fb]
    kinds = patch_int[bpatch, 0]
    mirror = np.zeros(nb, np.int32)
    for pi, a in sym_axes.items():
        mirror[bpatch == pi] = lay["axis_xor"][a]
    for b in np.flatnonzero(kinds == abi.BC_MAXWELL_WALL):
        for a in range(3):
            if abs(abs(g.face_normal[fb[b], a]) - 1.0) < 1e-10:
                mirror[b] = lay["axis_xor"][a]
    s["bface_owner"] = owner_b
    s["bface_kind"] = kinds
    s["bface_mirror_xor"] = mirror
    s["bface_patch"] = bpatch
    s["bface_geom"] = np.concatenate([g.face_normal[fb], (g.face_area[fb] / (L * L))[:, None],
                                      (g.face_center[fb] - g.cell_center[owner_b]) / L], 1).ravel()
    # volumes and pseudo time step (:449-469)
    vdt = np.zeros(nc)
    diag_scale = 1.0
    if params.pseudo_cfl > 0.0 and params.pseudo_time == "velocity":
        diag_scale = 1.0 + 1.0 / params.pseudo_cfl
    elif params.pseudo_cfl > 0.0:
        area_sum = np.zeros(nc)
        np.add.at(area_sum, cell, g.face_area[csr.faces])
        vdt = lay["xi_max"] * area_sum / (L * L) / params.pseudo_cfl
    s["volume"], s["vdt"] = volume, vdt
    s["block_offsets"] = block_offsets
    # per-direction sweep orders (:474-506)
    nd = len(dirs)
    s["n_sweep_dirs"] = nd
    if nd:
        order = np.empty((nd, nc), np.int32)
        pos = np.empty((nd, nc), np.int32)
        for gi in range(nd):
            dv = dirs[gi]
            key = dv[0] * g.cell_center[:, 0] + dv[1] * g.cell_center[:, 1] + dv[2] * g.cell_center[:, 2]
            for b in range(len(block_offsets) - 1):
                c0, c1 = block_offsets[b], block_offsets[b + 1]
                cs = np.arange(c0, c1)
                order[gi, c0:c1] = cs[np.lexsort((cs, key[c0:c1]))]
            pos[gi, order[gi]] = np.arange(nc)
        s["sweep_order"], s["sweep_pos"] = order.ravel(), pos.ravel()
        s["sweep_dir_of"] = sweep_direction_of(dirs, lay["xi"]).astype(np.uint8)
    # parameters
    s["limiter_mode"] = (abi.LIMITER_NONE if params.limiter == "none" else
                         abi.LIMITER_VENKAT_RELATIVE if params.limiter_eps == "relative" else
                         abi.LIMITER_VENKAT_ABSOLUTE)
    s["positivity"] = int(params.positivity_limiter)
    s["diag_scale"] = diag_scale
    s["interface_damping"] = params.interface_damping
    s["block_passes"] = params.block_passes
    s["negative_check_mode"] = abi.NEGATIVE_MODES[params.gsis_negative_check]
    s["velocity_chunk"] = params.velocity_chunk
    s["mu0"], s["omega"], s["Pr"] = d["mu_hat0"], gas.omega, gas.Pr
    s["cold_bgk_temperature"] = params.cold_bgk_temperature
    s["discrete_eq"] = int(params.equilibrium == "discrete")
    s["deq_fallback_collisionless"] = int(params.deq_fallback == "collisionless")
    s["deq_lo"] = tuple(float(x) for x in grid.lo)
    s["deq_hi"] = tuple(float(x) for x in grid.hi)
    s["deq_d"] = tuple(grid.delta(a) for a in range(3))
    s["deq_criterion"] = 27.0
    s["deq_tolerance"] = 1e-11 if params.precision == "fp64" else 1e-6
    s["deq_max_iterations"] = 20
    n_mw = int(np.sum(patch_int[bpatch, 0] == abi.BC_MAXWELL_WALL)) if nb else 0
    s["n_maxwell_faces"] = n_mw
    s["grid_n"] = tuple(grid.n)
    if n_mw:
        off = np.full(nb, -1, np.int64)
        frac = np.zeros(nb)
        slot = 0
        for b in range(nb):
            if kinds[b] == abi.BC_MAXWELL_WALL:
                off[b] = slot * nv
                frac[b] = 1.0 - patch_dbl[bpatch[b], 5]
                slot += 1
        s["maxwell_offset"], s["maxwell_specular_fraction"] = off, frac
        s["grid_to_storage"] = lay["grid_to_storage"]
    host = HostSetup(n_internal_faces=ni, owner=m.owner, cell_center=g.cell_center, face_center=g.face_center,
                     face_normal=g.face_normal, face_area=g.face_area, lsq=lsq, csr_faces=csr.faces,
                     patch_int=patch_int, patch_dbl=patch_dbl, patch_target=patch_target, cell_new_to_old=new_to_old,
                     bface_new_to_old=bface_new_to_old, storage_to_grid=lay["storage_to_grid"], length_scale=L,
                     gamma=gas.gamma, limiter_k=params.limiter_k, wall_relaxation=params.wall_relaxation,
                     convergence_u_floor=params.convergence_u_floor, mass_flow_scale=d["mass_flow_scale"],
                     closed_domain=closed, inner_sweeps=params.inner_sweeps,
                     inner_wall_update=params.inner_wall_update, boundary_iterations=params.boundary_iterations,
                     pressure_boundary_reconstruction=params.pressure_boundary_reconstruction,
                     patch_names=list(m.patch_names), ref_pressure=d["ref_pressure"], ref_velocity=d["ref_velocity"])
    return s, host
