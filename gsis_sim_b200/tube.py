"""O-grid hexahedral mesh of a circular tube discharging into a downstream reservoir, and the tube case.

Tube: radius R along x in [0, L]; cross-section = central square of n_c x n_c cells plus four blocks of
n_c x n_r cells reaching the circle (an O-grid). Reservoir: x in [L, L + L_res], cross-section [-H, H]^2, the tube
O-grid extended by four more blocks of n_c x n_o cells from the circle to the square. Patches: "inlet" (x = 0),
"wall" (tube wall), "back" (reservoir wall at x = L around the tube mouth), "outlet" (the other reservoir sides).
The default sizes give 134,528 cells (the ~135k-cell tube case of the kinetic benchmark).
"""
from __future__ import annotations

import math

import numpy as np

from . import kinetic_setup as ks
from .mesh import HEX_FACES, PolyMesh, build_from_cells


def _cross_section(n_c: int, rings: list, a: float):
    """2-D O-grid nodes and quads. rings: list of (n_layers, outer(t, side) -> (y, z)) from inside out.
    Returns points (P, 2), quads (Q, 4) counter-clockwise, ring index per quad (0 = square)."""
    pts = {}
    quads = []
    ring_of = []

    def node(key, yz):
        if key not in pts:
            pts[key] = (len(pts), yz)
        return pts[key][0]

    # square [-a, a]^2: key ("s", i, j)
    s = np.linspace(-a, a, n_c + 1)
    sq = {}
    for i in range(n_c + 1):
        for j in range(n_c + 1):
            sq[(i, j)] = node(("s", i, j), (s[i], s[j]))
    for i in range(n_c):
        for j in range(n_c):
            quads.append([sq[(i, j)], sq[(i + 1, j)], sq[(i + 1, j + 1)], sq[(i, j + 1)]])
            ring_of.append(0)
    # boundary loop of the square, counter-clockwise, 4 n_c segments; side s in 0..3, t in [0, 1]
    loop = []
    for k in range(n_c):
        loop.append((n_c, k))          # right side (y = a), z up
    for k in range(n_c):
        loop.append((n_c - k, n_c))    # top (z = a), y to the left
    for k in range(n_c):
        loop.append((0, n_c - k))      # left (y = -a), z down
    for k in range(n_c):
        loop.append((k, 0))            # bottom (z = -a), y to the right
    inner_ids = [sq[ij] for ij in loop]
    inner_xy = np.array([pts[("s",) + ij][1] for ij in loop])
    m = 4 * n_c
    layer0 = 0
    for r, (n_layers, outer) in enumerate(rings, start=1):
        outer_xy = np.array([outer(k / m) for k in range(m)])
        prev_ids = inner_ids
        for l in range(1, n_layers + 1):
            f = l / n_layers
            cur_xy = inner_xy + f * (outer_xy - inner_xy)
            cur_ids = [node(("r", layer0 + l, k), tuple(cur_xy[k])) for k in range(m)]
            for k in range(m):
                k1 = (k + 1) % m
                quads.append([prev_ids[k], cur_ids[k], cur_ids[k1], prev_ids[k1]])
                ring_of.append(r)
            prev_ids = cur_ids
        inner_ids, inner_xy = prev_ids, outer_xy
        layer0 += n_layers
    P = np.zeros((len(pts), 2))
    for _, (idx, yz) in pts.items():
        P[idx] = yz
    Q = np.array(quads, np.int64)
    # orient every quad counter-clockwise in (y, z)
    a2 = (P[Q[:, 1], 0] - P[Q[:, 0], 0]) * (P[Q[:, 2], 1] - P[Q[:, 0], 1]) - \
         (P[Q[:, 2], 0] - P[Q[:, 0], 0]) * (P[Q[:, 1], 1] - P[Q[:, 0], 1])
    Q[a2 < 0] = Q[a2 < 0][:, ::-1]
    return P, Q, np.array(ring_of)


def _circle(R):
    # point of the circle matching the square-loop parameter t (angle -pi/4 at t = 0, counter-clockwise)
    return lambda t: (R * math.cos(-math.pi / 4 + 2 * math.pi * t), R * math.sin(-math.pi / 4 + 2 * math.pi * t))


def _square(H):
    def f(t):
        u = (t * 4) % 4
        side, s = int(u), u - int(u)
        c = 2 * s - 1
        return [(H, H * c), (-H * c, H), (-H, -H * c), (H * c, -H)][side]
    return f


def tube_mesh(R=1.0, L=5.0, n_c=16, n_r=10, n_x=100, res_length=4.0, res_half=2.0, n_o=12, n_xr=27) -> PolyMesh:
    a = 0.5 * R
    P2t, Q2t, _ = _cross_section(n_c, [(n_r, _circle(R))], a)
    P2r, Q2r, ringr = _cross_section(n_c, [(n_r, _circle(R)), (n_o, _square(res_half))], a)
    # the reservoir cross-section contains the tube cross-section with the same node ids for its first nodes
    assert np.allclose(P2r[:len(P2t)], P2t)
    npr = len(P2r)
    xs = np.concatenate([np.linspace(0.0, L, n_x + 1), L + np.linspace(0.0, res_length, n_xr + 1)[1:]])
    pts = np.zeros((len(xs) * npr, 3))
    for i, x in enumerate(xs):
        pts[i * npr:(i + 1) * npr, 0] = x
        pts[i * npr:(i + 1) * npr, 1:] = P2r
    cells = []
    for i in range(len(xs) - 1):
        Q = Q2t if i < n_x else Q2r
        b, t = i * npr, (i + 1) * npr
        cells.append(np.concatenate([b + Q, t + Q], axis=1))
    hexes = np.concatenate(cells)
    # drop the points no cell uses (the reservoir rings exist in the cross-section table at every x station)
    used = np.unique(hexes)
    remap = np.full(len(pts), -1, np.int64)
    remap[used] = np.arange(len(used))
    pts = pts[used]
    hexes = remap[hexes]
    cell_faces = hexes[:, HEX_FACES]
    names = ["inlet", "wall", "back", "outlet"]
    tol = 1e-9 * (L + res_length)

    def classify(c):
        x, r2 = c[:, 0], c[:, 1] ** 2 + c[:, 2] ** 2
        out = np.full(len(c), 3)  # outlet: reservoir far end and sides
        out[x < tol] = 0
        out[(x > tol) & (x < L - tol)] = 1
        out[(np.abs(x - L) <= tol) & (r2 > (0.5 * R) ** 2)] = 2
        return out

    return build_from_cells(pts, cell_faces, names, classify)


def tube_case(delta=10.0, nv=32, vmax=5.0, precision="fp64", p_out=0.01, omega=0.81, mesh_kw=None, grid=None,
              **params):
    """The kinetic tube case: inlet p = 1, T = 1; reservoir outlet p = p_out; diffuse walls T = 1; rarefaction delta;
    uniform nv^3 velocity grid on [-vmax, vmax]^3 (units sqrt(R T0)) unless `grid` is given. Returns (setup, host)."""
    mesh = tube_mesh(**(mesh_kw or {}))
    gas = ks.Gas(omega=omega)
    cond = ks.Conditions(L_ref=1.0, T0=273.15, delta_rp=delta)
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("wall", "diffuse_wall", T=1.0),
           ks.BC("back", "diffuse_wall", T=1.0), ks.BC("outlet", "pressure_outlet", p=p_out)]
    if grid is None:
        grid = ks.VelocityGrid(n=(nv, nv, nv), lo=(-vmax,) * 3, hi=(vmax,) * 3)
    kp = ks.KineticParams(precision=precision, **params)
    return ks.build_kinetic_setup(mesh, gas, cond, bcs, grid, kp)
