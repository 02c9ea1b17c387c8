"""Face-based polyhedral meshes, finite-volume geometry and cell orderings (host side, numpy).

The mesh model is the `.pmesh` model (docs/pmesh_format.md of the reference): internal faces first, sorted by
(owner, neighbour) with owner < neighbour, then boundary faces grouped by patch; face nodes ordered so that the
right-hand normal points from owner to neighbour (outwards on the boundary). Geometry follows the reference's
`compute_geometry` (src/mesh/geometry.cpp:145-252: fan triangulation about the node average, pyramid
decomposition of cells), the cell-face CSR `build_cell_faces` (src/mesh/fv_geometry.cpp:271-310), the LSQ
gradient coefficients `build_lsq_gradient` (src/mesh/fv_geometry.cpp:350-395) and the RCB + block RCM ordering
of the kinetic setup (src/kinetic/kinetic_setup.cpp:44-178, src/mesh/ordering.cpp:74-279).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class PolyMesh:
    points: np.ndarray                 # (n_points, 3) [m]
    face_offsets: np.ndarray           # (n_faces + 1,) int64
    face_nodes: np.ndarray             # int32
    owner: np.ndarray                  # (n_faces,) int32
    neighbour: np.ndarray              # (n_internal,) int32
    n_cells: int
    patch_names: list = field(default_factory=list)
    patch_start: np.ndarray = None
    patch_count: np.ndarray = None
    patch_kinds: list = field(default_factory=list)  # .pmesh patch kinds (informational: wall, inlet, ...)
    metadata: dict = field(default_factory=dict)

    @property
    def n_faces(self) -> int:
        return len(self.owner)

    @property
    def n_internal(self) -> int:
        return len(self.neighbour)

    @property
    def n_boundary(self) -> int:
        return self.n_faces - self.n_internal

    def face(self, f: int) -> np.ndarray:
        return self.face_nodes[self.face_offsets[f]:self.face_offsets[f + 1]]

    def boundary_face_patches(self) -> np.ndarray:
        out = np.full(self.n_boundary, -1, np.int32)
        for p, (s, c) in enumerate(zip(self.patch_start, self.patch_count)):
            out[s - self.n_internal:s - self.n_internal + c] = p
        return out

    def as_dict(self) -> dict:
        return dict(points=self.points, face_offsets=self.face_offsets, face_nodes=self.face_nodes,
                    owner=self.owner, neighbour=self.neighbour, n_cells=self.n_cells,
                    patch_names=list(self.patch_names), patch_start=self.patch_start, patch_count=self.patch_count)


# outward faces of a hexahedron with vertices v0..v7 (v0-v3 bottom counter-clockwise, v4-v7 above them)
HEX_FACES = np.array([[0, 4, 7, 3], [1, 2, 6, 5], [0, 1, 5, 4], [3, 7, 6, 2], [0, 3, 2, 1], [4, 5, 6, 7]], np.int64)


def build_from_cells(points: np.ndarray, cell_faces: np.ndarray, patch_names: list, classify) -> PolyMesh:
    """Face-based mesh from cells given as outward faces of equal node count.

    cell_faces: (n_cells, n_faces_per_cell, k) node ids. classify(face_centers (m, 3)) -> patch index per face.
    Internal faces are sorted by (owner, neighbour, node key), boundary faces by (patch, owner, node key), the
    node order of an internal face is the owner's (the same conventions as the reference test mesher,
    tests/support/box_mesh.cpp:150-258)."""
    n_cells, nf, k = cell_faces.shape
    faces = cell_faces.reshape(-1, k)
    cell_of = np.repeat(np.arange(n_cells), nf)
    keys = np.sort(faces, axis=1)
    order = np.lexsort(keys.T[::-1])
    ks = keys[order]
    same_next = np.all(ks[1:] == ks[:-1], axis=1)
    first = np.ones(len(ks), bool)
    first[1:] = ~same_next
    group = np.cumsum(first) - 1
    counts = np.bincount(group)
    if np.any(counts > 2):
        raise ValueError("more than two cells share a face")
    gstart = np.flatnonzero(first)
    pair = counts[group[gstart]] == 2
    # internal faces
    a = order[gstart[pair]]
    b = order[gstart[pair] + 1]
    ca, cb = cell_of[a], cell_of[b]
    own_face = np.where(ca < cb, a, b)
    own = np.minimum(ca, cb)
    nei = np.maximum(ca, cb)
    ikey = keys[own_face]
    iord = np.lexsort(tuple(ikey.T[::-1]) + (nei, own))
    int_faces = faces[own_face[iord]]
    int_owner = own[iord]
    int_nei = nei[iord]
    # boundary faces
    bidx = order[gstart[~pair]]
    bfaces = faces[bidx]
    bown = cell_of[bidx]
    centers = face_geometry(points, np.arange(0, (len(bfaces) + 1) * k, k), bfaces.ravel())[1]
    bpatch = np.asarray(classify(centers), np.int64)
    if np.any(bpatch < 0) or np.any(bpatch >= len(patch_names)):
        raise ValueError("boundary face without a patch")
    bkey = keys[bidx]
    bord = np.lexsort(tuple(bkey.T[::-1]) + (bown, bpatch))
    all_faces = np.concatenate([int_faces, bfaces[bord]])
    owner = np.concatenate([int_owner, bown[bord]]).astype(np.int32)
    bp_sorted = bpatch[bord]
    n_int = len(int_faces)
    start = np.zeros(len(patch_names), np.int32)
    count = np.zeros(len(patch_names), np.int32)
    pos = n_int
    for p in range(len(patch_names)):
        c = int(np.sum(bp_sorted == p))
        start[p], count[p] = pos, c
        pos += c
    return PolyMesh(points=np.asarray(points, np.float64), face_offsets=np.arange(0, (len(all_faces) + 1) * k, k,
                                                                                 dtype=np.int64),
                    face_nodes=all_faces.ravel().astype(np.int32), owner=owner, neighbour=int_nei.astype(np.int32),
                    n_cells=n_cells, patch_names=list(patch_names), patch_start=start, patch_count=count)


def box_mesh(n, lo, hi, patch_names=("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")) -> PolyMesh:
    """Uniform hexahedral box (the undistorted case of tests/support/box_mesh.cpp:45-148). Sides with the same
    name form one patch, in order of first appearance."""
    nx, ny, nz = n
    xs = [lo[a] + (hi[a] - lo[a]) * np.arange(n[a] + 1) / n[a] for a in range(3)]
    for a in range(3):
        xs[a][0], xs[a][-1] = lo[a], hi[a]
    X, Y, Z = np.meshgrid(xs[0], xs[1], xs[2], indexing="ij")
    pts = np.stack([X.transpose(2, 1, 0).ravel(), Y.transpose(2, 1, 0).ravel(), Z.transpose(2, 1, 0).ravel()], 1)
    node = lambda i, j, k: i + (nx + 1) * (j + (ny + 1) * k)  # noqa: E731
    k_, j_, i_ = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i_, j_, k_ = i_.ravel(), j_.ravel(), k_.ravel()
    v = np.stack([node(i_, j_, k_), node(i_ + 1, j_, k_), node(i_ + 1, j_ + 1, k_), node(i_, j_ + 1, k_),
                  node(i_, j_, k_ + 1), node(i_ + 1, j_, k_ + 1), node(i_ + 1, j_ + 1, k_ + 1),
                  node(i_, j_ + 1, k_ + 1)], 1)
    cell_faces = v[:, HEX_FACES]
    names = []
    side_patch = []
    for s in range(6):
        if patch_names[s] not in names:
            names.append(patch_names[s])
        side_patch.append(names.index(patch_names[s]))
    size = np.asarray(hi, float) - np.asarray(lo, float)
    tol = 1e-9 * size.max()

    def classify(c):
        out = np.full(len(c), -1)
        for a in (2, 1, 0):  # the first matching axis wins, as in the reference classifier
            out = np.where(np.abs(c[:, a] - lo[a]) <= tol, side_patch[2 * a], out)
            out = np.where(np.abs(c[:, a] - hi[a]) <= tol, side_patch[2 * a + 1], out)
        return out

    return build_from_cells(pts, cell_faces, names, classify)


# ------------------------------------------------------------------------------------------------------------
# geometry
# ------------------------------------------------------------------------------------------------------------

def face_geometry(points, face_offsets, face_nodes):
    """Area vectors and centres of all faces (compute_face_geometry, src/mesh/geometry.cpp:145-186)."""
    sizes = np.diff(face_offsets)
    nf = len(sizes)
    S = np.zeros((nf, 3))
    X = np.zeros((nf, 3))
    for k in np.unique(sizes):
        idx = np.flatnonzero(sizes == k)
        nodes = face_nodes[face_offsets[idx][:, None] + np.arange(k)[None, :]]
        P = points[nodes]  # (m, k, 3)
        if k == 3:
            S[idx] = 0.5 * np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
            X[idx] = (P[:, 0] + P[:, 1] + P[:, 2]) / 3.0
            continue
        xbar = P.sum(axis=1) / k
        sum_n = np.zeros((len(idx), 3))
        tri_n = []
        for j in range(k):
            nj = np.cross(P[:, j] - xbar, P[:, (j + 1) % k] - xbar)
            tri_n.append(nj)
            sum_n += nj
        S[idx] = 0.5 * sum_n
        mag = np.sqrt(np.sum(sum_n * sum_n, axis=1))
        ok = mag > 0
        nhat = np.where(ok[:, None], sum_n / np.where(ok, mag, 1.0)[:, None], 0.0)
        sum_a = np.zeros(len(idx))
        sum_ac = np.zeros((len(idx), 3))
        for j in range(k):
            a = np.sum(tri_n[j] * nhat, axis=1)
            c = (P[:, j] + P[:, (j + 1) % k] + xbar) / 3.0
            sum_a += a
            sum_ac += a[:, None] * c
        X[idx] = np.where((np.abs(sum_a) > 0)[:, None], sum_ac / np.where(sum_a != 0, sum_a, 1.0)[:, None], xbar)
    return S, X


@dataclass
class Geometry:
    face_area_vector: np.ndarray
    face_area: np.ndarray
    face_normal: np.ndarray
    face_center: np.ndarray
    cell_volume: np.ndarray
    cell_center: np.ndarray


def compute_geometry(m: PolyMesh) -> Geometry:
    """compute_geometry (src/mesh/geometry.cpp:188-252)."""
    S, X = face_geometry(m.points, m.face_offsets, m.face_nodes)
    area = np.sqrt(np.sum(S * S, axis=1))
    if np.any(area <= 0):
        raise ValueError("face with zero area")
    normal = S / area[:, None]
    nc, ni = m.n_cells, m.n_internal
    cbar = np.zeros((nc, 3))
    nf = np.zeros(nc)
    np.add.at(cbar, m.owner, X)
    np.add.at(nf, m.owner, 1)
    np.add.at(cbar, m.neighbour, X[:ni])
    np.add.at(nf, m.neighbour, 1)
    cbar /= nf[:, None]
    vol = np.zeros(nc)
    mom = np.zeros((nc, 3))
    v_own = np.sum(S * (X - cbar[m.owner]), axis=1) / 3.0
    np.add.at(vol, m.owner, v_own)
    np.add.at(mom, m.owner, v_own[:, None] * (0.75 * X + 0.25 * cbar[m.owner]))
    v_nei = np.sum(-S[:ni] * (X[:ni] - cbar[m.neighbour]), axis=1) / 3.0
    np.add.at(vol, m.neighbour, v_nei)
    np.add.at(mom, m.neighbour, v_nei[:, None] * (0.75 * X[:ni] + 0.25 * cbar[m.neighbour]))
    center = np.where((np.abs(vol) > 0)[:, None], mom / np.where(vol != 0, vol, 1.0)[:, None], cbar)
    return Geometry(S, area, normal, X, vol, center)


@dataclass
class CellFaceCsr:
    offsets: np.ndarray  # (n_cells + 1,)
    faces: np.ndarray
    other: np.ndarray    # -1 on boundary faces
    sign: np.ndarray     # +1 owner, -1 neighbour


def build_cell_faces(m: PolyMesh) -> CellFaceCsr:
    """Cell -> face CSR in ascending face order (build_cell_faces, src/mesh/fv_geometry.cpp:271-310)."""
    nf, ni = m.n_faces, m.n_internal
    fo = np.arange(nf)
    cells = np.concatenate([m.owner, m.neighbour])
    faces = np.concatenate([fo, fo[:ni]])
    other = np.concatenate([np.concatenate([m.neighbour, np.full(nf - ni, -1, np.int32)]), m.owner[:ni]])
    sign = np.concatenate([np.ones(nf, np.int8), -np.ones(ni, np.int8)])
    order = np.lexsort((faces, cells))
    counts = np.bincount(cells, minlength=m.n_cells)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return CellFaceCsr(offsets, faces[order].astype(np.int32), other[order].astype(np.int32), sign[order])


def build_lsq(m: PolyMesh, g: Geometry, csr: CellFaceCsr, weight_power: float = 0.0) -> np.ndarray:
    """LSQ gradient coefficients c_k = w_k G^-1 r_k (build_lsq_gradient, src/mesh/fv_geometry.cpp:350-395)."""
    cell = np.repeat(np.arange(m.n_cells), np.diff(csr.offsets))
    r = np.where((csr.other >= 0)[:, None], g.cell_center[np.maximum(csr.other, 0)], g.face_center[csr.faces]) - \
        g.cell_center[cell]
    w = np.ones(len(r)) if weight_power == 0.0 else np.sqrt(np.sum(r * r, axis=1)) ** (-weight_power)
    a = {}
    for name, (i, j) in dict(a00=(0, 0), a01=(0, 1), a02=(0, 2), a11=(1, 1), a12=(1, 2), a22=(2, 2)).items():
        a[name] = np.zeros(m.n_cells)
        np.add.at(a[name], cell, w * r[:, i] * r[:, j])
    a00, a01, a02, a11, a12, a22 = (a[k] for k in ["a00", "a01", "a02", "a11", "a12", "a22"])
    det = a00 * (a11 * a22 - a12 * a12) - a01 * (a01 * a22 - a12 * a02) + a02 * (a01 * a12 - a11 * a02)
    tr3 = (a00 + a11 + a22) / 3.0
    cond = np.where(tr3 > 0, det / np.where(tr3 > 0, tr3, 1.0) ** 3, 0.0)
    if np.any(cond <= 1e-12):
        raise ValueError("LSQ gradient matrix nearly singular")
    i00 = (a11 * a22 - a12 * a12) / det
    i01 = (a02 * a12 - a01 * a22) / det
    i02 = (a01 * a12 - a02 * a11) / det
    i11 = (a00 * a22 - a02 * a02) / det
    i12 = (a01 * a02 - a00 * a12) / det
    i22 = (a00 * a11 - a01 * a01) / det
    c = cell
    x, y, z = r[:, 0], r[:, 1], r[:, 2]
    out = np.stack([i00[c] * x + i01[c] * y + i02[c] * z, i01[c] * x + i11[c] * y + i12[c] * z,
                    i02[c] * x + i12[c] * y + i22[c] * z], 1)
    return w[:, None] * out


# ------------------------------------------------------------------------------------------------------------
# orderings
# ------------------------------------------------------------------------------------------------------------

def cell_adjacency(m: PolyMesh):
    """Unique sorted neighbours per cell (build_cell_adjacency, src/mesh/ordering.cpp:74-105)."""
    a = np.concatenate([m.owner[:m.n_internal], m.neighbour])
    b = np.concatenate([m.neighbour, m.owner[:m.n_internal]])
    pairs = np.unique(np.stack([a, b], 1), axis=0)
    counts = np.bincount(pairs[:, 0], minlength=m.n_cells)
    off = np.concatenate([[0], np.cumsum(counts)])
    return off, pairs[:, 1].astype(np.int64)


def _bisect(cells: np.ndarray, P: int, centers: np.ndarray, out: list):
    """Recursive coordinate bisection (bisect, src/kinetic/kinetic_setup.cpp:46-80)."""
    if P <= 1 or len(cells) <= 1:
        out.append(cells)
        return
    x = centers[cells]
    ext = x.max(axis=0) - x.min(axis=0)
    axis = 0
    for a in (1, 2):
        if ext[a] > ext[axis]:
            axis = a
    P1 = P // 2
    n1 = int(np.floor(len(cells) * P1 / P + 0.5))
    order = np.lexsort((cells, x[:, axis]))
    left = np.sort(cells[order[:n1]])
    right = np.sort(cells[order[n1:]])
    _bisect(left, P1, centers, out)
    _bisect(right, P - P1, centers, out)


def _block_rcm(cells, adj_off, adj, block_of, b, placed):
    """Reverse Cuthill-McKee inside one block (block_rcm, src/kinetic/kinetic_setup.cpp:84-149)."""
    cells = [int(c) for c in cells]
    deg = {}
    for c in cells:
        nb = adj[adj_off[c]:adj_off[c + 1]]
        deg[c] = int(np.sum(block_of[nb] == b))
    key = lambda c: (deg[c], c)  # noqa: E731
    nbrs_of = {c: [int(x) for x in adj[adj_off[c]:adj_off[c + 1]] if block_of[x] == b] for c in cells}

    def last_level(start):
        seen = {start}
        level = [start]
        last = level
        while level:
            last = level
            nxt = []
            for c in level:
                for n in nbrs_of[c]:
                    if n not in seen:
                        seen.add(n)
                        nxt.append(n)
            level = nxt
        return last

    order = []
    for seed in sorted(cells, key=key):
        if placed[seed]:
            continue
        start = min(last_level(seed), key=key)
        first = len(order)
        order.append(start)
        placed[start] = True
        head = first
        while head < len(order):
            c = order[head]
            head += 1
            nb = [n for n in nbrs_of[c] if not placed[n]]
            for n in nb:
                placed[n] = True
            nb.sort(key=key)
            order.extend(nb)
    order.reverse()
    return order


def rcb_ordering(m: PolyMesh, g: Geometry, P: int):
    """RCB blocks with block-RCM inside (rcb_ordering, src/kinetic/kinetic_setup.cpp:152-178).
    Returns (new_to_old, block_offsets)."""
    groups = []
    _bisect(np.arange(m.n_cells), P, g.cell_center, groups)
    block_of = np.empty(m.n_cells, np.int64)
    for b, cs in enumerate(groups):
        block_of[cs] = b
    adj_off, adj = cell_adjacency(m)
    placed = np.zeros(m.n_cells, bool)
    new_to_old = []
    offsets = [0]
    for b, cs in enumerate(groups):
        new_to_old.extend(_block_rcm(cs, adj_off, adj, block_of, b, placed))
        offsets.append(len(new_to_old))
    return np.array(new_to_old, np.int32), np.array(offsets, np.int32)


def renumber_cells(m: PolyMesh, new_to_old: np.ndarray):
    """Renumbered mesh (renumber_cells, src/mesh/ordering.cpp:210-279). Returns (mesh, bface_new_to_old)."""
    old_to_new = np.empty_like(new_to_old)
    old_to_new[new_to_old] = np.arange(len(new_to_old), dtype=new_to_old.dtype)
    ni = m.n_internal
    o = old_to_new[m.owner[:ni]]
    n = old_to_new[m.neighbour]
    flip = o > n
    own = np.minimum(o, n)
    nei = np.maximum(o, n)
    iord = np.lexsort((nei, own))  # stable
    sizes = np.diff(m.face_offsets)
    new_nodes, new_off, new_owner = [], [0], []

    def append(f, flipped):
        nodes = m.face(f)
        if flipped:
            nodes = np.concatenate([nodes[:1], nodes[:0:-1]])
        new_nodes.append(nodes)
        new_off.append(new_off[-1] + len(nodes))

    for f in iord:
        append(f, bool(flip[f]))
    new_owner.extend(own[iord].tolist())
    bnew_to_old = []
    for s, c in zip(m.patch_start, m.patch_count):
        fs = np.arange(s, s + c)
        bo = old_to_new[m.owner[fs]]
        ordp = np.argsort(bo, kind="stable")
        for f in fs[ordp]:
            append(f, False)
            bnew_to_old.append(f - ni)
        new_owner.extend(bo[ordp].tolist())
    del sizes
    out = PolyMesh(points=m.points, face_offsets=np.array(new_off, np.int64),
                   face_nodes=np.concatenate(new_nodes).astype(np.int32), owner=np.array(new_owner, np.int32),
                   neighbour=nei[iord].astype(np.int32), n_cells=m.n_cells, patch_names=list(m.patch_names),
                   patch_start=m.patch_start.copy(), patch_count=m.patch_count.copy())
    return out, np.array(bnew_to_old, np.int32)
