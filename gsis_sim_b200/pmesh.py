"""Reader and writer of the reference's `.pmesh` mesh files (format v1, the reference's docs/pmesh_format.md;
reader/writer src/mesh/pmesh_io.cpp:1-470).

Layout: bytes 0-7 the magic "PMESH\\0\\0\\0"; bytes 8-15 a little-endian uint64 H; then H bytes of UTF-8 JSON (format,
version, length_unit, counts, patches, arrays with dtype / shape / absolute offset, optional metadata); then the arrays
at their 64-byte-aligned offsets. Faces: internal faces first (owner < neighbour, sorted by (owner, neighbour)),
then boundary faces patch by patch in the order of `patches`.

`read_pmesh` checks the file structure and the topology (as the reference reader does) and returns a `PolyMesh`;
`load_pmesh` also computes the geometry and checks closedness, positive volumes and internal-face orientation.
Violations raise `PmeshError`.
"""
from __future__ import annotations

import json
import struct
import warnings

import numpy as np

from .mesh import PolyMesh, compute_geometry

MAGIC = b"PMESH\x00\x00\x00"
VERSION = 1
PATCH_KINDS = ("wall", "inlet", "outlet", "symmetry", "patch")
_DTYPES = {"float64": np.dtype("<f8"), "int64": np.dtype("<i8"), "int32": np.dtype("<i4")}
_INDEX_ARRAYS = ("face_offsets", "face_nodes", "owner", "neighbour")


class PmeshError(ValueError):
    """A .pmesh file violates the format (the reference raises gsis::Error in the same places)."""


def _check(cond, msg):
    if not cond:
        raise PmeshError(msg)


def _read_array(buf: bytes, name: str, spec: dict, file_size: int) -> np.ndarray:
    _check(isinstance(spec, dict) and {"dtype", "shape", "offset"} <= set(spec), f"array {name}: dtype/shape/offset")
    dt = _DTYPES.get(spec["dtype"])
    _check(dt is not None, f"array {name}: unknown dtype {spec['dtype']!r}")
    if name == "points":
        _check(spec["dtype"] == "float64", "points must be float64")
    else:
        _check(spec["dtype"] in ("int32", "int64"), f"{name} must be int32 or int64")
    shape = tuple(int(x) for x in spec["shape"])
    off = int(spec["offset"])
    n = int(np.prod(shape)) if shape else 1
    _check(off >= 0 and off + n * dt.itemsize <= file_size, f"array {name} lies outside the file")
    a = np.frombuffer(buf, dtype=dt, count=n, offset=off).reshape(shape)
    return a.astype(np.float64) if name == "points" else a


def read_pmesh(path: str) -> PolyMesh:
    """Read a .pmesh file and check its structure and topology (not its geometry)."""
    with open(path, "rb") as fh:
        buf = fh.read()
    _check(len(buf) >= 16 and buf[:8] == MAGIC, f"{path}: not a .pmesh file (magic)")
    (hlen,) = struct.unpack("<Q", buf[8:16])
    _check(16 + hlen <= len(buf), f"{path}: header longer than the file")
    try:
        hdr = json.loads(buf[16:16 + hlen].decode("utf-8"))
    except (UnicodeDecodeError, json.JSONDecodeError) as e:
        raise PmeshError(f"{path}: header is not valid UTF-8 JSON: {e}") from e
    _check(hdr.get("format") == "pmesh", f"{path}: format is not 'pmesh'")
    _check(hdr.get("version") == VERSION, f"{path}: unsupported version {hdr.get('version')!r}")
    _check(hdr.get("length_unit", "m") == "m", f"{path}: length_unit must be 'm'")
    meta = hdr.get("metadata", {}) or {}
    for k, v in meta.items():
        if not isinstance(v, str):
            warnings.warn(f"{path}: metadata {k!r} is not a string and is skipped")
    n_points, n_faces = int(hdr["n_points"]), int(hdr["n_faces"])
    n_int, n_cells = int(hdr["n_internal_faces"]), int(hdr["n_cells"])
    arrays = hdr.get("arrays", {})
    for k in ("points", *_INDEX_ARRAYS):
        _check(k in arrays, f"{path}: array {k} missing")
    a = {k: _read_array(buf, k, arrays[k], len(buf)) for k in ("points", *_INDEX_ARRAYS)}
    mesh = PolyMesh(points=np.ascontiguousarray(a["points"].reshape(-1, 3)),
                    face_offsets=a["face_offsets"].astype(np.int64).ravel(),
                    face_nodes=a["face_nodes"].astype(np.int32).ravel(),
                    owner=a["owner"].astype(np.int32).ravel(),
                    neighbour=a["neighbour"].astype(np.int32).ravel(), n_cells=n_cells)
    _check(mesh.points.shape == (n_points, 3), f"{path}: points shape")
    _check(len(mesh.owner) == n_faces and len(mesh.face_offsets) == n_faces + 1, f"{path}: face array lengths")
    _check(len(mesh.neighbour) == n_int and 0 <= n_int <= n_faces, f"{path}: neighbour length")
    patches = hdr.get("patches", [])
    names, starts, counts, kinds = [], [], [], []
    expect = n_int
    for p in patches:
        name, kind, start, count = p["name"], p["kind"], int(p["start"]), int(p["count"])
        _check(kind in PATCH_KINDS, f"{path}: patch {name!r} has unknown kind {kind!r}")
        _check(name not in names, f"{path}: patch name {name!r} repeated")
        _check(start == expect and count >= 0, f"{path}: patch {name!r} does not follow the previous one")
        if count == 0:
            warnings.warn(f"{path}: patch {name!r} has no faces")
        names.append(name)
        kinds.append(kind)
        starts.append(start)
        counts.append(count)
        expect = start + count
    _check(expect == n_faces, f"{path}: patches do not cover the boundary faces")
    mesh.patch_names = names
    mesh.patch_kinds = kinds
    mesh.patch_start = np.array(starts, np.int64)
    mesh.patch_count = np.array(counts, np.int64)
    mesh.metadata = {k: v for k, v in meta.items() if isinstance(v, str)}
    check_topology(mesh)
    return mesh


def check_topology(mesh: PolyMesh) -> None:
    """Index ranges, face sizes and the internal-face order of the format (rules 1, 2, 4 and 6)."""
    fo, fn = mesh.face_offsets, mesh.face_nodes
    _check(fo[0] == 0 and np.all(np.diff(fo) >= 3) and fo[-1] == len(fn), "every face needs 3 or more nodes")
    _check(len(fn) == 0 or (fn.min() >= 0 and fn.max() < len(mesh.points)), "face node index out of range")
    for f in range(mesh.n_faces):
        nodes = fn[fo[f]:fo[f + 1]]
        _check(len(np.unique(nodes)) == len(nodes), f"face {f} repeats a node")
    _check(mesh.owner.min(initial=0) >= 0 and mesh.owner.max(initial=-1) < mesh.n_cells, "owner out of range")
    ni = mesh.n_internal
    if ni:
        o, nb = mesh.owner[:ni].astype(np.int64), mesh.neighbour.astype(np.int64)
        _check(nb.max() < mesh.n_cells, "neighbour out of range")
        _check(np.all(o < nb), "internal faces need owner < neighbour")
        key = o * mesh.n_cells + nb
        _check(np.all(np.diff(key) >= 0), "internal faces are not sorted by (owner, neighbour)")


def load_pmesh(path: str, closed_tol: float = 1e-10):
    """read_pmesh + the geometric checks of the reference loader: each cell closed (|sum S_out| <= 1e-10 sum |S|)
    and of positive volume; internal faces pointing from owner to neighbour are only counted (a warning).
    Returns (mesh, geometry, warnings)."""
    mesh = read_pmesh(path)
    g = compute_geometry(mesh)
    msgs = []
    ni = mesh.n_internal
    S = g.face_area_vector
    absS = np.linalg.norm(S, axis=1)
    acc = np.zeros((mesh.n_cells, 3))
    tot = np.zeros(mesh.n_cells)
    np.add.at(acc, mesh.owner, S)
    np.add.at(tot, mesh.owner, absS)
    np.add.at(acc, mesh.neighbour, -S[:ni])
    np.add.at(tot, mesh.neighbour, absS[:ni])
    bad = np.linalg.norm(acc, axis=1) > closed_tol * tot
    _check(not bad.any(), f"{path}: {int(bad.sum())} cells are not closed")
    _check(np.all(g.cell_volume > 0), f"{path}: non-positive cell volume")
    if ni:
        d = g.cell_center[mesh.neighbour] - g.cell_center[mesh.owner[:ni]]
        wrong = int(np.sum(np.einsum("ij,ij->i", S[:ni], d) <= 0))
        if wrong:
            msgs.append(f"{wrong} internal faces point from the neighbour to the owner")
            warnings.warn(f"{path}: {msgs[-1]}")
    return mesh, g, msgs


def write_pmesh(path: str, mesh: PolyMesh, metadata: dict | None = None) -> None:
    """Write a .pmesh file (points float64, face_offsets int64, the other index arrays int32), arrays packed at
    64-byte boundaries after the header, as the reference writer does."""
    check_topology(mesh)
    kinds = mesh.patch_kinds or ["patch"] * len(mesh.patch_names)
    arrays = [("points", np.ascontiguousarray(mesh.points, "<f8")),
              ("face_offsets", np.ascontiguousarray(mesh.face_offsets, "<i8")),
              ("face_nodes", np.ascontiguousarray(mesh.face_nodes, "<i4")),
              ("owner", np.ascontiguousarray(mesh.owner, "<i4")),
              ("neighbour", np.ascontiguousarray(mesh.neighbour, "<i4"))]
    names = {"<f8": "float64", "<i8": "int64", "<i4": "int32"}

    def header(offsets):
        h = {"format": "pmesh", "version": VERSION, "length_unit": "m", "n_points": int(len(mesh.points)),
             "n_faces": int(mesh.n_faces), "n_internal_faces": int(mesh.n_internal), "n_cells": int(mesh.n_cells),
             "patches": [{"name": n, "kind": k, "start": int(s), "count": int(c)}
                         for n, k, s, c in zip(mesh.patch_names, kinds, mesh.patch_start, mesh.patch_count)],
             "arrays": {n: {"dtype": names[a.dtype.str], "shape": list(a.shape), "offset": int(o)}
                        for (n, a), o in zip(arrays, offsets)}}
        if metadata:
            h["metadata"] = {str(k): str(v) for k, v in metadata.items()}
        return json.dumps(h, indent=2).encode("utf-8")

    # offsets depend on the header length, which depends on the offsets' digits: iterate to a fixed point
    offsets = [0] * len(arrays)
    for _ in range(4):
        hb = header(offsets)
        pos = 16 + len(hb)
        new = []
        for _, a in arrays:
            pos = (pos + 63) // 64 * 64
            new.append(pos)
            pos += a.nbytes
        if new == offsets:
            break
        offsets = new
    hb = header(offsets)
    with open(path, "wb") as fh:
        fh.write(MAGIC)
        fh.write(struct.pack("<Q", len(hb)))
        fh.write(hb)
        pos = 16 + len(hb)
        for (_, a), o in zip(arrays, offsets):
            fh.write(b"\x00" * (o - pos))
            fh.write(a.tobytes())
            pos = o + a.nbytes
