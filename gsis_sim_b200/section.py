"""Section cuts: the mass flow through a plane X = const along one axis (a diagnostic of the flow along a tube).

Follows the reference's src/mesh/section_cut.hpp / section_cut.cpp:
  * a cut at X on axis a is the set of internal faces whose two cells lie on opposite sides of X (cell centre
    x_c < X on one side, x_c >= X on the other) - a staircase on a general mesh, a plane on an aligned one. It splits
    the domain into {x_c < X} and the rest, so with a steady conservative discretisation the discrete flux through
    it equals the inlet / outlet flows (walls carry none);
  * `sign` is +1 when the face's area vector (owner -> neighbour) points from the x_c < X side to the other,
    -1 otherwise, so sum(sign * flux) is the flow in the +axis direction;
  * `area` is the total face area (L_ref^2), `projected_area` the sum of sign * S_axis, `face_position` the
    area-weighted mean face centre coordinate along the axis (X when the cut has no faces).
Positions are in L_ref units; the geometry is SI.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field

import numpy as np

_AXES = {"x": 0, "X": 0, "y": 1, "Y": 1, "z": 2, "Z": 2}


class SectionError(ValueError):
    """A malformed section specification (the reference raises gsis::Error in the same places)."""


@dataclass
class SectionSpec:
    """SectionSpec (src/mesh/section_cut.hpp): an axis (0, 1, 2) and positions in L_ref units, kept in the given
    order (repeats allowed)."""
    axis: int = 0
    positions: list = field(default_factory=list)

    def empty(self) -> bool:
        return len(self.positions) == 0


@dataclass
class SectionCut:
    """SectionCut (src/mesh/section_cut.hpp): the internal faces of one cut (mesh numbering) with their signs."""
    position: float
    axis: int
    faces: np.ndarray
    sign: np.ndarray
    area: float
    projected_area: float
    face_position: float


def parse_section_spec(positions: str, axis: str = "x") -> SectionSpec:
    """parse_section_spec (src/mesh/section_cut.cpp:11-38): positions separated by commas, semicolons, blanks or
    tabs; axis "x" / "y" / "z" (either case). An empty string gives no sections; a token that is not a finite
    number raises SectionError."""
    if axis not in _AXES:
        raise SectionError(f'section axis must be "x", "y" or "z" (got "{axis}")')
    vals = []
    for tok in re.split(r"[,; \t]+", positions):
        if not tok:
            continue
        try:
            v = float(tok)
        except ValueError:
            v = math.nan
        # the reference parses with from_chars, which takes neither "inf"/"nan" text nor a leading "+"
        if not math.isfinite(v) or tok.startswith("+") or not re.fullmatch(r"-?[0-9.]+([eE][-+]?[0-9]+)?", tok):
            raise SectionError(f'section position "{tok}" is not a number (in "{positions}")')
        vals.append(v)
    return SectionSpec(axis=_AXES[axis], positions=vals)


def section_axis_name(axis: int) -> str:
    """section_axis_name (src/mesh/section_cut.cpp:40-46)."""
    return {0: "x", 1: "y"}.get(axis, "z")


def build_section_cuts(owner, neighbour, cell_center, face_center, face_normal, face_area, length_scale: float,
                       spec: SectionSpec) -> list:
    """build_section_cuts (src/mesh/section_cut.cpp:48-81), vectorised over the internal faces.

    owner / neighbour: the internal faces' cells (len(neighbour) = number of internal faces); cell_center,
    face_center, face_area, face_normal (unit, owner -> neighbour): SI geometry; length_scale = L_ref [m]."""
    if spec.axis not in (0, 1, 2):
        raise SectionError(f"section axis {spec.axis} out of range")
    if not length_scale > 0.0:
        raise SectionError("the section length scale L_ref must be positive")
    a, L = spec.axis, float(length_scale)
    ni = len(neighbour)
    own = np.asarray(owner)[:ni]
    cc = np.asarray(cell_center)[:, a] / L
    xo, xn = cc[own], cc[np.asarray(neighbour)]
    A = np.asarray(face_area)[:ni] / (L * L)
    Sa = np.asarray(face_normal)[:ni, a] * np.asarray(face_area)[:ni] / (L * L)
    fc = np.asarray(face_center)[:ni, a] / L
    cuts = []
    for X in spec.positions:
        ob, nb = xo < X, xn < X
        faces = np.flatnonzero(ob != nb)
        sign = np.where(ob[faces], 1, -1).astype(np.int8)
        # sequential sums in face order, as the reference loop accumulates them
        area = _seq_sum(A[faces])
        proj = _seq_sum(sign * Sa[faces])
        sx = _seq_sum(A[faces] * fc[faces])
        cuts.append(SectionCut(position=float(X), axis=a, faces=faces.astype(np.int64), sign=sign, area=area,
                               projected_area=proj, face_position=sx / area if area > 0.0 else float(X)))
    return cuts


def _seq_sum(v: np.ndarray) -> float:
    s = 0.0
    for x in v.tolist():
        s += x
    return s


def section_flow(cut: SectionCut, face_flux) -> float:
    """section_flow (src/mesh/section_cut.cpp:83-91): sum of sign * face_flux[face] (face_flux indexed by internal
    face, owner -> neighbour)."""
    ff = np.asarray(face_flux)
    if len(cut.faces) and cut.faces.max() >= len(ff):
        raise SectionError("a section face lies outside the flux array")
    return _seq_sum(cut.sign * ff[cut.faces])


def owner_entries(csr_offsets, csr_other, csr_faces, owner, n_internal: int) -> tuple:
    """For every internal face: its neighbour cell and the CSR entry of the face in its owner's row, which is what
    the backend's internal_face_mass_flux reads (build_sections, src/kinetic/kinetic_solver.cpp:56-79).
    Raises SectionError if an internal face has no such entry."""
    offs = np.asarray(csr_offsets, np.int64)
    other = np.asarray(csr_other)
    cf = np.asarray(csr_faces, np.int64)
    own = np.asarray(owner)
    row_cell = np.repeat(np.arange(len(offs) - 1), np.diff(offs))
    e = np.flatnonzero((other >= 0) & (cf < n_internal))
    e = e[own[cf[e]] == row_cell[e]]
    neighbour = np.full(n_internal, -1, np.int64)
    entry = np.full(n_internal, -1, np.int64)
    neighbour[cf[e]] = other[e]
    entry[cf[e]] = e
    if n_internal and entry.min() < 0:
        f = int(np.flatnonzero(entry < 0)[0])
        raise SectionError(f"section face {f} is not in the face list of its owner cell {int(own[f])}")
    return neighbour, entry


@dataclass
class MassBalance:
    """MassBalance (src/kinetic/kinetic_output.hpp): inflow and outflow (both >= 0) and the imbalance
    (outflow - inflow) / max(inflow, outflow); valid when that scale is positive and every flow is finite."""
    inflow: float = 0.0
    outflow: float = 0.0
    imbalance: float = 0.0
    valid: bool = False


def mass_balance(patch_flow) -> MassBalance:
    """mass_balance (src/kinetic/kinetic_output.cpp:39-55): patch flows (nondimensional, outward positive) split
    into inflow (negative ones, negated) and outflow."""
    b = MassBalance()
    for F in np.asarray(patch_flow, float).tolist():
        if not math.isfinite(F):
            return b
        if F > 0.0:
            b.outflow += F
        else:
            b.inflow -= F
    scale = max(b.inflow, b.outflow)
    if scale > 0.0:
        b.imbalance = (b.outflow - b.inflow) / scale
        b.valid = True
    return b


def flow_spread(flows) -> float:
    """flow_spread (src/kinetic/kinetic_output.cpp:57-68): (max - min) / |mean| of at least two finite flows, else
    NaN (also NaN when the mean is 0)."""
    v = np.asarray(flows, float).tolist()
    if len(v) < 2 or not all(math.isfinite(x) for x in v):
        return math.nan
    s = 0.0
    for x in v:
        s += x
    mean = s / len(v)
    return (max(v) - min(v)) / abs(mean) if mean != 0.0 else math.nan
