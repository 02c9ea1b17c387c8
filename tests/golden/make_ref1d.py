"""Generates tests/golden/converged/couette_slab_ref1d.npz from the reference's independent 1-D solver (ref1d).

ref1d (verification/ref1d/src/ref1d in the reference tree) solves the same planar Couette problem as the 3-D
kinetic solver with the y and z velocity components integrated out analytically, a high-order (p = 3) discretisation
in x and only xi_x discretised. Run in a container that has the reference sources:
    python tests/golden/make_ref1d.py
The problem is the 200-cell slab of tests/golden/converged/couette_slab_200.npz: walls at T = 1 moving along y
at -+0.1 most-probable speeds (u = -+0.1 sqrt(2) sqrt(R T0)), delta = 1 (Kn = sqrt(pi) / 2), omega = 0.81,
Pr = 2/3, solved on ref1d's default 200-cell mesh with two velocity grids:
  * "mid24": the midpoint rule on 24 points in [-5, 5], the x-axis of the 3-D solver's 24^3 grid, so the two
    solvers differ only by their discretisation in x;
  * "gl": ref1d's default composite Gauss-Legendre grid on (0, 10] per half (velocity converged), the physical
    answer the 24-point grid approximates.
Stored per grid: node positions x and the nodal fields rho, u_y, T, q_x, q_y, P_xy.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.refpath import reference_path  # noqa: E402

REF1D = reference_path("verification", "ref1d", "src")
FIELDS = ["rho", "uy", "T", "qx", "qy", "Pxy"]


def main():
    sys.path.insert(0, REF1D)
    from ref1d.mesh import make_mesh
    from ref1d.solver import Problem, solve_case
    from ref1d.velocity import gauss_legendre, midpoint

    u = 0.1 * np.sqrt(2.0)
    problem = Problem(Kn=np.sqrt(np.pi) / 2.0, omega=0.81, u_L=-u, u_R=u)
    out = {"meta.problem": np.array([problem.Kn, problem.omega, problem.u_L, problem.u_R, problem.Pr])}
    for name, grid in (("mid24", midpoint(24, 5.0)), ("gl", gauss_legendre())):
        r = solve_case(problem, make_mesh(200), grid)
        assert r.converged, name
        out[f"{name}.x"] = r.x
        for f in FIELDS:
            out[f"{name}.{f}"] = r.col(f)
        out[f"{name}.residual"] = np.array(r.residual)
    os.makedirs(os.path.join(HERE, "converged"), exist_ok=True)
    path = os.path.join(HERE, "converged", "couette_slab_ref1d.npz")
    np.savez_compressed(path, **out)
    print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
