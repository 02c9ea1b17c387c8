"""The reference's case files: .pmesh meshes and TOML case definitions (no GPU needed).

Self-contained: .pmesh write/read round trip and the format's error cases; the TOML rules (required sections,
unknown keys, exactly one of delta_rp / Kn / p_ref). With the reference tree and its CPU library present (this
container): every case file of the reference parses, and the kinetic set-up built from a case file equals the one the
reference's own builder makes for the same mesh and conditions, array for array.
"""
import glob
import os
import struct

import numpy as np
import pytest

from gsis_sim_b200 import case
from gsis_sim_b200.mesh import box_mesh
from gsis_sim_b200.pmesh import PmeshError, load_pmesh, read_pmesh, write_pmesh
from oracle.refpath import reference_path

HERE = os.path.dirname(os.path.abspath(__file__))
CHANNEL = os.path.join(HERE, "golden", "case_channel", "channel.toml")
REF_CASES = reference_path("cases")


def _box():
    m = box_mesh((3, 2, 2), (0.0, 0.0, 0.0), (3.0, 2.0, 1.0), ("in", "out", "wall", "wall", "wall", "wall"))
    m.patch_kinds = ["inlet", "outlet", "wall"]
    return m


def test_pmesh_round_trip(tmp_path):
    m = _box()
    p = tmp_path / "box.pmesh"
    write_pmesh(str(p), m, {"note": "test"})
    r = read_pmesh(str(p))
    for k in ("points", "face_offsets", "face_nodes", "owner", "neighbour", "patch_start", "patch_count"):
        assert np.array_equal(getattr(m, k), getattr(r, k)), k
    assert r.patch_names == m.patch_names and r.patch_kinds == m.patch_kinds and r.metadata == {"note": "test"}
    _, g, warns = load_pmesh(str(p))
    assert abs(g.cell_volume.sum() - 6.0) < 1e-12 and warns == []
    data = p.read_bytes()
    (hlen,) = struct.unpack("<Q", data[8:16])
    assert data[:8] == b"PMESH\0\0\0" and all(o % 64 == 0 for o in _offsets(data[16:16 + hlen]))


def _offsets(header_bytes):
    import json

    return [a["offset"] for a in json.loads(header_bytes)["arrays"].values()]


def test_pmesh_errors(tmp_path):
    p = tmp_path / "x.pmesh"
    p.write_bytes(b"NOTPMESH" + b"\0" * 32)
    with pytest.raises(PmeshError):
        read_pmesh(str(p))
    m = _box()
    m.patch_kinds = ["inlet", "outlet", "wal"]
    with pytest.raises(PmeshError):
        write_pmesh(str(tmp_path / "k.pmesh"), m)
        read_pmesh(str(tmp_path / "k.pmesh"))
    m = _box()
    m.neighbour = m.neighbour[::-1].copy()  # internal faces no longer sorted / owner < neighbour broken
    with pytest.raises(PmeshError):
        write_pmesh(str(tmp_path / "s.pmesh"), m)


BASE = '''
[case]
name = "t"
mesh = "m.pmesh"
[gas]
molecular_mass = 6.63e-26
mu_ref = 2.117e-5
T_ref = 273.0
omega = 0.81
[conditions]
L_ref = 1.0
T0 = 273.0
{cond}
[[boundary]]
patch = "wall"
type = "diffuse_wall"
temperature = 273.0
{extra}
[velocity_grid]
n = [4, 4, 4]
range = [[-4.0, 4.0], [-4.0, 4.0], [-4.0, 4.0]]
'''


def test_toml_rules():
    c = case.parse_case_toml(BASE.format(cond="Kn = 0.1", extra=""))
    assert c.mode == "gsis" and c.conditions.Kn == 0.1 and c.velocity_grid["n"] == (4, 4, 4)
    with pytest.raises(case.CaseError):  # two of delta_rp / Kn / p_ref
        case.parse_case_toml(BASE.format(cond="Kn = 0.1\ndelta_rp = 1.0", extra=""))
    with pytest.raises(case.CaseError):  # unknown key in a typed section
        case.parse_case_toml(BASE.format(cond="Kn = 0.1", extra="colour = 3"))
    with pytest.raises(case.CaseError):  # missing required section
        case.parse_case_toml(BASE.format(cond="Kn = 0.1", extra="").replace("[velocity_grid]", "[velo]"))
    c = case.parse_case_toml(BASE.format(cond="Kn = 0.1", extra="") + "\n[kinetic]\nlimiter = \"nonsense\"\n")
    with pytest.raises(case.CaseError):
        case.kinetic_params(c)


def _kp(kinetic: str):
    return case.kinetic_params(case.parse_case_toml(BASE.format(cond="Kn = 0.1", extra="") + "\n[kinetic]\n" + kinetic))


def test_kinetic_params_defaults_and_values():
    """tests/kinetic/test_kinetic_params.cpp:44-71 and the [kinetic] part of test_kinetic_phase5.cpp:373-400."""
    d = case.kinetic_params(case.parse_case_toml(BASE.format(cond="Kn = 0.1", extra="")))
    assert d.pseudo_cfl == 0.0 and d.sweep_blocks == 0 and d.precision == "fp32" and d.boundary_iterations == 1
    assert d.cold_bgk_temperature == 0.0 and d.deq_fallback == "collisionless"
    assert d.pressure_boundary_reconstruction == "limited"
    p = _kp('pseudo_cfl = 50\nsweep_blocks = 8\nprecision = "fp64"\nbackend = "cpu"\nboundary_iterations = 8\n')
    assert p.pseudo_cfl == 50.0 and p.sweep_blocks == 8 and p.precision == "fp64" and p.boundary_iterations == 8
    q = _kp('limiter = "none"\nlimiter_eps = "relative"\ninitial_pressure = 0.5\ninitial_temperature = 1.2\n'
            'convergence_u_floor = 0.01\nlaunch_cells = 100\nsweep_cells_per_launch = 10\n')
    assert q.limiter == "none" and q.limiter_eps == "relative" and q.initial_pressure == 0.5
    assert q.initial_temperature == 1.2 and q.convergence_u_floor == 0.01
    c = _kp('cold_bgk_temperature = 0.1\ndeq_fallback = "continuous"\npressure_boundary_reconstruction = "cell"\n')
    assert c.cold_bgk_temperature == 0.1 and c.deq_fallback == "continuous"
    assert c.pressure_boundary_reconstruction == "cell"


@pytest.mark.parametrize("kinetic,word", [("boundary_iterations = 0", "boundary_iterations"),
                                          ("boundary_iterations = 1001", "boundary_iterations"),
                                          ("sweep_block = 8", "sweep_block"),
                                          ('precision = "fp16"', "kinetic.precision"),
                                          ('limiter = "minmod"', "kinetic.limiter"),
                                          ("initial_pressure = 0", "initial"),
                                          ('deq_fallback = "none"', "deq_fallback"),
                                          ("cold_bgk_temperature = -1", "cold_bgk_temperature")])
def test_kinetic_params_errors(kinetic, word):
    """tests/kinetic/test_kinetic_params.cpp:73-86 and test_kinetic_phase5.cpp:398-401: each bad value is an error
    that names the key."""
    with pytest.raises(case.CaseError, match=word):
        _kp(kinetic + "\n")


def test_channel_fixture_builds():
    cfg = case.load_case(CHANNEL)
    setup, host = case.case_setup(cfg)
    assert setup.n_cells == 72 and setup.nv == 12 * 12 * 8
    assert host.patch_dbl[0, 1] == 1.0 and 0.4 < host.patch_dbl[1, 1] < 0.6  # p_in = p_ref, pressure ratio ~2


_have_ref = os.path.isdir(REF_CASES)


@pytest.mark.skipif(not _have_ref, reason="reference tree not present")
def test_every_reference_case_file_parses():
    files = sorted(glob.glob(os.path.join(REF_CASES, "**", "*.toml"), recursive=True))
    assert files
    for f in files:
        case.load_case(f)


@pytest.mark.skipif(not _have_ref, reason="reference tree not present")
@pytest.mark.parametrize("rel", ["verification/kinetic/slab_couette_lin_Kn0p01_nx100.toml",
                                 "verification/kinetic/slab_heat_nl_Kn1_nx50.toml", "smoke/smoke.toml"])
def test_case_setup_matches_reference_builder(rel):
    from oracle import ref

    if not ref.available():
        pytest.skip("oracle/_ref/libgsisref.so not built")
    cfg = case.load_case(os.path.join(REF_CASES, rel))
    mesh = read_pmesh(cfg.mesh)
    setup, host = case.case_setup(cfg, precision="fp64", mesh=mesh)
    bcs = case.boundary_conditions(cfg, mesh.patch_names)
    c, vg = cfg.conditions, cfg.velocity_grid
    spec = ref.case_spec([(b.patch, b.type, dict(T=b.T, p=b.p, u=b.u, alpha=b.alpha)) for b in bcs], Kn=c.Kn,
                         delta_rp=c.delta_rp, nv=vg["n"], vlo=vg["lo"], vhi=vg["hi"],
                         kinetic=dict(cfg.kinetic, precision="fp64"), omega=cfg.gas.omega,
                         molecular_mass=cfg.gas.molecular_mass, mu_ref=cfg.gas.mu_ref, T_ref=cfg.gas.T_ref,
                         T0=c.T0, L_ref=c.L_ref)
    rc = ref.RefCase(ref.RefMesh.from_arrays(mesh.as_dict()), spec)
    for k, a in setup.arrays.items():
        b = rc.setup.arrays.get(k)
        assert (a is None) == (b is None), k
        if a is None:
            continue
        a, b = np.asarray(a), np.asarray(b)
        assert a.shape == b.shape, k
        if a.dtype.kind == "f":
            assert np.max(np.abs(a - b), initial=0.0) <= 1e-12 * max(np.max(np.abs(b), initial=0.0), 1e-300), k
        else:
            assert np.array_equal(a, b), k
    assert np.array_equal(host.patch_dbl, rc.patch_dbl)
