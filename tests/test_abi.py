"""The C-ABI library loads and exports every symbol include/gsis_b200.h declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

from gsis_sim_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "gsis_b200.h")).read()
    return sorted(set(re.findall(r"\b(kin_[a-z_0-9]+)\s*\(", text)))


def test_header_and_loader_agree():
    assert sorted(_lib.EXPORTED_SYMBOLS) == declared_symbols()


def test_header_constants_match_the_binding():
    """Every #define KIN_* value the Python binding copies equals the header's."""
    from gsis_sim_b200 import abi

    text = open(os.path.join(ROOT, "include", "gsis_b200.h")).read()
    defines = {k: int(v) for k, v in re.findall(r"#define\s+(KIN_[A-Z_0-9]+)\s+\(?(-?\d+)\)?", text)}
    assert "KIN_NOALLOC_MAX_STATES" in defines
    checked = [k for k in defines if hasattr(abi, k)]
    assert len(checked) >= 8, checked
    for k in checked:
        assert getattr(abi, k) == defines[k], (k, getattr(abi, k), defines[k])


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.fail(f"{_lib.LIB_PATH} missing: run __graft_entry__.build()")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_create_without_gpu_fails_loudly():
    """Without a device kin_create must return an error (no silent CPU fallback)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from tests import common
    from gsis_sim_b200.backend import B200Backend, KineticError

    _, setup = common.load("couette_fp64")
    with pytest.raises(KineticError):
        B200Backend(setup)
