"""Where the reference's source tree lies (TEST INFRASTRUCTURE: only the oracle build, fixture generators and tests
read it). The environment variable GSIS_REFERENCE names it; without it the oracle Makefile's default is used."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_root() -> str:
    """The reference tree: $GSIS_REFERENCE, else the REF default of oracle/Makefile."""
    env = os.environ.get("GSIS_REFERENCE")
    if env:
        return env
    try:
        out = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True, check=True)
        return out.stdout.strip()
    except (OSError, subprocess.CalledProcessError):
        return ""


def reference_path(*parts: str) -> str:
    """A path inside the reference tree ("" when the tree is unknown)."""
    root = reference_root()
    return os.path.join(root, *parts) if root else ""
