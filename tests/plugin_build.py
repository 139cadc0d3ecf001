"""Compiles the test plugins of tests/plugins with gcc (as the reference's own
plugin tests compile theirs, tests/noise/test_native_plugins.py:37-49)."""

import subprocess
from pathlib import Path

SRC = Path(__file__).resolve().parent / "plugins"

VARIANTS = {
    "uniform": ("test_plugins.c", []),
    "layered": ("test_plugins.c", ["-DLAYERED"]),
    "keyed": ("test_plugins.c", ["-DKEYED"]),
    "bad_abi": ("test_plugins.c", ["-DBAD_ABI"]),
    "unknown_depends": ("test_plugins.c", ["-DUNKNOWN_DEPENDS"]),
    "no_factor": ("test_plugins.c", ["-DNO_FACTOR"]),
    "no_destroy": ("test_plugins.c", ["-DNO_DESTROY"]),
    "truncator": ("test_truncator.c", []),
}


def build_all(out_dir: Path) -> dict:
    out = {}
    for name, (src, flags) in VARIANTS.items():
        so = out_dir / f"{name}.so"
        subprocess.run(["gcc", "-shared", "-fPIC", "-O2", *flags, "-o", str(so), str(SRC / src), "-lm"], check=True)
        out[name] = so
    return out
