"""Compile the reference's native helper (tme/external/bindings.cpp) into
``oracle/_ref/`` as a checker for the greedy distance filter.

    python oracle/build_ref.py [--reference /path/to/pyTME]

The source is compiled where it lies in the reference checkout (read-only); only
the shared object is written, to ``oracle/_ref/`` (git-ignored, shipped with the
working tree). Test infrastructure only: tests import it to cross-check
``find_candidate_indices``; nothing in the package uses it.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")


def build(reference: str) -> str:
    src = os.path.join(reference, "tme", "external", "bindings.cpp")
    if not os.path.exists(src):
        raise FileNotFoundError(src)
    os.makedirs(OUT_DIR, exist_ok=True)
    out = os.path.join(OUT_DIR, "extensions" + sysconfig.get_config_var("EXT_SUFFIX"))
    inc = subprocess.check_output([sys.executable, "-m", "pybind11", "--includes"],
                                  text=True).split()
    subprocess.check_call(["c++", "-O3", "-std=c++14", "-shared", "-fPIC", *inc, src, "-o", out])
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PYTME_REFERENCE", "/root/reference"))
    print(build(ap.parse_args().reference))
