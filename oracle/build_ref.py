"""Build the reference's code as test checkers and as the timed CPU baseline.

    python oracle/build_ref.py [--reference /path/to/pyTME] [--baseline]

* ``build``: compiles the reference's native helper (tme/external/bindings.cpp) where
  it lies in the reference checkout (read-only) into ``oracle/_ref/``, a checker for the
  greedy distance filter.
* ``install_baseline`` (``--baseline``): installs the reference package offline into
  ``baseline/_ref`` (``pip install --no-index --no-build-isolation --no-deps`` from a
  temporary copy, since its build writes into the source tree), then recompiles its
  pybind11 helper with portable flags: the package's own setup.py builds it with
  ``-march=native``, which would tie it to this machine's CPU, and the copy travels
  to other hosts. The GPU tests use it to drive tme's own ``scan_subsets`` through the
  B200 backend, and ``bench.py --impl reference`` times tme's own scoring loop with it.
  Its third-party imports that are not installed (pyFFTW, h5py, mrcfile, scikit-image)
  are provided by ``tests/golden/refshim``.

Both outputs are git-ignored and are not product code: nothing in ``pytme_b200``
imports them.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import sysconfig
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT_DIR = os.path.join(HERE, "_ref")
INSTALL_DIR = os.path.join(ROOT, "baseline", "_ref")
WHEELHOUSE = "/opt/wheelhouse"


def _compile_bindings(src: str, out: str) -> str:
    inc = subprocess.check_output([sys.executable, "-m", "pybind11", "--includes"],
                                  text=True).split()
    subprocess.check_call(["c++", "-O3", "-std=c++14", "-shared", "-fPIC", *inc, src, "-o", out])
    return out


def build(reference: str) -> str:
    src = os.path.join(reference, "tme", "external", "bindings.cpp")
    if not os.path.exists(src):
        raise FileNotFoundError(src)
    os.makedirs(OUT_DIR, exist_ok=True)
    out = os.path.join(OUT_DIR, "extensions" + sysconfig.get_config_var("EXT_SUFFIX"))
    return _compile_bindings(src, out)


def install_baseline(reference: str, force: bool = False) -> str:
    """Offline install of the reference package into baseline/_ref (see module doc)."""
    pkg = os.path.join(INSTALL_DIR, "tme")
    if os.path.isdir(pkg) and not force:
        return INSTALL_DIR
    if not os.path.isdir(os.path.join(reference, "tme")):
        raise FileNotFoundError(os.path.join(reference, "tme"))
    tmp = tempfile.mkdtemp(prefix="pytme_ref_src_")
    src = os.path.join(tmp, "src")
    shutil.copytree(reference, src, ignore=shutil.ignore_patterns(".git"))
    cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation",
           "--no-deps", "--upgrade", "--target", INSTALL_DIR, src]
    if os.path.isdir(WHEELHOUSE):
        cmd[4:4] = ["--find-links", WHEELHOUSE]
    subprocess.check_call(cmd, stdout=subprocess.DEVNULL)
    ext = os.path.join(pkg, "extensions" + sysconfig.get_config_var("EXT_SUFFIX"))
    _compile_bindings(os.path.join(src, "tme", "external", "bindings.cpp"), ext)
    shutil.rmtree(tmp, ignore_errors=True)
    return INSTALL_DIR


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PYTME_REFERENCE", "/root/reference"))
    ap.add_argument("--baseline", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.reference))
    if a.baseline:
        print(install_baseline(a.reference, force=a.force))
