"""Installs the unmodified reference package into baseline/_ref/.

bench.py's baseline legs import the reference's own optimizer from there
(core/lbfgs_torch_parallel.py: torch only, no cupy) to time the plain forms
the batched relaxation is compared with.  baseline/_ref/ is git-ignored; it
travels with the working tree to a GPU box, where the reference tree itself
is absent.  The install is pip's, offline, from a copy of the tree (the
build writes into its source directory, which must stay untouched):

    python baseline/install_ref.py [/path/to/reference]   (default: oracle.refsrc)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
TARGET = os.path.join(HERE, "_ref")


def install(ref: str) -> str:
    if not os.path.isdir(os.path.join(ref, "core")):
        raise FileNotFoundError(f"no reference tree at {ref}")
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "reference")
        shutil.copytree(ref, src, ignore=shutil.ignore_patterns("*.ipynb", "res", "analysis", ".git"))
        if os.path.isdir(TARGET):
            shutil.rmtree(TARGET)
        cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation", "--no-deps",
               "--find-links", "/opt/wheelhouse", "--target", TARGET, src]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("pip install of the reference failed:\n" + r.stderr[-4000:])
    return TARGET


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(HERE))
    from oracle.refsrc import reference_dir
    print(install(sys.argv[1] if len(sys.argv) > 1 else reference_dir()))
