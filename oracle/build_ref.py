"""Builds the reference's own CUDA kernels from its source into oracle/_ref/.

TEST INFRASTRUCTURE ONLY: the cubins are used by tests to compare this
package's kernels with the reference's kernels on the same inputs; nothing in
the product loads them.

The reference keeps its CUDA as Python string constants (core/pack_cuda.py:65,
core/pack_cuda_primitives.py:16, core/pack_cuda_lut.py:260, core/lap_batch.py:45)
and compiles them at run time with nvcc.  This recipe reads those strings
with ``ast`` (nothing is imported or executed), applies the same float32
substitutions the reference applies (pack_cuda.py:893-897,
pack_cuda_lut.py:713-726) and runs nvcc with the reference's flags
(pack_cuda.py:938-945) for sm_100a.  The extracted sources are written to a
temporary directory only; oracle/_ref/ receives the cubins.

    python oracle/build_ref.py [/path/to/reference]   (default: oracle.refsrc)
"""
from __future__ import annotations

import ast
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
FLAGS = ["-O3", "-use_fast_math", "--extra-device-vectorization", "-gencode", "arch=compute_100a,code=sm_100a"]


def _string_assign(path, name, env):
    tree = ast.parse(open(path).read())
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id == name for t in node.targets):
            return _eval(node.value, env)
    raise KeyError(f"{name} not found in {path}")


def _eval(node, env):
    """Evaluates string concatenations of literals, names and str(name)."""
    if isinstance(node, ast.Constant) and isinstance(node.value, str):
        return node.value
    if isinstance(node, ast.BinOp) and isinstance(node.op, ast.Add):
        return _eval(node.left, env) + _eval(node.right, env)
    if isinstance(node, ast.Call) and isinstance(node.func, ast.Name) and node.func.id == "str":
        return str(env[node.args[0].id])
    if isinstance(node, ast.Attribute):
        return env[f"{node.value.id}.{node.attr}"]
    if isinstance(node, ast.Name):
        return env[node.id]
    raise ValueError(f"unsupported expression {ast.dump(node)[:80]}")


def sources(ref_root):
    sys.path.insert(0, HERE)
    import oracle  # noqa: E402  (the FP64 restatement gives the tree radius)
    R = oracle.geometry()[3]
    core = os.path.join(ref_root, "core")
    prim = _string_assign(os.path.join(core, "pack_cuda_primitives.py"), "PRIMITIVE_SRC", {})
    env = {"MAX_OVERLAP_DIST_SQ": (2.0 * R) ** 2, "pack_cuda_primitives.PRIMITIVE_SRC": prim}
    pc = _string_assign(os.path.join(core, "pack_cuda.py"), "_CUDA_SRC", env).replace("double", "float")
    lut = _string_assign(os.path.join(core, "pack_cuda_lut.py"), "_CUDA_SRC", {})
    lut = lut.replace("$MAX_RADIUS$", str(R)).replace("double", "float")
    lut = lut.replace("sincos(", "sincosf(").replace("floor(", "floorf(")
    lut = re.sub(r"(\d+\.\d+)(?![eEf])", r"\1f", lut)
    lap = _string_assign(os.path.join(core, "lap_batch.py"), "_CUDA_SRC", {})
    return {"pack_cuda": pc, "pack_cuda_lut": lut, "lap_batch": lap}


def build(ref_root):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    os.makedirs(OUT, exist_ok=True)
    srcs = sources(ref_root)
    jobs = [("pack_cuda_area", "pack_cuda", ["-DENABLE_OVERLAP_AREA"]),
            ("pack_cuda_sep", "pack_cuda", ["-DENABLE_SEPARATION"]),
            ("pack_cuda_lut", "pack_cuda_lut", []),
            ("lap_batch", "lap_batch", [])]
    with tempfile.TemporaryDirectory() as tmp:
        for out_name, key, defs in jobs:
            cu = os.path.join(tmp, key + ".cu")
            with open(cu, "w") as f:
                f.write(srcs[key])
            cmd = [nvcc] + FLAGS + defs + ["-cubin", cu, "-o", os.path.join(OUT, out_name + ".cubin")]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {out_name}:\n{r.stderr[-2000:]}")
    return OUT


if __name__ == "__main__":
    # refsrc sits beside this script (imported by file: the package name
    # "oracle" would resolve to oracle/oracle.py from here)
    sys.path.insert(0, HERE)
    from refsrc import reference_dir
    print(build(sys.argv[1] if len(sys.argv) > 1 else reference_dir()))
