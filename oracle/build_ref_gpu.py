"""Build recipe of the reference's own GPU kernel (test and measurement
infrastructure, not the engine).

Reads cuPeriod's CUDA source string ``_BLS_CUDA_SRC`` and ``CUDA_BLOCK`` out of
the reference tree (``src/cuperiod/methods/_bls_core.py:64, 505-656``) without
importing or copying it into this repository, substitutes ``REAL`` and
``CUDA_BLOCK`` as the reference's ``_cuda_kernel`` does (``:661-672``) for its
double default and its float32 opt-in, and compiles both, with this
directory's own launcher (``ref_gpu_launcher.cu``), for sm_100a into
``oracle/_ref/libref_bls_block.so``.  The generated source lives in a temporary
directory outside the repository.

Usage: ``python oracle/build_ref_gpu.py [REFERENCE_ROOT]`` (default: the
``CUPERIOD_REFERENCE`` environment variable, else /root/reference).  Without a
reference tree it does nothing; the built library travels with the
repository's other built files.
"""

from __future__ import annotations

import ast
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libref_bls_block.so")
DEFAULT_ROOT = os.environ.get("CUPERIOD_REFERENCE", "/root/reference")


def _constants(path: str) -> tuple[str, int]:
    tree = ast.parse(open(path).read())
    src, block = None, None
    for node in tree.body:
        targets = []
        if isinstance(node, ast.Assign):
            targets = [t.id for t in node.targets if isinstance(t, ast.Name)]
        elif isinstance(node, ast.AnnAssign) and isinstance(node.target, ast.Name):
            targets = [node.target.id]
        value = getattr(node, "value", None)
        if "_BLS_CUDA_SRC" in targets and isinstance(value, ast.Constant):
            src = value.value
        if "CUDA_BLOCK" in targets and isinstance(value, ast.Constant):
            block = int(value.value)
    if src is None or block is None:
        raise RuntimeError(f"no _BLS_CUDA_SRC / CUDA_BLOCK in {path}")
    return src, block


def build(reference_root: str | None) -> str | None:
    if not reference_root:
        return None
    core = os.path.join(reference_root, "src", "cuperiod", "methods", "_bls_core.py")
    if not os.path.exists(core):
        return None
    src, block = _constants(core)
    deps = [core, os.path.join(HERE, "ref_gpu_launcher.cu"), os.path.abspath(__file__)]
    if os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in deps):
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        sources = []
        # one translation unit per precision (the kernel's block-scope
        # `extern __shared__` array must not meet its other-precision twin)
        for real, name in (("double", "bls_block_f64"), ("float", "bls_block_f32")):
            cu = os.path.join(tmp, f"{name}.cu")
            with open(cu, "w") as fh:
                fh.write(src.replace("CUDA_BLOCK", str(block)).replace("REAL", real)
                         .replace("bls_block", name))
            sources.append(cu)
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                        "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
                        f"-DREF_CUDA_BLOCK={block}", "-o", OUT, *sources,
                        os.path.join(HERE, "ref_gpu_launcher.cu")], check=True)
    return OUT


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else DEFAULT_ROOT
    out = build(root)
    print(out or "no reference tree: nothing built")
