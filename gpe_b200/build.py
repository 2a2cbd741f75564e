"""Build recipe for the in-tree CUDA library ``gpe_b200/libgpe_gpu.so``.

Compiles ``gpe_b200/csrc/*.cu`` for sm_100a only with nvcc (cross-compiles
without a GPU).  The CUDA runtime is linked statically and the driver entry
point for tensor-map encoding is resolved at run time, so the library loads on
a machine without a GPU driver (its calls then fail with GPE_ERR_NODEVICE).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libgpe_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# per-file flags: the line-length cells follow the reference's arithmetic
# operation by operation, so nothing may be contracted into an FMA
EXTRA = {"vortex.cu": ["-fmad=false"]}


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cuh", ".h")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return any(os.path.getmtime(d) > t for d in deps)


def local_deps(path: str, seen=None) -> set:
    """The file and every header of csrc/ or include/ it includes, transitively."""
    import re
    seen = set() if seen is None else seen
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        for name in re.findall(r'^\s*#\s*include\s+"([^"]+)"', f.read(), flags=re.M):
            for d in (CSRC, INCLUDE):
                cand = os.path.join(d, name)
                if os.path.exists(cand):
                    local_deps(cand, seen)
                    break
    return seen


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    cus = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]
    tmp = LIB + ".tmp"
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-I", INCLUDE, "-I", CSRC]
    if ptxas_info:
        common.insert(1, "-Xptxas=-v")
    objs, cmds = [], []
    for cu in cus:
        obj = os.path.join(objdir, os.path.basename(cu)[:-3] + ".o")
        objs.append(obj)
        # a translation unit is recompiled only when it or a header it
        # includes is newer than its object
        if (not force and not ptxas_info and os.path.exists(obj) and
                all(os.path.getmtime(d) <= os.path.getmtime(obj) for d in local_deps(cu))):
            continue
        cmds.append([*common, *EXTRA.get(os.path.basename(cu), []), "-c", cu, "-o", obj])
    # translation units compile in parallel, then one link
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
        results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    for r in results:
        sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, r.args)
    link = [nvcc_path(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, "-ldl"]
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
