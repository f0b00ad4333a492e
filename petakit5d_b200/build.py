"""Build libpkdecon.so (sm_100a) in-tree with nvcc.

``python -m petakit5d_b200.build`` compiles every ``csrc/*.cu`` into ``petakit5d_b200/lib/libpkdecon.so``
(``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``).  Objects are cached in ``_build/`` by
source hash so a rebuild only recompiles what changed.  ``--check`` builds the bounds-checked library
``lib/libpkdecon_check.so`` (``-DPK_CHECK``: the pass kernels test the indices of their global-memory
accesses and their shared-memory layout, record a failure and skip the access; the call returns
PK_ERR_INTERNAL); load it with ``PK_LIB=.../libpkdecon_check.so``.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpkdecon.so")
CHECK_LIB = os.path.join(LIBDIR, "libpkdecon_check.so")
OBJDIR = os.path.join(ROOT, "_build")

NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
              "-DPK_BUILD_LIB"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _digest(path, extra):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        h.update(f.read())
    for hdr in sorted(os.listdir(CSRC)):
        if hdr.endswith((".h", ".cuh")):
            with open(os.path.join(CSRC, hdr), "rb") as f:
                h.update(f.read())
    with open(os.path.join(ROOT, "include", "pkdecon.h"), "rb") as f:
        h.update(f.read())
    h.update(" ".join(extra).encode())
    return h.hexdigest()[:16]


def build(verbose=False, extra_flags=(), checked=False):
    nvcc = _nvcc()
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    flags = NVCC_FLAGS + list(extra_flags) + (["-DPK_CHECK"] if checked else [])
    lib_path = CHECK_LIB if checked else LIB
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))

    def compile_one(src):
        path = os.path.join(CSRC, src)
        # *_rdc.cu launch graphs from the device: relocatable device code, device-linked below
        fl = flags + (["-rdc=true"] if src.endswith("_rdc.cu") else [])
        obj = os.path.join(OBJDIR, f"{src}.{_digest(path, fl)}.o")
        if not os.path.exists(obj):
            cmd = [nvcc, *fl, "-I", os.path.join(ROOT, "include"), "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
            if verbose and r.stderr:
                print(r.stderr, flush=True)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(compile_one, srcs))
    rdc = [o for o, src in zip(objs, srcs) if src.endswith("_rdc.cu")]
    if rdc:
        dlink = os.path.join(OBJDIR, "dlink." + hashlib.sha256("".join(rdc).encode()).hexdigest()[:16] + ".o")
        cmd = [nvcc, "-dlink", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-o", dlink,
               *rdc, "-lcudadevrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"device link failed:\n{r.stdout}\n{r.stderr}")
        objs = objs + [dlink]
    tmp = lib_path + ".tmp"
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static", "-o", tmp, *objs,
           "-lcudadevrt", "-lz"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib_path)
    return lib_path


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, checked="--check" in sys.argv))
