"""Builds quantom_b200/liblima_b200.so in-tree with nvcc for sm_100a.

One shared library holds the C-ABI (include/lima_abi.h), the host engine
(C++) and the CUDA kernels.  Run ``python -m quantom_b200.build``.
"""
from __future__ import annotations

import hashlib
from concurrent.futures import ThreadPoolExecutor
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "liblima_b200.so"
BUILD = ROOT / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", f"-I{ROOT / 'include'}", f"-I{CSRC}"]
# Reference-semantics kernels reproduce the reference's host-compiled float
# operation order: no a*b+c contraction into FMA in that translation unit.
# The physics step kernel launches the list rebuild graph from the device
# (device graph launch): relocatable device code, linked with cudadevrt.
PER_FILE = {"kernels_reference.cu": ["-fmad=false"], "nlist_reference.cu": ["-fmad=false"],
            "kernels_physics.cu": ["-rdc=true"]}


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = Path(cuda) / "bin" / "nvcc"
    return str(p) if p.exists() else "nvcc"


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _stamp(cmd, src, headers) -> str:
    """Content hash of one object's inputs: the compile command, the source and
    every header (an object is reused only when none of them changed)."""
    h = hashlib.sha256(" ".join(cmd).encode())
    for f in [src, *sorted(headers)]:
        h.update(f.name.encode())
        h.update(f.read_bytes())
    return h.hexdigest()


# Library variants: extra defines for some sources, linked with the default
# objects of the others.  The staged variant reads the step kernel's list rows
# through shared memory (bulk copies); the engine loads it when LIMA_B200_LIB
# names it.
VARIANTS = {"staged": {"kernels_physics.cu": ["-DLIMA_STAGED_LIST=1"]}}


def variant_path(name: str) -> Path:
    return PKG / f"liblima_b200_{name}.so"


def build(verbose: bool = False, force: bool = False, variants=("staged",)) -> Path:
    """Compile every source to _build/*.o and link the library (and the named
    variants).  An object is recompiled when the content hash of its command,
    source and the headers differs from the one recorded beside it, or always
    with force=True."""
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    headers = [h for h in list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "lima_abi.h"]
               if h.exists()]
    objs = []
    jobs = []
    nvcc = _nvcc()
    var_objs = {v: [] for v in variants}

    def add(s, o, extra):
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, *PER_FILE.get(s.name, []), *extra, "-c", str(s), "-o", str(o)]
        if s.suffix == ".cpp":
            cmd = [nvcc, *NVCC_FLAGS, *extra, "-x", "cu", *ARCH, "-c", str(s), "-o", str(o)]
        stamp_file = o.with_suffix(".o.sha256")
        stamp = _stamp(cmd, s, headers)
        if not force and o.exists() and stamp_file.exists() and stamp_file.read_text() == stamp:
            return
        jobs.append((cmd, stamp_file, stamp))

    for s in srcs:
        o = BUILD / (s.name + ".o")
        objs.append(o)
        add(s, o, [])
        for v in variants:
            extra = VARIANTS[v].get(s.name)
            if extra:
                ov = BUILD / (s.name + f".{v}.o")
                add(s, ov, extra)
                var_objs[v].append(ov)
            else:
                var_objs[v].append(o)

    def compile_one(job):
        cmd, stamp_file, stamp = job
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        stamp_file.write_text(stamp)
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        list(pool.map(compile_one, jobs))
    for out, ol in [(OUT, objs)] + [(variant_path(v), var_objs[v]) for v in variants]:
        tmp = out.with_suffix(".so.tmp")
        cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, ol), "-lcudadevrt", "-lcudart", "-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, out)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(OUT)
