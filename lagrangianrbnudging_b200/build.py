"""Build liblbrb.so (the CUDA kernels + C-ABI) in-tree for sm_100a.

    python -m lagrangianrbnudging_b200.build [--verbose-ptxas]

All translation units are compiled with --fmad=false: the FP64 path keeps
the reference's rounding (no fused multiply-add contraction), which makes
its results bit-identical to the reference built with gcc -O2 on x86-64.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "liblbrb.so"
HOST = PKG / "lbrb_host"
SOURCES = ["lb_kernels.cu", "particle_kernels.cu", "nudge_kernels.cu", "aux_kernels.cu", "capi.cu",
           "adjoint_kernels.cu", "noalloc.cu", "ensemble_kernels.cu", "ensemble.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (Path(c).exists() or c == "nvcc"):
            return c
    return "nvcc"


def _stale() -> bool:
    if not LIB.exists() or not HOST.exists():
        return True
    for dep in (PKG / "host" / "lbrb_host.c", ROOT / "include" / "lbrb.h"):
        if dep.stat().st_mtime > HOST.stat().st_mtime:
            return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "lbrb.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs, cmds = [], []
    for s in SOURCES:
        o = objdir / (Path(s).stem + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(CSRC / s), "-o", str(o)]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(str(o))
    # translation units compile independently: run them side by side
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for r in ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args)
            if verbose_ptxas:
                sys.stderr.write(r.stderr)
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart", "-lpthread"], check=True)
    os.replace(tmp, LIB)
    # the host program, linked against the library next to it
    tmp = HOST.with_suffix(".tmp")
    import shutil

    cuda_inc = Path(shutil.which(nvcc()) or nvcc()).resolve().parent.parent / "include"
    subprocess.run(["gcc", "-std=gnu99", "-O2", "-Wall", f"-I{cuda_inc}", "-o", str(tmp),
                    str(PKG / "host" / "lbrb_host.c"), f"-L{PKG}", "-llbrb", "-Wl,-rpath,$ORIGIN",
                    "-lm", "-ldl"], check=True)
    os.replace(tmp, HOST)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose_ptxas="--verbose-ptxas" in sys.argv))
