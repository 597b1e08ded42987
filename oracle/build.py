"""Build recipes for the oracle (test infrastructure, not the product).

* ``build_oracle()`` compiles ``lbrb_oracle.c`` (the CPU restatement) into
  ``oracle/_build/liblbrb_oracle.so``.
* ``build_ref(program, params, tag)`` compiles the reference's OWN sources,
  read where they lie under the reference checkout, against the in-repo MPI and
  HDF5 stand-ins (``oracle/shim``).  Only compile-time parameters (the
  ``#define`` blocks at Trajectories/code/temppart_dump.c:15-31,
  Trajectories/code/mympi2.h:14-21, Nudging/code/tempvel_nudge.c:13-31) and
  hard-coded input paths (temppart_dump.c:374,454,535,615;
  tempvel_nudge.c:282,361,441,520,1415,2086-2101,2151) are rewritten.  The patched copies and
  the binaries go to ``oracle/_ref/<tag>/`` only (git-ignored; never
  committed).  Compiler: ``gcc -std=c99 -O2`` as the reference makefiles use.
"""
from __future__ import annotations

import hashlib
import os
import re
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SHIM = HERE / "shim"
BUILD = HERE / "_build"
REF_OUT = HERE / "_ref"
# the reference checkout: LBRB_REFERENCE_ROOT, else a checkout named
# `reference` beside this repository
REFERENCE_ROOT = Path(os.environ.get("LBRB_REFERENCE_ROOT", str(HERE.parent.parent / "reference")))

CFLAGS = ["-std=c99", "-O2", "-ffp-contract=off", "-fPIC"]

# reference sources per program: (main .c, header), relative to the checkout
PROGRAMS = {
    "temppart_dump": ("Trajectories/code/temppart_dump.c", "Trajectories/code/mympi2.h"),
    "tempvel_nudge": ("Nudging/code/tempvel_nudge.c", "Nudging/code/mympi2.h"),
}

# hard-coded absolute input paths in the reference -> run-directory relative
PATH_PATCHES = [
    ("/mnt/petaStor/agasthya/LagrangianNudging/High_Ra/St0.5/beta1/", "obs/"),
    ("/mnt/petaStor/agasthya/LagrangianNudging/High_Ra/", ""),
    ("../../St0.5/beta1/", "obs/"),
    ("../dump_Guo2/", ""),
]


def oracle_lib_path() -> Path:
    return BUILD / "liblbrb_oracle.so"


def build_oracle(force: bool = False) -> Path:
    """Compile the CPU restatement into a shared library (idempotent)."""
    src = HERE / "lbrb_oracle.c"
    out = oracle_lib_path()
    BUILD.mkdir(exist_ok=True)
    if not force and out.exists() and out.stat().st_mtime > max(
        src.stat().st_mtime, (HERE / "lbrb_oracle.h").stat().st_mtime
    ):
        return out
    tmp = out.with_suffix(".so.tmp")
    subprocess.run(["gcc", *CFLAGS, "-shared", "-o", str(tmp), str(src), "-lm"], check=True)
    os.replace(tmp, out)
    return out


def reference_available() -> bool:
    return all((REFERENCE_ROOT / p).exists() for pair in PROGRAMS.values() for p in pair)


def _fmt(v) -> str:
    if isinstance(v, bool):
        return "1" if v else "0"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        r = repr(float(v))
        return f"({r})" if v < 0 else r
    return str(v)


def _patch_defines(text: str, params: dict) -> tuple[str, set]:
    seen = set()
    out = []
    for line in text.splitlines(keepends=True):
        m = re.match(r"^#define\s+(\w+)\b", line)
        if m and m.group(1) in params:
            name = m.group(1)
            seen.add(name)
            line = f"#define {name} {_fmt(params[name])}\n"
        out.append(line)
    return "".join(out), seen


def build_ref(program: str, params: dict, tag: str | None = None) -> Path:
    """Patch the compile-time parameters of a reference program and build it
    against the shims.  Returns the path of the executable."""
    if not reference_available():
        raise FileNotFoundError(f"reference sources not found under {REFERENCE_ROOT}")
    csrc_rel, hdr_rel = PROGRAMS[program]
    csrc = (REFERENCE_ROOT / csrc_rel).read_text()
    hdr = (REFERENCE_ROOT / hdr_rel).read_text()
    shim = "".join((SHIM / n).read_text() for n in ("mpi.h", "mpi_shim.c", "hdf5.h", "hdf5_shim.c"))
    key = hashlib.sha1(repr((program, sorted(params.items()), csrc, hdr, shim, PATH_PATCHES)).encode()).hexdigest()[:12]
    tag = tag or f"{program}_{key}"
    d = REF_OUT / tag
    exe = d / program
    stamp = d / "stamp"
    if exe.exists() and stamp.exists() and stamp.read_text() == key:
        return exe
    d.mkdir(parents=True, exist_ok=True)
    csrc, seen_c = _patch_defines(csrc, params)
    hdr, seen_h = _patch_defines(hdr, params)
    missing = set(params) - seen_c - seen_h
    if missing:
        raise KeyError(f"parameters not defined in {program}: {sorted(missing)}")
    for a, b in PATH_PATCHES:
        csrc = csrc.replace(a, b)
    (d / Path(csrc_rel).name).write_text(csrc)
    (d / "mympi2.h").write_text(hdr)
    cmd = [
        "gcc", "-std=c99", "-O2", "-w", f"-I{d}", f"-I{SHIM}",
        str(d / Path(csrc_rel).name), str(SHIM / "mpi_shim.c"), str(SHIM / "hdf5_shim.c"),
        "-lm", "-o", str(exe),
    ]
    subprocess.run(cmd, check=True)
    stamp.write_text(key)
    return exe


if __name__ == "__main__":
    print(build_oracle(force=True))
