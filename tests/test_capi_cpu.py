"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/lbrb.h declares, and rejects bad parameters before touching CUDA."""
import ctypes as C
import re
from pathlib import Path

import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def L():
    build.build()
    return lb.lib()


def declared_symbols():
    text = (ROOT / "include" / "lbrb.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbrb_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(lb.EXPORTS)


def test_library_exports_every_declared_symbol(L):
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_abi_version(L):
    assert L.lbrb_abi_version() == 1


def test_defaults_follow_reference(L):
    p = lb.Params()
    L.lbrb_params_default(C.byref(p))
    # temppart_dump.c:16-28
    assert (p.nx, p.ny) == (1680, 840)
    assert p.relax == 0.502 and p.relaxg == 0.502
    assert p.Tup == -0.01 and p.Tdown == 0.01 and p.gravity == -0.00004


@pytest.mark.parametrize("bad", [dict(nx=50), dict(ny=2), dict(relax=0.5), dict(relaxg=0.4),
                                 dict(precision=7), dict(twall=3), dict(nudge="refbox", nobs=0),
                                 dict(nudge="refbox", nobs=4, ntempread=1),
                                 dict(gravity=float("nan"))])
def test_create_rejects_bad_parameters(L, bad):
    kw = dict(nx=64, ny=32)
    kw.update(bad)
    p = lb.make_params(**kw)
    h = C.c_void_p()
    assert L.lbrb_create(C.byref(p), C.byref(h)) == -1
    assert not h.value


def test_box_nudging_needs_fp64(L):
    p = lb.make_params(nx=64, ny=32, precision="fp32", nudge="refbox", nobs=16, ntempread=5)
    h = C.c_void_p()
    assert L.lbrb_create(C.byref(p), C.byref(h)) == -9


def test_host_program_rejects_bad_usage():
    import subprocess

    host = Path(build.__file__).resolve().parent / "lbrb_host"
    build.build()
    assert subprocess.run([str(host)], capture_output=True).returncode == 2
    assert subprocess.run([str(host), "trajectories", "nosuchparam=1"], capture_output=True).returncode == 2
    # the reference's contin=1 restart reads an uninitialised value; refused
    assert subprocess.run([str(host), "nudging", "contin=1"], capture_output=True).returncode == 2


def test_ensemble_create_rejects_bad_arguments(L):
    e = C.c_void_p()
    assert L.lbrb_ensemble_create(None, 0, C.byref(e)) == -1
    assert not e.value
    empty = (C.c_void_p * 1)(None)
    assert L.lbrb_ensemble_create(empty, 1, C.byref(e)) == -1
    assert L.lbrb_ensemble_nvariants() >= 1


def test_adjoint_store_rejects_bad_arguments(L):
    """the state-store switch of the adjoint window checks its arguments
    before touching a device"""
    assert L.lbrb_adjoint_set_store(None, 1) == -1
    assert L.lbrb_adjoint_get_store(None, None, None, None) == -1
