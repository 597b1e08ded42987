"""lbrb_stats_noalloc against the allocating entry points.

lbrb_stats_noalloc serves callers that cannot allocate device memory when
they ask for diagnostics (a framework that owns all device memory through its
own pool, a loop that must not allocate after start-up): it reads device
fields the caller owns and keeps its scratch in a fixed device array.  Here
it must give what lbrb_energy()/lbrb_nusselt() give on the same fields, to
the 1e-12 relative tolerance used for the compensated sums, on two calls in a
row (the second call reuses the scratch the first one left behind).

This file is collected last so that a run stopping at the first failure has
run every other test already; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _close(a, b):
    return abs(a - b) <= TOL * max(abs(b), 1e-300)


@pytest.mark.parametrize("precision,torch_dtype", [("fp64", "float64"), ("fp32", "float32")])
def test_stats_noalloc_matches_allocating_entry_points(precision, torch_dtype):
    import torch

    build.build()
    nx, ny = 200, 96
    base = lb.closure(nx, ny, Ra=1e6, Pr=1.0, U=0.1)
    with lb.Run(**base, precision=precision) as r:
        r.init_conduction(77, 5e-2)
        r.step(60)
        r.sync()
        ke, tm = r.energy()
        nu = r.nusselt()
        m = r.get_moments()
    dt = getattr(torch, torch_dtype)
    # caller-owned device fields (allocated by the caller, not by the entry point)
    fields = [torch.tensor(m[k], dtype=dt, device="cuda").contiguous() for k in ("rho", "u", "v", "T")]
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    for call in range(2):
        out = np.zeros(3)
        # the first call on a device may load the library's device code (and
        # the scratch array with it); a later call must take no device memory
        free_before = torch.cuda.mem_get_info()[0]
        rc = lb.lib().lbrb_stats_noalloc(
            *[C.c_void_p(t.data_ptr()) for t in fields], lb.PREC[precision], nx, ny, nx,
            base["relaxg"], base["Tup"], base["Tdown"], C.c_void_p(stream),
            out.ctypes.data_as(C.POINTER(C.c_double)))
        assert rc == 0, (call, rc)
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before, "the call took device memory"
        assert _close(out[0], ke), (call, out[0], ke)
        assert _close(out[1], tm), (call, out[1], tm)
        assert _close(out[2], nu), (call, out[2], nu)


def test_stats_noalloc_rejects_too_many_rows():
    import torch

    build.build()
    ny = 16385  # one row more than the scratch holds
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = np.zeros(3)
    p = C.c_void_p(t.data_ptr())
    rc = lb.lib().lbrb_stats_noalloc(p, p, p, p, 0, 4, ny, 4, 0.6, -0.5, 0.5, None,
                                      out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == -6
