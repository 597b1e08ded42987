"""The largest grids: 64-bit element offsets.

The fused kernels index the 18 population planes with 32-bit element
offsets while 36 planes of the grid fit below 2^32 elements, and with 64-bit
offsets beyond that (about 119.3 M nodes per plane, e.g. 16384 x 7296).  The
64-bit instantiations run only on such grids, so they are checked here
against the same domain cut into two y-slabs, whose planes take the 32-bit
path: the slabs advance exactly as the whole domain does (the property the
slab tests pin at small sizes), so T, u and v must agree bit for bit.

The whole domain needs about 23 GB of device memory in FP32 and 46 GB in
FP64; the whole handle is closed before the slabs are made."""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build

pytestmark = pytest.mark.gpu

NX, NY = 16384, 7296  # pitch 16384: 36 planes of 119.5 M elements pass 2^32
STEPS = 7             # three two-step launches and a single step


def test_grid_needs_64bit_offsets():
    plane = NX * NY  # nx is a multiple of 32: the pitch is nx
    assert 36 * plane >= 2 ** 32
    assert 36 * plane // 2 < 2 ** 32  # each slab's planes stay on the 32-bit path


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_64bit_offsets_match_slabs_on_32bit_offsets(precision):
    build.build()
    base = lb.closure(NX, NY, Ra=1e7, Pr=1.0, U=0.1)
    with lb.Run(**base, precision=precision) as r:
        r.init_conduction(11, 1e-2)
        r.step(STEPS)
        r.sync()
        m = r.get_moments()
        whole = {k: m[k] for k in ("u", "v", "T")}
        nu_whole = r.nusselt()
        del m
    with lb.SlabDomain([NY // 2, NY - NY // 2], **base, precision=precision) as d:
        d.init_conduction(11, 1e-2)
        d.step(STEPS)
        for s in d.slabs:
            s.sync()
        m = d.get_moments()
    assert np.isfinite(whole["T"]).all()
    assert np.abs(whole["v"]).max() > 0.0  # the flow has started
    for k in ("u", "v", "T"):
        np.testing.assert_array_equal(m[k], whole[k], err_msg=k)
    assert np.isfinite(nu_whole)
