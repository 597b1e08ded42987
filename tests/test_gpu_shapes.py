"""Every launch shape of the fused kernel -- block sizes, blocks per SM, the
interior fast path with 32-bit offsets and the general pull -- gives the same
state, bit for bit, on grids whose width is not a multiple of the block, in
both wall modes and both precisions, with u and v stored for particles."""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build

pytestmark = pytest.mark.gpu

NSHAPES = 10


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def run(precision, shape, nx, ny, twall, steps, nprtcl):
    kw = dict(**lb.closure(nx, ny, Ra=1e6, Pr=1.0, U=0.1), precision=precision, twall=twall, autotune=0,
              launch_shape=shape, nprtcl=nprtcl, noutconfig=0)
    with lb.Run(**kw) as r:
        r.set_graph(0)
        r.init_conduction(13, 3e-2)
        if nprtcl:
            rng = np.random.default_rng(2)
            x = rng.uniform(0.5, nx + 0.5, nprtcl)
            y = rng.uniform(1.0, ny, nprtcl)
            z = np.zeros(nprtcl)
            r.set_particles(np.arange(nprtcl, dtype=np.int32), x, y, z, z, np.zeros(nprtcl, np.int32), z)
        r.step(steps)
        f, g = r.get_populations()
        out = dict(f=f, g=g, **r.get_moments())
        if nprtcl:
            out.update({"p" + k: v for k, v in r.get_particles().items()})
        return out


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("twall", ["dirichlet", "adiabatic"])
@pytest.mark.parametrize("grid", [(200, 37), (64, 48)])
def test_every_launch_shape_gives_the_same_state(precision, twall, grid):
    nx, ny = grid
    shapes = range(NSHAPES)
    ref = run(precision, 7, nx, ny, twall, 23, 64)
    for sh in shapes:
        got = run(precision, sh, nx, ny, twall, 23, 64)
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"shape {sh}: {k}")


def test_launch_shape_out_of_range_is_rejected():
    with pytest.raises(lb.LbrbError):
        lb.Run(**lb.closure(64, 32, Ra=1e6, Pr=1.0, U=0.1), precision="fp32", autotune=0, launch_shape=NSHAPES)
