"""One domain cut into y-slabs (lbrb_slab_set / lbrb_slab_step): the slabs
advance exactly as the whole domain in one handle, bit for bit, in both
precisions and with uneven slab heights; the slabs' initial state is the
whole domain's; the height-weighted Nu is the whole domain's.  On one GPU the
slabs are handles on the same device: the exchange is the same peer copy as
across GPUs (cudaMemcpyPeerAsync), ordered by the same events."""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build

pytestmark = pytest.mark.gpu

NX, NY = 64, 48


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def params(precision):
    return dict(**lb.closure(NX, NY, Ra=1e6, Pr=1.0, U=0.1), precision=precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("heights", [(24, 24), (20, 17, 11), (3, 42, 3)])
def test_slabs_advance_as_the_whole_domain(precision, heights):
    with lb.Run(**params(precision)) as whole, lb.SlabDomain(heights, **params(precision)) as dom:
        whole.init_conduction(17, 2e-2)
        dom.init_conduction(17, 2e-2)
        fw, gw = whole.get_populations()
        fs, gs = dom.get_populations()
        np.testing.assert_array_equal(fs, fw)
        np.testing.assert_array_equal(gs, gw)
        for n in (1, 37, 300):
            whole.step(n)
            dom.step(n)
            fw, gw = whole.get_populations()
            fs, gs = dom.get_populations()
            np.testing.assert_array_equal(fs, fw)
            np.testing.assert_array_equal(gs, gw)
        mw, ms = whole.get_moments(), dom.get_moments()
        for k in ("rho", "u", "v", "T"):
            np.testing.assert_array_equal(ms[k], mw[k])
        assert dom.nusselt() == pytest.approx(whole.nusselt(), rel=1e-12, abs=1e-12)


def test_slabs_from_a_developed_state():
    """populations set from a whole-domain state after 2000 steps"""
    with lb.Run(**params("fp32")) as whole, lb.SlabDomain((16, 16, 16), **params("fp32")) as dom:
        whole.init_conduction(5, 5e-2)
        whole.step(2000)
        f, g = whole.get_populations()
        m = whole.get_moments()
        dom.set_populations(f, g)
        dom.set_moments(m["rho"], m["u"], m["v"], m["T"])
        # the whole run's state again from the same host copy (same rounding)
        whole.set_populations(f, g)
        whole.set_moments(m["rho"], m["u"], m["v"], m["T"])
        whole.step(500)
        dom.step(500)
        fw, gw = whole.get_populations()
        fs, gs = dom.get_populations()
        np.testing.assert_array_equal(fs, fw)
        np.testing.assert_array_equal(gs, gw)


def test_slab_mode_rejects_what_it_does_not_cover():
    with lb.Run(**dict(params("fp32"), ny=24)) as r:
        with pytest.raises(lb.LbrbError):
            r._ck(lb.lib().lbrb_slab_set(r.h, 30, NY))  # rows outside the domain
        r._ck(lb.lib().lbrb_slab_set(r.h, 0, NY))
        r.init_conduction(1, 1e-3)
        with pytest.raises(lb.LbrbError):
            r.step(2)  # one step per boundary exchange
    with lb.Run(**dict(params("fp32"), ny=24, nprtcl=8)) as r:
        with pytest.raises(lb.LbrbError):
            r._ck(lb.lib().lbrb_slab_set(r.h, 0, NY))  # particles are not covered
    with pytest.raises(ValueError):
        lb.SlabDomain((20, 20), **params("fp32"))  # heights must add up to ny
    with lb.SlabDomain((24, 24), **params("fp32")) as dom:
        dom.init_conduction(1, 1e-3)
        rev = (lb.C.c_void_p * 2)(dom.slabs[1].h, dom.slabs[0].h)
        assert lb.ERRORS[lb.lib().lbrb_slab_step(rev, 2, 1)] == "LBRB_ERR_ARG"  # slabs out of order
