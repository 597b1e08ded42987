"""The CUDA adjoint of the time step (lbrb_adjoint_window) against the FP64
tangent-linear model of the oracle, against central finite differences of the
GPU's own FP64 forward, and across checkpoint intervals, the two ways of
keeping the forward states (a store of every state, or checkpoints and
recompute) and precisions."""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build
from oracle.oracle import Oracle
from tests.golden.cases import adjoint_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    build.build()
    return adjoint_case(seed=3)


def gpu_window(c, precision, K, gradient=True, T0=None, store=-1):
    with lb.Run(**c["base"], precision=precision) as r:
        r.adjoint_set_store(store)
        r.adjoint_set_obs(c["steps"], c["ox"], c["oy"], c["oT"])
        out = r.adjoint_window(c["T0"] if T0 is None else T0, c["nsteps"], K, gradient=gradient)
        if gradient and store >= 0:
            assert r.adjoint_store()["used_last"] == store
        return out


def test_fp64_adjoint_matches_tangent_linear_model(case):
    c = case
    J, grad = gpu_window(c, "fp64", K=8)
    o = Oracle(c["params"], 0)
    rng = np.random.default_rng(23)
    for _ in range(3):
        d = rng.standard_normal(c["T0"].shape)
        Jt, dJ = o.tlm_window(c["T0"], d, c["nsteps"], c["steps"], c["ox"], c["oy"], c["oT"])
        assert abs(J - Jt) <= 1e-12 * Jt
        # <grad J, d> from the adjoint against the tangent-linear derivative
        assert abs(np.sum(grad * d) - dJ) <= 1e-9 * abs(dJ), (np.sum(grad * d), dJ)


def test_fp64_adjoint_matches_gpu_finite_differences(case):
    """central differences h = 1e-6 of the FP64 GPU forward (64x fewer
    directions than the configuration's 64, same tolerance 1e-4)"""
    c = case
    _, grad = gpu_window(c, "fp64", K=8)
    rng = np.random.default_rng(29)
    h = 1e-6
    for _ in range(2):
        d = rng.standard_normal(c["T0"].shape)
        Jp = gpu_window(c, "fp64", K=8, gradient=False, T0=c["T0"] + h * d)
        Jm = gpu_window(c, "fp64", K=8, gradient=False, T0=c["T0"] - h * d)
        fd = (Jp - Jm) / (2 * h)
        ad = np.sum(grad * d)
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)


def test_checkpoint_interval_does_not_change_the_gradient(case):
    c = case
    g1 = gpu_window(c, "fp64", K=1, store=0)[1]
    g7 = gpu_window(c, "fp64", K=7, store=0)[1]
    gall = gpu_window(c, "fp64", K=c["nsteps"], store=0)[1]
    np.testing.assert_array_equal(g1, g7)
    np.testing.assert_array_equal(g1, gall)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [None, (40, 13)])
def test_state_store_equals_checkpoint_recompute(case, precision, shape):
    """every state's moments kept (no recompute) against checkpoints every K
    steps with the segments recomputed: J and gradient bit-identical, on an
    even window (the 48x24 case) and an odd one (17 steps, partial strips)"""
    c = case if shape is None else adjoint_case(seed=9, nx=shape[0], ny=shape[1], nsteps=17, every=3,
                                                nobs=11)
    Js, gs = gpu_window(c, precision, K=5, store=1)
    for K in (1, 5, c["nsteps"]):
        Jr, gr = gpu_window(c, precision, K=K, store=0)
        assert Js == Jr
        np.testing.assert_array_equal(gs, gr)


def test_state_store_kept_for_the_next_window_and_freed(case):
    """the store stays with the handle across windows (the second window's
    gradient unchanged) and mode 0 frees it"""
    c = case
    with lb.Run(**c["base"], precision="fp32") as r:
        r.adjoint_set_store(1)
        r.adjoint_set_obs(c["steps"], c["ox"], c["oy"], c["oT"])
        _, g1 = r.adjoint_window(c["T0"], c["nsteps"], 8)
        st = r.adjoint_store()
        assert st["used_last"] == 1 and st["bytes"] > 0
        _, g2 = r.adjoint_window(c["T0"], c["nsteps"], 8)
        np.testing.assert_array_equal(g1, g2)
        r.adjoint_set_store(0)
        assert r.adjoint_store()["bytes"] == 0
        _, g3 = r.adjoint_window(c["T0"], c["nsteps"], 8)
        assert r.adjoint_store()["used_last"] == 0
        np.testing.assert_array_equal(g1, g3)


@pytest.mark.parametrize("store", [1, 0])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [None, (40, 13)])
def test_every_pair_kernel_variant_gives_the_same_gradient(case, precision, shape, store):
    """the tiled and the marching two-step kernels, every launch variant, on
    the 48x24 case and on a grid of partial strips and row groups, with the
    state store and with checkpoints"""
    c = case if shape is None else adjoint_case(seed=9, nx=shape[0], ny=shape[1], nsteps=17, every=3,
                                                nobs=11)
    grads = []
    for v in range(lb.Run.adjoint_variants()):
        with lb.Run(**c["base"], precision=precision) as r:
            r.adjoint_set_store(store)
            r.adjoint_set_variant(v)
            r.adjoint_set_obs(c["steps"], c["ox"], c["oy"], c["oT"])
            grads.append(r.adjoint_window(c["T0"], c["nsteps"], 8)[1])
            assert r.adjoint_variant() == v
    for g in grads[1:]:
        np.testing.assert_array_equal(g, grads[0])


def test_fp32_forward_adjoint_close_to_fp64(case):
    """FP32 shifted forward with FP64 adjoint accumulation: gradient within
    1e-3 (relative L2) of the FP64 one"""
    c = case
    J64, g64 = gpu_window(c, "fp64", K=8)
    J32, g32 = gpu_window(c, "fp32", K=8)
    assert abs(J32 - J64) <= 1e-4 * J64
    assert np.linalg.norm(g32 - g64) <= 1e-3 * np.linalg.norm(g64)


def test_autograd_wrapper_passes_gradcheck():
    """torch.autograd.gradcheck (central differences, FP64) through the
    C-ABI adjoint on a 16x8 window of 12 steps"""
    import torch
    from tests.adjoint_function import WindowMisfit

    c = adjoint_case(seed=5, nx=16, ny=8, nsteps=12, every=3, nobs=12)
    with lb.Run(**c["base"], precision="fp64") as r:
        r.adjoint_set_obs(c["steps"], c["ox"], c["oy"], c["oT"])
        T0 = torch.tensor(c["T0"], dtype=torch.float64, requires_grad=True)
        assert torch.autograd.gradcheck(lambda t: WindowMisfit.apply(t, r, c["nsteps"], 4), (T0,),
                                        eps=1e-6, atol=1e-9, rtol=1e-6)
        J = WindowMisfit.apply(T0, r, c["nsteps"], 4)
        J.backward()
        _, g = r.adjoint_window(c["T0"], c["nsteps"], 4)
        np.testing.assert_array_equal(T0.grad.numpy(), g)
