"""CUDA-graph replay inside lbrb_step (lbrb_set_graph): a run with graphs
ends bit-identical to the same run with every launch issued directly --
populations, moments, particles and records -- across record steps, the
u, v slot rotation, both precisions and both particle forms."""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build

pytestmark = pytest.mark.gpu

NX, NY, NP = 64, 32, 96


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def make(precision, graph, nprtcl, beta=0.0, full=0, noutconfig=10):
    r = lb.Run(**lb.closure(NX, NY, Ra=1e6, Pr=1.0, U=0.1), precision=precision, nprtcl=nprtcl,
               noutconfig=noutconfig if nprtcl else 0, record_slots=64, beta=beta, record_full=full)
    r.set_graph(graph)
    r.init_conduction(11, 2e-2)
    if nprtcl:
        rng = np.random.default_rng(5)
        x = rng.uniform(0.5, NX + 0.5, nprtcl)
        y = rng.uniform(1.0, NY, nprtcl)
        ptype = (np.arange(nprtcl) % 2).astype(np.int32)  # tracers and inertial particles
        invtau = np.where(ptype == 1, 1.0 / 50.0, 0.0)
        z = np.zeros(nprtcl)
        r.set_particles(np.arange(nprtcl, dtype=np.int32), x, y, z, z, ptype, invtau)
    return r


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("nprtcl,beta,full", [(0, 0.0, 0), (NP, 0.0, 0), (NP, 0.5, 1)])
def test_graph_replay_is_bit_identical(precision, nprtcl, beta, full):
    with make(precision, 0, nprtcl, beta, full) as a, make(precision, 1, nprtcl, beta, full) as b:
        for n in (1, 4, 7, 25, 58):  # crosses record steps and every buffer phase
            a.step(n)
            b.step(n)
            fa, ga = a.get_populations()
            fb, gb = b.get_populations()
            np.testing.assert_array_equal(fa, fb)
            np.testing.assert_array_equal(ga, gb)
            ma, mb = a.get_moments(), b.get_moments()
            for k in ma:
                np.testing.assert_array_equal(ma[k], mb[k])
            if nprtcl:
                pa, pb = a.get_particles(), b.get_particles()
                assert pa.keys() == pb.keys()
                for k in pa:
                    np.testing.assert_array_equal(pa[k], pb[k])
                sa, ra = a.drain_records_array()
                sb, rb = b.drain_records_array()
                np.testing.assert_array_equal(sa, sb)
                np.testing.assert_array_equal(ra, rb)
        assert a.istep == b.istep == 95


def test_graph_mode_argument_checked():
    with lb.Run(**lb.closure(NX, NY, Ra=1e6, Pr=1.0, U=0.1), precision="fp32") as r:
        with pytest.raises(lb.LbrbError):
            r.set_graph(2)


def test_steps_inside_a_callers_capture():
    """a caller that captures lbrb_step into its own graph gets the launches
    themselves (no nested capture): 6 steps without particles return the
    buffer phase, so three replays equal 18 direct steps"""
    import torch

    with make("fp32", -1, 0) as a, make("fp32", -1, 0) as b:
        s = torch.cuda.Stream()
        a.set_stream(s.cuda_stream)
        a.step(1)  # launch-shape tuning before the capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s, capture_error_mode="thread_local"):
            a.step(6)
        for _ in range(3):
            g.replay()
        torch.cuda.synchronize()
        a.set_stream(None)
        b.step(19)
        fa, ga = a.get_populations()
        fb, gb = b.get_populations()
        np.testing.assert_array_equal(fa, fb)
        np.testing.assert_array_equal(ga, gb)
