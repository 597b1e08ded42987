"""Twin experiment in small: run A records T along tracer trajectories every
step; run B (another initial perturbation) nudged toward those records with
bilinear-4 spreading ends much closer to A than a free run B does."""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build

pytestmark = pytest.mark.gpu


def test_nudging_toward_trajectory_records_tracks_the_truth():
    build.build()
    nx, ny, n, steps = 128, 64, 1024, 600
    base = lb.closure(nx, ny, Ra=1e6, Pr=1.0, U=0.1)
    rng = np.random.default_rng(3)
    x = rng.uniform(0.5, nx + 0.5, n)
    y = rng.uniform(1.0, ny, n)
    with lb.Run(**base, precision="fp32", nprtcl=n, noutconfig=1, record_slots=steps + 1) as a, \
            lb.Run(**base, precision="fp32") as free, \
            lb.Run(**base, precision="fp32", nudge="bilinear", alpha=1.0, nobs=n) as nud:
        a.init_conduction(11, 5e-2)
        a.set_particles(np.arange(n, dtype=np.int32), x, y, np.zeros(n), np.zeros(n),
                        np.zeros(n, np.int32), np.zeros(n))
        free.init_conduction(22, 5e-2)
        nud.init_conduction(22, 5e-2)
        a.step(steps)
        st, buf = a.drain_records_array()
        assert list(st) == list(range(1, steps + 1))
        nud.nudge_obs(1, buf[:, 0, :], buf[:, 1, :], buf[:, 8, :])
        free.step(steps)
        nud.step(steps)
        nud.sync()
        ta = a.get_moments()["T"]
        e_free = np.sqrt(np.mean((free.get_moments()["T"] - ta) ** 2))
        e_nud = np.sqrt(np.mean((nud.get_moments()["T"] - ta) ** 2))
    print(f"L2 error free {e_free:.3e} nudged {e_nud:.3e}")
    assert e_free > 0
    assert e_nud < 0.5 * e_free


def test_bilinear_nudging_is_deterministic():
    """the fixed-point innovation atomics make two identical nudged runs
    bit-identical whatever the order in which the atomics land"""
    build.build()
    nx, ny, n = 96, 48, 2048
    base = lb.closure(nx, ny, Ra=1e6, Pr=1.0, U=0.1)
    rng = np.random.default_rng(8)
    ox = rng.uniform(0.5, nx + 0.5, (50, n))
    oy = rng.uniform(1.0, ny, (50, n))
    oT = 0.5 - (oy - 0.5) / ny + 0.1 * rng.standard_normal((50, n))
    out = []
    for _ in range(2):
        with lb.Run(**base, precision="fp32", nudge="bilinear", alpha=0.5, nobs=n) as r:
            r.init_conduction(4, 1e-2)
            r.nudge_obs(1, ox, oy, oT)
            r.step(50)
            out.append(r.get_populations())
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
