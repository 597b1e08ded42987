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
