"""The FP64 tangent-linear model of the oracle against central finite
differences of the oracle's own forward (which is pinned to the reference):
the TLM is the CPU reference for the CUDA adjoint."""
import numpy as np

from tests.golden.cases import adjoint_case
from oracle.oracle import Oracle


def test_tlm_matches_central_differences():
    c = adjoint_case(seed=3)
    o = Oracle(c["params"], 0)
    rng = np.random.default_rng(17)
    h = 1e-6
    zero = np.zeros_like(c["T0"])
    for _ in range(3):
        d = rng.standard_normal(c["T0"].shape)
        J, dJ = o.tlm_window(c["T0"], d, c["nsteps"], c["steps"], c["ox"], c["oy"], c["oT"])
        Jp, _ = o.tlm_window(c["T0"] + h * d, zero, c["nsteps"], c["steps"], c["ox"], c["oy"], c["oT"])
        Jm, _ = o.tlm_window(c["T0"] - h * d, zero, c["nsteps"], c["steps"], c["ox"], c["oy"], c["oT"])
        fd = (Jp - Jm) / (2 * h)
        assert J > 0
        assert abs(fd - dJ) <= 1e-6 * abs(dJ), (fd, dJ)
