"""The specialised explicit-operator kernels (register windows along y and z, warp segments along
x, compile-time expression modes, 16-byte vectors) give the generic one-thread-per-value kernel's
results: the same bits for the 2-point (CD2) scheme, and within round-off for the 4-point (CD4)
one, whose two-term bulk formula the compiler may contract into a fused multiply-add differently
in the two kernel shapes; flow-only and heated, FP64 and mixed."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from chapsim2_b200 import solver as S

pytestmark = pytest.mark.gpu


def _run(case, precision, iacc, block, nc=(48, 18, 24), nsteps=2):
    if case == "heated":
        cfg, tc = C.heated_channel(nc=nc, iacc=iacc, dt=0.004)
    else:
        cfg, tc = C.channel(nc=nc, iacc=iacc, dt=0.004), None
    g = S.Solver(cfg, precision=precision)
    g.set_fields(*I.channel_fields(cfg))
    if tc is not None:
        g.thermo_init(tc)
    g.set_launch_shape(block, 0, 0)
    g.Solve_momentum_eq(0)
    g.step(nsteps)
    out = [x.copy() for x in g.get_fields()]
    if tc is not None:
        out += [v.copy() for v in g.get_thermo().values()]
    g.close()
    return out


@pytest.mark.parametrize("case", ["channel", "heated"])
@pytest.mark.parametrize("precision", [S.CHS_FP64, S.CHS_MIXED])
@pytest.mark.parametrize("iacc", [1, 2])
def test_specialised_match_generic(case, precision, iacc):
    a = _run(case, precision, iacc, 0)
    b = _run(case, precision, iacc, 256)
    for x, y in zip(a, b):
        if iacc == 1:
            assert np.array_equal(x, y)
        else:
            tol = 1e-12 if precision == S.CHS_FP64 else 1e-5
            assert np.max(np.abs(x - y)) <= tol * max(1.0, np.max(np.abs(y)))


def test_segments_of_lines_longer_and_shorter_than_a_warp_segment():
    # x lines of 48 (< 128, wrapped twice within a segment) and 192 (two segments) points
    for nc in ((48, 18, 24), (192, 18, 8)):
        a = _run("channel", S.CHS_FP64, 1, 0, nc=nc, nsteps=1)
        b = _run("channel", S.CHS_FP64, 1, 256, nc=nc, nsteps=1)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
