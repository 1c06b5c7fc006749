"""GPU compact line operators vs the oracle (FP64, every family/direction/bc)."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import solver as S
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

WALL_BCS = [(4, 4), (5, 5), (2, 3), (0, 0), (6, 6), (4, 5)]
TOL = 1e-12


def _fbc(rng, d, nin3):
    return rng.standard_normal({0: (nin3[2], nin3[1], 4), 1: (nin3[2], 4, nin3[0]), 2: (4, nin3[1], nin3[0])}[d])


@pytest.mark.parametrize("acc", [1, 2, 3, 4])
def test_ops_channel(acc):
    # ragged sizes: line counts not multiples of the CTA tile
    cfg = C.channel(nc=(24, 18, 12), iacc=acc)
    o = po.Oracle(cfg)
    g = S.Solver(cfg)
    rng = np.random.default_rng(acc)
    for d in (0, 1, 2):
        for fam in range(6):
            for ibc in (WALL_BCS if d == 1 else [(1, 1)]):
                nin3 = list(cfg.nc)
                if fam in (1, 3, 5):
                    nin3[d] = cfg.np_[d]
                fi = rng.standard_normal((nin3[2], nin3[1], nin3[0]))
                fb = _fbc(rng, d, nin3)
                for has in (False, True):
                    ref = o.op3d(d, fam, ibc, fi, fb if has else None)
                    got = g.op3d(d, fam, ibc, fi, fb if has else None)
                    err = np.abs(ref - got).max() / max(1.0, np.abs(ref).max())
                    assert err < TOL, (d, fam, ibc, has, err)
    g.close()


@pytest.mark.parametrize("acc", [1, 4])
def test_ops_periodic_long_lines(acc):
    # lines longer than 200 points use the 32-line tile
    cfg = C.taylor_green(16, iacc=acc)
    cfg.nc = (256, 16, 12)
    o = po.Oracle(cfg)
    g = S.Solver(cfg)
    rng = np.random.default_rng(7)
    for d in (0, 1, 2):
        for fam in range(6):
            nin3 = list(cfg.nc)
            fi = rng.standard_normal((nin3[2], nin3[1], nin3[0]))
            ref = o.op3d(d, fam, (1, 1), fi, None)
            got = g.op3d(d, fam, (1, 1), fi, None)
            assert np.abs(ref - got).max() / max(1.0, np.abs(ref).max()) < TOL
    g.close()
