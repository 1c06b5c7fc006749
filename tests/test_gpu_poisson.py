"""GPU Poisson solvers (FISHPACK x/z-FFT + y-TRID0, and the 3D-FFT poisson_000) vs the oracle."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import solver as S
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nc", [(16, 12, 8), (24, 18, 36), (128, 96, 128), (16, 192, 12), (24, 257, 8)])
def test_fishpack_poisson(nc):
    cfg = C.channel(nc=nc, iacc=1)
    o = po.Oracle(cfg)
    g = S.Solver(cfg)
    rng = np.random.default_rng(1)
    rhs = rng.standard_normal(o.shape_ccc)
    ref = o.poisson(rhs)
    got = g.solve_fft_poisson(rhs)
    assert np.abs(ref - got).max() / np.abs(ref).max() < 1e-11
    g.close()


@pytest.mark.parametrize("n,acc", [(16, 4), (24, 1), (64, 4)])
def test_poisson_000(n, acc):
    cfg = C.taylor_green(n, iacc=acc)
    cfg.nc = (n, n // 2 * 3 if n == 16 else n, n)
    o = po.Oracle(cfg)
    g = S.Solver(cfg)
    rng = np.random.default_rng(2)
    rhs = rng.standard_normal(o.shape_ccc)
    ref = o.poisson(rhs)
    got = g.solve_fft_poisson(rhs)
    assert np.abs(ref - got).max() / np.abs(ref).max() < 1e-11
    g.close()


@pytest.mark.parametrize("nc,acc,istret", [((16, 24, 12), 1, 2), ((32, 64, 24), 4, 2), ((24, 48, 16), 3, 1),
                                          ((16, 32, 8), 4, 0), ((16, 256, 8), 1, 2), ((64, 96, 64), 4, 2),
                                          ((18, 16, 27), 2, 2)])
def test_poisson_010(nc, acc, istret):
    """poisson_010 (y walls, 3FMD stretching or uniform) on the GPU vs the oracle, random rhs."""
    cfg = C.channel(nc=nc, iacc=acc, rstret=0.25, ifft=C.FFT_2DECOMP_3DFFT, istret=istret)
    o = po.Oracle(cfg)
    g = S.Solver(cfg)
    rng = np.random.default_rng(7)
    rhs = rng.standard_normal(o.shape_ccc)
    ref = o.poisson(rhs)
    got = g.solve_fft_poisson(rhs)
    assert np.abs(ref - got).max() / np.abs(ref).max() < 1e-11
    g.close()



@pytest.mark.parametrize("nc,istret", [((16, 24, 12), C.ISTRET_BOTTOM), ((16, 24, 12), C.ISTRET_TOP),
                                       ((16, 25, 12), C.ISTRET_2SIDES)])
def test_poisson_010_rejects_unsupported_setups(nc, istret):
    """chs_create refuses the 3D-FFT solver with y walls for istret 3 and 4 (whose reference matrices
    are not built for poisson_010's odd/even solves) and for an odd number of y cells."""
    cfg = C.channel(nc=nc, iacc=1, rstret=0.25, ifft=C.FFT_2DECOMP_3DFFT, istret=istret)
    with pytest.raises(RuntimeError, match="chs_create"):
        S.Solver(cfg)
