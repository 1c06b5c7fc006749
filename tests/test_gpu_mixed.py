"""Mixed-precision form (FP32 fields, operators, RHS and, with the FISHPACK solver, the x and z
transforms; FP64 wall-normal Poisson solves, mass-flux mean and divergence check) against the FP64
oracle and the FP64 GPU path."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from chapsim2_b200 import solver as S
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def xz_mean_profile(a):
    """x-z mean per y row of a (k, j, i) array (Calculate_xz_mean_yprofile, src/tools_solver.f90:104-158)."""
    return a.mean(axis=(0, 2))


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("acc,ifft", [(1, C.FFT_FISHPACK_2DFFT), (3, C.FFT_FISHPACK_2DFFT),
                                      (4, C.FFT_2DECOMP_3DFFT)])
def test_channel_mixed_profiles_vs_oracle(acc, ifft):
    if ifft == C.FFT_2DECOMP_3DFFT:
        cfg = C.channel(nc=(32, 24, 16), iacc=acc, dt=0.004, rstret=0.25, ifft=ifft)
    else:
        cfg = C.channel(nc=(32, 24, 16), iacc=acc, dt=0.004)
    f = I.channel_fields(cfg)
    o = po.Oracle(cfg)
    o.set_fields(*f)
    g = S.Solver(cfg, precision=S.CHS_MIXED)
    g.set_fields(*f)
    o.substep(0)
    g.Solve_momentum_eq(0)
    for _ in range(5):
        o.step()
    g.step(5)
    ref = o.get_fields()
    got = g.get_fields()
    shapes = cfg.shapes()
    for name, a, b, sh in zip(("qx", "qy", "qz"), got[:3], ref[:3], shapes[:3]):
        pa = xz_mean_profile(a.reshape(sh))
        pb = xz_mean_profile(b.reshape(sh))
        if name == "qx":
            # mean streamwise velocity profile: the mixed form's accuracy bound
            assert rel(pa, pb) < 1e-5, (name, rel(pa, pb))
        else:
            # the mean wall-normal and spanwise profiles are near zero: absolute check on the bulk scale
            assert np.abs(pa - pb).max() < 1e-5, (name, np.abs(pa - pb).max())
        # whole fields stay at FP32 round-off growth level
        assert rel(a, b) < 1e-4, (name, rel(a, b))
    d = g.diagnostics()
    assert abs(d["bulk_u"] - 1.0) < 1e-6
    assert d["nan_flag"] == 0
    if acc == 1:
        # CD2 operators are consistent with the FISHPACK projection: the FP64 check of the FP32
        # field sees only FP32 round-off (for compact schemes the post-projection divergence is
        # the O(h^2) scheme mismatch in both forms)
        assert d["max_div"] < 1e-3
    g.close()


def test_mixed_matches_fp64_gpu_on_bench_grid():
    cfg = C.channel(nc=(128, 96, 128), iacc=1, dt=0.02)
    f = I.channel_fields(cfg)
    g64 = S.Solver(cfg)
    g32 = S.Solver(cfg, precision=S.CHS_MIXED)
    for g in (g64, g32):
        g.set_fields(*f)
        g.Solve_momentum_eq(0)
        g.step(10)
    a = g32.get_fields()
    b = g64.get_fields()
    sh = cfg.shapes()[0]
    assert rel(xz_mean_profile(a[0].reshape(sh)), xz_mean_profile(b[0].reshape(sh))) < 1e-5
    d32, d64 = g32.diagnostics(), g64.diagnostics()
    assert abs(d32["bulk_ke"] - d64["bulk_ke"]) < 1e-5 * d64["bulk_ke"]
    g32.close()
    g64.close()


def test_tgv_mixed_energy_decay():
    cfg = C.taylor_green(32, iacc=4, dt=1e-3)
    g = S.Solver(cfg, precision=S.CHS_MIXED)
    g.set_fields(*I.taylor_green_fields(cfg))
    g.Solve_momentum_eq(0)
    e1 = g.diagnostics()["bulk_ke"]
    g.step(10)
    d = g.diagnostics()
    rate = (d["bulk_ke"] - e1) / (10 * cfg.dt)
    assert abs(rate + 0.75 / 1600) < 2e-2 * 0.75 / 1600
    g.close()


@pytest.mark.parametrize("nc", [(24, 192, 12), (36, 18, 36)])
def test_mixed_fp32_spectrum_grids(nc):
    """The FP32 spectrum of the mixed FISHPACK solver on grids that take the other kernel variants:
    columns taller than 160 rows (the in-place y solve) and radix-3 transform lengths; the mean
    streamwise profile after three RK3 steps against the FP64 path, and the FP64 divergence check."""
    cfg = C.channel(nc=nc, iacc=1, dt=0.002)
    f = I.channel_fields(cfg)
    out = []
    for prec in (S.CHS_FP64, S.CHS_MIXED):
        g = S.Solver(cfg, precision=prec)
        g.set_fields(*f)
        g.Solve_momentum_eq(0)
        g.step(3)
        out.append((g.get_fields(), g.diagnostics()))
        g.close()
    (a, _), (b, db) = out[1], out[0]
    sh = cfg.shapes()
    pa = xz_mean_profile(a[0].reshape(sh[0]))
    pb = xz_mean_profile(b[0].reshape(sh[0]))
    assert rel(pa, pb) < 1e-5, rel(pa, pb)
    assert rel(a[0], b[0]) < 1e-4
    assert out[1][1]["max_div"] < 1e-4 and out[1][1]["nan_flag"] == 0
