"""GPU RK3 substeps vs the oracle: Taylor-Green (CP6, 3D FFT) and channel (walls, FISHPACK, mass flux)."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from chapsim2_b200 import solver as S
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _pair(cfg, fields):
    o = po.Oracle(cfg)
    g = S.Solver(cfg)
    o.set_fields(*fields)
    g.set_fields(*fields)
    return o, g


def _compare(o, g, tol):
    ref = o.get_fields()
    got = g.get_fields()
    for name, a, b in zip(("qx", "qy", "qz", "p"), got[:4], ref[:4]):
        assert rel(a, b) < tol, (name, rel(a, b))
    # phi solves L phi = div(u*)/(alpha dt), where div(u*) cancels to round-off level; its error is
    # measured on the pressure scale
    err = np.linalg.norm(got[4] - ref[4]) / max(np.linalg.norm(ref[3]), 1e-300)
    assert err < tol, ("pcor", err)


@pytest.mark.parametrize("acc", [1, 3, 4])
def test_tgv_substeps(acc):
    cfg = C.taylor_green(24, iacc=acc, dt=2e-3)
    o, g = _pair(cfg, I.taylor_green_fields(cfg))
    o.substep(0)
    g.Solve_momentum_eq(0)
    _compare(o, g, 1e-12)
    for isub in (1, 2, 3, 1, 2, 3):
        o.substep(isub)
        g.Solve_momentum_eq(isub)
    _compare(o, g, 1e-11)
    g.close()


@pytest.mark.parametrize("acc", [1, 2, 3, 4])
def test_channel_substeps(acc):
    cfg = C.channel(nc=(24, 18, 16), iacc=acc, dt=0.004)
    o, g = _pair(cfg, I.channel_fields(cfg))
    o.substep(0)
    g.Solve_momentum_eq(0)
    _compare(o, g, 1e-11)
    for isub in (1, 2, 3):
        o.substep(isub)
        g.Solve_momentum_eq(isub)
    _compare(o, g, 1e-10)
    g.close()


def test_graph_replay_matches_direct_launches():
    cfg = C.channel(nc=(24, 18, 16), iacc=1, dt=0.004)
    f = I.channel_fields(cfg)
    g1 = S.Solver(cfg)
    g2 = S.Solver(cfg)
    for g in (g1, g2):
        g.set_fields(*f)
        g.Solve_momentum_eq(0)
    for isub in (1, 2, 3, 1, 2, 3):
        g1.Solve_momentum_eq(isub)
    g2.step(2)
    for a, b in zip(g1.get_fields(), g2.get_fields()):
        assert np.array_equal(a, b)
    g1.close()
    g2.close()


def test_host_dropin_matches_device_state():
    cfg = C.taylor_green(16, iacc=4, dt=2e-3)
    f = I.taylor_green_fields(cfg)
    g1 = S.Solver(cfg)
    g1.set_fields(*f)
    g1.Solve_momentum_eq(1)
    g2 = S.Solver(cfg)
    out = g2.Solve_momentum_eq_host(1, *[a.copy() for a in f])
    for a, b in zip(out, g1.get_fields()[:4]):
        assert np.array_equal(a, b)
    g1.close()
    g2.close()


def test_channel_full_size_step_vs_oracle():
    """128x96x128 channel (the benchmark grid), CD2: one RK3 step against the oracle, projection exact."""
    cfg = C.channel(nc=(128, 96, 128), iacc=1, dt=0.004)
    f = I.channel_fields(cfg)
    o, g = _pair(cfg, f)
    o.substep(0)
    g.Solve_momentum_eq(0)
    o.step()
    g.step(1)
    _compare(o, g, 1e-10)
    d = g.diagnostics()
    assert d["max_div"] < 1e-10
    assert abs(d["bulk_u"] - 1.0) < 1e-10
    assert d["nan_flag"] == 0
    g.close()


def test_tgv_energy_decay_gpu():
    """64^3 Taylor-Green (CP6): KE decays at the analytic initial rate, divergence at round-off."""
    cfg = C.taylor_green(64, iacc=4, dt=1e-3)
    g = S.Solver(cfg)
    g.set_fields(*I.taylor_green_fields(cfg))
    g.Solve_momentum_eq(0)
    e1 = g.diagnostics()["bulk_ke"]
    g.step(10)
    d = g.diagnostics()
    rate = (d["bulk_ke"] - e1) / (10 * cfg.dt)
    assert abs(rate + 0.75 / 1600) < 5e-3 * 0.75 / 1600
    assert d["max_div"] < 1e-10
    g.close()


@pytest.mark.parametrize("acc", [1, 4])
def test_channel_3fmd_substeps(acc):
    """Channel on the 3FMD-stretched grid with the 3D-FFT Poisson solver (poisson_010)."""
    cfg = C.channel(nc=(24, 32, 16), iacc=acc, dt=0.004, rstret=0.25, ifft=C.FFT_2DECOMP_3DFFT)
    o, g = _pair(cfg, I.channel_fields(cfg))
    o.substep(0)
    g.Solve_momentum_eq(0)
    _compare(o, g, 1e-11)
    for isub in (1, 2, 3):
        o.substep(isub)
        g.Solve_momentum_eq(isub)
    _compare(o, g, 1e-10)
    g.close()


def test_heated_channel_3fmd_substeps():
    """Variable-property channel (energy, table properties, g/q conversion) on the 3FMD grid."""
    cfg, tc = C.heated_channel(nc=(24, 32, 16), iacc=1, dt=0.004, rstret=0.25, t_ini=0.49,
                               ifft=C.FFT_2DECOMP_3DFFT)
    o, g = _pair(cfg, I.channel_fields(cfg))
    o.thermo_init(tc)
    g.thermo_init(tc)
    for isub in (0, 1, 2, 3, 1, 2, 3):
        o.substep(isub)
        g.substep(isub)
    ref, got = o.get_fields(), g.get_fields()
    for name, a, b in zip(("qx", "qy", "qz", "p"), got[:4], ref[:4]):
        assert rel(a, b) < 1e-10, (name, rel(a, b))
    th_o, th_g = o.get_thermo(), g.get_thermo()
    for k in ("rhoh", "h", "T", "k", "d", "m", "gx", "gy", "gz"):
        assert rel(th_g[k], th_o[k]) < 1e-10, (k, rel(th_g[k], th_o[k]))
    g.close()


@pytest.mark.parametrize("heated", [False, True])
def test_mass_conservation_monitors_vs_oracle(heated):
    """The three x-slab monitors of Check_element_mass_conservation (src/eq_continuity.f90:379-389):
    on the unprojected initial field (divergence O(1)) they match the oracle's; after the projection
    they sit at round-off like the oracle's."""
    if heated:
        cfg, tc = C.heated_channel(nc=(24, 18, 16), iacc=1, dt=0.004, t_ini=0.49)
    else:
        cfg, tc = C.channel(nc=(24, 18, 16), iacc=1, dt=0.004), None
    f = I.channel_fields(cfg)
    o, g = _pair(cfg, f)
    if tc is not None:
        o.thermo_init(tc)
        g.thermo_init(tc)
    ref = o.mass_conservation()
    got = g.diagnostics()["mcon"]
    assert max(ref) > 1e-3
    for a, b in zip(got, ref):
        assert abs(a - b) <= 1e-12 * max(ref), (got, ref)
    for isub in (0, 1, 2, 3):
        o.substep(isub)
        g.substep(isub)
    ref = o.mass_conservation()
    got = g.diagnostics()["mcon"]
    assert max(ref) < 1e-10 and max(got) < 1e-10, (got, ref)
    g.close()
