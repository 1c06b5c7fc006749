"""Variable-property (thermal) path of the oracle on the CPU: property lookups, the
constant-property limit, and the energy budget of the wall heat flux."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from oracle import pyoracle as po


def _interp(x, xp, fp):
    return np.interp(x, xp, fp)


def test_synthetic_table_is_monotonic_in_rhoh():
    t = C.synthetic_table()
    rh = t["d"] * t["h"]
    assert np.all(np.diff(rh) > 0)
    assert np.all(np.diff(t["h"]) > 0)
    assert abs(t["h"][0] + 0.5) < 1e-12 and abs(t["h"][-1] - 0.5) < 1e-12
    # cp is dh/dT
    dh = np.gradient(t["h"], t["t"])
    assert np.max(np.abs(dh - t["cp"])[5:-5] / t["cp"][5:-5]) < 2e-3


def test_ftp_from_dh_matches_two_pass_lookup():
    """rho*h -> h by table interpolation, then h -> rho, h = rho*h/rho, then h -> all
    (ftp_refresh_thermal_properties_from_DH, src/input_thermo.f90:393-446)."""
    cfg, tc = C.heated_channel(nc=(8, 8, 8))
    o = po.Oracle(cfg)
    o.set_fields(*I.channel_fields(cfg))
    o.thermo_init(tc)
    tb = tc.table
    rh_tab = tb["d"] * tb["h"]
    rng = np.random.default_rng(3)
    x = rng.uniform(rh_tab[0], rh_tab[-1], 500)
    h, T, d, m, k, cp = o.ftp_from_dh(x)
    h1 = _interp(x, rh_tab, tb["h"])
    d1 = _interp(h1, tb["h"], tb["d"])
    h2 = x / d1
    for got, col in ((T, "t"), (d, "d"), (m, "m"), (k, "k"), (cp, "cp")):
        ref = _interp(h2, tb["h"], tb[col])
        assert np.max(np.abs(got - ref)) < 1e-12, col
    assert np.max(np.abs(h - h2)) < 1e-14
    # clamping outside the table range
    h, T, d, *_ = o.ftp_from_dh(np.array([rh_tab[0] - 1.0, rh_tab[-1] + 1.0]))
    assert abs(T[0] - tb["t"][0]) < 1e-12 and abs(T[1] - tb["t"][-1]) < 1e-12


@pytest.mark.parametrize("acc", [1, 3])
def test_constant_properties_reproduce_the_flow_path(acc):
    cfg, tc = C.heated_channel(nc=(16, 12, 8), iacc=acc, dt=0.004, table=C.constant_table(), t_ini=0.3)
    f = I.channel_fields(cfg)
    a = po.Oracle(cfg)
    a.set_fields(*f)
    a.thermo_init(tc)
    cfg2 = C.channel(nc=(16, 12, 8), iacc=acc, dt=0.004)
    b = po.Oracle(cfg2)
    b.set_fields(*f)
    for isub in (0, 1, 2, 3):
        a.substep(isub)
        b.substep(isub)
    for x, y in zip(a.get_fields()[:4], b.get_fields()[:4]):
        assert np.max(np.abs(x - y)) <= 1e-13 * max(1.0, np.max(np.abs(y)))
    th = a.get_thermo()
    g = a.get_fields()
    assert np.max(np.abs(th["gx"] - g[0])) < 1e-13


def test_heat_flux_budget_at_rest():
    """Fluid at rest, uniform T: the first substep's change of the total rho*h equals the wall
    heat input rPrRen * (kappa dT/dy|top - kappa dT/dy|bottom) * area * dt * gamma_1."""
    cfg, tc = C.heated_channel(nc=(8, 16, 8), iacc=1, dt=1e-3)
    f = [np.zeros(s) for s in cfg.shapes()]
    o = po.Oracle(cfg)
    o.set_fields(*f)
    o.thermo_init(tc)
    geo = C.geometry(cfg)
    dy = np.diff(geo["yp"])
    h0 = o.get_thermo()["rhoh"]
    dx, dz = cfg.lxx / cfg.nc[0], cfg.lzz / cfg.nc[2]
    tot0 = np.sum(h0 * dy[None, :, None]) * dx * dz
    o.substep(1)
    th = o.get_thermo()
    tot1 = np.sum(th["rhoh"] * dy[None, :, None]) * dx * dz
    k_wall = np.interp(tc.t_ini, tc.table["t"], tc.table["k"])
    rpr = 1.0 / (cfg.ren * tc.prandtl)
    expect = rpr * k_wall * (tc.qw[1] - tc.qw[0]) * cfg.lxx * cfg.lzz * cfg.dt * (8.0 / 15.0)
    assert abs((tot1 - tot0) - expect) < 1e-3 * abs(expect)
