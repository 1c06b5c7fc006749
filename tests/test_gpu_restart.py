"""Restart files and running statistics: the files hold the raw FP64 fields in the reference's
layout and names, a run continued from them matches the uninterrupted run, and the running means
equal the reference's asymptotic averages of P2C-interpolated velocities computed by the oracle."""
import os

import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from chapsim2_b200 import solver as S
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _make(cfg, tc, f, precision=S.CHS_FP64):
    g = S.Solver(cfg, precision=precision)
    g.set_fields(*f)
    if tc is not None:
        g.thermo_init(tc)
    g.Solve_momentum_eq(0)
    return g


@pytest.mark.parametrize("iacc", [1, 3])
def test_flow_restart_continues_bit_for_bit(tmp_path, iacc):
    cfg = C.channel(nc=(24, 18, 16), iacc=iacc, dt=0.004)
    f = I.channel_fields(cfg)
    a = _make(cfg, None, f)
    a.step(4)
    b = _make(cfg, None, f)
    b.step(2)
    b.write_restart(tmp_path, 1, 2)
    for key, i in (("qx", 0), ("qy", 1), ("qz", 2), ("pr", 3)):
        raw = np.fromfile(S.data_file_name(tmp_path, 1, key, 2), dtype=np.float64)
        assert np.array_equal(raw, b.download(i).ravel())
    c = S.Solver(cfg)
    c.read_restart(tmp_path, 1, 2)
    c.step(2)
    for x, y in zip(a.get_fields(), c.get_fields()):
        assert np.array_equal(x, y)
    for g in (a, b, c):
        g.close()


def test_heated_restart_continues(tmp_path):
    cfg, tc = C.heated_channel(nc=(24, 18, 16), iacc=1, dt=0.004)
    f = I.channel_fields(cfg)
    a = _make(cfg, tc, f)
    a.step(3)
    b = _make(cfg, tc, f)
    b.step(1)
    b.write_restart(tmp_path, 1, 1)
    assert os.path.exists(S.data_file_name(tmp_path, 1, "rhoh", 1))
    assert os.path.exists(S.data_file_name(tmp_path, 1, "temp", 1))
    c = S.Solver(cfg)
    c.set_fields(*f)
    c.thermo_init(tc)
    c.read_restart(tmp_path, 1, 1)
    # the restored properties equal the state they were computed from
    tb, tc_ = b.get_thermo(), c.get_thermo()
    for key in ("T", "d", "m", "k", "h"):
        assert np.max(np.abs(tb[key] - tc_[key])) <= 1e-13 * np.max(np.abs(tb[key])), key
    c.step(2)
    # g is rebuilt from q and rho (one rounding), so the continuation agrees to round-off
    for x, y in zip(a.get_fields(), c.get_fields()):
        assert np.max(np.abs(x - y)) <= 1e-10 * max(1.0, np.max(np.abs(x)))
    ta, tcc = a.get_thermo(), c.get_thermo()
    assert np.max(np.abs(ta["T"] - tcc["T"])) <= 1e-10
    for g in (a, b, c):
        g.close()


@pytest.mark.parametrize("heated", [False, True])
def test_statistics_match_oracle_interpolations(tmp_path, heated):
    if heated:
        cfg, tc = C.heated_channel(nc=(24, 18, 16), iacc=1, dt=0.004)
    else:
        cfg, tc = C.channel(nc=(24, 18, 16), iacc=3, dt=0.004), None
    f = I.channel_fields(cfg)
    g = _make(cfg, tc, f)
    o = po.Oracle(cfg)
    bx, by, bz = cfg.nominal_bc[0, C.V_QX], cfg.nominal_bc[1, C.V_QY], cfg.nominal_bc[2, C.V_QZ]
    ref = {k: 0.0 for k in S.Solver.STATS}
    nstat = 0
    for step in range(3):
        g.step(1)
        nstat += 1
        g.stats_update(nstat)
        qx, qy, qz, p = g.get_fields()[:4]
        u = o.op3d(0, 5, tuple(bx), qx, None)
        fb = None
        if not cfg.periodic_y:
            n3, _, n1 = qy.shape
            fb = np.zeros((n3, 4, n1))
        v = o.op3d(1, 5, tuple(by), qy, fb)
        w = o.op3d(2, 5, tuple(bz), qz, None)
        ac, am = 1.0 / nstat, (nstat - 1.0) / nstat
        vals = {"pr": p, "ux": u, "uy": v, "uz": w, "uu": u * u, "vv": v * v, "ww": w * w, "uv": u * v,
                "uw": u * w, "vw": v * w}
        if heated:
            t = g.get_thermo()["T"].reshape(p.shape)
            vals["t"], vals["tt"] = t, t * t
        for k, x in vals.items():
            ref[k] = am * ref[k] + ac * x
    for k in vals:
        got = g.stats_get(k)
        assert np.max(np.abs(got - ref[k])) <= 1e-12 * max(1.0, np.max(np.abs(ref[k]))), k
    g.write_statistics(tmp_path, 1, 3)
    h = _make(cfg, tc, f)
    h.read_statistics(tmp_path, 1, 3)
    for k in vals:
        assert np.array_equal(h.stats_get(k), g.stats_get(k)), k
    g.close()
    h.close()
