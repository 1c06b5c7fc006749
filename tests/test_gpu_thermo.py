"""Variable-property (heated channel) path on the GPU against the FP64 oracle."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from chapsim2_b200 import solver as S
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _pair(cfg, tc, precision=S.CHS_FP64):
    f = I.channel_fields(cfg)
    o = po.Oracle(cfg)
    o.set_fields(*f)
    o.thermo_init(tc)
    g = S.Solver(cfg, precision=precision)
    g.set_fields(*f)
    g.thermo_init(tc)
    return o, g


@pytest.mark.parametrize("acc", [1, 3])
def test_heated_channel_substeps_vs_oracle(acc):
    cfg, tc = C.heated_channel(nc=(24, 18, 16), iacc=acc, dt=0.004, t_ini=0.49)
    o, g = _pair(cfg, tc)
    th_o, th_g = o.get_thermo(), g.get_thermo()
    for k in ("gx", "gy", "gz", "rhoh", "d"):
        assert rel(th_g[k], th_o[k]) < 1e-13, k
    o.substep(0)
    g.substep(0)
    for isub in (1, 2, 3, 1, 2, 3):
        o.substep(isub)
        g.substep(isub)
    ref, got = o.get_fields(), g.get_fields()
    for name, a, b in zip(("qx", "qy", "qz", "p"), got[:4], ref[:4]):
        assert rel(a, b) < 1e-10, (name, rel(a, b))
    th_o, th_g = o.get_thermo(), g.get_thermo()
    for k in ("rhoh", "h", "T", "k", "d", "m", "gx", "gy", "gz"):
        assert rel(th_g[k], th_o[k]) < 1e-10, (k, rel(th_g[k], th_o[k]))
    g.close()


def test_heated_channel_mixed_profiles():
    cfg, tc = C.heated_channel(nc=(32, 24, 16), iacc=1, dt=0.004, t_ini=0.49)
    o, g = _pair(cfg, tc, precision=S.CHS_MIXED)
    o.substep(0)
    g.substep(0)
    for _ in range(4):
        for isub in (1, 2, 3):
            o.substep(isub)
            g.substep(isub)
    sh = cfg.shapes()
    got, ref = g.get_fields(), o.get_fields()
    pu = lambda a: a.reshape(sh[0]).mean(axis=(0, 2))
    assert rel(pu(got[0]), pu(ref[0])) < 1e-5
    tg, to = g.get_thermo(), o.get_thermo()
    pt = lambda a: a.reshape(sh[3]).mean(axis=(0, 2))
    assert rel(pt(tg["T"]), pt(to["T"])) < 1e-5
    g.close()


def test_energy_and_momentum_entry_points_match_step():
    cfg, tc = C.heated_channel(nc=(24, 18, 16), iacc=1, dt=0.004)
    f = I.channel_fields(cfg)
    a = S.Solver(cfg)
    b = S.Solver(cfg)
    for g in (a, b):
        g.set_fields(*f)
        g.thermo_init(tc)
        g.Solve_momentum_eq(0)
    for isub in (1, 2, 3):
        a.Solve_energy_eq(isub)
        a.Solve_momentum_eq(isub)
    b.step(1)
    for x, y in zip(a.get_fields(), b.get_fields()):
        assert np.array_equal(x, y)
    ta, tb = a.get_thermo(), b.get_thermo()
    for k in ta:
        assert np.array_equal(ta[k], tb[k]), k
    a.close()
    b.close()


@pytest.mark.parametrize("nonuniform", [False, True])
def test_indexed_table_lookup_matches_oracle(nonuniform):
    """The device lookup starts its bisection from a per-bin bracket index; at the table nodes,
    their midpoints, the index's bin edges and one ulp either side, and random values, it gives the
    oracle's full-bisection lookup (tolerance 1e-13 of each column's range: the interpolation may
    use fused multiply-adds on the device)."""
    cfg, tc = C.heated_channel(nc=(16, 16, 16), iacc=1, dt=0.004)
    if nonuniform:
        # cluster the table rows towards the hot end so the index bins hold very different counts
        tb = tc.table
        s = np.linspace(0.0, 1.0, tb["t"].size) ** 3
        t_new = tb["t"][0] + (tb["t"][-1] - tb["t"][0]) * s
        for key in ("h", "d", "m", "k"):
            tb[key] = np.interp(t_new, tb["t"], tb[key])
        tb["t"] = t_new
    o, g = _pair(cfg, tc)
    g.mlp_params(np.random.default_rng(3).normal(0.0, 0.1, S.MLP_NPARAM).astype(np.float32))
    tb = tc.table
    rh_tab = tb["d"] * tb["h"]
    lo, hi = rh_tab[0], rh_tab[-1]
    nb = 2 * rh_tab.size
    edges = lo + np.arange(nb + 1) * ((hi - lo) / nb)
    rng = np.random.default_rng(11)
    x = np.concatenate([rh_tab, 0.5 * (rh_tab[1:] + rh_tab[:-1]), edges, np.nextafter(edges, -np.inf),
                        np.nextafter(edges, np.inf), rng.uniform(lo, hi, 20000)])
    x = np.clip(x, lo, hi)
    out, nfb = g.mlp_eval(x, tol=0.0)  # tolerance 0: every value takes the table lookup
    assert nfb == x.size
    h, T, d, m, k, cp = o.ftp_from_dh(x)
    for name, got, ref in zip(("T", "rho", "mu", "kappa", "h"), out, (T, d, m, k, h)):
        err = np.max(np.abs(got - ref))
        assert err <= 1e-13 * (ref.max() - ref.min()), (name, err)
    g.close()


@pytest.mark.parametrize("per_substep", [True, False])
@pytest.mark.parametrize("precision", [S.CHS_FP64, S.CHS_MIXED])
def test_host_fields_pipeline_matches_device_steps(precision, per_substep):
    """chs_time_steps_host_fields (pinned host state copied in and out around every substep, the two
    copy directions overlapped per field) and chs_time_rk3_host_fields (around every RK3 step) give
    the same state as device-resident steps."""
    cfg, tc = C.heated_channel(nc=(32, 24, 16), iacc=1, dt=0.004, t_ini=0.49)
    f = I.channel_fields(cfg)
    a = S.Solver(cfg, precision=precision)
    b = S.Solver(cfg, precision=precision)
    for g in (a, b):
        g.set_fields(*f)
        g.thermo_init(tc)
        g.substep(0)
    ids = [S.CHS_QX, S.CHS_QY, S.CHS_QZ, S.CHS_PRES, S.CHS_GX, S.CHS_GY, S.CHS_GZ, S.CHS_RHOH]
    host = {}
    for k in ids:
        x = b.download(k)
        h = b.pinned(x.shape)
        h[...] = x
        host[k] = h
    a.step(3)
    b.time_steps_host_fields(3, host, per_substep=per_substep)
    for k in ids:
        ref = a.download(k)
        assert np.array_equal(host[k], ref), k
        assert np.array_equal(b.download(k), ref), k
    a.close()
    b.close()


def _full_field_compare(o, g, tol):
    """u, v, w, p and rho*h, h, T, rho, mu, kappa, g against the oracle (p on its own scale)."""
    ref, got = o.get_fields(), g.get_fields()
    for name, a, b in zip(("qx", "qy", "qz", "p"), got[:4], ref[:4]):
        assert rel(a, b) < tol, (name, rel(a, b))
    th_o, th_g = o.get_thermo(), g.get_thermo()
    for k in ("rhoh", "h", "T", "d", "m", "k", "gx", "gy", "gz"):
        assert rel(th_g[k], th_o[k]) < tol, (k, rel(th_g[k], th_o[k]))


def test_heated_benchmark_workload_one_step_vs_oracle():
    """The benchmark's workload itself (heated channel 128x96x128, CD2, beta 1.5, Re_b 2800, isoflux
    walls, dt from CFL 0.8): the initial step and one RK3 step against the oracle, every field."""
    import bench
    cfg, f, tc = bench.workload("heated")
    o = po.Oracle(cfg)
    o.set_fields(*f)
    o.thermo_init(tc)
    g = S.Solver(cfg)
    g.set_fields(*f)
    g.thermo_init(tc)
    for isub in (0, 1, 2, 3):
        o.substep(isub)
    g.substep(0)
    g.step(1)
    _full_field_compare(o, g, 1e-10)
    d = g.diagnostics()
    assert d["max_div"] < 1e-10 and d["nan_flag"] == 0
    g.close()


def test_large_heated_channel_substep_vs_oracle():
    """Config 5 (384x256x384, beta 1.8, Re_b 6875, variable properties): the initial step and one
    substep against the oracle, every field (the oracle takes ~20 s per substep on 16 host cores)."""
    import bench
    cfg, f, tc = bench.workload("large")
    o = po.Oracle(cfg)
    o.set_fields(*f)
    o.thermo_init(tc)
    g = S.Solver(cfg)
    g.set_fields(*f)
    g.thermo_init(tc)
    for isub in (0, 1):
        o.substep(isub)
        g.substep(isub)
    _full_field_compare(o, g, 1e-10)
    g.close()
