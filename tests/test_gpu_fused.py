"""Fused CD2 momentum kernels (chs_set_fusion) against the operator path and the oracle.

The fused path evaluates every interpolation and derivative of Compute_momentum_rhs
(src/eq_momentum2.f90:101-1571) where the component sums need it, with the same plans as the
operator path; the two paths agree to round-off (the x/z pairs and the y bulk rows run one operator
on the combined convective + viscous expression).
"""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from chapsim2_b200 import solver as S
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


NAMES = ("qx", "qy", "qz", "p", "pcor", "rhoh", "T", "d", "m", "gx", "gy", "gz")


def _check(a, b, tol_q, tol_p):
    """Velocities, momenta and properties at tol_q; p and the pressure correction (whose solve
    amplifies round-off in every path alike) at tol_p, both measured against the pressure scale."""
    pn = max(np.linalg.norm(b[3]), 1e-300)
    for name, x, y in zip(NAMES, a, b):
        if name in ("p", "pcor"):
            err, tol = np.linalg.norm(x - y) / pn, tol_p
        else:
            err, tol = rel(x, y), tol_q
        assert err < tol, (name, err)


def _run(cfg, fields, tc, fused, precision=S.CHS_FP64, substeps=(0, 1, 2, 3, 1, 2, 3), graph_steps=0):
    g = S.Solver(cfg, precision=precision)
    g.set_fusion(fused)
    g.set_fields(*fields)
    if tc is not None:
        g.thermo_init(tc)
    for isub in substeps:
        g.substep(isub)
    if graph_steps:
        g.step(graph_steps)
    out = list(g.get_fields())
    if tc is not None:
        th = g.get_thermo()
        out += [th[k] for k in ("rhoh", "T", "d", "m", "gx", "gy", "gz")]
    g.close()
    return out


CASES = {
    "channel": lambda: (C.channel(nc=(24, 18, 16), iacc=C.IACCU_CD2, dt=0.004), None),
    "heated": lambda: C.heated_channel(nc=(24, 18, 16), iacc=C.IACCU_CD2, dt=0.004, t_ini=0.49),
    "channel3fmd": lambda: (C.channel(nc=(24, 32, 16), iacc=C.IACCU_CD2, dt=0.004, rstret=0.25,
                                      ifft=C.FFT_2DECOMP_3DFFT), None),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_fused_matches_operator_path(case):
    cfg, tc = CASES[case]()
    f = I.channel_fields(cfg)
    a = _run(cfg, f, tc, True, graph_steps=2)
    b = _run(cfg, f, tc, False, graph_steps=2)
    _check(a, b, 1e-13, 1e-9)


def test_fused_tgv_periodic_y():
    cfg = C.taylor_green(16, iacc=C.IACCU_CD2, dt=2e-3)
    f = I.taylor_green_fields(cfg)
    a = _run(cfg, f, None, True)
    b = _run(cfg, f, None, False)
    _check(a, b, 1e-13, 1e-11)
    o = po.Oracle(cfg)
    o.set_fields(*f)
    for isub in (0, 1, 2, 3, 1, 2, 3):
        o.substep(isub)
    _check(a, list(o.get_fields()), 1e-12, 1e-11)


@pytest.mark.parametrize("case", ["channel", "heated"])
def test_fused_mixed_matches_operator_path(case):
    cfg, tc = CASES[case]()
    f = I.channel_fields(cfg)
    a = _run(cfg, f, tc, True, precision=S.CHS_MIXED)
    b = _run(cfg, f, tc, False, precision=S.CHS_MIXED)
    # FP32 round-off: 1e-7 in the velocities, ~1e-3 in the pressure correction of both paths
    _check(a, b, 1e-5, 1e-2)
    sh = cfg.shapes()
    pu = lambda x: x.reshape(sh[0]).mean(axis=(0, 2))
    assert rel(pu(a[0]), pu(b[0])) < 1e-6


def test_fused_heated_vs_oracle_with_fewer_launches():
    cfg, tc = CASES["heated"]()
    f = I.channel_fields(cfg)
    o = po.Oracle(cfg)
    o.set_fields(*f)
    o.thermo_init(tc)
    g = S.Solver(cfg)
    g.set_fields(*f)
    g.thermo_init(tc)
    for isub in (0, 1, 2, 3, 1, 2, 3):
        o.substep(isub)
        g.substep(isub)
    got = list(g.get_fields())
    th = g.get_thermo()
    got += [th[k] for k in NAMES[5:]]
    ref = list(o.get_fields())
    tho = o.get_thermo()
    ref += [tho[k] for k in NAMES[5:]]
    _check(got, ref, 1e-13, 1e-10)
    n_fused = g.kernel_launches()
    g.close()
    h = S.Solver(cfg)
    h.set_fusion(False)
    h.set_fields(*f)
    h.thermo_init(tc)
    for isub in (0, 1, 2, 3, 1, 2, 3):
        h.substep(isub)
    assert n_fused < h.kernel_launches()
    h.close()
