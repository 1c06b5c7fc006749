"""Batched ensemble: one graph launch per substep advances members of different grids and
Reynolds numbers exactly as stepping each member alone; the autotuner keeps the solution."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from chapsim2_b200 import solver as S
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _members(precision):
    cfgs = C.ensemble_members(n=4, seed=7, nx=(16, 24), ny=(16, 12), nz=(16, 8))
    out = []
    for cfg in cfgs:
        f = I.channel_fields(cfg)
        cfg.dt = I.cfl_dt(cfg, *f[:3], cfl=0.5)
        g = S.Solver(cfg, precision=precision)
        g.set_fields(*f)
        g.Solve_momentum_eq(0)
        out.append(g)
    return out


@pytest.mark.parametrize("precision", [S.CHS_FP64, S.CHS_MIXED])
def test_ensemble_matches_members_stepped_alone(precision):
    a = _members(precision)
    b = _members(precision)
    assert len({m.cfg.nc for m in a}) > 1
    e = S.Ensemble(a)
    e.step(3)
    for m in b:
        m.step(3)
    for x, y in zip(a, b):
        for p, q in zip(x.get_fields(), y.get_fields()):
            assert np.array_equal(p, q)
    assert e.kernel_launches() > 0
    e.close()
    for m in a + b:
        m.close()


def test_autotune_keeps_the_state():
    cfg = C.channel(nc=(32, 24, 16), iacc=3, dt=0.004)
    f = I.channel_fields(cfg)
    a = S.Solver(cfg)
    b = S.Solver(cfg)
    for g in (a, b):
        g.set_fields(*f)
        g.Solve_momentum_eq(0)
    blk, lt, fu, ms = a.autotune(nsteps=2)
    assert blk in (0, 128, 256, 512) and lt in (16, 32, 64) and fu in (0, 1) and ms > 0
    for p, q in zip(a.get_fields(), b.get_fields()):
        assert np.array_equal(p, q)
    a.step(2)
    b.step(2)
    for p, q in zip(a.get_fields(), b.get_fields()):
        assert np.max(np.abs(p - q)) <= 1e-12 * max(1.0, np.max(np.abs(q)))
    a.close()
    b.close()


@pytest.mark.parametrize("heated", [False, True])
@pytest.mark.parametrize("precision", [S.CHS_FP64, S.CHS_MIXED])
def test_fused_sums_match_separate_operators(heated, precision):
    """The fused per-component passes (an autotuner choice) give the separate operators' result."""
    if heated:
        cfg, tc = C.heated_channel(nc=(24, 18, 16), iacc=1, dt=0.004)
    else:
        cfg, tc = C.channel(nc=(24, 18, 16), iacc=1, dt=0.004), None
    f = I.channel_fields(cfg)
    out = []
    for fused in (0, 1):
        g = S.Solver(cfg, precision=precision)
        g.set_fusion(False)  # the operator path, where the autotuner's fused sums apply
        g.set_fields(*f)
        if tc is not None:
            g.thermo_init(tc)
        g.set_launch_shape(0, 0, fused)
        g.Solve_momentum_eq(0)
        g.step(2)
        out.append([*g.get_fields()[:4]] + ([g.get_thermo()["T"]] if tc is not None else []))
        g.close()
    tol = 1e-12 if precision == S.CHS_FP64 else 1e-5
    for a, b in zip(*out):
        assert np.linalg.norm(a - b) <= tol * max(np.linalg.norm(b), 1e-30)


def test_ensemble_members_match_the_oracle():
    """Members of different grids and Reynolds numbers advanced together by the ensemble graph agree
    with the oracle stepping each member alone (FP64, two RK3 steps)."""
    cfgs = C.ensemble_members(n=3, seed=11, nx=(16, 24), ny=(16, 12), nz=(16, 8))
    members, oracles = [], []
    for cfg in cfgs:
        f = I.channel_fields(cfg)
        cfg.dt = I.cfl_dt(cfg, *f[:3], cfl=0.5)
        g = S.Solver(cfg)
        g.set_fields(*f)
        g.Solve_momentum_eq(0)
        members.append(g)
        o = po.Oracle(cfg)
        o.set_fields(*f)
        o.substep(0)
        oracles.append(o)
    e = S.Ensemble(members)
    e.step(2)
    for g, o in zip(members, oracles):
        o.step()
        o.step()
        got, ref = g.get_fields(), o.get_fields()
        for name, a, b in zip(("qx", "qy", "qz", "p"), got[:4], ref[:4]):
            err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
            assert err < 1e-10, (g.cfg.nc, name, err)
    e.close()
    for g in members:
        g.close()
