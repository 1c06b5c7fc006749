"""Host-side operator plans of the CUDA library, executed by a numpy emulation
of the line-operator kernel, against the oracle (CPU only; no GPU needed)."""
import numpy as np
import pytest

import planexec as PE
from chapsim2_b200 import config as C
from chapsim2_b200 import solver as S
from oracle import pyoracle as po

WALL_BCS = [(4, 4), (5, 5), (2, 3), (3, 2), (0, 0), (6, 6), (4, 5)]


def _cases():
    for acc in (1, 2, 3, 4):
        for kind in ("tgv", "chan"):
            for d in (0, 1, 2):
                for fam in range(6):
                    bcs = WALL_BCS if (kind == "chan" and d == 1) else [(1, 1)]
                    for ibc in bcs:
                        yield acc, kind, d, fam, ibc


@pytest.mark.parametrize("acc,kind,d,fam,ibc", list(_cases()))
def test_plan_matches_oracle(acc, kind, d, fam, ibc):
    cfg = C.taylor_green(12, iacc=acc) if kind == "tgv" else C.channel(nc=(12, 10, 8), iacc=acc)
    o = po.Oracle(cfg)
    rng = np.random.default_rng(acc * 100 + d * 10 + fam)
    nin3 = list(cfg.nc)
    if fam in (1, 3, 5):
        nin3[d] = cfg.np_[d]
    shp = (nin3[2], nin3[1], nin3[0])
    fi = rng.standard_normal(shp)
    fb = rng.standard_normal({0: (nin3[2], nin3[1], 4), 1: (nin3[2], 4, nin3[0]), 2: (4, nin3[1], nin3[0])}[d])
    for has in (False, True):
        p = S.plan_inspect(cfg, d, fam, ibc, has)
        ref = o.op3d(d, fam, ibc, fi, fb if has else None)
        got = PE.run_plan(p, fi, d, PE.fbc_ref_to_lines(fb, d, shp) if has else None)
        assert np.abs(ref - got).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_plan_rejects_short_lines():
    cfg = C.taylor_green(12)
    cfg.nc = (6, 12, 12)
    with pytest.raises(RuntimeError):
        S.plan_inspect(cfg, 0, 0, (1, 1), False)


def test_plan_boundary_rows_small():
    """Boundary rows touch only a few points near each end (or the wrap for periodic lines)."""
    cfg = C.channel(nc=(16, 24, 16), iacc=4)
    p = S.plan_inspect(cfg, 1, 2, (4, 4), True)
    assert p["nspec"] == 4
    for r in p["rows"]:
        assert len(r["idx"]) <= 6
        assert all((i < 6) or (i >= p["nin"] - 6) for i in r["idx"])


@pytest.mark.parametrize("acc", [1, 2, 3, 4])
@pytest.mark.parametrize("fam", range(6))
def test_periodic_explicit_plans_wrap(acc, fam):
    """Periodic explicit lines carry the wrap flag (every row through the bulk formula with
    wrapped indices); compact and wall-bounded lines never do."""
    cfg = C.channel(nc=(12, 10, 8), iacc=acc)
    for d in (0, 2):
        p = S.plan_inspect(cfg, d, fam, (1, 1), False)
        assert p["wrap"] == (1 if p["tdma"] == 0 else 0), (d, p["tdma"])
    for ibc in WALL_BCS:
        assert S.plan_inspect(cfg, 1, fam, ibc, True)["wrap"] == 0
