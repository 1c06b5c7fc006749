"""Dataflow-scheduled substep graphs (independent launches spread over several streams) give the
same bits as the one-stream graph and as eager substeps in program order."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from chapsim2_b200 import solver as S

pytestmark = pytest.mark.gpu


def _make(case, precision, iacc):
    if case == "heated":
        cfg, tc = C.heated_channel(nc=(24, 18, 16), iacc=iacc, dt=0.004)
    else:
        cfg, tc = C.channel(nc=(24, 18, 16), iacc=iacc, dt=0.004), None
    f = I.channel_fields(cfg)
    g = S.Solver(cfg, precision=precision)
    g.set_fields(*f)
    if tc is not None:
        g.thermo_init(tc)
    g.Solve_momentum_eq(0)
    return g, tc is not None


def _state(g, th):
    out = list(g.get_fields())
    if th:
        out += list(g.get_thermo().values())
    return out


@pytest.mark.parametrize("case", ["channel", "heated"])
@pytest.mark.parametrize("precision", [S.CHS_FP64, S.CHS_MIXED])
@pytest.mark.parametrize("iacc", [1, 3])
def test_lanes_match_program_order(case, precision, iacc):
    nsteps = 3
    # eager substeps, program order on one stream
    e, th = _make(case, precision, iacc)
    for _ in range(nsteps):
        for isub in (1, 2, 3):
            if th:
                e.Solve_energy_eq(isub)
            e.Solve_momentum_eq(isub)
    ref = _state(e, th)
    e.close()
    for lanes in (1, 2, 4, 8):
        g, th = _make(case, precision, iacc)
        g.set_lanes(lanes)
        g.step(nsteps)
        got = _state(g, th)
        g.close()
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), lanes


def test_set_lanes_rejects_out_of_range():
    g, _ = _make("channel", S.CHS_FP64, 1)
    for bad in (0, 9):
        with pytest.raises(RuntimeError):
            g.set_lanes(bad)
    g.close()
