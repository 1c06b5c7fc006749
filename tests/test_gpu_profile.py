"""Per-launch profiles of a substep: eager launches and one-stream graph replay give one record per
launch with the same classes and byte counts, and the graph profile advances the state exactly like
one substep."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from chapsim2_b200 import solver as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("heated", [False, True])
def test_graph_profile_matches_eager_profile(heated):
    if heated:
        cfg, tc = C.heated_channel(nc=(24, 18, 16), iacc=1, dt=0.004)
    else:
        cfg, tc = C.channel(nc=(24, 18, 16), iacc=3, dt=0.004), None
    f = I.channel_fields(cfg)
    gs = []
    for _ in range(2):
        g = S.Solver(cfg)
        g.set_fields(*f)
        if tc is not None:
            g.thermo_init(tc)
        g.Solve_momentum_eq(0)
        gs.append(g)
    a, b = gs
    pa = a.profile_substep(1)
    pb = b.profile_substep_graph(1)
    assert len(pa) == len(pb) > 10
    for x, y in zip(pa, pb):
        assert (x["kind"], x["dir"], x["bytes"]) == (y["kind"], y["dir"], y["bytes"])
        assert y["ms"] > 0.0
    for x, y in zip(a.get_fields(), b.get_fields()):
        assert np.array_equal(x, y)
    for g in gs:
        g.close()
