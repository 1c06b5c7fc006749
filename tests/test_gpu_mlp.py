"""MLP surrogate of the property update: the library's FP32 gradients against the numpy oracle,
training on the GPU, the tcgen05 BF16 inference against the FP32 network, the per-cell check with
table fallback against the oracle's table lookup, and what the network gains over the table."""
import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import initial as I
from chapsim2_b200 import solver as S
from oracle import mlp_ref as M
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _solver(nc=(16, 16, 16)):
    cfg, tc = C.heated_channel(nc=nc, iacc=1, dt=0.004)
    g = S.Solver(cfg)
    g.set_fields(*I.channel_fields(cfg))
    g.thermo_init(tc)
    return cfg, tc, g


def test_gradients_match_oracle():
    cfg, tc, g = _solver()
    rng = np.random.default_rng(5)
    p = rng.normal(0.0, 0.2, M.NPARAM).astype(np.float32)
    x = rng.uniform(-1, 1, 700).astype(np.float32)
    t = rng.uniform(-1, 1, (700, 4)).astype(np.float32)
    loss, grad = g.mlp_grad(p, x, t)
    lref, gref = M.loss_and_grad(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - lref) < 1e-5 * abs(lref)
    err = np.abs(grad - gref)
    assert np.max(err) < 1e-4 * np.max(np.abs(gref)) + 1e-7, np.max(err)
    g.close()


@pytest.fixture(scope="module")
def trained():
    cfg, tc, g = _solver()
    rep = g.mlp_train(nsamples=400000, batch=4096, epochs=12, lr=3e-3, seed=7)
    yield cfg, tc, g, rep
    g.close()


def test_training_converges(trained):
    cfg, tc, g, rep = trained
    print("training:", rep)
    assert rep["final_loss"] < 1e-3
    assert rep["steps"] == 12 * ((400000 + 4095) // 4096)


def test_tensor_core_inference_matches_fp32_network(trained):
    cfg, tc, g, rep = trained
    p = g.mlp_params()
    nm = g.mlp_norm()
    tb = tc.table
    rh = np.linspace((tb["d"] * tb["h"]).min(), (tb["d"] * tb["h"]).max(), 3001)
    out, nfb = g.mlp_eval(rh, tol=-1.0)
    assert nfb == 0
    y, _ = M.forward(p.astype(np.float64), nm["xa"] * rh + nm["xb"])
    ref = y * nm["ya"] + nm["yb"]
    # BF16 operands of the two 64x64 layers and the hardware tanh: a few 1e-3 of each range
    for j in range(4):
        e = np.max(np.abs(out[j] - ref[:, j])) / (2 * nm["ya"][j])
        assert e < 2e-2, (j, e)


def test_network_start_rows_judged_by_table(trained):
    """Mode-1 inference: the network's T picks the row where the table search starts and the table
    verifies it, so every output is the table lookup's; a wider error bound lets more starts
    through (fewer fallbacks)."""
    cfg, tc, g, rep = trained
    o = po.Oracle(cfg)
    o.set_fields(*I.channel_fields(cfg))
    o.thermo_init(tc)
    tb = tc.table
    rh_tab = tb["d"] * tb["h"]
    rng = np.random.default_rng(9)
    rh = rng.uniform(rh_tab.min(), rh_tab.max(), 20000)
    h, T, d, m, k, cp = o.ftp_from_dh(rh)
    raw, _ = g.mlp_eval(rh, tol=-1.0)
    e_raw = np.abs(raw[0] - T)
    fracs = []
    for tol in (0.0, 1e-4, 1e-3, 1e-2):
        out, nfb = g.mlp_eval(rh, tol=tol)
        for name, got, ref in zip(("T", "rho", "mu", "kappa", "h"), out, (T, d, m, k, h)):
            err = np.max(np.abs(got - ref))
            assert err <= 1e-13 * (ref.max() - ref.min()), (tol, name, err)
        fracs.append(nfb / rh.size)
    print(f"network T error vs table: max {e_raw.max():.3e} rms {np.sqrt(np.mean(e_raw**2)):.3e}; "
          f"fallback fraction at tol 0, 1e-4, 1e-3, 1e-2: {fracs}")
    assert fracs[0] == 1.0
    assert fracs[1] >= fracs[2] >= fracs[3]
    assert fracs[3] < 0.5


def test_network_in_the_time_loop(trained):
    """Heated-channel steps with the network-started property update give the table update's
    state bit for bit; the fallback count shows how often the network's start row was right."""
    cfg, tc, g, rep = trained
    f = I.channel_fields(cfg)
    a = S.Solver(cfg)
    b = S.Solver(cfg)
    for s in (a, b):
        s.set_fields(*f)
        s.thermo_init(tc)
    b.mlp_params(g.mlp_params())
    b.mlp_set_mode(1, tol=1e-4)
    for s in (a, b):
        s.Solve_momentum_eq(0)
        s.step(3)
    ta, tb_ = a.get_thermo(), b.get_thermo()
    for key in ta:
        assert np.array_equal(ta[key], tb_[key]), key
    for x, y in zip(a.get_fields(), b.get_fields()):
        assert np.array_equal(x, y)
    nfb = b.mlp_fallbacks()
    print(f"fallbacks {nfb} of {3 * 3 * cfg.ncell} cell updates")
    assert 0 <= nfb <= 3 * 3 * cfg.ncell
    a.close()
    b.close()
