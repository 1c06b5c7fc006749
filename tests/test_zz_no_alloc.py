"""chs_poisson_periodic_static (no device allocation, module-level work array) against the
handle's chs_poisson_solve_device on the same grid, scheme and right-hand sides.

The file name sorts last so that the GPU test also runs after every other test in one session.
"""
import dataclasses

import numpy as np
import pytest

from chapsim2_b200 import config as C
from chapsim2_b200 import solver as S


def _cfg(nc, iacc):
    return dataclasses.replace(C.taylor_green(16, iacc=iacc), nc=tuple(nc))


def _lengths(cfg):
    return (cfg.lxx, cfg.lyt - cfg.lyb, cfg.lzz)


@pytest.mark.parametrize("nc, msg", [((4096, 4096, 4096), "too large"), ((30, 24, 16), "2^a 3^b"),
                                      ((32, 5000, 16), "outside")])
def test_rejects_sizes_beyond_the_work_array(nc, msg):
    # the size checks return before any CUDA call, so they run without a GPU
    rc, text = S.poisson_periodic_static(1 << 20, nc, (1.0, 1.0, 1.0), 1)
    assert rc == S.CHS_ERR_ARG and msg in text, (rc, text)


def test_rejects_bad_scheme():
    rc, text = S.poisson_periodic_static(1 << 20, (32, 24, 16), (1.0, 1.0, 1.0), 7)
    assert rc == S.CHS_ERR_ARG and "iacc" in text


def _numpy_cd2(rhs, nc, lengths):
    """CD2 modified-wavenumber solution: phi_hat = -rhs_hat / k'^2 with the zero mode removed."""
    f = np.fft.fftn(rhs.reshape(nc[::-1]))
    k2 = 0.0
    for ax, (m, ln) in enumerate(zip(nc[::-1], lengths[::-1])):
        h = ln / m
        k = 2.0 * np.pi * np.fft.fftfreq(m, d=h)
        shape = [1, 1, 1]
        shape[ax] = m
        k2 = k2 + ((2.0 / h) * np.sin(k * h / 2.0)).reshape(shape) ** 2
    f = np.where(k2 < 1e-16, 0.0, -f / np.where(k2 < 1e-16, 1.0, k2))
    return np.real(np.fft.ifftn(f)).ravel()


def _handle_solve(nc, iacc, rhs):
    """The handle path's solve of the same right-hand side (None when the handle rejects the grid)."""
    import torch

    try:
        g = S.Solver(_cfg(nc, iacc))
    except Exception:
        return None
    a = torch.from_numpy(rhs).to("cuda")
    torch.cuda.synchronize()
    g._check(g.L.chs_poisson_solve_device(g.h, a.data_ptr()), "chs_poisson_solve_device")
    g.sync()
    out = a.cpu().numpy()
    g.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("iacc", [1, 2, 3, 4])
def test_matches_handle_solve_on_two_calls(iacc):
    """Two calls in a row on one grid, both equal to the handle path's solve bit for bit."""
    import torch

    nc = (48, 24, 32)
    cfg = _cfg(nc, iacc)
    rng = np.random.default_rng(7 + iacc)
    n = nc[0] * nc[1] * nc[2]
    b = torch.empty(n, dtype=torch.float64, device="cuda")
    for call in range(2):
        rhs = rng.standard_normal(n)
        ref = _handle_solve(nc, iacc, rhs)
        b.copy_(torch.from_numpy(rhs))
        torch.cuda.synchronize()
        rc, text = S.poisson_periodic_static(b.data_ptr(), nc, _lengths(cfg), iacc)
        assert rc == 0, text
        torch.cuda.synchronize()
        got = b.cpu().numpy()
        assert np.array_equal(got, ref), (call, np.abs(got - ref).max())
        if iacc == 1:
            phi = _numpy_cd2(rhs, nc, _lengths(cfg))
            assert np.abs(got - phi).max() < 1e-12 * np.abs(phi).max()


@pytest.mark.gpu
def test_alternating_grids_rewrite_the_tables():
    """Grid A, grid B (an odd 3^b length, another scheme), grid A again: every call that changes the
    grid or the scheme rewrites the tables, and each result matches the handle path (and, for CD2, the
    numpy solution)."""
    import torch

    seq = [((48, 24, 32), 1), ((27, 18, 16), 1), ((48, 24, 32), 1), ((27, 9, 12), 3), ((48, 24, 32), 2),
           ((48, 24, 32), 4)]
    rng = np.random.default_rng(11)
    for nc, iacc in seq:
        cfg = _cfg(nc, iacc)
        n = nc[0] * nc[1] * nc[2]
        rhs = rng.standard_normal(n)
        b = torch.from_numpy(rhs).to("cuda")
        torch.cuda.synchronize()
        rc, text = S.poisson_periodic_static(b.data_ptr(), nc, _lengths(cfg), iacc)
        assert rc == 0, (nc, iacc, text)
        torch.cuda.synchronize()
        got = b.cpu().numpy()
        ref = _handle_solve(nc, iacc, rhs)
        if ref is not None:
            assert np.array_equal(got, ref), (nc, iacc, np.abs(got - ref).max())
        if iacc == 1:
            phi = _numpy_cd2(rhs, nc, _lengths(cfg))
            assert np.abs(got - phi).max() < 1e-12 * np.abs(phi).max(), (nc, np.abs(got - phi).max())
        assert ref is not None or iacc == 1, f"no check for {nc} iacc {iacc}"
