"""Initial flow fields, mirroring src/initialisation.f90.

* Taylor-Green vortex: initialise_vortexgreen_3dflow (src/initialisation.f90:892-975).
* Channel: Generate_random_field + initialise_poiseuille_flow
  (src/initialisation.f90:161-247, :282-451).  The reference seeds gfortran's
  RNG per cell (src/tools_general.f90:420-601), which is not portable; a
  counter-based splitmix64 stream with a stated seed replaces it here.
"""
import numpy as np

from . import config as C

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x):
    """splitmix64 finaliser applied elementwise to uint64 counters."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return z ^ (z >> np.uint64(31))


def uniform_pm1(shape, seed, stream):
    """Uniform values in [-1, 1) for every cell of `shape`, reproducible from (seed, stream)."""
    n = int(np.prod(shape))
    ctr = np.arange(n, dtype=np.uint64) + (np.uint64(stream) << np.uint64(40)) + (np.uint64(seed) << np.uint64(52))
    bits = _splitmix64(ctr) >> np.uint64(11)
    u = bits.astype(np.float64) * (1.0 / 9007199254740992.0)
    return (2.0 * u - 1.0).reshape(shape)


def taylor_green_fields(cfg):
    """u = sin x cos y cos z, v = -cos x sin y cos z, w = 0, p = (cos2x + cos2y)(cos2z + 2)/16."""
    g = C.geometry(cfg)
    h = g["h"]
    nc = cfg.nc
    sqx, sqy, sqz, sp = cfg.shapes()
    xp = h[0] * np.arange(sqx[2])
    xc = h[0] * (np.arange(nc[0]) + 0.5)
    zc = h[2] * (np.arange(nc[2]) + 0.5)
    zp = h[2] * np.arange(sqz[0])
    yc = g["yc"]
    yp = g["yp"][: sqy[1]]
    qx = np.sin(xp)[None, None, :] * np.cos(yc)[None, :, None] * np.cos(zc)[:, None, None]
    qy = -np.cos(xc)[None, None, :] * np.sin(yp)[None, :, None] * np.cos(zc)[:, None, None]
    qz = np.zeros(sqz)
    p = (1.0 / 16.0) * (np.cos(2 * xc)[None, None, :] + np.cos(2 * yc)[None, :, None]) * \
        (np.cos(2 * zc)[:, None, None] + 2.0)
    del zp
    return np.ascontiguousarray(qx), np.ascontiguousarray(qy), qz, np.ascontiguousarray(p)


def volumetric_average(cfg, a):
    """Get_volumetric_average_3d_for_var_xcx (src/tools_general.f90:1202-1268) for a (k, j, i) array."""
    g = C.geometry(cfg)
    h = g["h"]
    dy = h[1] / g["mpcc"] if cfg.stretch_y else np.full(cfg.nc[1], h[1])
    w = dy[None, :, None] * h[0] * h[2]
    return float(np.sum(a * w) / np.sum(np.broadcast_to(w, a.shape)))


def channel_fields(cfg, noise=0.1, seed=20250101):
    """Poiseuille 1.5(1 - y^2) plus seeded uniform noise, walls enforced, bulk rescaled to 1."""
    sqx, sqy, sqz, sp = cfg.shapes()
    qx = noise * uniform_pm1(sqx, seed, 1)
    qy = noise * uniform_pm1(sqy, seed, 2)
    qz = noise * uniform_pm1(sqz, seed, 3)
    p = np.zeros(sp)
    # Dirichlet perturbation = 0 on the walls (enforce_velo_from_fbc without boundary values)
    if not cfg.periodic_y:
        qy[:, 0, :] = 0.0
        qy[:, -1, :] = 0.0
    g = C.geometry(cfg)
    ymax, ymin = g["yp"][-1], g["yp"][0]
    a = (ymax - ymin) * 0.5
    ux = (1.0 - g["yc"] ** 2 / a / a) * 1.5
    qx = qx + ux[None, :, None]
    ub = volumetric_average(cfg, qx)
    qx = qx / ub
    return qx, qy, qz, p


def cfl_dt(cfg, qx, qy, qz, cfl=0.8):
    """Time step giving the requested convective CFL on the given field.

    Uses second-order midpoint interpolation for the cell-centre velocities
    (the reference reports CFL with its compact interpolation,
    src/tools_solver.f90:273-375, and keeps dt fixed).
    """
    g = C.geometry(cfg)
    h = g["h"]
    u = 0.5 * (qx + np.roll(qx, -1, axis=2))
    if cfg.periodic_y:
        v = 0.5 * (qy + np.roll(qy, -1, axis=1))
    else:
        v = 0.5 * (qy[:, :-1, :] + qy[:, 1:, :])
    w = 0.5 * (qz + np.roll(qz, -1, axis=0))
    s = np.abs(u / h[0] + v * g["mpcc"][None, :, None] / h[1] + w / h[2])
    return float(cfl / s.max())
