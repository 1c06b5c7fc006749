"""Generate the long-horizon oracle fixtures of tests/golden/ (test infrastructure).

Runs the CPU FP64 oracle (oracle/, a restatement of the reference's time loop:
src/chapsim.f90:243-391 with Solve_energy_eq, src/eq_energy.f90:405-458, and
Solve_momentum_eq, src/eq_momentum2.f90:1799-1932) over the step counts of the
reference's example cases and stores what the GPU tests compare against:

* ``heated500``  -- the heated channel 128x96x128 (CD2, beta 1.5, Re_b 2800,
  isoflux walls, synthetic 4096-row table, dt from CFL 0.8 frozen: the
  benchmark workload), 500 RK3 steps;
* ``channel1000`` -- the flow-only channel 128x96x128 (CD2), 1000 RK3 steps;
* ``tgv200`` -- the Taylor-Green vortex 64^3, Re 1600, CP6, dt 1e-3,
  200 RK3 steps: kinetic energy (src/io_monitor.f90:209-241) and max |div|
  after every step;
* ``cp6fmd100`` -- the flow-only channel 64x64x64 on the 3FMD grid (beta 0.25)
  with CP6 operators and the 3D-FFT Poisson solver for y walls (poisson_010),
  100 RK3 steps: the compact schemes with a consistent Poisson solver.

Per checkpoint the channel cases store x-z-mean profiles
(Calculate_xz_mean_yprofile, src/tools_solver.f90:104-158) of u, p and, with
variable properties, T, h and rho; the y profiles of the u, v, w fluctuation
rms; bulk velocity, bulk kinetic energy and max |div|.  Every run starts with
the isub = 0 step of src/chapsim.f90:135 and then advances whole RK3 steps.

Usage:  python tests/golden/make_long_runs.py [case ...]   (all cases by default)
The heated and flow-only channels take ~35 min each on 8 host cores.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from chapsim2_b200 import config as C  # noqa: E402
from chapsim2_b200 import initial as I  # noqa: E402
from oracle import pyoracle as po  # noqa: E402


def case(name):
    """(cfg, fields, thermo config or None, steps, checkpoint interval) of one fixture case."""
    if name == "heated500":
        cfg, tc = C.heated_channel(nc=(128, 96, 128), iacc=C.IACCU_CD2)
        f = I.channel_fields(cfg)
        cfg.dt = I.cfl_dt(cfg, *f[:3], cfl=0.8)
        return cfg, f, tc, 500, 50
    if name == "channel1000":
        cfg = C.channel(nc=(128, 96, 128), iacc=C.IACCU_CD2)
        f = I.channel_fields(cfg)
        cfg.dt = I.cfl_dt(cfg, *f[:3], cfl=0.8)
        return cfg, f, None, 1000, 100
    if name == "tgv200":
        cfg = C.taylor_green(64, iacc=C.IACCU_CP6, dt=1e-3)
        return cfg, I.taylor_green_fields(cfg), None, 200, 1
    if name == "cp6fmd100":
        cfg = C.channel(nc=(64, 64, 64), iacc=C.IACCU_CP6, rstret=0.25, ifft=C.FFT_2DECOMP_3DFFT)
        f = I.channel_fields(cfg)
        cfg.dt = I.cfl_dt(cfg, *f[:3], cfl=0.8)
        return cfg, f, None, 100, 10
    raise ValueError(name)


def xz_mean(a):
    return a.mean(axis=(0, 2))


def xz_rms(a):
    return np.sqrt(((a - a.mean(axis=(0, 2), keepdims=True)) ** 2).mean(axis=(0, 2)))


def snapshot(cfg, fields, thermo, div, bulk_ke):
    """Per-checkpoint record from (qx, qy, qz, p) and optional thermo dict."""
    qx, qy, qz, p = fields[:4]
    r = {"u_mean": xz_mean(qx), "p_mean": xz_mean(p), "u_rms": xz_rms(qx), "v_rms": xz_rms(qy),
         "w_rms": xz_rms(qz), "bulk_u": I.volumetric_average(cfg, qx), "bulk_ke": bulk_ke,
         "max_div": float(np.abs(div).max())}
    if thermo is not None:
        r["T_mean"] = xz_mean(thermo["T"])
        r["h_mean"] = xz_mean(thermo["h"])
        r["rho_mean"] = xz_mean(thermo["d"])
    return r


def run(name):
    cfg, f, tc, steps, every = case(name)
    o = po.Oracle(cfg)
    o.set_fields(*f)
    if tc is not None:
        o.thermo_init(tc)
    o.substep(0)
    recs, marks = [], []
    t0 = time.time()

    def record(step):
        if name == "tgv200":
            # the Taylor-Green check is the kinetic-energy curve: scalars only
            recs.append({"bulk_ke": o.bulk_ke(), "max_div": float(np.abs(o.divergence()).max())})
        else:
            th = o.get_thermo() if tc is not None else None
            recs.append(snapshot(cfg, o.get_fields(), th, o.divergence(), o.bulk_ke()))
        marks.append(step)

    record(0)
    for s in range(1, steps + 1):
        o.step()
        if s % every == 0:
            record(s)
            if name != "tgv200" or s % 20 == 0:
                print(f"{name}: step {s}/{steps}  {time.time() - t0:.0f} s  ke {recs[-1]['bulk_ke']:.10e}",
                      flush=True)
    out = {"steps": np.array(marks), "dt": np.array(cfg.dt)}
    for k in recs[0]:
        out[k] = np.array([r[k] for r in recs])
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}")


if __name__ == "__main__":
    for n in (sys.argv[1:] or ["tgv200", "cp6fmd100", "heated500", "channel1000"]):
        run(n)
