"""Run a few substeps of the channel, heated channel or Taylor-Green case for profilers.

Launches every kernel individually (no graph replay), so a profiler sees one
launch per operator.  Example:
    python chapsim2_b200/profile_case.py --nc 128 96 128 --substeps 3
    python chapsim2_b200/profile_case.py --case heated --precision mixed --mlp-epochs 4
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from chapsim2_b200 import config as C  # noqa: E402
from chapsim2_b200 import initial as I  # noqa: E402
from chapsim2_b200 import solver as S  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="channel", choices=["channel", "heated", "tgv"])
    ap.add_argument("--nc", type=int, nargs=3, default=[128, 96, 128])
    ap.add_argument("--iacc", type=int, default=C.IACCU_CD2)
    ap.add_argument("--substeps", type=int, default=3)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--mlp-epochs", type=int, default=0,
                    help="heated case: train the property surrogate for this many epochs and use it")
    ap.add_argument("--graph-profile", action="store_true",
                    help="after the substeps, print a per-launch profile of substep 1 replayed as a graph")
    ap.add_argument("--fusion", type=int, default=1, choices=[0, 1],
                    help="CD2 fused substep kernels (1, the default) or the operator path (0)")
    ap.add_argument("--poisson", default="fishpack", choices=["fishpack", "3dfft"],
                    help="channel cases: FISHPACK with tanh stretching, or the 3D-FFT solver (poisson_010) "
                         "with 3FMD stretching (rstret 0.25)")
    a = ap.parse_args()
    tc = None
    wall = {} if a.poisson == "fishpack" else dict(ifft=C.FFT_2DECOMP_3DFFT, rstret=0.25)
    if a.case == "channel":
        cfg = C.channel(nc=tuple(a.nc), iacc=a.iacc, **wall)
        f = I.channel_fields(cfg)
        cfg.dt = I.cfl_dt(cfg, *f[:3], cfl=0.8)
    elif a.case == "heated":
        cfg, tc = C.heated_channel(nc=tuple(a.nc), iacc=a.iacc, **wall)
        f = I.channel_fields(cfg)
        cfg.dt = I.cfl_dt(cfg, *f[:3], cfl=0.8)
    else:
        cfg = C.taylor_green(a.nc[0], iacc=a.iacc)
        f = I.taylor_green_fields(cfg)
    g = S.Solver(cfg, precision=S.CHS_MIXED if a.precision == "mixed" else S.CHS_FP64)
    g.set_fusion(a.fusion)
    g.set_fields(*f)
    if tc is not None:
        g.thermo_init(tc)
        if a.mlp_epochs > 0:
            g.mlp_train(nsamples=200000, batch=4096, epochs=a.mlp_epochs, lr=3e-3, seed=7)
            g.mlp_set_mode(1, tol=1e-4)
    g.Solve_momentum_eq(0)
    for i in range(a.substeps):
        g.substep(1 + i % 3)
    if a.graph_profile:
        kinds = ("line_op", "fft", "ysolve", "elementwise", "fused_momentum")
        prof = g.profile_substep_graph(1)
        for i, r in enumerate(prof):
            print(f"{i:3d} {kinds[r['kind']]:11s} dir {r['dir']:2d} {r['bytes'] / 1e6:9.1f} MB {r['ms'] * 1e3:9.1f} us "
                  f"{r['bytes'] / r['ms'] / 1e6:7.0f} GB/s")
        print(f"substep total {sum(r['ms'] for r in prof):.3f} ms over {len(prof)} launches")
    d = g.diagnostics()
    print(f"{a.case} {cfg.nc} iacc={a.iacc}: {a.substeps} substeps, launches={g.kernel_launches()}, "
          f"max_div={d['max_div']:.3e}, nan={d['nan_flag']}")
    g.close()
    if d["nan_flag"]:
        sys.exit(1)


if __name__ == "__main__":
    main()
