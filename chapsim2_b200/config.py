"""Domain configuration mirroring CHAPSim2's input parameters and set-up.

Codes follow src/modules.f90 (boundary conditions :223-229, accuracies
:248-251, stretching :207-212, FFT libraries :169-173).  Geometry follows
src/geometry.f90:151-269 and :410-530; boundary-condition reassignment follows
src/bc_general.f90:137-248 and src/input_general.f90:405-460.
"""
from dataclasses import dataclass, field

import numpy as np

# boundary-condition codes (src/modules.f90:223-229)
IBC_INTERIOR, IBC_PERIODIC, IBC_SYMMETRIC, IBC_ASYMMETRIC, IBC_DIRICHLET, IBC_NEUMANN, IBC_INTRPL = range(7)
# accuracy codes (src/modules.f90:248-251)
IACCU_CD2, IACCU_CD4, IACCU_CP4, IACCU_CP6 = 1, 2, 3, 4
# stretching (src/modules.f90:207-212)
ISTRET_NO, ISTRET_CENTRE, ISTRET_2SIDES, ISTRET_BOTTOM, ISTRET_TOP = 0, 1, 2, 3, 4
# Poisson solvers (src/modules.f90:169-170)
FFT_FISHPACK_2DFFT, FFT_2DECOMP_3DFFT = 2, 3
# flow driving (src/modules.f90:260-264)
IDRVF_NO, IDRVF_X_MASSFLUX = 0, 1
# variable slots of the nominal bc table
V_QX, V_QY, V_QZ, V_PR, V_TM = range(5)


@dataclass
class DomainConfig:
    """One CHAPSim2 domain: grid, boundary conditions, schemes and time step."""
    nc: tuple
    lxx: float
    lyt: float
    lyb: float
    lzz: float
    istret: int = ISTRET_NO
    rstret: float = 0.0
    iacc: int = IACCU_CP6
    ifft: int = FFT_FISHPACK_2DFFT
    idriven: int = IDRVF_NO
    ren: float = 1600.0
    dt: float = 1.0e-3
    # nominal bc codes [dir x,y,z][var qx,qy,qz,pr,Tm][side]
    nominal_bc: np.ndarray = field(default_factory=lambda: np.full((3, 5, 2), IBC_PERIODIC, np.int32))
    # constant y-wall values [var][side] (fbcy_const, src/input_general.f90:420-424)
    fbcy_const: np.ndarray = field(default_factory=lambda: np.zeros((5, 2)))
    name: str = "domain"

    @property
    def periodic_y(self):
        return bool(np.any(self.nominal_bc[1] == IBC_PERIODIC))

    @property
    def stretch_y(self):
        return self.istret != ISTRET_NO

    @property
    def np_(self):
        """Point counts per direction: nc for periodic directions, nc + 1 otherwise."""
        n = list(self.nc)
        if not self.periodic_y:
            n[1] = self.nc[1] + 1
        return tuple(n)

    def shapes(self):
        """numpy (C-order, k-j-i) shapes of qx, qy, qz, p."""
        nc, n = self.nc, self.np_
        return ((nc[2], nc[1], n[0]), (nc[2], n[1], nc[0]), (n[2], nc[1], nc[0]), (nc[2], nc[1], nc[0]))

    @property
    def ncell(self):
        return int(self.nc[0]) * int(self.nc[1]) * int(self.nc[2])


def taylor_green(n=64, iacc=IACCU_CP6, dt=1.0e-3, ren=1600.0):
    """3D Taylor-Green vortex box: triply periodic, uniform, 3D-FFT Poisson.

    The reference forces the box to x, z in [0, 2 pi], y in [-pi, pi]
    (src/input_general.f90:376-382).
    """
    return DomainConfig(nc=(n, n, n), lxx=2 * np.pi, lyt=np.pi, lyb=-np.pi, lzz=2 * np.pi, iacc=iacc,
                        ifft=FFT_2DECOMP_3DFFT, idriven=IDRVF_NO, ren=ren, dt=dt, name=f"tgv{n}")


def channel(nc=(128, 96, 128), rstret=0.075, ren=2800.0, iacc=IACCU_CP6, dt=None, lxx=4 * np.pi,
            lzz=4 * np.pi / 3, ifft=FFT_FISHPACK_2DFFT, istret=ISTRET_2SIDES):
    """Periodic turbulent channel with no-slip y walls and constant mass flux.

    With the FISHPACK Poisson solver (default) the stretching is the reference's
    tanh mapping with beta = 20 * rstret (src/geometry.f90:237); rstret = 0.075
    is beta = 1.5.  With ifft = FFT_2DECOMP_3DFFT the mapping is the 3FMD one
    (src/geometry.f90:287-408, beta = rstret, e.g. 0.25 as in the reference's
    channel example) and the Poisson solver is poisson_010
    (src/input_general.f90:552-553, src/poisson_1stderivcomp.f90:1457-1816).
    """
    bc = np.full((3, 5, 2), IBC_PERIODIC, np.int32)
    bc[1, V_QX] = IBC_DIRICHLET
    bc[1, V_QY] = IBC_DIRICHLET
    bc[1, V_QZ] = IBC_DIRICHLET
    bc[1, V_PR] = IBC_NEUMANN
    bc[1, V_TM] = IBC_DIRICHLET
    cfg = DomainConfig(nc=tuple(nc), lxx=lxx, lyt=1.0, lyb=-1.0, lzz=lzz, istret=istret, rstret=rstret,
                       iacc=iacc, ifft=ifft, idriven=IDRVF_X_MASSFLUX, ren=ren,
                       dt=dt if dt is not None else 1.0e-3, nominal_bc=bc, name=f"channel{nc[0]}x{nc[1]}x{nc[2]}")
    return cfg


# ---------------------------------------------------------------------------
# variable-property (thermal) runs
# ---------------------------------------------------------------------------
T_PC = 0.5  # pseudo-critical temperature of the synthetic fluid


def _h_of_t(t):
    """h(T) = integral of cp from T_PC (closed form for cp = 1 + 4/(1+((T-0.5)/0.02)^2))."""
    x = np.asarray(t, np.float64) - T_PC
    return x + 0.08 * np.arctan(x / 0.02)


def synthetic_table(n=4096):
    """Nondimensional property table of the heated-channel case, sorted by T.

    cp(T) = 1 + 4/(1+((T-0.5)/0.02)^2), h = integral of cp dT, rho = 1 - 0.6 (1+tanh((T-0.5)/0.03))/2,
    mu = rho^0.7, kappa = cp^0.5, beta = -(1/rho) drho/dT.  h is measured from the pseudo-critical
    point and the T range is symmetric about it with h spanning a unit interval, h in [-1/2, 1/2];
    with h = 0 at T = 0.5 the table's rho*h is monotonic in T, which the reference's rho*h lookup
    requires (src/input_thermo.f90:560-598).  Columns are (T, h, rho, mu, kappa, cp, beta), the
    nondimensional form of the reference's table file (P H T D M K CP B, src/input_thermo.f90:640-657).
    """
    lo, hi = 0.0, 0.5
    for _ in range(200):  # x + 0.08 atan(x/0.02) = 1/2
        mid = 0.5 * (lo + hi)
        if _h_of_t(T_PC + mid) < 0.5:
            lo = mid
        else:
            hi = mid
    x = 0.5 * (lo + hi)
    t = np.linspace(T_PC - x, T_PC + x, n)
    h = _h_of_t(t)
    cp = 1.0 + 4.0 / (1.0 + ((t - T_PC) / 0.02) ** 2)
    th = np.tanh((t - T_PC) / 0.03)
    d = 1.0 - 0.6 * (1.0 + th) / 2.0
    m = d ** 0.7
    k = cp ** 0.5
    b = (0.3 / 0.03) * (1.0 - th * th) / d
    return dict(t=t, h=h, d=d, m=m, k=k, cp=cp, b=b)


def constant_table(n=256):
    """Constant-property table (rho = mu = kappa = cp = 1, h = T): the variable-property path then
    reproduces the constant-property momentum solution."""
    t = np.linspace(-1.0, 2.0, n)
    one = np.ones(n)
    return dict(t=t, h=t.copy(), d=one, m=one.copy(), k=one.copy(), cp=one.copy(), b=np.zeros(n))


@dataclass
class ThermoConfig:
    """Thermal set-up of a variable-property run (input_thermo / [thermo] section)."""
    table: dict
    t_ini: float = 0.47
    prandtl: float = 1.0  # rPrRen = 1/(Re Pr) with unit reference properties (src/tools_solver.f90:63)
    qw: tuple = (-1.0, 1.0)  # dT/dy at the y walls: heat flux q_w = 1 into the fluid at both walls


def heated_channel(nc=(128, 96, 128), iacc=IACCU_CD2, dt=None, rstret=0.075, ren=2800.0, table=None, t_ini=0.47,
                   ifft=FFT_FISHPACK_2DFFT):
    """Heated channel with variable properties (same grid and flow as the channel) and isoflux
    y walls: T is Neumann at the walls, so the property BC is Dirichlet there
    (src/bc_general.f90:182-186).  Returns (DomainConfig, ThermoConfig)."""
    cfg = channel(nc=nc, rstret=rstret, ren=ren, iacc=iacc, dt=dt, ifft=ifft)
    cfg.nominal_bc[1, V_TM] = IBC_NEUMANN
    cfg.name = f"heated{nc[0]}x{nc[1]}x{nc[2]}"
    tc = ThermoConfig(table=table if table is not None else synthetic_table(), t_ini=t_ini)
    cfg.fbcy_const[V_TM] = tc.qw
    return cfg, tc


def ensemble_members(n=48, seed=4242, nx=(64, 96, 128), ny=(64, 96), nz=(64, 96, 128), re=(2000.0, 5000.0),
                     iacc=IACCU_CD2):
    """Members of the batched ensemble: periodic channels 4pi x 2 x 4pi/3 with tanh stretching
    beta = 1.5 whose grids (Nx, Ny, Nz) and bulk Reynolds numbers are drawn by a seeded splitmix64
    stream."""
    state = [seed & 0xFFFFFFFFFFFFFFFF]

    def u():
        state[0] = (state[0] + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = state[0]
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z ^= z >> 31
        return (z >> 11) / float(1 << 53)

    out = []
    for _ in range(n):
        g = (nx[int(u() * len(nx))], ny[int(u() * len(ny))], nz[int(u() * len(nz))])
        r = re[0] + (re[1] - re[0]) * u()
        out.append(channel(nc=g, ren=r, iacc=iacc))
    return out


# ---------------------------------------------------------------------------
# geometry (src/geometry.f90)
# ---------------------------------------------------------------------------
def _tanh_mapping(cfg, node, n):
    if node:
        shift, delta_eta = 0.0, 1.0 / (n - 1)
    else:
        shift, delta_eta = 0.5 / n, 1.0 / n
    eta = shift + np.arange(n) * delta_eta
    gamma, delta, ymin, ymax = {ISTRET_2SIDES: (0.5, 0.5, -1.0, 1.0), ISTRET_BOTTOM: (-1.0, 1.0, 0.0, 1.0),
                                ISTRET_TOP: (1.0, 0.0, 0.0, 1.0)}[cfg.istret]
    beta = cfg.rstret * 20.0
    mm = np.tanh(beta * gamma)
    y = np.tanh(beta * (eta - delta)) / mm
    m1 = 1.0 - y * y * mm * mm
    small = (m1 < 1e-20) & (m1 > -1e-20)
    m1 = np.where(small, 1.0, mm / beta / np.where(small, 1.0, m1))
    ff = (cfg.lyt - cfg.lyb) / (ymax - ymin)
    return (y - ymin) * ff + cfg.lyb, m1 / ff


def _heaviside(r):
    """heaviside_step (src/modules.f90:960-971)."""
    return np.where(r > 1.0e-20, 1.0, np.where(r < -1.0e-20, 0.0, 0.5))


def _fmd_mapping(cfg, node, n):
    """Buildup_grid_mapping_1D_3fmd (src/geometry.f90:287-408): y and yMapping(:,1) = d eta/dy."""
    if node:
        shift, delta_eta = 0.0, 1.0 / (n - 1)
    else:
        shift, delta_eta = 0.5 / n, 1.0 / n
    eta = shift + np.arange(n) * delta_eta
    gamma, delta = {ISTRET_CENTRE: (1.0, 0.0), ISTRET_2SIDES: (1.0, 0.5), ISTRET_BOTTOM: (0.5, 0.5),
                    ISTRET_TOP: (0.5, 0.0)}[cfg.istret]
    beta = cfg.rstret
    alpha = (-1.0 + np.sqrt(1.0 + 4.0 * np.pi * np.pi * beta * beta)) / beta * 0.5
    cc = np.sqrt(alpha * beta + 1.0) / np.sqrt(beta)
    dd = cc / np.sqrt(alpha)
    ee = cc * np.sqrt(alpha)
    st1 = (1.0 - 2.0 * delta) / gamma * 0.5
    st2 = (3.0 - 2.0 * delta) / gamma * 0.5
    mm = np.pi * (gamma * eta + delta)
    y = (np.arctan(dd * np.tan(mm)) - np.arctan(dd * np.tan(np.pi * delta))
         + np.pi * (_heaviside(eta - st1) + _heaviside(eta - st2)))
    y = 1.0 / (gamma * ee) * y
    if node:
        y[0], y[-1] = 0.0, 1.0
    ly = cfg.lyt - cfg.lyb
    return y * ly + cfg.lyb, (alpha / np.pi + np.sin(mm) * np.sin(mm) / np.pi / beta) / ly


def geometry(cfg):
    """Return dict with h(3), yp(np_geo), yc(nc), mppt, mpcc (yMapping(:,1))."""
    nc = cfg.nc
    h = np.array([cfg.lxx / nc[0], (cfg.lyt - cfg.lyb) / nc[1], cfg.lzz / nc[2]])
    if cfg.stretch_y:
        h[1] = 1.0 / nc[1]
        # the 3D-FFT solver selects the 3FMD mapping, FISHPACK the tanh one (src/input_general.f90:552-553)
        mapping = _fmd_mapping if cfg.ifft == FFT_2DECOMP_3DFFT else _tanh_mapping
        yp, mppt = mapping(cfg, True, nc[1] + 1)
        yc, mpcc = mapping(cfg, False, nc[1])
    else:
        yp = np.arange(nc[1] + 1) * h[1] + cfg.lyb
        yc = np.arange(nc[1]) * h[1] + h[1] * 0.5 + cfg.lyb
        mppt = np.ones(nc[1] + 1)
        mpcc = np.ones(nc[1])
    return dict(h=h, yp=yp, yc=yc, mppt=mppt, mpcc=mpcc)


def calculated_bcs(cfg):
    """Apply config_calc_basic_ibc (src/bc_general.f90:137-184) to the nominal table.

    Returns (ibc[3][5][2], fbcy_const[5][2]).
    """
    ibc = np.array(cfg.nominal_bc, np.int32, copy=True)
    fb = np.array(cfg.fbcy_const, np.float64, copy=True)
    for n in range(2):
        if ibc[0, V_QX, n] == IBC_SYMMETRIC:
            ibc[0, V_QX, n] = IBC_ASYMMETRIC
        if ibc[1, V_QY, n] == IBC_SYMMETRIC:
            ibc[1, V_QY, n] = IBC_ASYMMETRIC
        if ibc[2, V_QZ, n] == IBC_SYMMETRIC:
            ibc[2, V_QZ, n] = IBC_ASYMMETRIC
        if ibc[0, V_QX, n] == IBC_DIRICHLET:
            ibc[0, V_PR, n] = IBC_NEUMANN
        if ibc[1, V_QY, n] == IBC_DIRICHLET:
            ibc[1, V_PR, n] = IBC_NEUMANN
            fb[V_PR, n] = 0.0
        if ibc[2, V_QZ, n] == IBC_DIRICHLET:
            ibc[2, V_PR, n] = IBC_NEUMANN
    return ibc, fb
