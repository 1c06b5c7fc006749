"""ctypes binding of libchapsim_gpu.so, mirroring the reference's Fortran interface.

The calls follow the routines that src/chapsim.f90 drives each time step:
``Solve_momentum_eq(isub)`` (src/eq_momentum2.f90:1799), ``solve_fft_poisson``
(src/poisson_interface.f90:119) and the post-step checks.  There is no CPU
fallback: if the CUDA library is missing or no GPU is present the calls raise.
"""
import ctypes
import os

import numpy as np

from . import config as C

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libchapsim_gpu.so")

CHS_QX, CHS_QY, CHS_QZ, CHS_PRES, CHS_PCOR, CHS_MX_RHS0, CHS_MY_RHS0, CHS_MZ_RHS0 = range(8)
(CHS_GX, CHS_GY, CHS_GZ, CHS_RHOH, CHS_HENTH, CHS_TTEMP, CHS_KCOND, CHS_DDENS, CHS_MVISC,
 CHS_ENE_RHS0) = range(8, 18)
CHS_FP64, CHS_MIXED = 0, 1
CHS_OK, CHS_ERR_ARG, CHS_ERR_CUDA, CHS_ERR_STATE, CHS_ERR_NUMERIC = range(5)
_D = ctypes.POINTER(ctypes.c_double)


class ChsConfig(ctypes.Structure):
    _fields_ = [
        ("nc", ctypes.c_int * 3),
        ("iacc", ctypes.c_int),
        ("istret", ctypes.c_int),
        ("ifft", ctypes.c_int),
        ("idriven", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("lxx", ctypes.c_double), ("lyt", ctypes.c_double), ("lyb", ctypes.c_double), ("lzz", ctypes.c_double),
        ("rstret", ctypes.c_double), ("dt", ctypes.c_double), ("ren", ctypes.c_double),
        ("nominal_bc", ctypes.c_int * 30),
        ("fbcy_const", ctypes.c_double * 10),
        ("yp", _D), ("yc", _D), ("ymap_pt", _D), ("ymap_cc", _D),
    ]


class ChsThermo(ctypes.Structure):
    _fields_ = [("ntable", ctypes.c_int), ("t", _D), ("h", _D), ("d", _D), ("m", _D), ("k", _D), ("cp", _D),
                ("b", _D), ("rPrRen", ctypes.c_double), ("t_ini", ctypes.c_double)]


class ChsMlpTrainCfg(ctypes.Structure):
    _fields_ = [("nsamples", ctypes.c_int), ("batch", ctypes.c_int), ("epochs", ctypes.c_int),
                ("lr", ctypes.c_double), ("seed", ctypes.c_ulonglong)]


class ChsMlpReport(ctypes.Structure):
    _fields_ = [("final_loss", ctypes.c_double), ("train_ms", ctypes.c_double), ("steps", ctypes.c_int)]


MLP_NPARAM = 8708


class ChsDiag(ctypes.Structure):
    _fields_ = [("max_div", ctypes.c_double), ("bulk_ke", ctypes.c_double), ("bulk_u", ctypes.c_double),
                ("last_bulk_rhs", ctypes.c_double), ("nan_flag", ctypes.c_int), ("mcon", ctypes.c_double * 3)]


EXPORTED = ["chs_create", "chs_destroy", "chs_upload_field", "chs_download_field", "chs_momentum_substep",
            "chs_step", "chs_poisson_solve", "chs_poisson_solve_device", "chs_diagnostics", "chs_op3d",
            "chs_plan_inspect", "chs_sync", "chs_kernel_launches", "chs_last_error", "chs_momentum_substep_host",
            "chs_time_steps", "chs_time_steps_host", "chs_host_alloc", "chs_host_free", "chs_profile_substep",
            "chs_poisson_periodic_static", "chs_thermo_init", "chs_energy_substep", "chs_time_steps_host_fields",
            "chs_time_rk3_host_fields",
            "chs_mlp_train", "chs_mlp_set_mode", "chs_mlp_fallbacks", "chs_mlp_params", "chs_mlp_grad",
            "chs_mlp_eval", "chs_mlp_norm", "chs_ensemble_create", "chs_ensemble_step", "chs_ensemble_time_steps",
            "chs_ensemble_kernel_launches", "chs_ensemble_destroy", "chs_autotune", "chs_set_launch_shape",
            "chs_set_lanes", "chs_profile_substep_graph", "chs_write_restart", "chs_read_restart",
            "chs_stats_update", "chs_stats_get", "chs_write_statistics", "chs_read_statistics",
            "chs_data_file_name", "chs_set_fusion", "chs_profile_class"]


class ChsKprof(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("dir", ctypes.c_int), ("bytes", ctypes.c_double), ("ms", ctypes.c_float)]

_lib = None


def load():
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run chapsim2_b200/build.py (no CPU fallback exists)")
    L = ctypes.CDLL(LIB_PATH)
    L.chs_create.argtypes = [ctypes.POINTER(ChsConfig), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.chs_destroy.argtypes = [ctypes.c_void_p]
    L.chs_upload_field.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_size_t]
    L.chs_download_field.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_size_t]
    L.chs_momentum_substep.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.chs_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.chs_poisson_solve.argtypes = [ctypes.c_void_p, _D]
    L.chs_poisson_solve_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.chs_diagnostics.argtypes = [ctypes.c_void_p, ctypes.POINTER(ChsDiag)]
    L.chs_op3d.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D,
                           ctypes.POINTER(ctypes.c_int), _D]
    L.chs_plan_inspect.argtypes = [ctypes.POINTER(ChsConfig), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, _D, ctypes.c_size_t]
    L.chs_sync.argtypes = [ctypes.c_void_p]
    L.chs_kernel_launches.restype = ctypes.c_longlong
    L.chs_kernel_launches.argtypes = [ctypes.c_void_p]
    L.chs_last_error.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    L.chs_momentum_substep_host.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D, _D]
    L.chs_time_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.chs_time_steps_host.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D, _D, ctypes.POINTER(ctypes.c_float)]
    L.chs_host_alloc.restype = ctypes.c_void_p
    L.chs_host_alloc.argtypes = [ctypes.c_size_t]
    L.chs_host_free.argtypes = [ctypes.c_void_p]
    L.chs_profile_substep.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ChsKprof), ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int)]
    L.chs_profile_substep_graph.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ChsKprof), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int)]
    L.chs_thermo_init.argtypes = [ctypes.c_void_p, ctypes.POINTER(ChsThermo)]
    _F = ctypes.POINTER(ctypes.c_float)
    L.chs_mlp_train.argtypes = [ctypes.c_void_p, ctypes.POINTER(ChsMlpTrainCfg), ctypes.POINTER(ChsMlpReport)]
    L.chs_mlp_set_mode.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
    L.chs_mlp_fallbacks.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong)]
    L.chs_mlp_params.argtypes = [ctypes.c_void_p, _F, ctypes.c_int, ctypes.c_int]
    L.chs_mlp_grad.argtypes = [ctypes.c_void_p, _F, ctypes.c_int, _F, _F, _F, _F]
    L.chs_mlp_eval.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_double, _D,
                               ctypes.POINTER(ctypes.c_ulonglong)]
    L.chs_mlp_norm.argtypes = [ctypes.c_void_p, _D]
    L.chs_set_launch_shape.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.chs_set_lanes.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.chs_set_fusion.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.chs_profile_class.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_float)]
    for fn in ("chs_write_restart", "chs_read_restart", "chs_write_statistics", "chs_read_statistics"):
        getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
    L.chs_stats_update.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.chs_stats_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t]
    L.chs_data_file_name.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p,
                                     ctypes.c_size_t]
    L.chs_ensemble_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.chs_ensemble_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.chs_ensemble_time_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.chs_ensemble_kernel_launches.restype = ctypes.c_longlong
    L.chs_ensemble_kernel_launches.argtypes = [ctypes.c_void_p]
    L.chs_ensemble_destroy.argtypes = [ctypes.c_void_p]
    L.chs_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_float)]
    L.chs_time_steps_host_fields.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_D),
                                             ctypes.POINTER(ctypes.c_float)]
    L.chs_time_rk3_host_fields.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_D),
                                           ctypes.POINTER(ctypes.c_float)]
    L.chs_energy_substep.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.chs_poisson_periodic_static.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_char_p, ctypes.c_size_t]
    _lib = L
    return L


def poisson_periodic_static(d_rhs, nc, lengths, iacc, stream=None):
    """Periodic Poisson solve in place on a device array (address d_rhs) with no device allocation.

    Returns (status, message); status 0 is success.
    """
    L = load()
    n = (ctypes.c_int * 3)(*[int(v) for v in nc])
    ln = (ctypes.c_double * 3)(*[float(v) for v in lengths])
    err = ctypes.create_string_buffer(512)
    rc = L.chs_poisson_periodic_static(ctypes.c_void_p(d_rhs), n, ln, int(iacc), stream, err, 512)
    return rc, err.value.decode()


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_D)


def make_config(cfg, precision=CHS_FP64):
    """Fill a ChsConfig from a DomainConfig; returns (struct, keep-alive arrays)."""
    g = C.geometry(cfg)
    keep = [np.ascontiguousarray(g[k], np.float64) for k in ("yp", "yc", "mppt", "mpcc")]
    s = ChsConfig()
    for d in range(3):
        s.nc[d] = int(cfg.nc[d])
    s.iacc, s.istret, s.ifft, s.idriven = int(cfg.iacc), int(cfg.istret), int(cfg.ifft), int(cfg.idriven)
    s.precision = int(precision)
    s.lxx, s.lyt, s.lyb, s.lzz = float(cfg.lxx), float(cfg.lyt), float(cfg.lyb), float(cfg.lzz)
    s.rstret, s.dt, s.ren = float(cfg.rstret), float(cfg.dt), float(cfg.ren)
    nb = np.ascontiguousarray(cfg.nominal_bc, np.int32).ravel()
    for i in range(30):
        s.nominal_bc[i] = int(nb[i])
    fb = np.ascontiguousarray(cfg.fbcy_const, np.float64).ravel()
    for i in range(10):
        s.fbcy_const[i] = float(fb[i])
    s.yp, s.yc, s.ymap_pt, s.ymap_cc = [_ptr(a) for a in keep]
    return s, keep


def data_file_name(directory, idom, keyword, iteration):
    """Restart/statistics file name of the reference's naming (host only)."""
    L = load()
    buf = ctypes.create_string_buffer(4096)
    rc = L.chs_data_file_name(str(directory).encode(), int(idom), str(keyword).encode(), int(iteration), buf, 4096)
    if rc != 0:
        raise RuntimeError(f"chs_data_file_name failed ({rc})")
    return buf.value.decode()


def plan_inspect(cfg, d, fam, ibc, has_fbc):
    """Host-only view of one operator plan (dict of numpy arrays)."""
    L = load()
    s, keep = make_config(cfg)
    n = cfg.np_[d] if fam in (1, 2, 4) else cfg.nc[d]
    buf = np.zeros(128 + 5 * n + 8)
    rc = L.chs_plan_inspect(ctypes.byref(s), d, fam, int(ibc[0]), int(ibc[1]), int(bool(has_fbc)), _ptr(buf),
                            buf.size)
    if rc != 0:
        raise RuntimeError(f"chs_plan_inspect failed ({rc})")
    h = buf[:20]
    p = dict(fam=int(h[0]), nin=int(h[1]), nout=int(h[2]), b_lo=int(h[3]), b_hi=int(h[4]),
             off=[int(x) for x in h[5:9]], sgn=h[9], r1=h[10], r2=h[11], dd=h[12], nspec=int(h[13]),
             tdma=int(h[14]), b1=h[15], an=h[16], cn=h[17], inv_den=h[18], neu1=(int(h[19]) // 2) % 2,
             neu2=int(h[19]) % 2, wrap=int(h[19]) // 4)
    rows = []
    for k in range(p["nspec"]):
        o = buf[20 + 26 * k: 46 + 26 * k]
        nt = int(o[1])
        rows.append(dict(row=int(o[0]), idx=o[2:2 + nt].astype(int), w=o[12:12 + nt].copy(), wb=o[22:26].copy()))
    p["rows"] = rows
    arr = buf[128:128 + 5 * n]
    p["a"], p["c"], p["d"], p["x1"], p["map"] = [arr[i * n:(i + 1) * n].copy() for i in range(5)]
    return p


class Solver:
    """One domain resident on the GPU (a chs_handle)."""

    def __init__(self, cfg, device=0, precision=CHS_FP64):
        self.cfg = cfg
        self.L = load()
        self._s, self._keep = make_config(cfg, precision)
        h = ctypes.c_void_p()
        rc = self.L.chs_create(ctypes.byref(self._s), int(device), ctypes.byref(h))
        if rc != 0 or not h.value:
            raise RuntimeError(f"chs_create failed with status {rc}")
        self.h = h
        self.shapes = cfg.shapes()

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.chs_destroy(self.h)
            self.h = None
        for p in self.__dict__.pop("_pinned", []):
            self.L.chs_host_free(p)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            buf = ctypes.create_string_buffer(1024)
            self.L.chs_last_error(self.h, buf, 1024)
            raise RuntimeError(f"{what} failed ({rc}): {buf.value.decode()}")

    # ---- state
    def upload(self, field, a):
        a = np.ascontiguousarray(a, np.float64)
        self._check(self.L.chs_upload_field(self.h, field, _ptr(a), a.size), "chs_upload_field")

    def download(self, field):
        shp = {CHS_QX: 0, CHS_MX_RHS0: 0, CHS_QY: 1, CHS_MY_RHS0: 1, CHS_QZ: 2, CHS_MZ_RHS0: 2,
               CHS_PRES: 3, CHS_PCOR: 3, CHS_GX: 0, CHS_GY: 1, CHS_GZ: 2}.get(field, 3)
        a = np.zeros(self.shapes[shp])
        self._check(self.L.chs_download_field(self.h, field, _ptr(a), a.size), "chs_download_field")
        return a

    def thermo_init(self, tc):
        """Start a variable-property run (after set_fields): table, 1/(Re Pr) and T_ini."""
        tb = tc.table
        self._tcols = [np.ascontiguousarray(tb[k], np.float64) for k in ("t", "h", "d", "m", "k", "cp", "b")]
        th = ChsThermo()
        th.ntable = len(self._tcols[0])
        th.t, th.h, th.d, th.m, th.k, th.cp, th.b = [_ptr(c) for c in self._tcols]
        th.rPrRen = 1.0 / (self.cfg.ren * tc.prandtl)
        th.t_ini = float(tc.t_ini)
        self._check(self.L.chs_thermo_init(self.h, ctypes.byref(th)), "chs_thermo_init")

    def Solve_energy_eq(self, isub):
        """Energy equation and property update of one RK3 substep (isub 1..3)."""
        self._check(self.L.chs_energy_substep(self.h, int(isub)), "chs_energy_substep")

    def substep(self, isub):
        """One substep of the time loop: energy (variable-property runs) then momentum."""
        if getattr(self, "_tcols", None) is not None and isub >= 1:
            self.Solve_energy_eq(isub)
        self.Solve_momentum_eq(isub)

    def autotune(self, nsteps=2):
        """Pick the fastest launch shapes for this handle; returns (block, lt_max, fused, ms per nsteps)."""
        b, l, fu, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        self._check(self.L.chs_autotune(self.h, int(nsteps), ctypes.byref(b), ctypes.byref(l), ctypes.byref(fu),
                                        ctypes.byref(ms)), "chs_autotune")
        return b.value, l.value, fu.value, ms.value

    def set_launch_shape(self, block=0, lt_max=0, fused=0):
        self._check(self.L.chs_set_launch_shape(self.h, int(block), int(lt_max), int(fused)), "chs_set_launch_shape")

    def set_lanes(self, lanes):
        """Streams a captured substep spreads its independent launches over (1..8)."""
        self._check(self.L.chs_set_lanes(self.h, int(lanes)), "chs_set_lanes")

    def set_fusion(self, on):
        """Fused CD2 substep kernels (True, the default) or the operator path (False)."""
        self._check(self.L.chs_set_fusion(self.h, 1 if on else 0), "chs_set_fusion")

    # ---- MLP surrogate of the property update
    def mlp_train(self, nsamples=1000000, batch=4096, epochs=20, lr=2e-3, seed=20250101):
        cfg = ChsMlpTrainCfg(int(nsamples), int(batch), int(epochs), float(lr), int(seed))
        rep = ChsMlpReport()
        self._check(self.L.chs_mlp_train(self.h, ctypes.byref(cfg), ctypes.byref(rep)), "chs_mlp_train")
        return dict(final_loss=rep.final_loss, train_ms=rep.train_ms, steps=rep.steps)

    def mlp_set_mode(self, mode, tol=-1.0):
        self._check(self.L.chs_mlp_set_mode(self.h, int(mode), float(tol)), "chs_mlp_set_mode")

    def mlp_fallbacks(self):
        c = ctypes.c_ulonglong()
        self._check(self.L.chs_mlp_fallbacks(self.h, ctypes.byref(c)), "chs_mlp_fallbacks")
        return int(c.value)

    def mlp_params(self, values=None):
        _F = ctypes.POINTER(ctypes.c_float)
        if values is None:
            out = np.zeros(MLP_NPARAM, np.float32)
            self._check(self.L.chs_mlp_params(self.h, out.ctypes.data_as(_F), MLP_NPARAM, 0), "chs_mlp_params")
            return out
        v = np.ascontiguousarray(values, np.float32)
        self._check(self.L.chs_mlp_params(self.h, v.ctypes.data_as(_F), MLP_NPARAM, 1), "chs_mlp_params")

    def mlp_grad(self, params, x, t):
        _F = ctypes.POINTER(ctypes.c_float)
        p = np.ascontiguousarray(params, np.float32)
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(MLP_NPARAM, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(self.L.chs_mlp_grad(self.h, p.ctypes.data_as(_F), len(x), x.ctypes.data_as(_F),
                                        t.ctypes.data_as(_F), g.ctypes.data_as(_F), loss.ctypes.data_as(_F)),
                    "chs_mlp_grad")
        return float(loss[0]), g

    def mlp_eval(self, rhoh, tol=-1.0):
        """(out[5][n] = T, rho, mu, kappa, h; number of table fallbacks)."""
        r = np.ascontiguousarray(rhoh, np.float64).ravel()
        out = np.zeros((5, r.size))
        c = ctypes.c_ulonglong()
        self._check(self.L.chs_mlp_eval(self.h, r.size, _ptr(r), float(tol), _ptr(out), ctypes.byref(c)),
                    "chs_mlp_eval")
        return out, int(c.value)

    def mlp_norm(self):
        o = np.zeros(10)
        self._check(self.L.chs_mlp_norm(self.h, _ptr(o)), "chs_mlp_norm")
        return dict(xa=o[0], xb=o[1], ya=o[2:6].copy(), yb=o[6:10].copy())

    def get_thermo(self):
        """dict of rhoh, h, T, k, d, m (ccc) and gx, gy, gz."""
        ids = dict(rhoh=CHS_RHOH, h=CHS_HENTH, T=CHS_TTEMP, k=CHS_KCOND, d=CHS_DDENS, m=CHS_MVISC, gx=CHS_GX,
                   gy=CHS_GY, gz=CHS_GZ)
        return {k: self.download(v) for k, v in ids.items()}

    def set_fields(self, qx, qy, qz, p):
        for f, a in ((CHS_QX, qx), (CHS_QY, qy), (CHS_QZ, qz), (CHS_PRES, p)):
            self.upload(f, a)

    def get_fields(self):
        return tuple(self.download(f) for f in (CHS_QX, CHS_QY, CHS_QZ, CHS_PRES, CHS_PCOR))

    # ---- reference-facing calls
    def Solve_momentum_eq(self, isub):
        """One RK3 substep (isub 1..3) or the initial Euler step (isub 0)."""
        self._check(self.L.chs_momentum_substep(self.h, int(isub)), "chs_momentum_substep")

    def step(self, nsteps=1):
        self._check(self.L.chs_step(self.h, int(nsteps)), "chs_step")

    def solve_fft_poisson(self, rhs):
        r = np.array(rhs, np.float64, copy=True, order="C")
        self._check(self.L.chs_poisson_solve(self.h, _ptr(r)), "chs_poisson_solve")
        return r

    def diagnostics(self):
        d = ChsDiag()
        self._check(self.L.chs_diagnostics(self.h, ctypes.byref(d)), "chs_diagnostics")
        return dict(max_div=d.max_div, bulk_ke=d.bulk_ke, bulk_u=d.bulk_u, last_bulk_rhs=d.last_bulk_rhs,
                    nan_flag=d.nan_flag, mcon=[d.mcon[0], d.mcon[1], d.mcon[2]])

    def op3d(self, d, fam, ibc, fi, fbc2d=None):
        fi = np.ascontiguousarray(fi, np.float64)
        nin = (ctypes.c_int * 3)(fi.shape[2], fi.shape[1], fi.shape[0])
        nout = [fi.shape[2], fi.shape[1], fi.shape[0]]
        nout[d] = self.cfg.np_[d] if fam in (1, 2, 4) else self.cfg.nc[d]
        fo = np.zeros((nout[2], nout[1], nout[0]))
        fb = None if fbc2d is None else np.ascontiguousarray(fbc2d, np.float64)
        self._check(self.L.chs_op3d(self.h, d, fam, int(ibc[0]), int(ibc[1]), _ptr(fb), _ptr(fi), nin, _ptr(fo)),
                    "chs_op3d")
        return fo

    def Solve_momentum_eq_host(self, isub, qx, qy, qz, p):
        """Drop-in substep on host arrays (updated in place)."""
        arrs = [np.ascontiguousarray(a, np.float64) for a in (qx, qy, qz, p)]
        for a, s in zip(arrs, self.shapes):
            assert a.shape == s
        self._check(self.L.chs_momentum_substep_host(self.h, int(isub), *[_ptr(a) for a in arrs]),
                    "chs_momentum_substep_host")
        return arrs

    def time_steps(self, nsteps):
        ms = ctypes.c_float()
        self._check(self.L.chs_time_steps(self.h, int(nsteps), ctypes.byref(ms)), "chs_time_steps")
        return float(ms.value)

    def pinned(self, shape):
        """numpy view of a page-locked host buffer (freed with the Solver)."""
        n = int(np.prod(shape))
        p = self.L.chs_host_alloc(n * 8)
        if not p:
            raise RuntimeError("chs_host_alloc failed")
        self.__dict__.setdefault("_pinned", []).append(p)
        buf = (ctypes.c_double * n).from_address(p)
        return np.ndarray(shape, np.float64, buffer=buf)

    def time_steps_host(self, nsteps, qx, qy, qz, p):
        ms = ctypes.c_float()
        self._check(self.L.chs_time_steps_host(self.h, int(nsteps), _ptr(qx), _ptr(qy), _ptr(qz), _ptr(p),
                                               ctypes.byref(ms)), "chs_time_steps_host")
        return float(ms.value)

    def time_steps_host_fields(self, nsteps, fields, per_substep=True):
        """fields: dict {chs_field id: pinned host array}; returns ms of nsteps steps with the arrays
        copied in and out every substep (per_substep) or every RK3 step."""
        ids = (ctypes.c_int * len(fields))(*[int(k) for k in fields])
        bufs = (_D * len(fields))(*[_ptr(a) for a in fields.values()])
        ms = ctypes.c_float()
        fn, name = ((self.L.chs_time_steps_host_fields, "chs_time_steps_host_fields") if per_substep else
                    (self.L.chs_time_rk3_host_fields, "chs_time_rk3_host_fields"))
        self._check(fn(self.h, int(nsteps), len(fields), ids, bufs, ctypes.byref(ms)), name)
        return float(ms.value)

    def profile_substep(self, isub=1, maxk=512):
        arr = (ChsKprof * maxk)()
        n = ctypes.c_int()
        self._check(self.L.chs_profile_substep(self.h, int(isub), arr, maxk, ctypes.byref(n)), "chs_profile_substep")
        return [dict(kind=arr[i].kind, dir=arr[i].dir, bytes=arr[i].bytes, ms=arr[i].ms) for i in range(n.value)]

    # ---- restart files and running statistics
    def write_restart(self, directory, idom, iteration):
        self._check(self.L.chs_write_restart(self.h, str(directory).encode(), int(idom), int(iteration)),
                    "chs_write_restart")

    def read_restart(self, directory, idom, iteration):
        self._check(self.L.chs_read_restart(self.h, str(directory).encode(), int(idom), int(iteration)),
                    "chs_read_restart")

    def stats_update(self, nstat):
        self._check(self.L.chs_stats_update(self.h, int(nstat)), "chs_stats_update")

    STATS = ("pr", "ux", "uy", "uz", "uu", "vv", "ww", "uv", "uw", "vw", "t", "tt")

    def stats_get(self, which):
        """Running mean `which` (index or name of STATS) as a (nz, ny, nx) array."""
        k = self.STATS.index(which) if isinstance(which, str) else int(which)
        out = np.zeros(self.shapes[3])
        self._check(self.L.chs_stats_get(self.h, k, _ptr(out), out.size), "chs_stats_get")
        return out

    def write_statistics(self, directory, idom, iteration):
        self._check(self.L.chs_write_statistics(self.h, str(directory).encode(), int(idom), int(iteration)),
                    "chs_write_statistics")

    def read_statistics(self, directory, idom, iteration):
        self._check(self.L.chs_read_statistics(self.h, str(directory).encode(), int(idom), int(iteration)),
                    "chs_read_statistics")

    def profile_substep_graph(self, isub=1, maxk=512):
        """Per-launch profile of one substep replayed as a CUDA graph (advances the state)."""
        arr = (ChsKprof * maxk)()
        n = ctypes.c_int()
        self._check(self.L.chs_profile_substep_graph(self.h, int(isub), arr, maxk, ctypes.byref(n)),
                    "chs_profile_substep_graph")
        return [dict(kind=arr[i].kind, dir=arr[i].dir, bytes=arr[i].bytes, ms=arr[i].ms) for i in range(n.value)]

    def profile_class(self, kind, isub=1, reps=20):
        """ms of one graph replay of substep isub holding only kernel class `kind` (-1: all)."""
        ms = ctypes.c_float()
        self._check(self.L.chs_profile_class(self.h, int(isub), int(kind), int(reps), ctypes.byref(ms)),
                    "chs_profile_class")
        return ms.value

    def sync(self):
        self._check(self.L.chs_sync(self.h), "chs_sync")

    def kernel_launches(self):
        return int(self.L.chs_kernel_launches(self.h))


class Ensemble:
    """Independent Solvers advanced together: one CUDA-graph launch per RK3 substep for all members."""

    def __init__(self, solvers):
        self.L = load()
        self.members = list(solvers)
        arr = (ctypes.c_void_p * len(self.members))(*[m.h.value for m in self.members])
        e = ctypes.c_void_p()
        rc = self.L.chs_ensemble_create(arr, len(self.members), ctypes.byref(e))
        if rc != 0 or not e.value:
            raise RuntimeError(f"chs_ensemble_create failed with status {rc}")
        self.e = e

    def step(self, nsteps=1):
        rc = self.L.chs_ensemble_step(self.e, int(nsteps))
        if rc != 0:
            raise RuntimeError(f"chs_ensemble_step failed with status {rc}")

    def time_steps(self, nsteps):
        ms = ctypes.c_float()
        rc = self.L.chs_ensemble_time_steps(self.e, int(nsteps), ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"chs_ensemble_time_steps failed with status {rc}")
        return float(ms.value)

    def kernel_launches(self):
        return int(self.L.chs_ensemble_kernel_launches(self.e))

    def close(self):
        if getattr(self, "e", None) and self.e.value:
            self.L.chs_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
