"""ctypes binding of the CPU FP64 oracle (test infrastructure only).

The oracle restates CHAPSim2's flow path in C++ (see the .cpp headers for the
reference file:line each routine follows).  Only tests/, the smoke check and
bench.py's CPU baseline may import this module; the product path never does.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liborc.so")
_lib = None

D = ctypes.POINTER(ctypes.c_double)
I = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile liborc.so from the oracle sources (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_tdma.argtypes = [ctypes.c_int, D, D, D, D, ctypes.c_int]
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [I, D, I, D]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_geometry.argtypes = [ctypes.c_void_p, D, D, D, D, I, D]
        L.orc_bcs.argtypes = [ctypes.c_void_p, I, I]
        L.orc_op3d.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               D, D, I, D]
        L.orc_op1d.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               D, D, D]
        L.orc_set_fields.argtypes = [ctypes.c_void_p, D, D, D, D]
        L.orc_get_fields.argtypes = [ctypes.c_void_p, D, D, D, D, D]
        L.orc_get_rhs0.argtypes = [ctypes.c_void_p, D, D, D]
        L.orc_momentum_rhs.argtypes = [ctypes.c_void_p, D, D, D, D, D, D]
        L.orc_momentum_substep.argtypes = [ctypes.c_void_p, ctypes.c_int, D]
        L.orc_poisson.argtypes = [ctypes.c_void_p, D]
        L.orc_divergence.argtypes = [ctypes.c_void_p, D]
        L.orc_bulk_ke.restype = ctypes.c_double
        L.orc_bulk_ke.argtypes = [ctypes.c_void_p]
        L.orc_vol_average_pcc.restype = ctypes.c_double
        L.orc_vol_average_pcc.argtypes = [ctypes.c_void_p, D]
        L.orc_thermo_init.argtypes = [ctypes.c_void_p, ctypes.c_int, D, D, D, D, D, D, D, ctypes.c_double, D,
                                      ctypes.c_double]
        L.orc_substep.argtypes = [ctypes.c_void_p, ctypes.c_int, D]
        L.orc_get_thermo.argtypes = [ctypes.c_void_p, D, D, D, D, D, D, D, D, D]
        L.orc_ftp_from_dh.argtypes = [ctypes.c_void_p, ctypes.c_int, D, D]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(D) if a is not None else None


def tdma(a, b, c, r, cyclic):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    c = np.ascontiguousarray(c, np.float64)
    x = np.array(r, np.float64)
    lib().orc_tdma(int(cyclic), _p(a), _p(b), _p(c), _p(x), len(x))
    return x


class Oracle:
    """One CHAPSim2 domain + flow state held by the oracle.

    Arrays are Fortran-ordered (x fastest); numpy views use shape (n3, n2, n1)
    in C order, i.e. ``a[k, j, i]``.
    """

    def __init__(self, cfg):
        self.cfg = cfg
        ints = np.zeros(16, np.int32)
        ints[:8] = [cfg.nc[0], cfg.nc[1], cfg.nc[2], cfg.iacc, cfg.istret, cfg.idriven, cfg.ifft,
                    1 if cfg.periodic_y else 0]
        dbl = np.zeros(16, np.float64)
        dbl[:7] = [cfg.lxx, cfg.lyt, cfg.lyb, cfg.lzz, cfg.rstret, cfg.dt, cfg.ren]
        nom = np.ascontiguousarray(cfg.nominal_bc, np.int32)
        fbc = np.ascontiguousarray(cfg.fbcy_const, np.float64)
        self.h = lib().orc_create(ints.ctypes.data_as(I), _p(dbl), nom.ctypes.data_as(I), _p(fbc))
        if not self.h:
            raise RuntimeError("orc_create failed")
        nc = cfg.nc
        self.np = np.zeros(3, np.int32)
        hh = np.zeros(3)
        self.yp = np.zeros(nc[1] + 1)
        self.yc = np.zeros(nc[1])
        self.mppt = np.zeros(nc[1] + 1)
        self.mpcc = np.zeros(nc[1])
        lib().orc_geometry(self.h, _p(self.yp), _p(self.yc), _p(self.mppt), _p(self.mpcc),
                           self.np.ctypes.data_as(I), _p(hh))
        self.hgrid = hh
        n = self.np
        self.shape_pcc = (nc[2], nc[1], n[0])
        self.shape_cpc = (nc[2], n[1], nc[0])
        self.shape_ccp = (n[2], nc[1], nc[0])
        self.shape_ccc = (nc[2], nc[1], nc[0])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def bcs(self):
        ibc = np.zeros(30, np.int32)
        mbc = np.zeros(36, np.int32)
        lib().orc_bcs(self.h, ibc.ctypes.data_as(I), mbc.ctypes.data_as(I))
        return ibc.reshape(3, 5, 2), mbc.reshape(18, 2)

    def op3d(self, d, fam, ibc, fi, fbc2d=None):
        fi = np.ascontiguousarray(fi, np.float64)
        nin = np.array([fi.shape[2], fi.shape[1], fi.shape[0]], np.int32)
        nout = nin.copy()
        to_p = fam in (1, 2, 4)
        nout[d] = self.np[d] if to_p else self.cfg.nc[d]
        fo = np.zeros((nout[2], nout[1], nout[0]))
        fb = None if fbc2d is None else np.ascontiguousarray(fbc2d, np.float64)
        rc = lib().orc_op3d(self.h, d, fam, int(ibc[0]), int(ibc[1]), _p(fb), _p(fi), nin.ctypes.data_as(I),
                            _p(fo))
        if rc != 0:
            raise RuntimeError("orc_op3d failed")
        return fo

    def op1d(self, d, fam, ibc, fi, nout, fbc=None):
        fi = np.ascontiguousarray(fi, np.float64)
        fo = np.zeros(nout)
        fb = None if fbc is None else np.ascontiguousarray(fbc, np.float64)
        lib().orc_op1d(self.h, d, fam, int(ibc[0]), int(ibc[1]), _p(fb), _p(fi), _p(fo))
        return fo

    def set_fields(self, qx, qy, qz, p):
        a = [np.ascontiguousarray(x, np.float64) for x in (qx, qy, qz, p)]
        lib().orc_set_fields(self.h, *[_p(x) for x in a])

    def get_fields(self):
        qx = np.zeros(self.shape_pcc)
        qy = np.zeros(self.shape_cpc)
        qz = np.zeros(self.shape_ccp)
        p = np.zeros(self.shape_ccc)
        pc = np.zeros(self.shape_ccc)
        lib().orc_get_fields(self.h, _p(qx), _p(qy), _p(qz), _p(p), _p(pc))
        return qx, qy, qz, p, pc

    def get_rhs0(self):
        mx = np.zeros(self.shape_pcc)
        my = np.zeros(self.shape_cpc)
        mz = np.zeros(self.shape_ccp)
        lib().orc_get_rhs0(self.h, _p(mx), _p(my), _p(mz))
        return mx, my, mz

    def momentum_rhs(self):
        out = [np.zeros(s) for s in (self.shape_pcc, self.shape_cpc, self.shape_ccp,
                                     self.shape_pcc, self.shape_cpc, self.shape_ccp)]
        if lib().orc_momentum_rhs(self.h, *[_p(x) for x in out]) != 0:
            raise RuntimeError("orc_momentum_rhs failed")
        return out

    def thermo_init(self, tc):
        """Start a variable-property run (call after set_fields): table, 1/(Re Pr), wall fluxes, T_ini."""
        tb = tc.table
        cols = [np.ascontiguousarray(tb[k], np.float64) for k in ("t", "h", "d", "m", "k", "cp", "b")]
        qw = np.ascontiguousarray(tc.qw, np.float64)
        rpr = 1.0 / (self.cfg.ren * tc.prandtl)
        if lib().orc_thermo_init(self.h, len(cols[0]), *[_p(c) for c in cols], rpr, _p(qw), float(tc.t_ini)) != 0:
            raise RuntimeError("orc_thermo_init failed")
        self._keep_table = cols

    def get_thermo(self):
        """dict of rhoh, h, T, k, d, m (ccc) and gx, gy, gz."""
        out = {k: np.zeros(self.shape_ccc) for k in ("rhoh", "h", "T", "k", "d", "m")}
        out["gx"] = np.zeros(self.shape_pcc)
        out["gy"] = np.zeros(self.shape_cpc)
        out["gz"] = np.zeros(self.shape_ccp)
        lib().orc_get_thermo(self.h, *[_p(out[k]) for k in ("rhoh", "h", "T", "k", "d", "m", "gx", "gy", "gz")])
        return out

    def ftp_from_dh(self, rhoh):
        """Property lookup from rho*h: (h, T, rho, mu, kappa, cp) arrays."""
        r = np.ascontiguousarray(rhoh, np.float64).ravel()
        out = np.zeros((6, r.size))
        lib().orc_ftp_from_dh(self.h, r.size, _p(r), _p(out))
        return out

    def substep(self, isub):
        """One substep of the time loop: energy (variable-property runs) then momentum."""
        bulk = np.zeros(1)
        if lib().orc_substep(self.h, int(isub), _p(bulk)) != 0:
            raise RuntimeError("orc_substep failed")
        return float(bulk[0])

    def step(self):
        for isub in (1, 2, 3):
            self.substep(isub)

    def poisson(self, rhs):
        r = np.array(rhs, np.float64, copy=True)
        lib().orc_poisson(self.h, _p(r))
        return r

    def divergence(self):
        d = np.zeros(self.shape_ccc)
        lib().orc_divergence(self.h, _p(d))
        return d

    def mass_conservation(self):
        """Check_element_mass_conservation (src/eq_continuity.f90:337-397): max |div + drho/dt| over
        the x slabs 1:4, 5:n-4 and n-5:n (1-based, :379-389), i.e. fl%mcon(1:3).  drho/dt is zero
        there: the property update has already set rho_m1 = rho (src/eq_energy.f90:48-49)."""
        import numpy as np
        d = np.abs(self.divergence())
        n = d.shape[2]
        return [float(d[:, :, 0:4].max()), float(d[:, :, 4:n - 4].max()), float(d[:, :, n - 6:n].max())]

    def bulk_ke(self):
        return lib().orc_bulk_ke(self.h)

    def vol_average_pcc(self, a):
        a = np.ascontiguousarray(a, np.float64)
        return lib().orc_vol_average_pcc(self.h, _p(a))
