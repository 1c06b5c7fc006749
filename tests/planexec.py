"""numpy emulation of the GPU line-operator kernel (test support).

Executes a plan returned by chapsim2_b200.solver.plan_inspect on every line of
a 3D array, step for step as line_op_kernel does (special rows, bulk stencil,
Thomas forward/backward, cyclic closure, y metric, Neumann overrides), so the
host-side plan builder can be checked against the oracle without a GPU.
"""
import numpy as np


def run_plan(p, fi3d, d, fbc_lines=None):
    """fi3d: numpy (k, j, i) array; d: direction; fbc_lines: (4, nlines) or None."""
    a = np.moveaxis(fi3d, 2 - d, -1)          # lines along last axis
    shp = a.shape[:-1]
    lines = a.reshape(-1, a.shape[-1])
    nl = lines.shape[0]
    nin, nout = p["nin"], p["nout"]
    assert lines.shape[1] == nin
    if d == 1:  # kernel line order for y is i + n1*k; here lines are ordered (k, i) -> same
        pass
    out = np.zeros((nl, nout))
    off = p["off"]
    for L in range(nl):
        f = lines[L]
        sv = []
        for r in p["rows"]:
            v = float(np.dot(r["w"], f[r["idx"]])) if len(r["idx"]) else 0.0
            for u in range(4):
                if r["wb"][u] != 0.0:
                    v += r["wb"][u] * fbc_lines[u, L]
            sv.append(v * p["dd"])
        rows = {r["row"]: sv[k] for k, r in enumerate(p["rows"])}
        y = np.zeros(nout)
        nsw = nout - 1 if p["tdma"] == 2 else nout
        prev = 0.0
        for i in range(nout):
            if p.get("wrap", 0):
                g = lambda o: f[(i + o) % nin]
                rr = (p["r1"] * (g(off[0]) + p["sgn"] * g(off[1])) + p["r2"] * (g(off[2]) + p["sgn"] * g(off[3]))) * p["dd"]
            elif p["b_lo"] <= i <= p["b_hi"]:
                g = lambda o: f[i + o]
                rr = (p["r1"] * (g(off[0]) + p["sgn"] * g(off[1])) + p["r2"] * (g(off[2]) + p["sgn"] * g(off[3]))) * p["dd"]
            else:
                rr = rows[i]
            yy = rr
            if p["tdma"] and i < nsw:
                yy = rr / p["b1"] if i == 0 else (rr - p["a"][i] * prev) * p["d"][i]
                prev = yy
            y[i] = yy
        if p["tdma"]:
            for i in range(nsw - 2, -1, -1):
                y[i] = y[i] - p["c"][i] * y[i + 1]
            if p["tdma"] == 2:
                y[nout - 1] = (y[nout - 1] - p["cn"] * y[0] - p["an"] * y[nout - 2]) * p["inv_den"]
                y[:nout - 1] += p["x1"][:nout - 1] * y[nout - 1]
        if np.any(p["map"] != 0):
            y = y * p["map"]
        if p["neu1"]:
            y[0] = fbc_lines[0, L]
        if p["neu2"]:
            y[nout - 1] = fbc_lines[1, L]
        out[L] = y
    res = out.reshape(*shp, nout)
    return np.ascontiguousarray(np.moveaxis(res, -1, 2 - d))


def fbc_ref_to_lines(fbc_ref, d, shape_in):
    """Reference-layout planes -> (4, nlines) in the kernel's line order.

    shape_in is the numpy (k, j, i) shape of the input array; the reference
    layouts are fbcx(4,n2,n3) -> numpy (n3, n2, 4), fbcy(n1,4,n3) -> (n3, 4, n1),
    fbcz(n1,n2,4) -> (4, n2, n1).
    """
    n3, n2, n1 = shape_in
    if d == 0:
        return np.ascontiguousarray(fbc_ref.reshape(n3, n2, 4).reshape(-1, 4).T)
    if d == 1:
        return np.ascontiguousarray(fbc_ref.reshape(n3, 4, n1).transpose(1, 0, 2).reshape(4, -1))
    return np.ascontiguousarray(fbc_ref.reshape(4, n2, n1).reshape(4, -1))
