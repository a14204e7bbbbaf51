"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes front end of the CPU restatement in oracle.cpp (see its header for what
it restates and why its parity is pinned by analytic tests rather than by
reference fixtures).  Imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_build", "liboracle.so")

sys.path.insert(0, os.path.join(os.path.dirname(_HERE), "mg-glam-durham_b200"))
from mgglam_b200 import MggConfig, MggReport  # noqa: E402  (shared plain-C struct layouts)

_lib = None


def build():
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.POINTER
        f = P(ctypes.c_float)
        d = P(ctypes.c_double)
        i64 = ctypes.c_int64
        ci = ctypes.c_int
        cf = ctypes.c_float
        cfg = P(MggConfig)
        L.orc_rfft1f.argtypes = [d, ci]
        L.orc_rfft1b.argtypes = [d, ci]
        L.orc_density_f.argtypes = [f, f, f, i64, ci, f, ci]
        L.orc_density_d.argtypes = [f, f, f, i64, ci, d, ci]
        L.orc_potential_f.argtypes = [f, ci, cf, cf, cf, ci]
        L.orc_potential_d.argtypes = [d, ci, cf, cf, cf, ci]
        L.orc_potential_mg_f.argtypes = [f, f, cfg, cf, ci]
        L.orc_potential_mg_d.argtypes = [d, d, cfg, cf, ci]
        L.orc_move_f.argtypes = [f, f, f, f, f, f, f, f, i64, cfg, cf, cf, cf, d, ci, ci]
        L.orc_move_f.restype = ctypes.c_double
        L.orc_move_d.argtypes = [d, d, f, f, f, f, f, f, i64, cfg, cf, cf, cf, d, ci, ci]
        L.orc_move_d.restype = ctypes.c_double
        L.orc_scalar_field_f.argtypes = [f, f, cfg, cf, ci, P(MggReport), ci, d, ci]
        L.orc_scalar_field_d.argtypes = [d, d, cfg, cf, ci, P(MggReport), ci, d, ci]
        L.orc_power_f.argtypes = [f, ci, cf, ci, d, d, d, d, d, d, ci]
        L.orc_power_pol_f.argtypes = [f, ci, cf, ci, d, d, d, ci, ci]
        L.orc_density_rsd_f.argtypes = [f, f, f, f, f, f, i64, ci, ci, ci, cf, cf, cf, f]
        L.orc_density_pdf_f.argtypes = [f, ci, P(ctypes.c_int64), d, d, d]
        L.orc_power_rsd_f.argtypes = [f, f, f, f, f, f, i64, ci, cf, cf, cf, cf, ci, d, d, d, d, d, ci]
        L.orc_mg_op_f.argtypes = [f, f, cfg, cf, ci, ci]
        L.orc_mg_op_f.restype = ctypes.c_double
        L.orc_kmf_operator_f.argtypes = [f, f, cfg, cf, d, d, ci]
        L.orc_dgp_root_density_f.argtypes = [f, cfg, cf, d]
        L.orc_dgp_root_density_f.restype = i64
        L.orc_max_threads.restype = ci
        L.orc_set_sweep_order.argtypes = [ci]
        _lib = L
    return _lib


def threads() -> int:
    return int(lib().orc_max_threads())


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _fp(a):
    return _p(a, ctypes.c_float)


def _dp(a):
    return _p(a, ctypes.c_double)


def rfft1f(r):
    r = np.array(r, dtype=np.float64)
    lib().orc_rfft1f(_dp(r), r.size)
    return r


def rfft1b(r):
    r = np.array(r, dtype=np.float64)
    lib().orc_rfft1b(_dp(r), r.size)
    return r


def density(x, y, z, ngrid, fp64=False, nthreads=1):
    """DENSIT; nthreads>1 uses the reference's unordered atomic scatter."""
    x, y, z = (np.ascontiguousarray(a, dtype=np.float32) for a in (x, y, z))
    if fp64:
        fi = np.empty(ngrid ** 3, dtype=np.float64)
        lib().orc_density_d(_fp(x), _fp(y), _fp(z), x.size, ngrid, _dp(fi), nthreads)
    else:
        fi = np.empty(ngrid ** 3, dtype=np.float32)
        lib().orc_density_f(_fp(x), _fp(y), _fp(z), x.size, ngrid, _fp(fi), nthreads)
    return fi


def potential(fi, ngrid, aexpn, om, omb, nthreads=None):
    nt = nthreads or threads()
    if fi.dtype == np.float64:
        out = np.array(fi, dtype=np.float64)
        lib().orc_potential_d(_dp(out), ngrid, aexpn, om, omb, nt)
    else:
        out = np.array(fi, dtype=np.float32)
        lib().orc_potential_f(_fp(out), ngrid, aexpn, om, omb, nt)
    return out


def potential_mg(fi, fi2, cfg, aexpn, nthreads=None):
    nt = nthreads or threads()
    if fi.dtype == np.float64:
        out = np.array(fi, dtype=np.float64)
        lib().orc_potential_mg_d(_dp(out), _dp(np.ascontiguousarray(fi2, dtype=np.float64)), ctypes.byref(cfg),
                                 aexpn, nt)
    else:
        out = np.array(fi, dtype=np.float32)
        lib().orc_potential_mg_f(_fp(out), _fp(np.ascontiguousarray(fi2, dtype=np.float32)), ctypes.byref(cfg),
                                 aexpn, nt)
    return out


def move(fi, fi2, parts, cfg, aexpn, astep, factv, bg=None, nthreads=None):
    """MOVE; parts = [x, y, z, vx, vy, vz] float32 arrays (copied); returns (parts, enkin)."""
    nt = nthreads or threads()
    p = [np.array(a, dtype=np.float32) for a in parts]
    bgp = None if bg is None else _dp(np.ascontiguousarray(bg, dtype=np.float64))
    rows = 0 if bg is None else bg.shape[0]
    if fi.dtype == np.float64:
        f2 = np.ascontiguousarray(fi2 if fi2 is not None else fi, dtype=np.float64)
        e = lib().orc_move_d(_dp(fi), _dp(f2), *[_fp(a) for a in p], p[0].size, ctypes.byref(cfg), aexpn, astep,
                             factv, bgp, rows, nt)
    else:
        f2 = np.ascontiguousarray(fi2 if fi2 is not None else fi, dtype=np.float32)
        e = lib().orc_move_f(_fp(np.ascontiguousarray(fi, dtype=np.float32)), _fp(f2), *[_fp(a) for a in p],
                             p[0].size, ctypes.byref(cfg), aexpn, astep, factv, bgp, rows, nt)
    return p, e


class _sweep_order:
    """Context manager selecting the nDGP / k-mouflage sweep order: 'serial' (the
    reference's single-thread in-place order) or 'snapshot' (each colour sweep
    reads the field as it was before the sweep)."""

    def __init__(self, order):
        if order not in ("serial", "snapshot"):
            raise ValueError(order)
        self.flag = int(order == "snapshot")

    def __enter__(self):
        lib().orc_set_sweep_order(self.flag)

    def __exit__(self, *exc):
        lib().orc_set_sweep_order(0)


def scalar_field(fi, fi2, cfg, aexpn, i_step, nthreads=None, bg=None, order="serial"):
    """scalar_field(i_step); returns (fi2_new, report).  fi is not modified.
    bg: BackgroundEvolution table (rows x 6) for k-mouflage / csf.
    order: 'serial' or 'snapshot' sweep order of the nDGP / k-mouflage relaxations."""
    with _sweep_order(order):
        return _scalar_field(fi, fi2, cfg, aexpn, i_step, nthreads, bg)


def _scalar_field(fi, fi2, cfg, aexpn, i_step, nthreads=None, bg=None):
    nt = nthreads or threads()
    rep = MggReport()
    bgp, rows = (None, 0) if bg is None else (_dp(np.ascontiguousarray(bg, dtype=np.float64)), bg.shape[0])
    if bg is not None:
        bg = np.ascontiguousarray(bg, dtype=np.float64)
        bgp = _dp(bg)
    if fi.dtype == np.float64:
        f = np.array(fi, dtype=np.float64)
        u = np.array(fi2, dtype=np.float64)
        lib().orc_scalar_field_d(_dp(f), _dp(u), ctypes.byref(cfg), aexpn, i_step, ctypes.byref(rep), nt, bgp, rows)
    else:
        f = np.array(fi, dtype=np.float32)
        u = np.array(fi2, dtype=np.float32)
        lib().orc_scalar_field_f(_fp(f), _fp(u), ctypes.byref(cfg), aexpn, i_step, ctypes.byref(rep), nt, bgp, rows)
    return u, rep


def mg_op(fi, fi2, cfg, aexpn, op, nthreads=None, order="serial"):
    """Single MG building block on level 0: 0 red sweep, 1 black sweep, 2 residual RMS, 3 one V-cycle."""
    nt = nthreads or threads()
    f = np.array(fi, dtype=np.float32)
    u = np.array(fi2, dtype=np.float32)
    with _sweep_order(order):
        r = lib().orc_mg_op_f(_fp(f), _fp(u), ctypes.byref(cfg), aexpn, op, nt)
    return u, r


def kmf_operator(fi, fi2, cfg, aexpn, bg):
    """The level-0 k-mouflage operator at every cell (float64), for density fi and field fi2."""
    f = np.array(fi, dtype=np.float32)
    u = np.array(fi2, dtype=np.float32)
    out = np.empty(f.size, dtype=np.float64)
    b = np.ascontiguousarray(bg, dtype=np.float64)
    lib().orc_kmf_operator_f(_fp(f), _fp(u), ctypes.byref(cfg), aexpn, _dp(out), _dp(b), b.shape[0])
    return out


def dgp_root_density(fi2, cfg, aexpn):
    """(density contrast for which the level-0 nDGP operator vanishes at every cell of fi2,
    number of cells without a root)."""
    u = np.array(fi2, dtype=np.float32)
    out = np.empty(u.size, dtype=np.float64)
    bad = lib().orc_dgp_root_density_f(_fp(u), ctypes.byref(cfg), aexpn, _dp(out))
    return out, int(bad)


def power(fi, ngrid, box, nbins=None, nthreads=None):
    nt = nthreads or threads()
    nb = nbins or ngrid // 2
    f = np.array(fi, dtype=np.float32)
    outs = [np.zeros(nb) for _ in range(6)]
    lib().orc_power_f(_fp(f), ngrid, box, nb, *[_dp(a) for a in outs], nt)
    return dict(k=outs[0], nmodes=outs[1], pk=outs[2], klog=outs[3], nmodeslog=outs[4], pklog=outs[5])


def power_pol(fi, ngrid, box, pol, nbins=None, nthreads=None):
    """POWERfft5(iPol, 0): pol = 0 monopole, 1 quadrupole about the z (third) axis."""
    nt = nthreads or threads()
    nb = nbins or ngrid // 2
    f = np.array(fi, dtype=np.float32)
    outs = [np.zeros(nb) for _ in range(3)]
    lib().orc_power_pol_f(_fp(f), ngrid, box, nb, *[_dp(a) for a in outs], pol, nt)
    return dict(k=outs[0], nmodes=outs[1], pk=outs[2])


def density_rsd(parts, ngrid_old, ngrid, iswitch, aexpn, om, oml):
    """DENSITrsd(iSwitch, NGRID_old) with sigv = 0 on the ngrid mesh."""
    p = [np.ascontiguousarray(a, dtype=np.float32) for a in parts]
    fi = np.empty(ngrid ** 3, dtype=np.float32)
    lib().orc_density_rsd_f(*[_fp(a) for a in p], p[0].size, ngrid_old, ngrid, iswitch, aexpn, om, oml, _fp(fi))
    return fi


def density_pdf(fi, ngrid):
    """DensDistr: (ncells[4003], den_sum[4003], rms, mean) for bins i = -2001..2001."""
    f = np.ascontiguousarray(fi, dtype=np.float32)
    nc = np.zeros(4003, dtype=np.int64)
    den = np.zeros(4003)
    rms = ctypes.c_double()
    mean = ctypes.c_double()
    lib().orc_density_pdf_f(_fp(f), ngrid, nc.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _dp(den),
                            ctypes.byref(rms), ctypes.byref(mean))
    return nc, den, rms.value, mean.value


def power_rsd(parts, ngrid, box, aexpn, om, oml, nbins=None, nthreads=None):
    """GetPower(1) with sigv = 0: dict of k, nmodes, preal, p0, p2 on the ngrid/2 mesh."""
    nt = nthreads or threads()
    nb = nbins or ngrid // 4
    p = [np.ascontiguousarray(a, dtype=np.float32) for a in parts]
    outs = [np.zeros(nb) for _ in range(5)]
    lib().orc_power_rsd_f(*[_fp(a) for a in p], p[0].size, ngrid, box, aexpn, om, oml, nb,
                          *[_dp(a) for a in outs], nt)
    return dict(k=outs[0], nmodes=outs[1], preal=outs[2], p0=outs[3], p2=outs[4])
