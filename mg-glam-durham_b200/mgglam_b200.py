"""Host-side mirror of MG-GLAM's particle-mesh step over the sm_100a C ABI.

The reference drives one box from ``Program PMP`` (PMP2main.f90:17-89) through
parameterless subroutines that share module globals (Module Tools,
PMP2mod_tools.f90:8-111).  :class:`Box` holds the same state on one GPU and
exposes one method per subroutine with the reference's name, argument meaning
and order of use::

    box.density()           DENSIT            PMP2mod_density.f90:17
    box.scalar_field(i)     scalar_field(i)   PMP2extradof.f90:12
    box.potential()         POTENTfft5        PMP2main.f90:705
    box.potential_mg()      POTENT_FOR_MG     PMP2main.f90:869
    box.move(factv)         MOVE(FactV)       PMP2main.f90:304
    box.power()             GetPower(0)       PMP2mod_power.f90:20

:func:`step_table` restates the time-step table of ``Initialize``
(PMP2main.f90:154-184) and :meth:`Box.pm_step` the body of the main loop
(PMP2main.f90:36-81).  Every call goes to ``libmgglam_b200.so``; there is no CPU
path, and a missing library or device raises :class:`MGGError`.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmgglam_b200.so")

# status codes (include/mgglam.h)
MGG_OK = 0
ERR_NAMES = {1: "ARG", 2: "CUDA", 3: "NOMEM", 4: "STATE", 5: "UNSUPPORTED", 6: "NUMERIC", 7: "NO_DEVICE"}
MODEL_FR, MODEL_DGP, MODEL_SYMMETRON, MODEL_KMOUFLAGE, MODEL_CSF = 1, 2, 3, 4, 5
PREC_PLAIN, PREC_MIXED = 0, 1
PDF_BINS = 4003   # MGG_PDF_BINS: DensDistr bins i = -2001..2001
GRID_FI, GRID_FI2 = 0, 1
T_TOTAL, T_FORCE, T_MOVE, T_DENSITY, T_POWER, T_MG, T_NBUCKETS = 0, 1, 2, 3, 4, 8, 11

EXPORTED_SYMBOLS = (
    "mgg_create", "mgg_destroy", "mgg_last_error", "mgg_set_time", "mgg_upload_particles",
    "mgg_download_particles", "mgg_density", "mgg_scalar_field", "mgg_potential", "mgg_potential_mg",
    "mgg_move", "mgg_power", "mgg_upload_grid", "mgg_download_grid", "mgg_set_background",
    "mgg_synchronize", "mgg_timing", "mgg_profile", "mgg_profile_count", "mgg_profile_read",
    "mgg_profile_reset", "mgg_timer_start", "mgg_timer_stop", "mgg_make_ics", "mgg_version",
    "mgg_background_table", "mgg_density_noalloc", "mgg_step", "mgg_step_host", "mgg_step_batch", "mgg_get_config",
    "mgg_reconfigure", "mgg_box_bytes", "mgg_server_create", "mgg_server_submit", "mgg_server_wait",
    "mgg_server_destroy", "mgg_server_error", "mgg_pm_write", "mgg_pm_read_header", "mgg_pm_read",
    "mgg_pm_last_error", "mgg_power_rsd", "mgg_density_pdf", "mgg_cic_keys", "mgg_step_host_pipelined",
    "mgg_run_steps",
)


class MGGError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mgg error {code} ({ERR_NAMES.get(code, '?')}): {msg}")
        self.code = code


class MggConfig(ctypes.Structure):
    _fields_ = [
        ("ngrid", ctypes.c_int32), ("nrow", ctypes.c_int32), ("box", ctypes.c_float),
        ("om", ctypes.c_float), ("oml", ctypes.c_float), ("omb", ctypes.c_float),
        ("mg_flag", ctypes.c_int32), ("mg_model", ctypes.c_int32),
        ("vcycle", ctypes.c_int32), ("fcycle", ctypes.c_int32), ("wcycle", ctypes.c_int32),
        ("iter_count_max", ctypes.c_int32), ("res_conv", ctypes.c_double),
        ("fr_n", ctypes.c_int32), ("fr0", ctypes.c_double),
        ("n_branch", ctypes.c_int32), ("s_branch", ctypes.c_int32), ("h0rc", ctypes.c_double),
        ("sym_astar", ctypes.c_double), ("sym_xi", ctypes.c_double), ("sym_beta", ctypes.c_double),
        ("kmf_power_law", ctypes.c_int32), ("kmf_born_infeld", ctypes.c_int32), ("kmf_n", ctypes.c_int32),
        ("kmf_k0", ctypes.c_double), ("kmf_beta", ctypes.c_double), ("kmf_lambda", ctypes.c_double),
        ("csf_coupling", ctypes.c_int32), ("csf_potential", ctypes.c_int32),
        ("csf_alpha", ctypes.c_double), ("csf_beta", ctypes.c_double), ("csf_lambda", ctypes.c_double),
        ("precision", ctypes.c_int32), ("device", ctypes.c_int32),
    ]


class MggReport(ctypes.Structure):
    _fields_ = [("cycles", ctypes.c_int32), ("exit_reason", ctypes.c_int32),
                ("residual", ctypes.c_double * 64)]


class MggIcParams(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("sigma8", ctypes.c_double), ("hubble", ctypes.c_double),
                ("ns", ctypes.c_double), ("aexpn", ctypes.c_float), ("astep", ctypes.c_float)]


class MggStepState(ctypes.Structure):
    """AEXPN, ASTEP, StepFactor, ISTEP of Module Tools plus the last step's outputs."""
    _fields_ = [("aexpn", ctypes.c_float), ("astep", ctypes.c_float), ("step_factor", ctypes.c_float),
                ("istep", ctypes.c_int32), ("ekin", ctypes.c_double), ("report", MggReport)]


class MggRequest(ctypes.Structure):
    _fields_ = [("cfg", MggConfig), ("ic", MggIcParams), ("nsteps", ctypes.c_int32)]


class MggPmHeader(ctypes.Structure):
    """Header record of PMcrd.DAT (PMP2mod_tools.f90:258-262, 431-435)."""
    _fields_ = [("header", ctypes.c_char * 45), ("aexpn", ctypes.c_float), ("aexp0", ctypes.c_float),
                ("amplt", ctypes.c_float), ("astep", ctypes.c_float), ("istep", ctypes.c_int32),
                ("partw", ctypes.c_float), ("tintg", ctypes.c_float), ("ekin", ctypes.c_float),
                ("ekin1", ctypes.c_float), ("ekin2", ctypes.c_float), ("au0", ctypes.c_float),
                ("aeu0", ctypes.c_float), ("nrow", ctypes.c_int32), ("ngrid", ctypes.c_int32),
                ("nrealization", ctypes.c_int32), ("nseed", ctypes.c_int32), ("om", ctypes.c_float),
                ("oml", ctypes.c_float), ("hubble", ctypes.c_float), ("nparticles", ctypes.c_int64),
                ("extras", ctypes.c_float * 100)]


class MggResultInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("nbins", ctypes.c_int32), ("aexpn", ctypes.c_float),
                ("steps", ctypes.c_int32), ("cycles", ctypes.c_int64), ("ekin", ctypes.c_double),
                ("t_submit_ms", ctypes.c_double), ("t_admit_ms", ctypes.c_double), ("t_done_ms", ctypes.c_double)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load the sm_100a library; raise MGGError when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise MGGError(7, f"{path} is missing: build it with `make -C mg-glam-durham_b200`")
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    f32p = P(ctypes.c_float)
    f64p = P(ctypes.c_double)
    vp = ctypes.c_void_p
    sig = {
        "mgg_create": (ctypes.c_int, [P(MggConfig), P(vp)]),
        "mgg_destroy": (ctypes.c_int, [vp]),
        "mgg_last_error": (ctypes.c_char_p, [vp]),
        "mgg_set_time": (ctypes.c_int, [vp, ctypes.c_float, ctypes.c_float]),
        "mgg_upload_particles": (ctypes.c_int, [vp] + [f32p] * 6 + [ctypes.c_int64]),
        "mgg_download_particles": (ctypes.c_int, [vp] + [f32p] * 6 + [ctypes.c_int64]),
        "mgg_density": (ctypes.c_int, [vp]),
        "mgg_scalar_field": (ctypes.c_int, [vp, ctypes.c_int32, P(MggReport)]),
        "mgg_potential": (ctypes.c_int, [vp]),
        "mgg_potential_mg": (ctypes.c_int, [vp]),
        "mgg_move": (ctypes.c_int, [vp, ctypes.c_float, f64p]),
        "mgg_power": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32] + [f64p] * 6),
        "mgg_power_rsd": (ctypes.c_int, [vp, ctypes.c_int32] + [f64p] * 5),
        "mgg_density_pdf": (ctypes.c_int, [vp, ctypes.c_int32, P(ctypes.c_int64), f64p, f64p]),
        "mgg_upload_grid": (ctypes.c_int, [vp, ctypes.c_int32, f32p]),
        "mgg_download_grid": (ctypes.c_int, [vp, ctypes.c_int32, f32p]),
        "mgg_set_background": (ctypes.c_int, [vp, f64p, ctypes.c_int32]),
        "mgg_synchronize": (ctypes.c_int, [vp]),
        "mgg_timing": (ctypes.c_int, [vp, f64p]),
        "mgg_profile": (ctypes.c_int, [vp, ctypes.c_int32]),
        "mgg_profile_count": (ctypes.c_int, []),
        "mgg_profile_read": (ctypes.c_int, [vp, ctypes.c_int32, P(ctypes.c_char_p), P(ctypes.c_int64),
                                            f64p, f64p]),
        "mgg_profile_reset": (ctypes.c_int, [vp]),
        "mgg_timer_start": (ctypes.c_int, [vp]),
        "mgg_timer_stop": (ctypes.c_int, [vp, f64p]),
        "mgg_make_ics": (ctypes.c_int, [vp, P(MggIcParams)]),
        "mgg_version": (ctypes.c_char_p, []),
        "mgg_background_table": (ctypes.c_int, [P(MggConfig), ctypes.c_double, f64p, ctypes.c_int32,
                                                P(ctypes.c_int32), f64p]),
        "mgg_density_noalloc": (ctypes.c_int, [vp, vp, vp, ctypes.c_int64, ctypes.c_int32, vp, vp]),
        "mgg_cic_keys": (ctypes.c_int, [vp, P(ctypes.c_uint32), P(ctypes.c_uint32), P(ctypes.c_uint32)]),
        "mgg_step": (ctypes.c_int, [vp, P(MggStepState)]),
        "mgg_run_steps": (ctypes.c_int, [vp, P(MggStepState), ctypes.c_int32, P(MggReport), P(ctypes.c_double)]),
        "mgg_step_host": (ctypes.c_int, [vp, P(MggStepState)] + [f32p] * 6 + [ctypes.c_int64]),
        "mgg_step_host_pipelined": (ctypes.c_int, [vp, P(MggStepState)] + [f32p] * 6 + [ctypes.c_int64]),
        "mgg_step_batch": (ctypes.c_int, [P(vp), P(MggStepState), ctypes.c_int32]),
        "mgg_get_config": (ctypes.c_int, [vp, P(MggConfig)]),
        "mgg_reconfigure": (ctypes.c_int, [vp, P(MggConfig)]),
        "mgg_box_bytes": (ctypes.c_int64, [P(MggConfig)]),
        "mgg_server_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_double, ctypes.c_int32, P(vp)]),
        "mgg_server_submit": (ctypes.c_int, [vp, P(MggRequest), P(ctypes.c_int64)]),
        "mgg_server_wait": (ctypes.c_int, [vp, ctypes.c_int64, P(MggResultInfo), f64p, f64p, f64p, ctypes.c_int32]),
        "mgg_server_destroy": (ctypes.c_int, [vp]),
        "mgg_server_error": (ctypes.c_char_p, [vp, ctypes.c_int64]),
        "mgg_pm_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, P(MggPmHeader)] + [f32p] * 6),
        "mgg_pm_read_header": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, P(MggPmHeader)]),
        "mgg_pm_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, P(MggPmHeader)] + [f32p] * 6 +
                        [ctypes.c_int64]),
        "mgg_pm_last_error": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _dptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_config(ngrid: int, nrow: int, box: float, om: float = 0.3089, oml: float = 0.6911,
                omb: float = 0.0486, mg_model: int = MODEL_FR, mg_flag: int = 1, fr_n: int = 1,
                fr0: float = -1.0e-5, cycle: str = "V", iter_count_max: int = 4, res_conv: float = 1.0e-8,
                precision: int = PREC_PLAIN, device: int = 0, **kw) -> MggConfig:
    """Setup.dat contents (ReadSetup, PMP2mod_tools.f90:114-231) as an mgg_config."""
    c = MggConfig()
    c.ngrid, c.nrow, c.box = ngrid, nrow, box
    c.om, c.oml, c.omb = om, oml, omb
    c.mg_flag, c.mg_model = mg_flag, mg_model
    c.vcycle, c.fcycle, c.wcycle = int(cycle == "V"), int(cycle == "F"), int(cycle == "W")
    c.iter_count_max, c.res_conv = iter_count_max, res_conv
    c.fr_n, c.fr0 = fr_n, fr0
    c.n_branch, c.s_branch, c.h0rc = 1, 0, 1.0
    c.sym_astar, c.sym_xi, c.sym_beta = 0.5, 1.0 / 2997.92458, 1.0
    c.kmf_power_law, c.kmf_born_infeld, c.kmf_n = 1, 0, 3
    c.kmf_k0, c.kmf_beta, c.kmf_lambda = 1.0, 0.1, 1.0
    c.csf_coupling, c.csf_potential = 1, 1
    c.csf_alpha, c.csf_beta, c.csf_lambda = 0.1, -0.2, 1.0
    c.precision, c.device = precision, device
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def step_table(aexpn0: float, astep0: float):
    """Alist of Initialize (PMP2main.f90:154-171) in Real*4 arithmetic."""
    f32 = np.float32
    step_factor = f32(f32(astep0) / f32(aexpn0))
    da, a = f32(astep0), f32(aexpn0)
    alist = [a]
    while True:
        if da < f32(step_factor / f32(1.25)) * a and a < f32(0.3):
            da = f32(f32(1.5) * da)
        a = f32(a + da)
        alist.append(a)
        if len(alist) > 2001:
            raise ValueError("Too many timesteps")
        if a >= f32(1.0):
            break
    return np.array(alist, dtype=np.float32)


def astep_for_nsteps(aexpn0: float, nsteps: int) -> float:
    """Initial step ASTEP0 whose table (PMP2main.f90:161-171) reaches a=1 in exactly nsteps.

    The step count is not monotonic in ASTEP0 (the x1.5 growth of the early steps
    switches off at a = 0.3), so a bisection on it can land on a neighbouring
    count; when it does, the largest ASTEP0 of a fine geometric scan that gives
    exactly nsteps is taken.  ValueError when no ASTEP0 gives nsteps."""
    def count(a):
        return len(step_table(aexpn0, a)) - 1

    lo, hi = 1e-6, 1.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if count(mid) > nsteps:
            lo = mid
        else:
            hi = mid
    a = float(np.float32(hi))
    if count(a) == nsteps:
        return a
    for cand in np.geomspace(1.0 - aexpn0, 1e-6, 40000):
        c = float(np.float32(cand))
        if count(c) == nsteps:
            return c
    raise ValueError(f"no initial step gives {nsteps} steps from a = {aexpn0}")


@dataclass
class StepState:
    """AEXPN, ASTEP, ISTEP and the step factor of Module Tools."""
    aexpn: float
    astep: float
    istep: int = 0
    step_factor: float = 0.0
    ekin: float = 0.0
    reports: list = field(default_factory=list)


class Box:
    """One simulation box resident on one GPU (an ``mgg_ctx``)."""

    def __init__(self, cfg: MggConfig):
        self.lib = load_library()
        self.cfg = cfg
        h = ctypes.c_void_p()
        rc = self.lib.mgg_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != MGG_OK:
            raise MGGError(rc, self.lib.mgg_last_error(None).decode())
        self.h = h
        self.ngrid = cfg.ngrid
        self.np = cfg.nrow ** 3

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc: int):
        if rc != MGG_OK:
            raise MGGError(rc, self.lib.mgg_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.mgg_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- Module Tools state ----------------------------------------------
    def set_time(self, aexpn: float, astep: float):
        self._check(self.lib.mgg_set_time(self.h, aexpn, astep))

    def upload_particles(self, x, y, z, vx, vy, vz):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (x, y, z, vx, vy, vz)]
        self._check(self.lib.mgg_upload_particles(self.h, *[_fptr(a) for a in arrs], self.np))

    def download_particles(self):
        out = [np.empty(self.np, dtype=np.float32) for _ in range(6)]
        self._check(self.lib.mgg_download_particles(self.h, *[_fptr(a) for a in out], self.np))
        return out

    def upload_grid(self, which: int, grid: np.ndarray):
        g = np.ascontiguousarray(grid, dtype=np.float32).reshape(-1)
        if g.size != self.ngrid ** 3:
            raise ValueError("grid size mismatch")
        self._check(self.lib.mgg_upload_grid(self.h, which, _fptr(g)))

    def download_grid(self, which: int) -> np.ndarray:
        g = np.empty(self.ngrid ** 3, dtype=np.float32)
        self._check(self.lib.mgg_download_grid(self.h, which, _fptr(g)))
        return g

    def set_background(self, table: np.ndarray):
        t = np.ascontiguousarray(table, dtype=np.float64)
        self._check(self.lib.mgg_set_background(self.h, _dptr(t), t.shape[0]))

    def synchronize(self):
        self._check(self.lib.mgg_synchronize(self.h))

    # -- the reference's subroutines -------------------------------------
    def density(self):
        """DENSIT (PMP2mod_density.f90:17-301)."""
        self._check(self.lib.mgg_density(self.h))

    def scalar_field(self, i_step: int) -> MggReport:
        """scalar_field(i_step) (PMP2extradof.f90:12-178)."""
        rep = MggReport()
        self._check(self.lib.mgg_scalar_field(self.h, i_step, ctypes.byref(rep)))
        return rep

    def potential(self):
        """POTENTfft5 (PMP2main.f90:705-867)."""
        self._check(self.lib.mgg_potential(self.h))

    def potential_mg(self):
        """POTENT_FOR_MG (PMP2main.f90:869-1015)."""
        self._check(self.lib.mgg_potential_mg(self.h))

    def move(self, factv: float) -> float:
        """MOVE(FactV) (PMP2main.f90:304-685); returns ENKIN."""
        e = ctypes.c_double(0.0)
        self._check(self.lib.mgg_move(self.h, factv, ctypes.byref(e)))
        return e.value

    def power(self, recompute_density: bool = True, nbins: int | None = None):
        """GetPower(0) (PMP2mod_power.f90:20-66): dict of k, nmodes, pk (+ log bins)."""
        nb = nbins or self.ngrid // 2
        outs = [np.zeros(nb, dtype=np.float64) for _ in range(6)]
        self._check(self.lib.mgg_power(self.h, int(recompute_density), nb, *[_dptr(a) for a in outs]))
        return dict(k=outs[0], nmodes=outs[1], pk=outs[2], klog=outs[3], nmodeslog=outs[4], pklog=outs[5])

    def power_rsd(self, nbins: int | None = None):
        """GetPower(1) with sigv = 0 (PMP2mod_power.f90:20-108): dict of k, nmodes, preal, p0, p2
        on the NGRID/2 mesh (the PowerDM.Z columns).  Overwrites FI."""
        nb = nbins or self.ngrid // 4
        outs = [np.zeros(nb, dtype=np.float64) for _ in range(5)]
        self._check(self.lib.mgg_power_rsd(self.h, nb, *[_dptr(a) for a in outs]))
        return dict(k=outs[0], nmodes=outs[1], preal=outs[2], p0=outs[3], p2=outs[4])

    def density_pdf(self, level: int = 0):
        """DensDistr (PMP2mod_density.f90:1041-1126) on the NGRID/2^level mesh (level 0: FI as it
        stands).  Returns the reference's table columns per bin i = -2001..2001 (dens_left,
        dens_right, density, dens*dN/d(dens)/Ncells, cells) and the RMS and mean of 1 + delta."""
        nc = np.zeros(PDF_BINS, dtype=np.int64)
        den = np.zeros(PDF_BINS, dtype=np.float64)
        st = np.zeros(2, dtype=np.float64)
        self._check(self.lib.mgg_density_pdf(self.h, level, nc.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                             _dptr(den), _dptr(st)))
        i = np.arange(PDF_BINS) - 2001
        d1 = (10.0 ** (i * 0.001)).astype(np.float32).astype(np.float64)
        d1[0] = 0.0
        d2 = (10.0 ** ((i + 1) * 0.001)).astype(np.float32).astype(np.float64)
        mean_bin = den / np.maximum(nc, 1)
        ng = self.ngrid >> level
        return dict(dens_left=d1, dens_right=d2, density=mean_bin,
                    f=nc / (d2 - d1) / float(ng) ** 3 * mean_bin, ncells=nc, den_sum=den,
                    rms=float(st[0]), mean=float(st[1]))

    def cic_keys(self, cells: bool = True):
        """Integer keys of the last density on the NGRID mesh (mgg_cic_keys): row counts
        (NGRID^2, row = (J-1) + NGRID (K-1)), row offsets (NGRID^2 + 1) and, with cells,
        per-cell counts (NGRID^3, cell = (I-1) + NGRID row) recounted from the row buckets."""
        n = self.ngrid
        rc = np.zeros(n * n, dtype=np.uint32)
        rs = np.zeros(n * n + 1, dtype=np.uint32)
        cc = np.zeros(n ** 3, dtype=np.uint32) if cells else None
        u32 = ctypes.POINTER(ctypes.c_uint32)
        self._check(self.lib.mgg_cic_keys(self.h, rc.ctypes.data_as(u32), rs.ctypes.data_as(u32),
                                          None if cc is None else cc.ctypes.data_as(u32)))
        return rc, rs, cc

    def make_ics(self, seed: int, aexpn: float, astep: float, sigma8: float = 0.8159,
                 hubble: float = 0.6774, ns: float = 0.9667):
        p = MggIcParams(seed, sigma8, hubble, ns, aexpn, astep)
        self._check(self.lib.mgg_make_ics(self.h, ctypes.byref(p)))

    # -- the main loop body ----------------------------------------------
    def start(self, aexpn0: float, astep0: float) -> StepState:
        """ISTEP/AEXPN/ASTEP after Initialize; StepFactor = ASTEP0/AEXPN0 (PMP2main.f90:124)."""
        f32 = np.float32
        return StepState(aexpn=float(f32(aexpn0)), astep=float(f32(astep0)), istep=0,
                         step_factor=float(f32(f32(astep0) / f32(aexpn0))))

    def new_state(self, aexpn0: float, astep0: float) -> MggStepState:
        """Step state after Initialize (PMP2main.f90:124) for mgg_step."""
        st = MggStepState()
        st.aexpn, st.astep = aexpn0, astep0
        st.step_factor = float(np.float32(np.float32(astep0) / np.float32(aexpn0)))
        st.istep = 0
        return st

    def step(self, st: MggStepState) -> MggStepState:
        """One main-loop iteration in one C-ABI call (mgg_step)."""
        self._check(self.lib.mgg_step(self.h, ctypes.byref(st)))
        return st

    def run_steps(self, st: MggStepState, nsteps: int):
        """nsteps main-loop iterations queued as CUDA graphs with no host round trip (mgg_run_steps); returns
        the per-step reports and ENKIN values."""
        reps = (MggReport * max(nsteps, 1))()
        ek = (ctypes.c_double * max(nsteps, 1))()
        self._check(self.lib.mgg_run_steps(self.h, ctypes.byref(st), nsteps, reps, ek))
        return list(reps)[:nsteps], list(ek)[:nsteps]

    def step_host(self, st: MggStepState, parts) -> MggStepState:
        """mgg_step with host particle arrays (float32, updated in place)."""
        assert all(a.dtype == np.float32 and a.flags.c_contiguous and a.size == self.np for a in parts)
        self._check(self.lib.mgg_step_host(self.h, ctypes.byref(st), *[_fptr(a) for a in parts], self.np))
        return st

    def step_host_pipelined(self, st: MggStepState, parts) -> MggStepState:
        """mgg_step_host_pipelined: positions back on return; the velocities (parts[3:])
        are complete after synchronize()."""
        assert all(a.dtype == np.float32 and a.flags.c_contiguous and a.size == self.np for a in parts)
        self._check(self.lib.mgg_step_host_pipelined(self.h, ctypes.byref(st), *[_fptr(a) for a in parts], self.np))
        return st

    def pm_step(self, st: StepState, i: int) -> StepState:
        """One iteration of the main loop (PMP2main.f90:36-60)."""
        f32 = np.float32
        self.set_time(st.aexpn, st.astep)
        self.density()
        if self.cfg.mg_flag == 1:
            st.reports.append(self.scalar_field(i))
        self.potential()
        factv = f32(1.0)
        if f32(st.astep) < f32(f32(st.step_factor) / f32(1.25)) * f32(st.aexpn) and f32(st.aexpn) < f32(0.3):
            st.astep = float(f32(f32(1.5) * f32(st.astep)))
            factv = f32(1.2)
        if self.cfg.mg_flag == 1:
            self.potential_mg()
        self.set_time(st.aexpn, st.astep)
        st.ekin = self.move(float(factv))
        # ADDTIME (PMP2main.f90:256-261)
        st.istep += 1
        st.aexpn = float(f32(f32(st.aexpn) + f32(st.astep)))
        return st

    # -- measurement -----------------------------------------------------
    def timing(self) -> np.ndarray:
        out = np.zeros(T_NBUCKETS, dtype=np.float64)
        self._check(self.lib.mgg_timing(self.h, _dptr(out)))
        return out

    def profile(self, enable: bool):
        self._check(self.lib.mgg_profile(self.h, int(enable)))

    def profile_reset(self):
        self._check(self.lib.mgg_profile_reset(self.h))

    def profile_read(self) -> dict:
        res = {}
        for i in range(self.lib.mgg_profile_count()):
            name = ctypes.c_char_p()
            n = ctypes.c_int64()
            ms = ctypes.c_double()
            b = ctypes.c_double()
            self._check(self.lib.mgg_profile_read(self.h, i, ctypes.byref(name), ctypes.byref(n),
                                                  ctypes.byref(ms), ctypes.byref(b)))
            res[name.value.decode()] = dict(launches=n.value, ms=ms.value, bytes=b.value)
        return res

    def timer_start(self):
        self._check(self.lib.mgg_timer_start(self.h))

    def timer_stop(self) -> float:
        ms = ctypes.c_double()
        self._check(self.lib.mgg_timer_stop(self.h, ctypes.byref(ms)))
        return ms.value


def background_table(cfg: MggConfig, hubble: float = 0.6774):
    """BackgroundEvolution table and lambda of the k-mouflage / csf models (host computation).

    Sets cfg.kmf_lambda or cfg.csf_lambda like Fix_Parameter_lambda does
    (PMP2mod_MGbackground.f90:141-146); returns (table[rows, 6], lambda)."""
    lib = load_library()
    cap = 100020
    tab = np.zeros((cap, 6), dtype=np.float64)
    rows = ctypes.c_int32(0)
    lam = ctypes.c_double(0.0)
    rc = lib.mgg_background_table(ctypes.byref(cfg), hubble, _dptr(tab), cap, ctypes.byref(rows), ctypes.byref(lam))
    if rc != MGG_OK:
        raise MGGError(rc, lib.mgg_last_error(None).decode())
    return tab[: rows.value], lam.value


def density_noalloc(x: int, y: int, z: int, np_: int, ngrid: int, fi: int, stream: int = 0) -> None:
    """CIC density of device arrays without any device allocation (mgg_density_noalloc).

    For callers that cannot call cudaMalloc (their device memory comes from their
    own pool, or they must not allocate mid-run).  x, y, z, fi are device
    addresses on the current device (e.g. torch tensor .data_ptr()); fi receives
    NGRID^3 floats.  Limits: NGRID a power of two in [16, 256], at most 2^21
    particles; scratch is a fixed device array of 40.5 MiB shared by every
    call, so calls that overlap on the GPU race.  Returns when the grid is done."""
    lib = load_library()
    rc = lib.mgg_density_noalloc(x, y, z, np_, ngrid, fi, stream or None)
    if rc != MGG_OK:
        raise MGGError(rc, lib.mgg_last_error(None).decode())


def step_batch(boxes, states, raise_on_error: bool = True):
    """Batched form: one main-loop step of every box, concurrently (mgg_step_batch).

    Returns the indices of the boxes whose step failed (each box's error is its
    mgg_last_error); with raise_on_error, a failure raises MGGError instead."""
    lib = load_library()
    n = len(boxes)
    hs = (ctypes.c_void_p * n)(*[b.h.value for b in boxes])
    arr = (MggStepState * n)(*states)
    rc = lib.mgg_step_batch(hs, arr, n)
    for i in range(n):
        ctypes.memmove(ctypes.byref(states[i]), ctypes.byref(arr[i]), ctypes.sizeof(MggStepState))
    if rc == MGG_OK:
        return []
    failed = [i for i, b in enumerate(boxes) if lib.mgg_last_error(b.h)]
    if raise_on_error:
        raise MGGError(rc, "; ".join(f"box {i}: {lib.mgg_last_error(boxes[i].h).decode()}" for i in failed))
    return failed


class Server:
    """Serving form (mgg_server_*): continuous admission of whole simulations
    by device-memory budget, run side by side on one GPU."""

    def __init__(self, device: int = 0, hbm_budget_gb: float = 64.0, max_active: int = 8):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.mgg_server_create(device, hbm_budget_gb, max_active, ctypes.byref(h))
        if rc != MGG_OK:
            raise MGGError(rc, "mgg_server_create failed")
        self.h = h

    def submit(self, cfg: MggConfig, seed: int, aexpn0: float, astep0: float, nsteps: int,
               sigma8: float = 0.8159, hubble: float = 0.6774, ns: float = 0.9667) -> int:
        r = MggRequest()
        r.cfg = cfg
        r.ic = MggIcParams(seed, sigma8, hubble, ns, aexpn0, astep0)
        r.nsteps = nsteps
        rid = ctypes.c_int64()
        rc = self.lib.mgg_server_submit(self.h, ctypes.byref(r), ctypes.byref(rid))
        if rc != MGG_OK:
            raise MGGError(rc, "mgg_server_submit failed")
        return rid.value

    def wait(self, rid: int, nbins: int):
        """(info, k, nmodes, pk) of request rid, blocking until it is done."""
        info = MggResultInfo()
        k, nm, pk = (np.zeros(nbins) for _ in range(3))
        rc = self.lib.mgg_server_wait(self.h, rid, ctypes.byref(info), _dptr(k), _dptr(nm), _dptr(pk), nbins)
        if rc != MGG_OK:
            raise MGGError(rc, self.lib.mgg_server_error(self.h, rid).decode())
        return info, k, nm, pk

    def close(self):
        if self.h:
            self.lib.mgg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pm_header(cfg: MggConfig, aexpn: float, astep: float, istep: int, aexpn0: float, ekin: float = 0.0,
              title: str = "mgglam-b200 snapshot", nrealization: int = 1, nseed: int = 0,
              hubble: float = 0.6774) -> MggPmHeader:
    """PMcrd header for a box (WriteDataPM, PMP2mod_tools.f90:426-435); extras(100) = Box."""
    h = MggPmHeader()
    h.header = title.encode()[:45].ljust(45)
    h.aexpn, h.aexp0, h.amplt, h.astep, h.istep = aexpn, aexpn0, 0.0, astep, istep
    h.partw = float(np.float32(np.float32(cfg.ngrid) ** 3 / np.float32(cfg.nrow ** 3)))
    h.ekin = ekin
    h.nrow, h.ngrid, h.nrealization, h.nseed = cfg.nrow, cfg.ngrid, nrealization, nseed
    h.om, h.oml, h.hubble = cfg.om, cfg.oml, hubble
    h.nparticles = cfg.nrow ** 3
    h.extras[99] = cfg.box
    return h


def pm_write(directory: str, moment: int, header: MggPmHeader, parts) -> None:
    """WriteDataPM: PMcrd[.NNNN].DAT + PMcrs<i>[.NNNN].DAT (moment < 0: no step number)."""
    lib = load_library()
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in parts]
    rc = lib.mgg_pm_write(directory.encode(), moment, ctypes.byref(header), *[_fptr(a) for a in arrs])
    if rc != MGG_OK:
        raise MGGError(rc, lib.mgg_pm_last_error().decode())


def pm_read(directory: str, moment: int):
    """ReadDataPM: (header, [x, y, z, vx, vy, vz])."""
    lib = load_library()
    h = MggPmHeader()
    rc = lib.mgg_pm_read_header(directory.encode(), moment, ctypes.byref(h))
    if rc != MGG_OK:
        raise MGGError(rc, lib.mgg_pm_last_error().decode())
    arrs = [np.empty(h.nparticles, dtype=np.float32) for _ in range(6)]
    rc = lib.mgg_pm_read(directory.encode(), moment, ctypes.byref(h), *[_fptr(a) for a in arrs], h.nparticles)
    if rc != MGG_OK:
        raise MGGError(rc, lib.mgg_pm_last_error().decode())
    return h, arrs


def version() -> str:
    return load_library().mgg_version().decode()
