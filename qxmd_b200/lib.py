"""ctypes binding of the C ABI (include/qxmd_b200.h) and a thin host-side
context that mirrors the reference routines the hot path replaces.

The library is loaded from qxmd_b200/_lib/libqxmd_b200.so; if it is missing
or fails to load, every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build
from . import cell

_lib = None

QX_PREC_FP64 = 0
QX_PREC_MIXED = 1
QX_NL_NONE, QX_NL_GSPACE, QX_NL_RSPACE = 0, 1, 2
QX_HPSI_KINETIC, QX_HPSI_NONLOCAL, QX_HPSI_ACCUMULATE = 1, 2, 4
QX_ERR = {1: "ARG", 2: "CUDA", 3: "NOTPD", 4: "EIG", 5: "STATE"}

# Every symbol the header declares (checked by the CPU test suite).
EXPORTS = [
    "qx_last_error", "qx_version", "qx_launch_count", "qx_create", "qx_destroy", "qx_set_glocal", "qx_set_kb_g",
    "qx_set_kb_builder", "qx_build_kb_g", "qx_get_kb_g", "qx_set_kb_r_builder", "qx_set_kb_r_channel_radii", "qx_build_kb_r", "qx_get_kb_r",
    "qx_forces_nl_r", "qxgpu_fnnlcl2",
    "qx_set_kb_r", "qx_set_nlmode", "qx_set_occ", "qx_put_psi", "qx_get_psi", "qx_put_hpsi",
    "qx_get_hpsi", "qx_get_eig", "qx_get_rho", "qx_put_rho", "qx_get_glocal", "qx_dev_ptr",
    "qx_sync", "qx_hpsi", "qx_ekinetic", "qx_enonloc", "qx_hmatrix", "qx_gradres", "qx_untryt",
    "qx_untryhc", "qx_eigen", "qx_hmatrix_static", "qx_schmidt", "qx_softchg", "qx_scf_init", "qx_scf_mixing", "qx_set_force_tables", "qx_forces",
    "qx_tddft_store", "qx_tddft_overlap", "qx_autotune", "qx_refine_from", "qx_scf_launch", "qx_scf_result",
    "qxgpu_kbnlpp_frc2",
    "qx_scf_rho_from_psi", "qx_scf_iteration", "qx_scf_iteration_host", "qxgpu_hcnonloc", "qxgpu_hckbpp_g", "qxgpu_enonloc", "qxgpu_eigen",
    "qxgpu_schmidt", "qxgpu_hmatrix", "qxgpu_untryt", "qxgpu_softchg", "qxgpu_rfft3",
    "qx_fssh_init", "qx_fssh_step", "qx_fssh_state", "qx_build_vloc", "qx_gemm_fallbacks",
]


class QxError(RuntimeError):
    def __init__(self, code, where):
        self.code = code
        super().__init__(f"{where}: QX_ERR_{QX_ERR.get(code, code)}: {last_error()}")


class CgParm(C.Structure):
    _fields_ = [("itermx", C.c_int), ("iteremx", C.c_int), ("noband", C.c_int),
                ("tolera", C.c_double), ("roughfzan", C.c_double), ("roughfeig", C.c_double),
                ("threinn", C.c_double), ("wdinner", C.c_double), ("ccreal4", C.c_int),
                ("sequential", C.c_int)]

    @classmethod
    def defaults(cls, noband, **kw):
        """Defaults of modules.f90:171-182."""
        p = dict(itermx=4, iteremx=4, noband=noband, tolera=1e-10, roughfzan=0.3,
                 roughfeig=0.3, threinn=0.0, wdinner=0.9, ccreal4=0, sequential=0)
        p.update(kw)
        return cls(**p)


class FsshParm(C.Structure):
    """qx_fssh_parm: band window, MD step and substep (Rydberg time units),
    Boltzmann factor and its temperature (Ry), hops on/off, rnd00 seed."""
    _fields_ = [("b0", C.c_int), ("nstate", C.c_int), ("dtmd", C.c_double), ("dttddft", C.c_double),
                ("boltzmann", C.c_int), ("treq", C.c_double), ("hop", C.c_int), ("seed", C.c_double)]


class ScfOut(C.Structure):
    _fields_ = [("etot", C.c_double), ("eband", C.c_double), ("ehartree", C.c_double),
                ("exc", C.c_double), ("evxc", C.c_double), ("resid", C.c_double),
                ("zmax", C.c_double), ("ncg_hpsi", C.c_int), ("eig_clusters", C.c_int)]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_vp = C.c_void_p
_ctx = C.c_void_p


def lib(build_if_missing: bool = True):
    """Load the C-ABI library (building it first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise RuntimeError(f"qxmd_b200 library missing: {path}")
        _build.build()
    L = C.CDLL(path)
    sig = {
        "qx_last_error": ([], C.c_char_p),
        "qx_version": ([], C.c_int),
        "qx_launch_count": ([], C.c_long),
        "qx_create": ([C.POINTER(_ctx), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _ip, _dp, C.c_int, _vp], C.c_int),
        "qx_destroy": ([_ctx], C.c_int),
        "qx_set_glocal": ([_ctx, _dp], C.c_int),
        "qx_set_kb_g": ([_ctx, C.c_int, _dp, _dp], C.c_int),
        "qx_set_kb_builder": ([_ctx, C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _ip, _ip, _dp, _ip], C.c_int),
        "qx_build_kb_g": ([_ctx, C.c_int, _ip, _dp], C.c_int),
        "qx_get_kb_g": ([_ctx, _dp, _dp], C.c_int),
        "qx_set_kb_r_channel_radii": ([_ctx, _dp], C.c_int),
        "qx_set_kb_r_builder": ([_ctx, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _vp, _ip, _dp, C.c_double, _dp],
                                C.c_int),
        "qx_forces_nl_r": ([_ctx, _dp], C.c_int),
        "qxgpu_fnnlcl2": ([_ctx, _dp, _dp], C.c_int),
        "qx_build_kb_r": ([_ctx, C.c_int, _ip, _dp], C.c_int),
        "qx_get_kb_r": ([_ctx, C.POINTER(C.c_int), _vp, _vp, _vp], C.c_int),
        "qx_set_kb_r": ([_ctx, C.c_int, C.c_int, _ip, _ip, _dp, _dp, C.c_double], C.c_int),
        "qx_set_nlmode": ([_ctx, C.c_int], C.c_int),
        "qx_set_occ": ([_ctx, _dp, C.c_double], C.c_int),
        "qx_put_psi": ([_ctx, _dp], C.c_int),
        "qx_get_psi": ([_ctx, _dp], C.c_int),
        "qx_put_hpsi": ([_ctx, _dp], C.c_int),
        "qx_get_hpsi": ([_ctx, _dp], C.c_int),
        "qx_get_eig": ([_ctx, _dp], C.c_int),
        "qx_get_rho": ([_ctx, _dp], C.c_int),
        "qx_put_rho": ([_ctx, _dp], C.c_int),
        "qx_get_glocal": ([_ctx, _dp], C.c_int),
        "qx_dev_ptr": ([_ctx, C.c_int], C.c_void_p),
        "qx_sync": ([_ctx], C.c_int),
        "qx_hpsi": ([_ctx, _vp, _vp, C.c_int, C.c_int], C.c_int),
        "qx_ekinetic": ([_ctx, _vp, _vp], C.c_int),
        "qx_enonloc": ([_ctx], C.c_int),
        "qx_hmatrix": ([_ctx, _vp], C.c_int),
        "qx_hmatrix_static": ([_vp, _vp, C.c_int, C.c_int, _vp, _vp], C.c_int),
        "qx_gradres": ([_ctx, _vp, _vp, _vp], C.c_int),
        "qx_untryt": ([_ctx, _vp], C.c_int),
        "qx_untryhc": ([_ctx], C.c_int),
        "qx_eigen": ([_ctx, C.POINTER(CgParm), _vp, _vp], C.c_int),
        "qx_schmidt": ([_ctx], C.c_int),
        "qx_softchg": ([_ctx], C.c_int),
        "qx_scf_init": ([_ctx, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_double], C.c_int),
        "qx_scf_mixing": ([_ctx, C.c_int, C.c_double], C.c_int),
        "qx_set_force_tables": ([_ctx, C.c_int, C.c_int, _ip, _dp, C.c_int, _ip, _ip, _dp, _dp, _dp], C.c_int),
        "qx_forces": ([_ctx, _dp, _dp], C.c_int),
        "qx_tddft_store": ([_ctx], C.c_int),
        "qx_autotune": ([_ctx, C.c_char_p, C.c_int], C.c_int),
        "qx_refine_from": ([_ctx, _ctx], C.c_int),
        "qx_scf_launch": ([_ctx, C.POINTER(CgParm)], C.c_int),
        "qx_scf_result": ([_ctx, C.POINTER(ScfOut)], C.c_int),
        "qx_tddft_overlap": ([_ctx, _dp], C.c_int),
        "qxgpu_kbnlpp_frc2": ([_ctx, _dp, _dp], C.c_int),
        "qx_scf_rho_from_psi": ([_ctx], C.c_int),
        "qx_scf_iteration": ([_ctx, C.POINTER(CgParm), C.POINTER(ScfOut)], C.c_int),
        "qx_scf_iteration_host": ([_ctx, C.POINTER(CgParm), C.POINTER(ScfOut), _vp, _vp, _vp, _vp], C.c_int),
        "qxgpu_hcnonloc": ([_ctx, _dp, _dp, C.c_int], C.c_int),
        "qxgpu_hckbpp_g": ([_ctx, _dp, _dp, C.c_int], C.c_int),
        "qxgpu_enonloc": ([_ctx, _dp, _dp, _vp], C.c_int),
        "qxgpu_eigen": ([_ctx, _dp, _dp, _vp, _vp, C.POINTER(CgParm)], C.c_int),
        "qxgpu_schmidt": ([_ctx, _dp], C.c_int),
        "qxgpu_hmatrix": ([_ctx, _dp, _dp, _vp, _vp], C.c_int),
        "qxgpu_untryt": ([_ctx, _dp, _dp, _vp], C.c_int),
        "qxgpu_softchg": ([_ctx, _dp, _dp], C.c_int),
        "qxgpu_rfft3": ([_ctx, C.c_int, _dp, _dp], C.c_int),
        "qx_fssh_init": ([_ctx, C.POINTER(FsshParm), _dp], C.c_int),
        "qx_build_vloc": ([_ctx], C.c_int),
        "qx_gemm_fallbacks": ([], C.c_long),
        "qx_fssh_step": ([_ctx, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "qx_fssh_state": ([_ctx, _vp, _vp, _vp, _vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def gemm_fallbacks() -> int:
    """FP32 contractions so far that ran on the CUDA-core GEMM (qx_gemm_fallbacks)."""
    return int(lib().qx_gemm_fallbacks())


def launch_count() -> int:
    return int(lib().qx_launch_count())


def last_error() -> str:
    if _lib is None:
        return ""
    m = _lib.qx_last_error()
    return m.decode() if m else ""


def _ck(code, where):
    if code:
        raise QxError(code, where)


def _ptr(a):
    return None if a is None else a.ctypes.data


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One cell's device-resident hot-path state (qx_ctx).

    Arrays use the Fortran layouts: wavefunctions (nband, nplwex) in numpy
    row-major = gdcr(nplwex, nband) column-major.
    """

    def __init__(self, sys, precision: int = QX_PREC_FP64, nlmode: int = QX_NL_GSPACE,
                 nband: int | None = None, stream: int = 0):
        L = lib()
        gs = sys.gs
        self.sys = sys
        self.nb = nband or sys.nband
        self.ne = gs.nplwex
        self.n = gs.kfft0
        self.precision = precision
        h = _ctx()
        ijkgd = np.ascontiguousarray(gs.ijkgd()[gs.nplw5 - gs.nplw: gs.nplw5 + gs.nplw + 1], dtype=np.int32)
        _ck(L.qx_create(C.byref(h), precision, gs.grid[0], gs.grid[1], gs.grid[2], gs.nplw, ijkgd,
                        _f64(gs.dkgnrm()), self.nb, stream), "qx_create")
        self.h = h
        self.L = L
        _ck(L.qx_set_glocal(h, _f64(sys.vloc)), "qx_set_glocal")
        _ck(L.qx_set_kb_g(h, sys.kb_g.shape[1], _f64(sys.kb_g.T), _f64(sys.vclalp)), "qx_set_kb_g")
        kr = sys.kb_r
        self._kbr_lmx = int(np.asarray(kr.vnl).shape[1])
        _ck(L.qx_set_kb_r(h, sys.cell.natom, self._kbr_lmx, np.ascontiguousarray(kr.off, dtype=np.int32),
                          np.ascontiguousarray(kr.mesh, dtype=np.int32), _f64(kr.vnl), _f64(kr.clalp),
                          kr.rdelv), "qx_set_kb_r")
        _ck(L.qx_set_nlmode(h, nlmode), "qx_set_nlmode")
        occ = np.zeros(self.nb)
        occ[: min(self.nb, sys.occ.size)] = sys.occ[: self.nb]
        _ck(L.qx_set_occ(h, occ, gs.rvol), "qx_set_occ")

    def close(self):
        if getattr(self, "h", None):
            self.L.qx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- transfers -----------------------------------------------------------
    def put_psi(self, x):
        _ck(self.L.qx_put_psi(self.h, _f64(x)), "qx_put_psi")

    def get_psi(self):
        out = np.empty((self.nb, self.ne))
        _ck(self.L.qx_get_psi(self.h, out), "qx_get_psi")
        return out

    def put_hpsi(self, x):
        _ck(self.L.qx_put_hpsi(self.h, _f64(x)), "qx_put_hpsi")

    def get_hpsi(self):
        out = np.empty((self.nb, self.ne))
        _ck(self.L.qx_get_hpsi(self.h, out), "qx_get_hpsi")
        return out

    def get_eig(self):
        out = np.empty(self.nb)
        _ck(self.L.qx_get_eig(self.h, out), "qx_get_eig")
        return out

    def get_rho(self):
        out = np.empty(self.n)
        _ck(self.L.qx_get_rho(self.h, out), "qx_get_rho")
        return out

    def put_rho(self, x):
        _ck(self.L.qx_put_rho(self.h, _f64(x)), "qx_put_rho")

    def get_glocal(self):
        out = np.empty(self.n)
        _ck(self.L.qx_get_glocal(self.h, out), "qx_get_glocal")
        return out

    def set_glocal(self, g):
        _ck(self.L.qx_set_glocal(self.h, _f64(g)), "qx_set_glocal")

    def set_nlmode(self, m):
        _ck(self.L.qx_set_nlmode(self.h, m), "qx_set_nlmode")

    def dev_ptr(self, which):
        return self.L.qx_dev_ptr(self.h, which)

    def sync(self):
        _ck(self.L.qx_sync(self.h), "qx_sync")

    # -- hot path --------------------------------------------------------------
    def hpsi_dev(self, cptr, hcptr, nb, flags):
        _ck(self.L.qx_hpsi(self.h, cptr, hcptr, nb, flags), "qx_hpsi")

    def ekinetic(self):
        e = C.c_double()
        ekib = np.empty(self.nb)
        _ck(self.L.qx_ekinetic(self.h, C.addressof(e), ekib.ctypes.data), "qx_ekinetic")
        return e.value, ekib

    def enonloc(self):
        _ck(self.L.qx_enonloc(self.h), "qx_enonloc")

    def hmatrix(self):
        hm = np.empty((self.nb, self.nb))
        _ck(self.L.qx_hmatrix(self.h, hm.ctypes.data), "qx_hmatrix")
        return hm.T.copy()     # column-major -> (row, col)

    def gradres(self):
        prod = np.empty(self.nb)
        zm, zs = C.c_double(), C.c_double()
        _ck(self.L.qx_gradres(self.h, prod.ctypes.data, C.addressof(zm), C.addressof(zs)), "qx_gradres")
        return prod, zm.value, zs.value

    def untryt(self):
        ev = np.empty(self.nb)
        _ck(self.L.qx_untryt(self.h, ev.ctypes.data), "qx_untryt")
        return ev

    def untryhc(self):
        _ck(self.L.qx_untryhc(self.h), "qx_untryhc")

    def eigen(self, parm: CgParm):
        nri = np.zeros(self.nb, dtype=np.int32)
        nh = C.c_int()
        _ck(self.L.qx_eigen(self.h, C.byref(parm), nri.ctypes.data, C.addressof(nh)), "qx_eigen")
        return nri, nh.value

    def schmidt(self):
        _ck(self.L.qx_schmidt(self.h), "qx_schmidt")

    def softchg(self):
        _ck(self.L.qx_softchg(self.h), "qx_softchg")

    # -- SCF -------------------------------------------------------------------
    def scf_init(self, mixbeta=0.3, kerker_q0=1.0):
        s = self.sys
        _ck(self.L.qx_scf_init(self.h, _f64(s.vloc), _f64(s.gs.cross.ravel(order="F")),
                               s.gs.ecutdens, s.eewald, mixbeta, kerker_q0), "qx_scf_init")

    def refine_from(self, src: "Context"):
        """qx_refine_from: take over src's converged state (this context FP64)."""
        _ck(self.L.qx_refine_from(self.h, src.h), "qx_refine_from")

    def autotune(self) -> str:
        """qx_autotune; returns its one-line report."""
        buf = C.create_string_buffer(2048)
        _ck(self.L.qx_autotune(self.h, buf, 2048), "qx_autotune")
        return buf.value.decode()

    def tddft_store(self):
        """Keep the current psi as the previous MD step's wavefunctions."""
        _ck(self.L.qx_tddft_store(self.h), "qx_tddft_store")

    def tddft_overlap(self):
        """aij[i, j] = <prev_i|psi_j> (Gamma metric), (nband, nband)."""
        out = np.zeros((self.nb, self.nb))
        _ck(self.L.qx_tddft_overlap(self.h, out), "qx_tddft_overlap")
        return out.T.copy()   # column-major (i + j nband) -> [i, j]

    def fssh_init(self, parm: FsshParm, occ):
        """qx_fssh_init: start surface hopping on the band window of parm."""
        self._fssh_n = parm.nstate
        _ck(self.L.qx_fssh_init(self.h, C.byref(parm), _f64(occ)), "qx_fssh_init")

    def fssh_step(self, phis=None, eig=None):
        """qx_fssh_step; phis[k, j] = <psi_k(t)|psi_j(t+dt)> (None: the device
        overlap of the kept and the current psi).  Returns (transition None or
        (s, news), occ (nstate), bkl (nstate, 7))."""
        n = getattr(self, "_fssh_n", 1)
        ph = None if phis is None else np.ascontiguousarray(np.asarray(phis, dtype=np.float64).T)
        ev = None if eig is None else _f64(eig)
        occ = np.zeros(n)
        tr = C.c_int(-1)
        bkl = np.zeros((n, 7))
        _ck(self.L.qx_fssh_step(self.h, None if ph is None else ph.ctypes.data,
                                None if ev is None else ev.ctypes.data, occ.ctypes.data, C.addressof(tr),
                                bkl.ctypes.data), "qx_fssh_step")
        return (None if tr.value < 0 else divmod(tr.value, n)), occ, bkl

    def fssh_state(self):
        """(dnr, dni (nstate, 7, 7), accum[news, s], rndx)."""
        n = self._fssh_n
        dnr, dni = np.zeros((n, 7, 7)), np.zeros((n, 7, 7))
        acc = np.zeros((n, n))
        r = C.c_double()
        _ck(self.L.qx_fssh_state(self.h, dnr.ctypes.data, dni.ctypes.data, acc.ctypes.data, C.addressof(r)),
            "qx_fssh_state")
        return dnr, dni, acc.T.copy(), r.value

    def set_kb_builder(self, b: dict):
        """qx_set_kb_builder from the dict of cell.kb_builder_tables."""
        _ck(self.L.qx_set_kb_builder(self.h, b["ntype"], b["lmx"], b["mxqlm"], _f64(b["dlqlm"]), _f64(b["tbqlm"]),
                                     b["nlm"], _f64(b["qlm"]), np.ascontiguousarray(b["lmidx"], dtype=np.int32),
                                     np.ascontiguousarray(b["even"], dtype=np.int32), _f64(b["vclalp"]),
                                     np.ascontiguousarray(b["ngabc"], dtype=np.int32)), "qx_set_kb_builder")

    def build_kb_g(self, ityp, satm):
        """qx_build_kb_g: the G-space KB tables of the geometry satm (natom, 3) fractional."""
        satm = _f64(satm)
        _ck(self.L.qx_build_kb_g(self.h, satm.shape[0], np.ascontiguousarray(ityp, dtype=np.int32), satm),
            "qx_build_kb_g")

    def get_kb_g(self, nproj):
        """(eqlmr_ (nplwex, nproj), vclalp (nproj)) read back from the device."""
        tab = np.zeros((nproj, self.ne))
        vcl = np.zeros(nproj)
        _ck(self.L.qx_get_kb_g(self.h, tab, vcl), "qx_get_kb_g")
        return tab.T.copy(), vcl

    def set_kb_r_builder(self, b: dict):
        """qx_set_kb_r_builder from the dict of cell.kbr_builder_tables."""
        dt = _f64(b["dtabnl"]) if b.get("dtabnl") is not None else None
        lmx = int(b.get("lmx", 4))
        _ck(self.L.qx_set_kb_r_builder(self.h, b["ntype"], lmx, b["mxnl"], _f64(b["dltnl"]), _f64(b["rcut"]),
                                       _f64(b["tabnl"]), None if dt is None else dt.ctypes.data,
                                       np.ascontiguousarray(b["poly"], dtype=np.int32),
                                       _f64(b["clalp"]), b["rdelv"], _f64(b["rba"])), "qx_set_kb_r_builder")
        self._kbr_lmx = lmx
        if b.get("rcut_l") is not None:
            self.set_kb_r_channel_radii(b["rcut_l"])

    def set_kb_r_channel_radii(self, rcl):
        """qx_set_kb_r_channel_radii: rcl (lmx * ntype,) radius of each projector's channel."""
        _ck(self.L.qx_set_kb_r_channel_radii(self.h, _f64(rcl)), "qx_set_kb_r_channel_radii")

    def forces_nl_r(self):
        """Real-space KB forces (natom, 3) Ry/bohr of the current psi."""
        f = np.zeros(3 * self.sys.cell.natom)
        _ck(self.L.qx_forces_nl_r(self.h, f), "qx_forces_nl_r")
        return f.reshape(-1, 3)

    def build_kb_r(self, ityp, satm):
        """qx_build_kb_r: the real-space KB tables of the geometry satm (natom, 3) fractional."""
        satm = _f64(satm)
        _ck(self.L.qx_build_kb_r(self.h, satm.shape[0], np.ascontiguousarray(ityp, dtype=np.int32), satm),
            "qx_build_kb_r")

    def get_kb_r(self, natom):
        """(off (natom+1), mesh (npts), vnl (npts, lmx)) read back from the device."""
        n = C.c_int(0)
        _ck(self.L.qx_get_kb_r(self.h, C.byref(n), None, None, None), "qx_get_kb_r")
        off = np.zeros(natom + 1, dtype=np.int32)
        mesh = np.zeros(max(n.value, 1), dtype=np.int32)
        vnl = np.zeros((max(n.value, 1), self._kbr_lmx))
        _ck(self.L.qx_get_kb_r(self.h, C.byref(n), off.ctypes.data, mesh.ctypes.data, vnl.ctypes.data),
            "qx_get_kb_r")
        return off, mesh[: n.value], vnl[: n.value]

    def set_force_tables(self):
        """qx_set_force_tables from the system's geometry (one species)."""
        t = cell.force_tables(self.sys)
        _ck(self.L.qx_set_force_tables(self.h, t["natom"], t["ntype"], np.ascontiguousarray(t["ityp"], dtype=np.int32),
                                       _f64(t["satm"]), t["n5"], np.ascontiguousarray(t["ijk5"], dtype=np.int32),
                                       np.ascontiguousarray(t["ngabc"], dtype=np.int32), _f64(t["gvec5"]),
                                       _f64(t["svco"]), _f64(t["gw"])), "qx_set_force_tables")

    def build_vloc(self):
        """qx_build_vloc: the local pseudopotential of the force tables' geometry."""
        _ck(self.L.qx_build_vloc(self.h), "qx_build_vloc")

    def forces(self):
        """(floc, fnl) of the current psi, each (natom, 3) Ry/bohr."""
        nat = self.sys.cell.natom
        fl = np.zeros((nat, 3))
        fn = np.zeros((nat, 3))
        _ck(self.L.qx_forces(self.h, fl, fn), "qx_forces")
        return fl, fn

    def kbnlpp_frc2_host(self, cgjr):
        """qxgpu_kbnlpp_frc2: the G-space KB forces of host wavefunctions."""
        out = np.zeros((self.sys.cell.natom, 3))
        _ck(self.L.qxgpu_kbnlpp_frc2(self.h, _f64(cgjr), out), "qxgpu_kbnlpp_frc2")
        return out

    def scf_mixing(self, itratn=10, cmetric=20.0):
        """Pulay mixing with the reference defaults (itratn 10, cmetric 20);
        itratn <= 1 returns to Kerker-filtered linear mixing."""
        _ck(self.L.qx_scf_mixing(self.h, int(itratn), float(cmetric)), "qx_scf_mixing")

    def scf_rho_from_psi(self):
        _ck(self.L.qx_scf_rho_from_psi(self.h), "qx_scf_rho_from_psi")

    def scf_launch(self, parm: CgParm):
        """Enqueue one SCF iteration on this context's stream."""
        _ck(self.L.qx_scf_launch(self.h, C.byref(parm)), "qx_scf_launch")

    def scf_result(self) -> dict:
        out = ScfOut()
        _ck(self.L.qx_scf_result(self.h, C.byref(out)), "qx_scf_result")
        return out.asdict()

    def scf_iteration(self, parm: CgParm) -> dict:
        out = ScfOut()
        _ck(self.L.qx_scf_iteration(self.h, C.byref(parm), C.byref(out)), "qx_scf_iteration")
        return out.asdict()

    def scf_iteration_host(self, parm: CgParm, psi_in=None, psi_out=None, rho_out=None, eig_out=None) -> dict:
        """qx_scf_iteration_host on host float64 arrays (C-contiguous; the
        outputs are written in place; None skips one)."""
        def ptr(a, n, out):
            if a is None:
                return None
            assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"] and a.size == n
            assert not out or a.flags["WRITEABLE"]
            return a.ctypes.data
        n = self.nb * self.sys.gs.nplwex
        out = ScfOut()
        _ck(self.L.qx_scf_iteration_host(self.h, C.byref(parm), C.byref(out), ptr(psi_in, n, False),
                                         ptr(psi_out, n, True), ptr(rho_out, self.sys.gs.kfft0, True),
                                         ptr(eig_out, self.nb, True)), "qx_scf_iteration_host")
        return out.asdict()

    # -- drop-in shims (host arrays) ----------------------------------------
    def hcnonloc_host(self, cgjr, rhcr):
        out = _f64(rhcr).copy()
        _ck(self.L.qxgpu_hcnonloc(self.h, _f64(cgjr), out, cgjr.shape[0]), "qxgpu_hcnonloc")
        return out

    def hckbpp_g_host(self, cgjr, rhcr):
        out = _f64(rhcr).copy()
        _ck(self.L.qxgpu_hckbpp_g(self.h, _f64(cgjr), out, cgjr.shape[0]), "qxgpu_hckbpp_g")
        return out

    def enonloc_host(self, cgjr):
        out = np.empty_like(_f64(cgjr))
        ekib = np.empty(self.nb)
        _ck(self.L.qxgpu_enonloc(self.h, _f64(cgjr), out, ekib.ctypes.data), "qxgpu_enonloc")
        return out, ekib

    def eigen_host(self, gdcr, rhcr, ekib, parm):
        x = _f64(gdcr).copy()
        hx = _f64(rhcr).copy()
        eig = np.empty(self.nb)
        ek = _f64(ekib)
        _ck(self.L.qxgpu_eigen(self.h, x, hx, ek.ctypes.data, eig.ctypes.data, C.byref(parm)), "qxgpu_eigen")
        return x, hx, eig

    def schmidt_host(self, cgjr):
        x = _f64(cgjr).copy()
        _ck(self.L.qxgpu_schmidt(self.h, x), "qxgpu_schmidt")
        return x

    def softchg_host(self, cgjr):
        rho = np.empty(self.n)
        _ck(self.L.qxgpu_softchg(self.h, _f64(cgjr), rho), "qxgpu_softchg")
        return rho

    def rfft3_host(self, key, fft3x, fft3y):
        x = _f64(fft3x).copy()
        y = _f64(fft3y).copy()
        _ck(self.L.qxgpu_rfft3(self.h, key, x, y), "qxgpu_rfft3")
        return x, y
