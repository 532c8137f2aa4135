"""ORACLE -- test infrastructure only (the checker, never the product).

ctypes front end to ``qxmd_oracle.c``, the CPU FP64 restatement of QXMD's
Kohn-Sham hot path.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
``cpu_baseline`` leg import this package.

PARITY UNPINNED: the reference (Fortran + FFTW 3.3.8) cannot be built here and
ships no golden vectors; see the header of qxmd_oracle.c.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_cp = np.ctypeslib.ndpointer(dtype=np.complex128, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile the oracle with gcc into oracle/_build/liboracle.so."""
    src = os.path.join(_HERE, "qxmd_oracle.c")
    if not force and os.path.exists(_SO) and os.path.getmtime(_SO) >= os.path.getmtime(src):
        return _SO
    os.makedirs(os.path.dirname(_SO), exist_ok=True)
    # -ffp-contract=off keeps every multiply and add as written; -fopenmp
    # runs the band loops on host threads (results independent of the count).
    tmp = _SO + ".tmp"
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", "-fopenmp",
                           "-ffp-contract=off", "-o", tmp, src, "-lm"])
    os.replace(tmp, _SO)
    return _SO


class _Ham(C.Structure):
    _fields_ = [("k1", C.c_int), ("k2", C.c_int), ("k3", C.c_int),
                ("nplw", C.c_int), ("nplwex", C.c_int),
                ("ijk_pos", C.c_void_p), ("ijk_neg", C.c_void_p),
                ("dkgnrm", C.c_void_p), ("glocal", C.c_void_p),
                ("nlmode", C.c_int), ("nproj", C.c_int),
                ("kbg", C.c_void_p), ("vclalp", C.c_void_p),
                ("natom", C.c_int), ("lmx", C.c_int),
                ("off", C.c_void_p), ("mesh", C.c_void_p),
                ("vnl", C.c_void_p), ("clalp", C.c_void_p),
                ("rdelv", C.c_double)]


class _CGParm(C.Structure):
    _fields_ = [("itermx", C.c_int), ("iteremx", C.c_int), ("noband", C.c_int),
                ("tolera", C.c_double), ("roughfzan", C.c_double),
                ("roughfeig", C.c_double), ("threinn", C.c_double),
                ("wdinner", C.c_double), ("ccreal4", C.c_int), ("sequential", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        L.orc_fft3.argtypes = [_cp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_fft1.argtypes = [_cp, C.c_int, C.c_int]
        L.orc_dot.argtypes = [_dp, _dp, C.c_int]
        L.orc_dot.restype = C.c_double
        L.orc_wvg2r.argtypes = [_dp, C.c_int, _ip, _ip, C.c_int, C.c_int, C.c_int, _dp]
        L.orc_hpsi.argtypes = [C.POINTER(_Ham), _dp, _dp, C.c_int]
        L.orc_hcnonloc.argtypes = [C.POINTER(_Ham), _dp, _dp]
        L.orc_hckbpp.argtypes = [C.POINTER(_Ham), _dp, _dp, C.c_void_p]
        L.orc_calnlc.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, _dp, C.c_double, _dp, _dp, C.c_void_p]
        L.orc_ekinetic.argtypes = [C.POINTER(_Ham), _dp, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_ekinetic.restype = C.c_double
        L.orc_eigen_bkl.argtypes = [C.POINTER(_Ham), C.POINTER(_CGParm), C.c_int, _dp, _dp, _dp,
                                    _dp, _dp, _ip]
        L.orc_cholinv.argtypes = [_dp, C.c_int]
        L.orc_cholinv.restype = C.c_int
        L.orc_schmidt.argtypes = [_dp, C.c_int, C.c_int, C.c_void_p]
        L.orc_schmidt.restype = C.c_int
        L.orc_hmatrix.argtypes = [_dp, _dp, C.c_int, C.c_int, _dp, _dp]
        L.orc_gradres.argtypes = [_dp, _dp, _dp, _dp, C.c_int, C.c_int, _dp,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_jacobi.argtypes = [_dp, C.c_int, _dp, _dp, C.c_int]
        L.orc_jacobi.restype = C.c_int
        L.orc_rotate.argtypes = [_dp, C.c_int, C.c_int, _dp]
        L.orc_softchg.argtypes = [C.POINTER(_Ham), _dp, C.c_int, _dp, C.c_double, _dp]
        L.orc_xclda.argtypes = [_dp, C.c_long, C.c_double, _dp, C.c_void_p, _dp]
        L.orc_fssh_dm.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                                  _dp, _dp, _dp, _dp, C.POINTER(C.c_double), C.c_void_p]
        L.orc_fssh_dm.restype = C.c_int
        L.orc_rnd00.argtypes = [C.POINTER(C.c_double)]
        L.orc_rnd00.restype = C.c_double
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
    return _lib


def set_threads(n: int) -> None:
    """Host threads of the oracle's band loops (results do not depend on it)."""
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Fssh:
    """State of tddft_fssh_dm (tddft_fssh.f90:1989-2402) for a window of nst
    states: density matrices dn (nst, 7, 7) complex (initially 1 at the centre),
    accumulated probabilities accum[news, s], occupations and the rnd00 state."""

    def __init__(self, occ, seed, dtmd, dttddft=0.02, boltzmann=True, treq=0.0019, hop=True):
        self.nst = len(occ)
        self.dnr = np.zeros((self.nst, 7, 7))
        self.dni = np.zeros((self.nst, 7, 7))
        self.dnr[:, 3, 3] = 1.0
        self.accum = np.zeros((self.nst, self.nst), order="F")
        self.occ = np.array(occ, dtype=np.float64)
        self.rndx = C.c_double(seed)
        self.dtmd, self.dttddft, self.boltz, self.treq, self.hop = dtmd, dttddft, boltzmann, treq, hop

    def step(self, phis, eig):
        """One MD step; phis[k, j] = <psi_k(t)|psi_j(t+dt)>.  Returns
        (transition: None or (s, news), bkl (nst, 7))."""
        bkl = np.zeros((self.nst, 7))
        acc = np.ascontiguousarray(self.accum.T)          # [s, news] row-major = (news, s) column-major
        ph = np.ascontiguousarray(np.asarray(phis, dtype=np.float64).T)   # column-major phis(k, j)
        t = lib().orc_fssh_dm(self.nst, ph, _f64(eig), self.dtmd, self.dttddft, int(self.boltz), self.treq,
                              int(self.hop), self.dnr, self.dni, acc, self.occ, C.byref(self.rndx),
                              bkl.ctypes.data)
        self.accum = acc.T.copy()
        return (None if t < 0 else divmod(t, self.nst)), bkl


def rnd00(rndx: float, n: int):
    """n successive draws of the Park-Miller rnd00 from state rndx."""
    x = C.c_double(rndx)
    return np.array([lib().orc_rnd00(C.byref(x)) for _ in range(n)])


class Ham:
    """Oracle Hamiltonian built from a qxmd_b200.cell.System.

    nlmode: 0 no nonlocal part, 1 G-space KB (hckbpp_ib_g), 2 real-space KB (calnlc).
    """

    def __init__(self, sys, nlmode: int = 1, glocal=None):
        gs = sys.gs
        self.sys = sys
        self.nplwex = gs.nplwex
        self._keep = {
            "ijk_pos": np.ascontiguousarray(gs.ijk_pos, dtype=np.int32),
            "ijk_neg": np.ascontiguousarray(gs.ijk_neg, dtype=np.int32),
            "dkgnrm": _f64(gs.dkgnrm()),
            "glocal": _f64(sys.vloc if glocal is None else glocal),
            "kbg": _f64(sys.kb_g.T),             # projector-major
            "vclalp": _f64(sys.vclalp),
            "off": np.ascontiguousarray(sys.kb_r.off, dtype=np.int32),
            "mesh": np.ascontiguousarray(sys.kb_r.mesh, dtype=np.int32),
            "vnl": _f64(sys.kb_r.vnl),
            "clalp": _f64(sys.kb_r.clalp),
        }
        k = self._keep
        h = _Ham()
        h.k1, h.k2, h.k3 = gs.grid
        h.nplw, h.nplwex = gs.nplw, gs.nplwex
        h.ijk_pos = k["ijk_pos"].ctypes.data
        h.ijk_neg = k["ijk_neg"].ctypes.data
        h.dkgnrm = k["dkgnrm"].ctypes.data
        h.glocal = k["glocal"].ctypes.data
        h.nlmode = nlmode
        h.nproj = sys.kb_g.shape[1]
        h.kbg = k["kbg"].ctypes.data
        h.vclalp = k["vclalp"].ctypes.data
        h.natom = sys.cell.natom
        h.lmx = int(k["vnl"].shape[1]) if k["vnl"].ndim == 2 else sys.pp.lmx   # projectors per point
        h.off = k["off"].ctypes.data
        h.mesh = k["mesh"].ctypes.data
        h.vnl = k["vnl"].ctypes.data
        h.clalp = k["clalp"].ctypes.data
        h.rdelv = sys.kb_r.rdelv
        self.h = h

    def set_glocal(self, glocal):
        self._keep["glocal"] = _f64(glocal)
        self.h.glocal = self._keep["glocal"].ctypes.data

    # -- hot-path routines ---------------------------------------------------
    def hpsi(self, c):
        c = _f64(c)
        nb = c.shape[0]
        hc = np.zeros_like(c)
        lib().orc_hpsi(C.byref(self.h), c, hc, nb)
        return hc

    def hcnonloc(self, c, rhcr):
        out = _f64(rhcr).copy()
        lib().orc_hcnonloc(C.byref(self.h), _f64(c), out)
        return out

    def hckbpp(self, c, rhcr):
        out = _f64(rhcr).copy()
        slm = np.zeros(self.h.nproj)
        lib().orc_hckbpp(C.byref(self.h), _f64(c), out, slm.ctypes.data)
        return out, slm

    def ekinetic(self, c, occ=None):
        c = _f64(c)
        ekib = np.zeros(c.shape[0])
        occ_a = None if occ is None else _f64(occ)
        e = lib().orc_ekinetic(C.byref(self.h), c, c.shape[0],
                               None if occ_a is None else occ_a.ctypes.data, ekib.ctypes.data)
        return e, ekib

    def eigen(self, gdcr, rhcr, ekib, noband, itermx=4, iteremx=4, tolera=1e-10,
              roughfzan=0.3, roughfeig=0.3, threinn=0.0, wdinner=0.9, ccreal4=False,
              sequential=False):
        x = _f64(gdcr).copy()
        hx = _f64(rhcr).copy()
        nb = x.shape[0]
        p = _CGParm(itermx, iteremx, noband, tolera, roughfzan, roughfeig, threinn, wdinner,
                    int(ccreal4), int(sequential))
        eig = np.zeros(nb)
        bzan = np.zeros(nb)
        nri = np.zeros(nb, dtype=np.int32)
        lib().orc_eigen_bkl(C.byref(self.h), C.byref(p), nb, x, hx, _f64(ekib), eig, bzan, nri)
        return x, hx, eig, bzan, nri

    def softchg(self, c, occ):
        rho = np.zeros(self.sys.gs.kfft0)
        c = _f64(c)
        lib().orc_softchg(C.byref(self.h), c, c.shape[0], _f64(occ), self.sys.gs.rvol, rho)
        return rho


def fft3(a, grid, sign):
    """Unscaled 3D transform of a (k3,k2,k1)-shaped or flat complex grid."""
    z = np.ascontiguousarray(a, dtype=np.complex128).ravel().copy()
    lib().orc_fft3(z, grid[0], grid[1], grid[2], sign)
    return z


def wvg2r(gs, c):
    out = np.zeros(gs.kfft0)
    lib().orc_wvg2r(_f64(c), gs.nplw, np.ascontiguousarray(gs.ijk_pos, dtype=np.int32),
                    np.ascontiguousarray(gs.ijk_neg, dtype=np.int32), *gs.grid, out)
    return out


def calnlc(kbr, lmx, natom, psir):
    apk = np.zeros_like(_f64(psir))
    sumr = np.zeros(natom * lmx)
    lib().orc_calnlc(natom, lmx, np.ascontiguousarray(kbr.off, dtype=np.int32),
                     np.ascontiguousarray(kbr.mesh, dtype=np.int32), _f64(kbr.vnl),
                     _f64(kbr.clalp), kbr.rdelv, _f64(psir), apk, sumr.ctypes.data)
    return apk, sumr


def dot(x, y):
    return lib().orc_dot(_f64(x), _f64(y), x.shape[-1])


def cholinv(s):
    """Lower-triangular L^-1 of S = L L^T (column-major semantics); returns (Linv, rc)."""
    n = s.shape[0]
    a = np.asfortranarray(_f64(s)).ravel(order="F").copy()
    rc = lib().orc_cholinv(a, n)
    return a.reshape(n, n, order="F"), rc


def schmidt(c):
    c = _f64(c).copy()
    nb, ne = c.shape
    linv = np.zeros(nb * nb)
    rc = lib().orc_schmidt(c, ne, nb, linv.ctypes.data)
    return c, linv.reshape(nb, nb, order="F"), rc


def hmatrix(c, hc):
    c = _f64(c)
    nb, ne = c.shape
    hm = np.zeros(nb * nb)
    eig = np.zeros(nb)
    lib().orc_hmatrix(c, _f64(hc), ne, nb, hm, eig)
    return hm.reshape(nb, nb, order="F"), eig


def gradres(c, hc, eig, occ):
    c = _f64(c)
    nb, ne = c.shape
    prod = np.zeros(nb)
    zm = C.c_double()
    zs = C.c_double()
    lib().orc_gradres(c, _f64(hc), _f64(eig), _f64(occ), ne, nb, prod, C.byref(zm), C.byref(zs))
    return prod, zm.value, zs.value


def jacobi(a, maxsweep=60):
    n = a.shape[0]
    aa = np.asfortranarray(_f64(a)).ravel(order="F").copy()
    w = np.zeros(n)
    v = np.zeros(n * n)
    sw = lib().orc_jacobi(aa, n, w, v, maxsweep)
    return w, v.reshape(n, n, order="F"), sw


def rotate(c, u):
    c = _f64(c).copy()
    nb, ne = c.shape
    lib().orc_rotate(c, ne, nb, np.asfortranarray(_f64(u)).ravel(order="F").copy())
    return c


def xclda(rho, rdelv):
    rho = _f64(rho)
    v = np.zeros_like(rho)
    e = np.zeros_like(rho)
    en = np.zeros(4)
    lib().orc_xclda(rho, rho.size, rdelv, v, e.ctypes.data, en)
    return v, e, en
