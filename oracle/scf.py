"""ORACLE -- test infrastructure only.  One SCF iteration in the order of
pwlda_md (pwlda.f90:1628-3700) on the C oracle's hot-path routines, with the
density side (Hartree harting engrad.f90:1673-1743, PZ LDA vxc.f90:961-1018,
Kerker-filtered linear mixing or Pulay mixing mxchgg_pulay
chgdns.f90:954-1120) restated in numpy.  Checker for the device
qx_scf_iteration.  PARITY UNPINNED (see qxmd_oracle.c).
"""
from __future__ import annotations

import math

import numpy as np

from . import Ham, hmatrix, jacobi, rotate, schmidt, xclda


def grid_g2(gs):
    """|G|^2 on the FFT grid, -1 outside the density sphere (qx_scf.cu k_grid_g2)."""
    k1, k2, k3 = gs.grid
    i1 = np.arange(k1)
    i2 = np.arange(k2)
    i3 = np.arange(k3)
    d1 = np.where(i1 <= k1 // 2, i1, i1 - k1).astype(float)
    d2 = np.where(i2 <= k2 // 2, i2, i2 - k2).astype(float)
    d3 = np.where(i3 <= k3 // 2, i3, i3 - k3).astype(float)
    D3, D2, D1 = np.meshgrid(d3, d2, d1, indexing="ij")
    c = gs.cross
    gx = c[0, 0] * D1 + c[0, 1] * D2 + c[0, 2] * D3
    gy = c[1, 0] * D1 + c[1, 1] * D2 + c[1, 2] * D3
    gz = c[2, 0] * D1 + c[2, 1] * D2 + c[2, 2] * D3
    s = (gx * gx + gy * gy + gz * gz).ravel()
    return np.where(s <= gs.ecutdens, s, -1.0)


def pulay_factq1(g2, cmetric):
    """Metric parameter of the mixing residual (mxchgg_alloc, chgdns.f90:661-668):
    w(G) = (G^2 + q1)/G^2 with q1 from the smallest and largest nonzero |G|^2 of
    the density sphere (reclat.f90:205)."""
    m = g2 > 0
    g2min, g2max = float(g2[m].min()), float(g2[m].max())
    bbb = g2max - cmetric * g2min
    return (cmetric - 1.0) * g2max * g2min / bbb if bbb > 1.0e-5 else 0.0


def invers(a):
    """INVERS (funcs.f90:1-56): inverse of a, error 1 when the determinant of
    a / max|a_ij| is below 1e-30."""
    elmax = np.abs(a).max()
    if abs(np.linalg.det(a / elmax)) < 1.0e-30:
        return None
    return np.linalg.inv(a / elmax) / elmax


class Pulay:
    """mxchgg_pulay (chgdns.f90:954-1120) with lmixhold = .false.: history of
    input densities u_i and residuals d_i = rho_out - rho_in in G space, the
    metric a_ij = Omega sum_{G != 0} Re(d_i^* d_j) (G^2 + q1)/G^2, new density
    sum_i c_i (u_i + K(G) d_i) with c = rowsums(A^-1)/sum(A^-1) and
    K(G) = aslh G^2/(G^2 + bslh).  A singular A drops the oldest entry; a
    tiny centre element restarts the history; after itratn entries the next
    call starts over with one Kerker step."""

    def __init__(self, g2, rvol, itratn=10, aslh=0.8, bslh=0.64, cmetric=20.0):
        self.m = g2 > 0
        self.w = np.zeros_like(g2)
        q1 = pulay_factq1(g2, cmetric)
        self.w[self.m] = (g2[self.m] + q1) / g2[self.m]
        self.k = np.zeros_like(g2)
        self.k[self.m] = aslh * g2[self.m] / (g2[self.m] + bslh)
        self.rvol, self.itratn = rvol, itratn
        self.u, self.d = [], []
        self.reset_next = True

    def dot(self, a, b):
        return self.rvol * float(np.sum((np.conj(a) * b).real * self.w))

    def mix(self, rin_g, rout_g):
        if self.reset_next or len(self.u) >= self.itratn:
            self.u, self.d = [], []
            self.reset_next = False
        d = np.where(self.m, rout_g - rin_g, 0.0)
        self.u.append(rin_g.copy())
        self.d.append(d)
        while True:
            n = len(self.u)
            if n == 1:
                c = np.ones(1)
                break
            a = np.array([[self.dot(x, y) for y in self.d] for x in self.d])
            amax = abs(a[(n + 1) // 2 - 1, (n + 1) // 2 - 1])
            if amax < 1.0e-15:
                self.u, self.d = self.u[-1:], self.d[-1:]
                continue
            inv = invers(a / amax)
            if inv is None:
                self.u, self.d = self.u[1:], self.d[1:]
                continue
            c = inv.sum(axis=1) / inv.sum()
            break
        new = sum(ci * (u + self.k * d) for ci, u, d in zip(c, self.u, self.d))
        if len(self.u) == self.itratn:
            self.reset_next = True
        return new


class ScfState:
    def __init__(self, sys, psi, nlmode=1, mixbeta=0.3, kerker_q0=1.0, pulay=0, cmetric=20.0):
        self.sys = sys
        self.ham = Ham(sys, nlmode)
        self.psi = np.array(psi, dtype=np.float64)
        self.g2 = grid_g2(sys.gs)
        self.beta = mixbeta
        self.q02 = kerker_q0 ** 2
        self.rho_in = self.ham.softchg(self.psi, sys.occ)
        self.pulay = Pulay(self.g2, sys.gs.rvol, pulay, mixbeta, self.q02, cmetric) if pulay > 1 else None

    def _fft(self, r):
        k1, k2, k3 = self.sys.gs.grid
        return np.fft.fftn(r.reshape(k3, k2, k1)).ravel() / r.size

    def _ifft(self, z):
        k1, k2, k3 = self.sys.gs.grid
        return np.fft.ifftn(z.reshape(k3, k2, k1)).ravel() * z.size

    def potential(self):
        gs = self.sys.gs
        rg = self._fft(self.rho_in)
        m = self.g2 > 0
        vg = np.zeros_like(rg)
        vg[m] = 8.0 * math.pi * rg[m] / self.g2[m]
        eh = 0.5 * gs.rvol * np.sum((vg * np.conj(rg)).real)
        vh = self._ifft(vg).real
        vxc, _, en = xclda(self.rho_in, gs.rvol / gs.kfft0)
        glocal = self.sys.vloc + vh + vxc
        return glocal, eh, en[0] + en[2], en[1] + en[3]

    def iteration(self, noband, itermx=4, iteremx=4, sequential=False):
        sys = self.sys
        glocal, eh, exc, evxc = self.potential()
        self.ham.set_glocal(glocal)
        hc = self.ham.hpsi(self.psi)
        _, ekib = self.ham.ekinetic(self.psi)
        hm, _ = hmatrix(self.psi, hc)
        w, u, sweeps = jacobi(hm)
        psi = rotate(self.psi, u)
        hc = rotate(hc, u)
        eband = float(np.sum(sys.occ[: w.size] * w))
        psi, hc, eig, _, nri = self.ham.eigen(psi, hc, ekib, noband, itermx=itermx, iteremx=iteremx,
                                              sequential=sequential)
        psi, _, rc = schmidt(psi)
        if rc:
            raise RuntimeError(f"oracle schmidt: not positive definite ({rc})")
        rho_out = self.ham.softchg(psi, sys.occ)
        d = rho_out - self.rho_in
        resid = float(np.sum(d * d) * sys.gs.rvol / sys.gs.kfft0)
        if self.pulay is not None:
            self.rho_in = self._ifft(self.pulay.mix(self._fft(self.rho_in), self._fft(rho_out))).real
        else:
            dg = self._fft(d)
            f = np.zeros_like(self.g2)
            m = self.g2 > 0
            f[m] = self.g2[m] / (self.g2[m] + self.q02)
            self.rho_in = self.rho_in + self.beta * self._ifft(dg * f).real
        self.psi = psi
        return dict(etot=eband - eh + exc - evxc + sys.eewald, eband=eband, ehartree=eh, exc=exc,
                    evxc=evxc, resid=resid, ncg_hpsi=int(nri.sum()), jacobi_sweeps=sweeps, eig=eig)
