"""ORACLE -- test infrastructure only.  One SCF iteration in the order of
pwlda_md (pwlda.f90:1628-3700) on the C oracle's hot-path routines, with the
density side (Hartree harting engrad.f90:1673-1743, PZ LDA vxc.f90:961-1018,
Kerker-filtered linear mixing) restated in numpy.  Checker for the device
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


class ScfState:
    def __init__(self, sys, psi, nlmode=1, mixbeta=0.3, kerker_q0=1.0):
        self.sys = sys
        self.ham = Ham(sys, nlmode)
        self.psi = np.array(psi, dtype=np.float64)
        self.g2 = grid_g2(sys.gs)
        self.beta = mixbeta
        self.q02 = kerker_q0 ** 2
        self.rho_in = self.ham.softchg(self.psi, sys.occ)

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

    def iteration(self, noband, itermx=4, iteremx=4):
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
        psi, hc, eig, _, nri = self.ham.eigen(psi, hc, ekib, noband, itermx=itermx, iteremx=iteremx)
        psi, _, rc = schmidt(psi)
        if rc:
            raise RuntimeError(f"oracle schmidt: not positive definite ({rc})")
        rho_out = self.ham.softchg(psi, sys.occ)
        d = rho_out - self.rho_in
        resid = float(np.sum(d * d) * sys.gs.rvol / sys.gs.kfft0)
        dg = self._fft(d)
        f = np.zeros_like(self.g2)
        m = self.g2 > 0
        f[m] = self.g2[m] / (self.g2[m] + self.q02)
        self.rho_in = self.rho_in + self.beta * self._ifft(dg * f).real
        self.psi = psi
        return dict(etot=eband - eh + exc - evxc + sys.eewald, eband=eband, ehartree=eh, exc=exc,
                    evxc=evxc, resid=resid, ncg_hpsi=int(nri.sum()), jacobi_sweeps=sweeps, eig=eig)
