"""ORACLE -- test infrastructure only.  Hellmann-Feynman forces restated in
numpy (FP64) from the reference:

* flocal_g (nlkbpp.f90:1037-1120): local pseudopotential in G space,
  F_a = 2 sum_{G != 0} svco(G) (Re rho(G) sin(G.R_a) + Im rho(G) cos(G.R_a)) G,
  cos/sin(G.R_a) from the per-dimension recurrence of stscfn
  (bulk.f90:2086-2175);
* kbnlpp_frc2 (nlkbpp.f90:1878-2130, the lbigmm2 branch with the eqlmr_
  table): for every band n, projector l of atom a,
  fsl = sum_{g >= 1} (beta(2g) psi(2g+1) - beta(2g+1) psi(2g)) G(g),
  F_a += 2 * fsl * slmir * occ_n * 2 * vclalp_l, slmir = <beta|psi> with the
  KB metric 2 sum - b0 c0 - 2 b1 c1 (hckbpp_ib_g, nlkbpp.f90:1678-1713);
* fnnlcl2 (nlkbppr.f90:2024-3120): real-space KB on the projector points of
  setnlc, F_a = 2 sum_n occ_n / Omega sum_l clalp_l P_l D_l with P_l and its
  gradient sum D_l over the fixed point set.

The ion-ion term is qxmd_b200.cell.ewald_forces.  PARITY UNPINNED (see
qxmd_oracle.c); the sum of the three terms is pinned by central differences
of the self-consistent total energy in the CPU tests.
"""
from __future__ import annotations

import math

import numpy as np


def phase_tables(satm: np.ndarray, kmax: int):
    """dcq/dsq[a, dim, k + kmax] = cos/sin(2 pi k s_dim(a)) by the angle-addition
    recurrence of stscfn."""
    nat = satm.shape[0]
    dcq = np.zeros((nat, 3, 2 * kmax + 1))
    dsq = np.zeros((nat, 3, 2 * kmax + 1))
    for a in range(nat):
        for d in range(3):
            ph = satm[a, d] * 2.0 * math.pi
            c1, s1 = math.cos(ph), math.sin(ph)
            dcq[a, d, kmax] = 1.0
            if kmax >= 1:
                dcq[a, d, kmax + 1] = c1
                dsq[a, d, kmax + 1] = s1
                dcq[a, d, kmax - 1] = c1
                dsq[a, d, kmax - 1] = -s1
            cp, sp = c1, s1
            for k in range(2, kmax + 1):
                cn, sn = c1 * cp - s1 * sp, s1 * cp + c1 * sp
                dcq[a, d, kmax + k], dsq[a, d, kmax + k] = cn, sn
                dcq[a, d, kmax - k], dsq[a, d, kmax - k] = cn, -sn
                cp, sp = cn, sn
    return dcq, dsq


def floc_g(t: dict, rho_r: np.ndarray, grid) -> np.ndarray:
    """flocal_g on the density rho(r) (flat grid, k1 fastest); (natom, 3) Ry/bohr."""
    k1, k2, k3 = grid
    rg = (np.fft.fftn(rho_r.reshape(k3, k2, k1)) / rho_r.size).ravel()
    ng = t["ngabc"]
    kmax = int(np.abs(ng).max())
    dcq, dsq = phase_tables(t["satm"], kmax)
    r = rg[t["ijk5"]]
    f = np.zeros((t["natom"], 3))
    g = slice(1, t["n5"])
    k = ng[g] + kmax
    for a in range(t["natom"]):
        c1, c2, c3 = dcq[a, 0, k[:, 0]], dcq[a, 1, k[:, 1]], dcq[a, 2, k[:, 2]]
        s1, s2, s3 = dsq[a, 0, k[:, 0]], dsq[a, 1, k[:, 1]], dsq[a, 2, k[:, 2]]
        cc12 = c1 * c2 - s1 * s2
        sc12 = s1 * c2 + c1 * s2
        zc = cc12 * c3 - sc12 * s3
        zs = sc12 * c3 + cc12 * s3
        ftmp = t["svco"][g] * (r[g].real * zs + r[g].imag * zc)
        f[a] = 2.0 * (ftmp[:, None] * t["gvec5"][g]).sum(axis=0)
    return f


def fnl_r(off: np.ndarray, mesh: np.ndarray, vnl: np.ndarray, dvnl: np.ndarray, clalp: np.ndarray,
          rdelv: float, rvol: float, psir: np.ndarray, occ: np.ndarray) -> np.ndarray:
    """fnnlcl2 (nlkbppr.f90:2024-3120): real-space KB forces (natom, 3) Ry/bohr
    on a fixed point set.  For band n with psi_n(r) (psir (nb, kfft0), the
    unscaled inverse transform wvg2r) and atom a:
      sumr_l = clalp_l P_l,  P_l = rdelv sum_points vnl_l psi_n  (svsumr of calnlc),
      sumxr_l = D_l = rdelv sum_points grad vnl_l psi_n,
      F_a += sum_l sumr_l sumxr_l * 2 occ_n / Omega       (nlkbppr.f90:3025-3043).
    vnl (npts, 4) and dvnl (npts, 4, 3) from oracle.tables.setnlc(grad=True)."""
    nat = off.size - 1
    lmx = vnl.shape[1]
    f = np.zeros((nat, 3))
    for n in range(psir.shape[0]):
        if abs(occ[n]) <= 1e-15:
            continue
        w = 2.0 * occ[n] / rvol
        for a in range(nat):
            sl = slice(off[a], off[a + 1])
            ps = psir[n, mesh[sl]]
            p = rdelv * (ps @ vnl[sl])                               # (lmx,)
            dd = rdelv * np.einsum("p,plx->lx", ps, dvnl[sl])       # (lmx, 3)
            f[a] += w * ((clalp[:lmx] * p)[:, None] * dd).sum(axis=0)
    return f


def fnl_kb(t: dict, kb_g: np.ndarray, vclalp: np.ndarray, psi: np.ndarray, occ: np.ndarray) -> np.ndarray:
    """kbnlpp_frc2 for psi (nb, nplwex); kb_g (nplwex, nproj), projector
    j = l + lmx * atom; (natom, 3) Ry/bohr."""
    nat = t["natom"]
    nproj = kb_g.shape[1]
    lmx = nproj // nat
    gw = t["gw"]
    # slmir: KB metric projections (nproj, nb)
    p = 2.0 * kb_g.T @ psi.T - np.outer(kb_g[0], psi[:, 0]) - 2.0 * np.outer(kb_g[1], psi[:, 1])
    br, bi = kb_g[2::2], kb_g[3::2]                 # g >= 1
    cr, ci = psi[:, 2::2], psi[:, 3::2]
    f = np.zeros((nat, 3))
    for a in range(nat):
        for l in range(lmx):
            j = l + lmx * a
            fzz = br[:, j][None, :] * ci - bi[:, j][None, :] * cr   # (nb, nplw)
            fsl = fzz @ gw[1:]                                    # (nb, 3)
            w = occ * 2.0 * vclalp[j] * p[j]                      # (nb,)
            f[a] += 2.0 * (w[:, None] * fsl).sum(axis=0)
    return f
