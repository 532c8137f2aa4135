"""ORACLE -- test infrastructure only.  The G-space KB projector table
eqlmr_ restated in numpy (FP64) from the reference's table builders:

* setqlm (nlkbpp.f90:2196-2247): radial table tbqlm at |G| by the
  three-point forward-difference interpolation, m = 2 int(|G|/(2 dl)),
  d = (|G|/dl - m)/2, f = d((d-1) a_m + t_{m+2} - t_m) + t_m, with
  a_m = tbqlma = 2(t_m + t_{m+2} - 2 t_{m+1}) (ppkb.f90:3228-3236), times the
  channel's angular factor;
* stscfn_pw (pwlda.f90:5711-5850): cos/sin(G.R_a) composed from the
  per-dimension angle-addition tables (phase_tables of oracle.forces);
* setbgq (nlkbpp.f90:2135-2187): even l -> (cos f, -sin f), odd l ->
  (-sin f, -cos f) per half-sphere G, projector j = l + lmx * a.

* setnlc (nlkbppr.f90:1010-1560): for each atom the grid points of the box
  around its nearest grid point (x fastest, periodic wrap in place of the
  reference's image atoms) within the projector radius, the radial table
  interpolated at r by the same three-point formula (tabnl/tabnla) times the
  channel's real solid-harmonic polynomial of the displacement; and the
  x-line index of those points ordered by point.

PARITY UNPINNED as the rest of the oracle; the tests tie these builders to the
analytic model tables that the H|psi> parity tests use.
"""
from __future__ import annotations

import numpy as np

from .forces import phase_tables


def setqlm(ag: np.ndarray, dl: float, tb: np.ndarray, ang: np.ndarray) -> np.ndarray:
    """Interpolated radial table times the angular factor at |G| = ag."""
    m = 2 * (ag / (2.0 * dl)).astype(np.int64)
    d = 0.5 * (ag / dl - m)
    t0, t1, t2 = tb[m], tb[m + 1], tb[m + 2]
    a = 2.0 * (t0 + t2 - 2.0 * t1)
    return (d * ((d - 1.0) * a + t2 - t0) + t0) * ang


def structure_phases(satm: np.ndarray, ngabc: np.ndarray):
    """ycos, ysin (natom, nG) of stscfn_pw for integer G coordinates ngabc (nG, 3)."""
    kmax = int(np.abs(ngabc).max())
    dcq, dsq = phase_tables(satm, kmax)
    k = ngabc + kmax
    nat = satm.shape[0]
    yc = np.empty((nat, ngabc.shape[0]))
    ys = np.empty_like(yc)
    for a in range(nat):
        c1, c2, c3 = dcq[a, 0, k[:, 0]], dcq[a, 1, k[:, 1]], dcq[a, 2, k[:, 2]]
        s1, s2, s3 = dsq[a, 0, k[:, 0]], dsq[a, 1, k[:, 1]], dsq[a, 2, k[:, 2]]
        cc12 = c1 * c2 - s1 * s2
        sc12 = s1 * c2 + c1 * s2
        yc[a] = cc12 * c3 - sc12 * s3
        ys[a] = sc12 * c3 + cc12 * s3
    return yc, ys


def setbgq(b: dict, ityp: np.ndarray, satm: np.ndarray):
    """eqlmr_ (nplwex, nproj) and vclalp (nproj) from the builder arguments
    b (the dict of qxmd_b200.cell.kb_builder_tables) and a geometry."""
    ag = np.sqrt(b["g2"])
    lmx, ntype = b["lmx"], b["ntype"]
    zzz = np.empty((ntype * lmx, ag.size))
    for ch in range(ntype * lmx):
        zzz[ch] = setqlm(ag, b["dlqlm"][ch // lmx], b["tbqlm"][ch], b["qlm"][b["lmidx"][ch]])
    yc, ys = structure_phases(satm, b["ngabc"])
    nat = satm.shape[0]
    tab = np.zeros((2 * ag.size, lmx * nat))
    vcl = np.zeros(lmx * nat)
    for a in range(nat):
        it = int(ityp[a])
        for l in range(lmx):
            ch = l + lmx * it
            f = zzz[ch]
            j = l + lmx * a
            if b["even"][ch]:
                tab[0::2, j], tab[1::2, j] = yc[a] * f, -ys[a] * f
            else:
                tab[0::2, j], tab[1::2, j] = -ys[a] * f, -yc[a] * f
            vcl[j] = b["vclalp"][ch]
    return tab, vcl


def _poly(c: int, x, y, z):
    return [np.ones_like(x), x, y, z, x * y, y * z, z * x, x * x - y * y, 3 * z * z - (x * x + y * y + z * z)][c]


def _poly_grad(c: int, x, y, z):
    """Gradient (npts, 3) of the solid-harmonic polynomial of _poly."""
    o, z0 = np.ones_like(x), np.zeros_like(x)
    g = [(z0, z0, z0), (o, z0, z0), (z0, o, z0), (z0, z0, o), (y, x, z0), (z0, z, y), (z, z0, x),
         (2 * x, -2 * y, z0), (-2 * x, -2 * y, 4 * z)][c]
    return np.stack(g, axis=1)


def box_halfwidths(rba: np.ndarray, grid, rmax: float):
    binv = np.linalg.inv(rba)
    return [int(rmax * np.linalg.norm(binv[i]) * grid[i] + 0.5) + 1 for i in range(3)]


def setnlc(b: dict, ityp: np.ndarray, satm: np.ndarray, grad: bool = False):
    """(off (natom+1), mesh (npts), vnl (npts, lmx)) in box order; b is the dict
    of qxmd_b200.cell.kbr_builder_tables, with optional per-projector channel
    radii b["rcut_l"] (lmx * ntype, each at most the species radius b["rcut"]);
    b["lmx"] projectors per atom (4 when absent).  With grad, also dvnl (npts, lmx, 3):
    the gradient of each projector value with respect to the displacement d
    of the point from its atom, as fnnlcl2 builds it from the radial table
    and its derivative table (nlkbppr.f90:2200-2240):
    grad(g(r) P(d)) = (g'(r)/r) d P(d) + g(r) grad P(d), both radial tables
    interpolated by the three-point formula of setqlm."""
    k = np.array(b["grid"])
    lmx = int(b.get("lmx", 4))
    nd = box_halfwidths(b["rba"], b["grid"], float(np.max(b["rcut"])))
    o3, o2, o1 = np.meshgrid(np.arange(-nd[2], nd[2] + 1), np.arange(-nd[1], nd[1] + 1),
                             np.arange(-nd[0], nd[0] + 1), indexing="ij")
    o = np.stack([o1.ravel(), o2.ravel(), o3.ravel()], axis=1)
    offs, meshes, vals, grads = [0], [], [], []
    for a in range(satm.shape[0]):
        it = int(ityp[a])
        s = satm[a]
        n = np.floor(s * k + 0.5).astype(np.int64) + o
        f = n / k - s
        d = f @ b["rba"].T
        r2 = np.einsum("ij,ij->i", d, d)
        sel = r2 <= b["rcut"][it] ** 2
        n, d = n[sel], d[sel]
        w = n % k
        meshes.append((w[:, 0] + k[0] * (w[:, 1] + k[1] * w[:, 2])).astype(np.int32))
        r = np.sqrt(r2[sel])
        # projector l belongs to the channel of radius rcut_l[ch] (rmxnlc of
        # nlkbppr.f90:1405-1431): zero at the points outside it, so that the
        # sums over the species sphere equal the sums over each channel's list
        rl2 = r2[sel]
        inside = [rl2 <= (b["rcut_l"][l + lmx * it] ** 2 if b.get("rcut_l") is not None else np.inf)
                  for l in range(lmx)]
        v = np.empty((r.size, lmx))
        for l in range(lmx):
            ch = l + lmx * it
            v[:, l] = setqlm(r, b["dltnl"][it], b["tabnl"][ch], _poly(int(b["poly"][ch]), d[:, 0], d[:, 1], d[:, 2]))
            v[:, l] = np.where(inside[l], v[:, l], 0.0)
        vals.append(v)
        if grad:
            gv = np.empty((r.size, lmx, 3))
            one = np.ones_like(r)
            for l in range(lmx):
                ch = l + lmx * it
                c = int(b["poly"][ch])
                g = setqlm(r, b["dltnl"][it], b["tabnl"][ch], one)
                dg = setqlm(r, b["dltnl"][it], b["dtabnl"][ch], one)
                p = _poly(c, d[:, 0], d[:, 1], d[:, 2])
                gv[:, l, :] = (dg * p)[:, None] * d + g[:, None] * _poly_grad(c, d[:, 0], d[:, 1], d[:, 2])
                gv[:, l, :] = np.where(inside[l][:, None], gv[:, l, :], 0.0)
            grads.append(gv)
        offs.append(offs[-1] + r.size)
    out = (np.asarray(offs, dtype=np.int32), np.concatenate(meshes), np.concatenate(vals, axis=0))
    if grad:
        out = out + (np.concatenate(grads, axis=0),)
    return out
