"""Caller-side set-up for the Kohn-Sham hot path: cell, G half-sphere, FFT grid,
model pseudopotential tables and the random initial wavefunctions.

In QXMD all of this is computed by the Fortran host before the hot path runs
(`reclat.f90`, `modules.f90:set_rciprl`, `nlkbpp.f90:setbgq`,
`nlkbppr.f90:setnlc`, `savedd.f90:rdwfns`).  The hot path only consumes the
resulting read-only arrays, so this module produces exactly those arrays in the
layouts the Fortran code uses:

* ``nga/ngb/ngc`` and ``recnrm`` for G = 0..nplw5, sorted by |G|^2 as
  ``strvec`` sorts them (`reclat.f90:500-875`, stable order of equal keys);
* ``ijkgd(-nplw5:nplw5)``: the FFT-grid index of +G and -G
  (`reclat.f90:254-274`), kept 0-based here;
* ``dkgnrm(2*(nplw+1))``: |G|^2 duplicated for (Re, Im) (`modules.f90:1557-1562`);
* wavefunctions as the real Gamma-point half sphere ``gdcr(nplwex, nband)`` with
  nplwex = 2*(nplw+1), column-major, component 2 (Im c(G=0)) identically 0.

The pseudopotential is an analytic model with the table layout of QXMD's
norm-conserving KB path: an Appelbaum-Hamann-form local potential and
Gaussian s/p Kleinman-Bylander projectors.  Reading Troullier-Martins files
and the King-Smith filter (`ppkb.f90`, `ppkbr.f90`) are table builders outside
the hot path; the projector tables produced here have the same meaning as
``eqlmr_``/``vclalp`` (`nlkbpp.f90:2135-2187`, `:1262`) and
``meshnl``/``vnlcr``/``clalp_ncr`` (`nlkbppr.f90:1773-1900`).

Units are Rydberg atomic units (|G|^2 in Ry, e^2 = 2), as in QXMD.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# FFT sizes accepted by chkftm for the FFTW3 build: every 2^a 3^b 5^c 7^d up to
# 4900 (`reclat.f90:889-918`).  Generated rather than tabulated.
def _fftw3_sizes(limit: int = 4900) -> list[int]:
    out = []
    for n in range(1, limit + 1):
        m = n
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        if m == 1:
            out.append(n)
    return out


_NPWRNM = _fftw3_sizes()


def chkftm(k1: int, k2: int, k3: int) -> tuple[int, int, int]:
    """Round FFT mesh sizes up to the next allowed size (`reclat.f90:1007-1084`).

    The first axis takes the first table entry >= k1; axes 2 and 3 search from
    the second entry; axes equal to axis 1 on input stay equal to it.
    """
    def up(k, start):
        for n in _NPWRNM[start:]:
            if n >= k:
                return n
        raise ValueError(f"FFT mesh {k} beyond the chkftm table")

    d1 = up(k1, 0)
    d2 = up(k2, 1)
    d3 = up(k3, 1)
    if k2 == k1:
        d2 = d1
    if k3 == k1:
        d3 = d1
    return d1, d2, d3


def rciprl(a: np.ndarray) -> tuple[np.ndarray, float]:
    """Reciprocal vectors b (a_i . b_j = delta_ij, columns) and |volume|
    (`reclat.f90:1089-1132`).  ``a[:, i]`` is lattice vector i."""
    b = np.empty((3, 3))
    b[0, 0] = a[1, 1] * a[2, 2] - a[2, 1] * a[1, 2]
    b[1, 0] = a[2, 1] * a[0, 2] - a[0, 1] * a[2, 2]
    b[2, 0] = a[0, 1] * a[1, 2] - a[1, 1] * a[0, 2]
    v = a[0, 0] * b[0, 0] + a[1, 0] * b[1, 0] + a[2, 0] * b[2, 0]
    vr = 1.0 / v
    b[:, 0] *= vr
    b[0, 1] = (a[1, 2] * a[2, 0] - a[2, 2] * a[1, 0]) * vr
    b[1, 1] = (a[2, 2] * a[0, 0] - a[0, 2] * a[2, 0]) * vr
    b[2, 1] = (a[0, 2] * a[1, 0] - a[1, 2] * a[0, 0]) * vr
    b[0, 2] = (a[1, 0] * a[2, 1] - a[2, 0] * a[1, 1]) * vr
    b[1, 2] = (a[2, 0] * a[0, 1] - a[0, 0] * a[2, 1]) * vr
    b[2, 2] = (a[0, 0] * a[1, 1] - a[1, 0] * a[0, 1]) * vr
    return b, abs(v)


def _half_space_candidates(kmaxm: int, kmaxm1: tuple[int, int, int]) -> np.ndarray:
    """Integer triples of one member of each +-G pair, in the enumeration order
    of `reclat.f90:626-763` (ih >= jh >= kh >= 0, ih >= 1, with the signed
    permutations chosen by the coincidence pattern of ih, jh, kh)."""
    out = []
    for ih in range(1, kmaxm + 1):
        for jh in range(0, ih + 1):
            for kh in range(0, jh + 1):
                kzero = kh == 0
                keqj = kh == jh
                ieqj = ih == jh
                pat = 1 + (1 if kzero else 0) + (2 if keqj else 0) + (4 if ieqj else 0)
                cand = [(ih, jh, kh)]
                if pat != 7:
                    cand += [(kh, ih, jh), (jh, kh, ih)]
                if pat != 4:
                    cand += [(-ih, jh, kh), (kh, -ih, jh), (jh, kh, -ih)]
                    if pat not in (6, 7):
                        if pat != 2:
                            cand += [(ih, -jh, kh), (kh, ih, -jh), (-jh, kh, ih),
                                     (ih, jh, -kh), (-kh, ih, jh), (jh, -kh, ih)]
                        if pat not in (3, 5):
                            cand += [(ih, kh, jh), (jh, ih, kh), (kh, jh, ih),
                                     (-ih, kh, jh), (jh, -ih, kh), (kh, jh, -ih)]
                            if pat != 2:
                                cand += [(ih, kh, -jh), (-jh, ih, kh), (kh, -jh, ih),
                                         (ih, -kh, jh), (jh, ih, -kh), (-kh, jh, ih)]
                for t in cand:
                    if (abs(t[0]) <= kmaxm1[0] + 1 and abs(t[1]) <= kmaxm1[1] + 1
                            and abs(t[2]) <= kmaxm1[2] + 1):
                        out.append(t)
    return np.asarray(out, dtype=np.int64).reshape(-1, 3)


@dataclasses.dataclass
class GSphere:
    """Reciprocal-space set-up of one cell (the outputs of strvec/reclat)."""
    rba: np.ndarray          # (3,3) lattice vectors as columns, bohr
    cross: np.ndarray        # (3,3) 2*pi*b, columns are reciprocal vectors
    rvol: float
    ecut: float
    ecutdens: float
    nplw: int                # wavefunction half sphere (G=0 excluded from the count)
    nplw5: int               # density half sphere
    nga: np.ndarray          # int (nplw5+1,)
    ngb: np.ndarray
    ngc: np.ndarray
    gvec: np.ndarray         # (nplw5+1, 3) cartesian G
    recnrm: np.ndarray       # |G|^2 (nplw5+1,)
    grid: tuple[int, int, int]
    ijk_pos: np.ndarray      # 0-based grid index of +G, (nplw5+1,)
    ijk_neg: np.ndarray      # 0-based grid index of -G, (nplw5+1,)

    @property
    def nplwex(self) -> int:
        return 2 * (self.nplw + 1)

    @property
    def kfft0(self) -> int:
        return self.grid[0] * self.grid[1] * self.grid[2]

    def dkgnrm(self) -> np.ndarray:
        """|G|^2 per real component of the wavefunction half sphere."""
        return np.repeat(self.recnrm[: self.nplw + 1], 2).copy()

    def ijkgd(self) -> np.ndarray:
        """ijkgd(-nplw5:nplw5) as a 0-based array of length 2*nplw5+1
        (entry nplw5+m is G index m)."""
        out = np.empty(2 * self.nplw5 + 1, dtype=np.int32)
        out[self.nplw5:] = self.ijk_pos
        out[: self.nplw5 + 1] = self.ijk_neg[::-1]
        return out


def strvec(rba: np.ndarray, ecut: float, ecutdens: float) -> GSphere:
    """Enumerate, sort and index the G half sphere (`reclat.f90:500-875`,
    `modules.f90:1402-1562`, grid from `reclat.f90:254-291`)."""
    b, rvol = rciprl(rba)
    dpi = 2.0 * math.acos(-1.0)
    cross = dpi * b
    gxfft = math.sqrt(ecutdens) / dpi
    kmaxm1 = []
    perm = ((1, 2, 0), (2, 0, 1), (0, 1, 2))
    for i in range(3):
        p1, p2, p3 = perm[i]
        a1x = b[1, p1] * b[2, p2] - b[2, p1] * b[1, p2]
        a1y = b[2, p1] * b[0, p2] - b[0, p1] * b[2, p2]
        a1z = b[0, p1] * b[1, p2] - b[1, p1] * b[0, p2]
        aaa = 1.0 / math.sqrt(a1x * a1x + a1y * a1y + a1z * a1z)
        pk3 = b[0, p3] * a1x * aaa + b[1, p3] * a1y * aaa + b[2, p3] * a1z * aaa
        kmaxm1.append(int(abs(gxfft / pk3)))
    kmaxm = max(kmaxm1)
    t = _half_space_candidates(kmaxm, tuple(kmaxm1))
    d = t.astype(np.float64)
    gs1 = cross[0, 0] * d[:, 0] + cross[0, 1] * d[:, 1] + cross[0, 2] * d[:, 2]
    gs2 = cross[1, 0] * d[:, 0] + cross[1, 1] * d[:, 1] + cross[1, 2] * d[:, 2]
    gs3 = cross[2, 0] * d[:, 0] + cross[2, 1] * d[:, 1] + cross[2, 2] * d[:, 2]
    gss = gs1 * gs1 + gs2 * gs2 + gs3 * gs3
    fctmax = 1.0e9 / np.max(np.abs(gss))
    key = np.trunc(fctmax * gss).astype(np.int64)
    order = np.argsort(key, kind="stable")
    gss_s = gss[order]
    nplw5 = int(np.count_nonzero(gss_s <= ecutdens))
    nplw = int(np.count_nonzero(gss_s <= ecut))
    sel = order[:nplw5]
    nga = np.concatenate([[0], t[sel, 0]]).astype(np.int64)
    ngb = np.concatenate([[0], t[sel, 1]]).astype(np.int64)
    ngc = np.concatenate([[0], t[sel, 2]]).astype(np.int64)
    gvec = np.zeros((nplw5 + 1, 3))
    gvec[1:, 0] = gs1[sel]
    gvec[1:, 1] = gs2[sel]
    gvec[1:, 2] = gs3[sel]
    recnrm = np.concatenate([[0.0], gss_s[:nplw5]])
    kd = (int(np.max(np.abs(nga))), int(np.max(np.abs(ngb))), int(np.max(np.abs(ngc))))
    grid = chkftm(2 * kd[0] + 1, 2 * kd[1] + 1, 2 * kd[2] + 1)
    k1, k2, k3 = grid
    ijk_pos = (np.mod(nga, k1) + (np.mod(ngb, k2) + np.mod(ngc, k3) * k2) * k1).astype(np.int32)
    ijk_neg = (np.mod(-nga, k1) + (np.mod(-ngb, k2) + np.mod(-ngc, k3) * k2) * k1).astype(np.int32)
    return GSphere(rba=np.array(rba, dtype=np.float64), cross=cross, rvol=rvol,
                   ecut=ecut, ecutdens=ecutdens, nplw=nplw, nplw5=nplw5,
                   nga=nga, ngb=ngb, ngc=ngc, gvec=gvec, recnrm=recnrm, grid=grid,
                   ijk_pos=ijk_pos, ijk_neg=ijk_neg)


# --------------------------------------------------------------------------
# Cells
# --------------------------------------------------------------------------

_DIAMOND_BASIS = np.array([
    [0.00, 0.00, 0.00], [0.00, 0.50, 0.50], [0.50, 0.00, 0.50], [0.50, 0.50, 0.00],
    [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75], [0.75, 0.75, 0.25],
])


@dataclasses.dataclass
class Cell:
    rba: np.ndarray          # (3,3) lattice vectors as columns
    pos: np.ndarray          # (natom, 3) cartesian bohr
    zv: float = 4.0          # valence charge per atom

    @property
    def natom(self) -> int:
        return self.pos.shape[0]

    @property
    def nel(self) -> int:
        return int(round(self.zv * self.natom))


def diamond_si(reps=(1, 1, 1), a: float = 10.26, seed: int = 1,
               disp: float = 0.05, strain=None) -> Cell:
    """Diamond-cubic Si supercell with seeded uniform displacements
    (``default_rng(seed).uniform(-disp, disp, (natom, 3))`` bohr) and an
    optional per-axis strain factor."""
    reps = tuple(int(r) for r in reps)
    frac = []
    for i in range(reps[0]):
        for j in range(reps[1]):
            for k in range(reps[2]):
                frac.append((_DIAMOND_BASIS + np.array([i, j, k])) / np.array(reps))
    frac = np.concatenate(frac, axis=0)
    lengths = a * np.array(reps, dtype=np.float64)
    if strain is not None:
        lengths = lengths * np.asarray(strain, dtype=np.float64)
    rba = np.diag(lengths)
    rng = np.random.default_rng(seed)
    pos = frac @ rba.T + rng.uniform(-disp, disp, (frac.shape[0], 3))
    return Cell(rba=rba, pos=pos)


# --------------------------------------------------------------------------
# Model pseudopotential (Rydberg units)
# --------------------------------------------------------------------------

@dataclasses.dataclass(frozen=True)
class ModelPP:
    """Appelbaum-Hamann-form local part and Gaussian s/p KB projectors, in Ry.

    v_loc(r) = -(2Z/r) erf(sqrt(alpha) r) + (v1 + v2 r^2) exp(-alpha r^2)
    beta_s(r) = A_s exp(-r^2/(2 sig^2)) Y_00,  beta_p(r) = A_p r exp(-r^2/(2 sig^2)) Y_1m
    normalised so that int beta_l(r)^2 r^2 dr = 1; KB energies e_s, e_p.
    v1, v2 are Appelbaum and Hamann's Si values (3.042, -1.372 Hartree) in
    Rydberg.  With these KB energies the Si cells keep a gap between the
    occupied and the empty bands, so a fixed-occupation SCF converges.
    """
    zv: float = 4.0
    alpha: float = 0.6102
    v1: float = 6.084
    v2: float = -2.744
    sig: float = 0.8
    e_s: float = 0.3
    e_p: float = 0.15
    rcut: float = 4.0       # real-space projector sphere radius (bohr)

    @property
    def lmx(self) -> int:
        return 4            # s + three p, the Si projector count

    @property
    def a_s(self) -> float:
        return math.sqrt(4.0 / (math.sqrt(math.pi) * self.sig ** 3))

    @property
    def a_p(self) -> float:
        return math.sqrt(8.0 / (3.0 * math.sqrt(math.pi) * self.sig ** 5))

    def vloc_g(self, g2: np.ndarray) -> np.ndarray:
        """Per-atom Fourier transform of v_loc without 1/Omega; the G = 0
        entry is the finite (non-Coulomb) limit."""
        g2 = np.asarray(g2, dtype=np.float64)
        a = self.alpha
        ex = np.exp(-g2 / (4.0 * a))
        gauss = (math.pi / a) ** 1.5 * ex * (self.v1 + self.v2 * (1.5 / a - g2 / (4.0 * a * a)))
        out = np.empty_like(g2)
        nz = g2 > 1e-12
        out[nz] = -8.0 * math.pi * self.zv * ex[nz] / g2[nz] + gauss[nz]
        out[~nz] = 2.0 * math.pi * self.zv / a + gauss[~nz]
        return out

    def radial_g(self, g: np.ndarray):
        """4*pi * int r^2 j_l(g r) beta_l(r) dr for l = 0 and, divided by g,
        for l = 1 (so that multiplying by G_m gives the p-channel value)."""
        s = self.sig
        ex = np.exp(-0.5 * g * g * s * s)
        f0 = 4.0 * math.pi * self.a_s * math.sqrt(math.pi / 2.0) * s ** 3 * ex
        f1_over_g = 4.0 * math.pi * self.a_p * math.sqrt(math.pi / 2.0) * s ** 5 * ex
        return f0, f1_over_g


Y00 = 1.0 / math.sqrt(4.0 * math.pi)
Y1 = math.sqrt(3.0 / (4.0 * math.pi))


def structure_phase(gs: GSphere, cell: Cell, n: int):
    """ycos/ysin(0:n, natom): cos and sin of G.R (`pwlda.f90:1296` stscfn_pw)."""
    gr = gs.gvec[: n + 1] @ cell.pos.T           # (n+1, natom)
    return np.cos(gr), np.sin(gr)


def kb_tables_g(gs: GSphere, cell: Cell, pp: ModelPP):
    """eqlmr_(nplwex, lmx, natom) and vclalp(lmx) as in `nlkbpp.f90:2135-2187`.

    eqlmr_ = (-i)^l * 4 pi Y_lm(G^) F_l(|G|) * exp(-i G.R), stored (Re, Im)
    per G of the half sphere; projector order per atom is s, p_x, p_y, p_z.
    Returned as a (nplwex, nproj) column-major-friendly array with
    nproj = lmx * natom (projector index = l + lmx * atom).
    """
    n = gs.nplw
    g = gs.gvec[: n + 1]
    gn = np.sqrt(gs.recnrm[: n + 1])
    f0, f1g = pp.radial_g(gn)
    ycos, ysin = structure_phase(gs, cell, n)
    nproj = pp.lmx * cell.natom
    tab = np.zeros((gs.nplwex, nproj))
    for ia in range(cell.natom):
        c = ycos[:, ia]
        s = ysin[:, ia]
        # s channel: even l -> (cos f, -sin f)
        f = f0 * Y00
        tab[0::2, 4 * ia + 0] = c * f
        tab[1::2, 4 * ia + 0] = -s * f
        for m in range(3):
            f = f1g * Y1 * g[:, m]
            # odd l -> (-sin f, -cos f)
            tab[0::2, 4 * ia + 1 + m] = -s * f
            tab[1::2, 4 * ia + 1 + m] = -c * f
    vclalp = np.tile(np.array([pp.e_s, pp.e_p, pp.e_p, pp.e_p]), cell.natom) / gs.rvol
    return tab, vclalp


def kb_builder_tables(gs: GSphere, cell: Cell, pp: ModelPP, dl: float = 0.005) -> dict:
    """Arguments of qx_set_kb_builder / qx_build_kb_g for the model
    pseudopotential (one species): radial tables tbqlm on |G| = k dl (s:
    F_0 Y_00; p: F_1/|G| Y_1, so that the angular factor of p_m is G_m), the
    angular factors qlm (1, gx, gy, gz) per half-sphere G, the parities of
    setbgq and the KB energies; plus the geometry (fractional coordinates)
    and |G|^2 for the oracle.  Arrays are in numpy row-major order of the
    C interface's column-major arguments."""
    n = gs.nplw
    g2 = np.ascontiguousarray(gs.recnrm[: n + 1])
    mxqlm = 2 * int(math.sqrt(float(g2.max())) / (2.0 * dl)) + 6
    k = np.arange(mxqlm + 1) * dl
    f0, f1g = pp.radial_g(k)
    tbqlm = np.ascontiguousarray(np.stack([f0 * Y00, f1g * Y1, f1g * Y1, f1g * Y1]))
    g = gs.gvec[: n + 1]
    qlm = np.ascontiguousarray(np.stack([np.ones(n + 1), g[:, 0], g[:, 1], g[:, 2]]))
    satm = np.ascontiguousarray(np.linalg.solve(gs.rba, cell.pos.T).T)
    return dict(ntype=1, lmx=4, mxqlm=mxqlm, dlqlm=np.array([dl]), tbqlm=tbqlm, nlm=4, qlm=qlm,
                lmidx=np.arange(4, dtype=np.int32), even=np.array([1, 0, 0, 0], dtype=np.int32),
                vclalp=np.array([pp.e_s, pp.e_p, pp.e_p, pp.e_p]) / gs.rvol,
                ngabc=np.ascontiguousarray(np.stack([gs.nga[: n + 1], gs.ngb[: n + 1], gs.ngc[: n + 1]],
                                                    axis=1).astype(np.int32)),
                ityp=np.zeros(cell.natom, dtype=np.int32), satm=satm, g2=g2)


def kbr_builder_tables(gs: GSphere, cell: Cell, pp: ModelPP, dl: float = 0.002) -> dict:
    """Arguments of qx_set_kb_r_builder / qx_build_kb_r for the model
    pseudopotential (one species): radial tables on r = k dl (s: A_s
    exp(-r^2/2 sig^2) Y_00; p: A_p exp(-r^2/2 sig^2) Y_1, times the
    displacement component through poly 1-3) and their g'(r)/r tables for the
    force gradients, the projector radius, the KB
    energies and the volume per grid point; plus the geometry."""
    mxnl = 2 * int(pp.rcut / (2.0 * dl)) + 6
    r = np.arange(mxnl + 1) * dl
    ex = np.exp(-0.5 * r * r / pp.sig ** 2)
    tabnl = np.ascontiguousarray(np.stack([pp.a_s * ex * Y00] + [pp.a_p * ex * Y1] * 3))
    # g'(r)/r of the Gaussian radial parts: -g(r)/sig^2
    dtabnl = np.ascontiguousarray(-tabnl / pp.sig ** 2)
    satm = np.ascontiguousarray(np.linalg.solve(gs.rba, cell.pos.T).T)
    return dict(ntype=1, mxnl=mxnl, dltnl=np.array([dl]), rcut=np.array([pp.rcut]), tabnl=tabnl, dtabnl=dtabnl,
                poly=np.arange(4, dtype=np.int32), clalp=np.array([pp.e_s, pp.e_p, pp.e_p, pp.e_p]),
                rdelv=gs.rvol / gs.kfft0, rba=np.ascontiguousarray(gs.rba, dtype=np.float64),
                grid=tuple(gs.grid), ityp=np.zeros(cell.natom, dtype=np.int32), satm=satm)


@dataclasses.dataclass
class KBReal:
    """Real-space KB tables (the meaning of meshnl/npmsnl/numsnl/vnlcr in
    `nlkbppr.f90:1773-1900`): for atom a, grid points mesh[off[a]:off[a+1]]
    with projector values vnl[off[a]+mm, l]."""
    off: np.ndarray          # int32 (natom+1,)
    mesh: np.ndarray         # int32 (npts,) 0-based grid index
    vnl: np.ndarray          # float64 (npts, lmx)
    clalp: np.ndarray        # (lmx,) KB energies per projector (clalp_ncr)
    rdelv: float             # volume per grid point


def kb_tables_r(gs: GSphere, cell: Cell, pp: ModelPP) -> KBReal:
    k1, k2, k3 = gs.grid
    a = gs.rba
    # Fortran order: ijk = n1 + (n2 + n3*k2)*k1 with n1 fastest.
    idx = np.arange(k1 * k2 * k3)
    n1 = idx % k1
    n2 = (idx // k1) % k2
    n3 = idx // (k1 * k2)
    frac = np.stack([n1 / k1, n2 / k2, n3 / k3], axis=1)
    ainv = np.linalg.inv(a)
    offs = [0]
    meshes, vals = [], []
    for ia in range(cell.natom):
        fr = ainv @ cell.pos[ia]
        df = frac - fr
        df -= np.round(df)                      # nearest periodic image
        dr = df @ a.T
        r2 = np.einsum("ij,ij->i", dr, dr)
        sel = np.nonzero(r2 <= pp.rcut ** 2)[0]
        d = dr[sel]
        ex = np.exp(-0.5 * r2[sel] / pp.sig ** 2)
        v = np.empty((sel.size, 4))
        v[:, 0] = pp.a_s * ex * Y00
        v[:, 1] = pp.a_p * ex * Y1 * d[:, 0]
        v[:, 2] = pp.a_p * ex * Y1 * d[:, 1]
        v[:, 3] = pp.a_p * ex * Y1 * d[:, 2]
        meshes.append(sel.astype(np.int32))
        vals.append(v)
        offs.append(offs[-1] + sel.size)
    return KBReal(off=np.asarray(offs, dtype=np.int32), mesh=np.concatenate(meshes),
                  vnl=np.concatenate(vals, axis=0),
                  clalp=np.array([pp.e_s, pp.e_p, pp.e_p, pp.e_p]),
                  rdelv=gs.rvol / gs.kfft0)


def vloc_grid(gs: GSphere, cell: Cell, pp: ModelPP) -> np.ndarray:
    """Local pseudopotential on the FFT grid (real, kfft0), from the density
    sphere: v(r) = sum_G V(G) e^{iGr} with V(G) = (1/Omega) sum_a v_a(G) e^{-iG.R_a}."""
    n5 = gs.nplw5
    vg = pp.vloc_g(gs.recnrm[: n5 + 1]) / gs.rvol
    ycos, ysin = structure_phase(gs, cell, n5)
    sr = ycos.sum(axis=1)
    si = -ysin.sum(axis=1)
    z = np.zeros(gs.kfft0, dtype=np.complex128)
    z[gs.ijk_pos] = vg * (sr + 1j * si)
    z[gs.ijk_neg[1:]] = np.conj(z[gs.ijk_pos[1:]])
    k1, k2, k3 = gs.grid
    zz = z.reshape(k3, k2, k1)
    r = np.fft.ifftn(zz) * gs.kfft0
    return np.ascontiguousarray(r.real.ravel())


def ewald_energy(cell: Cell, gs: GSphere, eta: float | None = None) -> float:
    """Ion-ion energy (Ry) by Ewald summation for point charges zv."""
    a = gs.rba
    vol = gs.rvol
    z = cell.zv
    nat = cell.natom
    if eta is None:
        eta = (math.sqrt(math.pi) * nat ** (1 / 6) / vol ** (1 / 3)) ** 2
    # real space
    rc = 6.0 / math.sqrt(eta)
    nmax = [int(math.ceil(rc / np.linalg.norm(a[:, i]))) + 1 for i in range(3)]
    er = 0.0
    shifts = []
    for i in range(-nmax[0], nmax[0] + 1):
        for j in range(-nmax[1], nmax[1] + 1):
            for k in range(-nmax[2], nmax[2] + 1):
                shifts.append(a @ np.array([i, j, k], dtype=np.float64))
    shifts = np.array(shifts)
    from scipy.special import erfc as verfc
    d = cell.pos[:, None, :] - cell.pos[None, :, :]
    for s in shifts:
        rr = np.linalg.norm(d + s, axis=2)
        m = (rr > 1e-10) & (rr < rc)
        er += float(np.sum(verfc(math.sqrt(eta) * rr[m]) / rr[m]))
    er *= 0.5 * z * z
    # reciprocal space over the density sphere (half sphere, x2)
    g2 = gs.recnrm[1:]
    gv = gs.gvec[1:]
    sf = np.exp(-1j * (gv @ cell.pos.T)).sum(axis=1)
    eg = 2.0 * np.sum(4.0 * math.pi / vol * np.exp(-g2 / (4 * eta)) / g2 * np.abs(sf) ** 2) * 0.5 * z * z
    eself = -z * z * nat * math.sqrt(eta / math.pi)
    ebg = -0.5 * math.pi * (z * nat) ** 2 / (eta * vol)
    return 2.0 * (er + eg + eself + ebg)        # Hartree -> Rydberg


def ewald_forces(cell: Cell, gs: GSphere, eta: float | None = None) -> np.ndarray:
    """Ion-ion forces (Ry/bohr, (natom, 3)): minus the gradient of
    ewald_energy with respect to each atom position, term by term (real-space
    erfc sum and reciprocal sum over the density half sphere)."""
    a = gs.rba
    vol = gs.rvol
    z = cell.zv
    nat = cell.natom
    if eta is None:
        eta = (math.sqrt(math.pi) * nat ** (1 / 6) / vol ** (1 / 3)) ** 2
    from math import erfc
    se = math.sqrt(eta)
    rc = 6.0 / se
    nmax = [int(math.ceil(rc / np.linalg.norm(a[:, i]))) + 1 for i in range(3)]
    shifts = []
    for i in range(-nmax[0], nmax[0] + 1):
        for j in range(-nmax[1], nmax[1] + 1):
            for k in range(-nmax[2], nmax[2] + 1):
                shifts.append(a @ np.array([i, j, k], dtype=np.float64))
    shifts = np.array(shifts)
    f = np.zeros((nat, 3))
    for ia in range(nat):
        d = cell.pos[ia] - cell.pos
        for s in shifts:
            v = d + s
            rr = np.linalg.norm(v, axis=1)
            m = (rr > 1e-10) & (rr < rc)
            r = rr[m]
            g = np.array([erfc(se * x) for x in r]) / r ** 2 + 2.0 * se / math.sqrt(math.pi) * np.exp(-eta * r * r) / r
            f[ia] += z * z * np.sum((g / r)[:, None] * v[m], axis=0)
    g2 = gs.recnrm[1:]
    gv = gs.gvec[1:]
    ph = gv @ cell.pos.T                                   # (ng, natom)
    sf = np.exp(-1j * ph).sum(axis=1)                      # S(G)
    w = 4.0 * math.pi / vol * np.exp(-g2 / (4 * eta)) / g2  # both +G and -G: x2 over the half sphere
    for ia in range(nat):
        im = np.imag(np.exp(-1j * ph[:, ia]) * np.conj(sf))
        f[ia] += -2.0 * z * z * np.sum((w * im)[:, None] * gv, axis=0)
    return 2.0 * f                                        # Hartree -> Rydberg


def force_tables(s: "System") -> dict:
    """Arguments of qx_set_force_tables for a system of one species: fractional
    coordinates, the density half sphere (grid indices, integer and cartesian
    G), the local form factor svco(G) = v_loc(|G|) (Ry, the per-atom
    transform without 1/Omega) and the wavefunction half sphere's G."""
    gs = s.gs
    n5 = gs.nplw5 + 1
    satm = np.linalg.solve(gs.rba, s.cell.pos.T).T
    return dict(natom=s.cell.natom, ntype=1, ityp=np.zeros(s.cell.natom, dtype=np.int32),
                satm=np.ascontiguousarray(satm), n5=n5, ijk5=gs.ijk_pos.astype(np.int32),
                ngabc=np.ascontiguousarray(np.stack([gs.nga, gs.ngb, gs.ngc], axis=1).astype(np.int32)),
                gvec5=np.ascontiguousarray(gs.gvec), svco=s.pp.vloc_g(gs.recnrm).astype(np.float64),
                gw=np.ascontiguousarray(gs.gvec[: gs.nplw + 1]))


def random_wavefunctions(nplwex: int, nband: int, seed: float = 25.0) -> np.ndarray:
    """Initial gdcr(nplwex, nband) from the Park-Miller generator rnd00
    (`funcs.f90:1673-1689`) with seed 25.0 (`savedd.f90:289, 911-918`):
    gdcr(i, n) = rn - 0.5 in band order, then gdcr(2, n) = 0.  Returned with
    shape (nband, nplwex) (row n = band n, the column-major Fortran layout)."""
    a = 16807
    m = 2147483647
    out = np.empty((nband, nplwex))
    flat = out.reshape(-1)
    total = flat.size
    # x_{k+1} = a x_k mod m is exact in binary64 (products below 2^53) and in
    # int64, so the states are computed in blocks of B: x_{k+B} = (a^B mod m)
    # x_k mod m (products below 2^62), giving the same values as the
    # one-by-one recurrence of the reference.
    B = min(total, 4096)
    first = np.empty(B, dtype=np.int64)
    x = int(seed)
    for i in range(B):
        x = (a * x) % m
        first[i] = x
    jump = pow(a, B, m)
    states = np.empty(total, dtype=np.int64)
    cur = first
    for k0 in range(0, total, B):
        n = min(B, total - k0)
        states[k0:k0 + n] = cur[:n]
        cur = (cur * jump) % m
    flat[:] = states.astype(np.float64) / float(m) - 0.5
    out[:, 1] = 0.0
    return out


def occupations(nband: int, nel: int) -> np.ndarray:
    """Non-metallic occupations (lfermi = 1): two electrons per band from the
    bottom."""
    occ = np.zeros(nband)
    nfull = nel // 2
    occ[:nfull] = 2.0
    if nel % 2:
        occ[nfull] = 1.0
    return occ


@dataclasses.dataclass
class System:
    """Everything the hot path reads for one cell."""
    cell: Cell
    gs: GSphere
    pp: ModelPP
    nband: int
    occ: np.ndarray
    vloc: np.ndarray             # (kfft0,)
    kb_g: np.ndarray             # (nplwex, nproj)
    vclalp: np.ndarray           # (nproj,)
    kb_r: KBReal
    eewald: float


def build_system(cell: Cell, ecut: float, ecutdens: float, nband: int,
                 pp: ModelPP | None = None, with_ewald: bool = True) -> System:
    pp = pp or ModelPP()
    gs = strvec(cell.rba, ecut, ecutdens)
    kb_g, vclalp = kb_tables_g(gs, cell, pp)
    return System(cell=cell, gs=gs, pp=pp, nband=nband,
                  occ=occupations(nband, cell.nel),
                  vloc=vloc_grid(gs, cell, pp), kb_g=kb_g, vclalp=vclalp,
                  kb_r=kb_tables_r(gs, cell, pp),
                  eewald=ewald_energy(cell, gs) if with_ewald else 0.0)


# Named workloads (sizes from the hot-path scope table).
def si8(with_ewald=True) -> System:
    return build_system(diamond_si((1, 1, 1), seed=1), 12.0, 48.0, 16, with_ewald=with_ewald)


def si64(ecutdens: float = 64.0, with_ewald=True) -> System:
    return build_system(diamond_si((2, 2, 2), seed=2), 16.0, ecutdens, 160, with_ewald=with_ewald)


def batch_cell(i: int, with_ewald: bool = False) -> System:
    """Cell i of the batch of independent cells: with default_rng(100 + i),
    Si8, Si16 (2x1x1) or Si32 (2x2x1), a uniform +-3% strain per axis, Ecut
    drawn from {10, 12, 14, 16} Ry (density cutoff 4 Ecut) and 0-16 empty
    bands above the occupied ones (at most 80 bands); the displacements use
    the same seed."""
    rng = np.random.default_rng(100 + i)
    reps = ((1, 1, 1), (2, 1, 1), (2, 2, 1))[int(rng.integers(3))]
    strain = 1.0 + rng.uniform(-0.03, 0.03, 3)
    ecut = float(rng.choice([10.0, 12.0, 14.0, 16.0]))
    c = diamond_si(reps, seed=100 + i, strain=strain)
    nocc = c.nel // 2
    nband = min(80, nocc + int(rng.integers(0, 17)))
    return build_system(c, ecut, 4.0 * ecut, nband, with_ewald=with_ewald)


def si512(with_ewald=False) -> System:
    return build_system(diamond_si((4, 4, 4), seed=3), 12.0, 48.0, 1100, with_ewald=with_ewald)
