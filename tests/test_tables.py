"""The oracle's restatement of the G-space KB table builders (setqlm
nlkbpp.f90:2196-2247, stscfn_pw pwlda.f90:5711-5850, setbgq
nlkbpp.f90:2135-2187) on the CPU: a known answer for the interpolation, the
recurrence phases against direct cosines, and the assembled table against the
analytic model tables that the H|psi> parity tests use."""
import dataclasses
import math

import numpy as np

from oracle import tables
from qxmd_b200 import cell


def test_setqlm_interpolation_is_exact_for_quadratics():
    """The three-point formula reproduces a quadratic table exactly: with
    t_k = 1.5 - 0.25 k + 0.125 k^2 the value at |G| is that polynomial in |G|/dl."""
    dl = 0.05
    k = np.arange(64, dtype=np.float64)
    tb = 1.5 - 0.25 * k + 0.125 * k * k
    ag = np.linspace(0.0, 2.9, 301)
    x = ag / dl
    got = tables.setqlm(ag, dl, tb, np.ones_like(ag))
    assert np.max(np.abs(got - (1.5 - 0.25 * x + 0.125 * x * x))) < 1e-11


def test_structure_phases_match_direct_cosines():
    rng = np.random.default_rng(5)
    satm = rng.uniform(-0.5, 1.5, (3, 3))
    ng = rng.integers(-9, 10, (200, 3)).astype(np.int32)
    yc, ys = tables.structure_phases(satm, ng)
    ph = 2.0 * math.pi * satm @ ng.T.astype(np.float64)
    assert np.max(np.abs(yc - np.cos(ph))) < 1e-12
    assert np.max(np.abs(ys - np.sin(ph))) < 1e-12


def test_builder_matches_model_tables():
    """Si8 displaced (seed 1) and moved again: the interpolated table equals
    the analytic one within the interpolation error of dl = 0.005 (5e-8 of
    the largest entry), the KB energies exactly."""
    s = cell.si8(with_ewald=False)
    b = cell.kb_builder_tables(s.gs, s.cell, s.pp)
    for shift in (0.0, 0.07):
        c = dataclasses.replace(s.cell, pos=s.cell.pos + shift * np.array([1.0, -0.5, 0.25]))
        ref, vref = cell.kb_tables_g(s.gs, c, s.pp)
        satm = np.linalg.solve(s.gs.rba, c.pos.T).T
        tab, vcl = tables.setbgq(b, b["ityp"], satm)
        assert np.max(np.abs(tab - ref)) / np.max(np.abs(ref)) < 5e-8
        assert np.array_equal(vcl, vref)


def test_real_space_builder_matches_model_tables():
    """setnlc restated (box search with periodic wrap) against the nearest-image
    full-grid tables of the model: the same points per atom and the same
    projector values within the interpolation error (1e-8 of the largest)."""
    s = cell.si8(with_ewald=False)
    b = cell.kbr_builder_tables(s.gs, s.cell, s.pp)
    for shift in (0.0, 0.11):
        c = dataclasses.replace(s.cell, pos=s.cell.pos + shift * np.array([0.3, 1.0, -0.7]))
        ref = cell.kb_tables_r(s.gs, c, s.pp)
        satm = np.linalg.solve(s.gs.rba, c.pos.T).T
        off, mesh, vnl = tables.setnlc(b, b["ityp"], satm)
        assert np.array_equal(off, ref.off)
        scale = np.max(np.abs(ref.vnl))
        for a in range(c.natom):
            o = np.argsort(mesh[off[a]:off[a + 1]])
            p = np.argsort(ref.mesh[ref.off[a]:ref.off[a + 1]])
            assert np.array_equal(mesh[off[a]:off[a + 1]][o], ref.mesh[ref.off[a]:ref.off[a + 1]][p])
            got = vnl[off[a]:off[a + 1]][o]
            want = ref.vnl[ref.off[a]:ref.off[a + 1]][p]
            assert np.max(np.abs(got - want)) / scale < 1e-8


def test_channel_radii_reproduce_calnlc_per_channel_lists():
    """setnlc gives each angular channel its own point list, the points within
    rmxnlc(la) (nlkbppr.f90:1405-1431), and calnlc sums each projector over
    its channel's list (nlkbppr.f90:1812-1818, 1862-1868).  The device keeps
    one list per atom (the species radius, the largest channel's) with each
    projector zero beyond its own channel's radius.  Restated here both ways
    for s and p channels of different radii: the nonzero part of the union
    list is the channel list (same points, same order, same values), and the
    projections sumr and the scattered rk agree to rounding."""
    s = cell.si8(with_ewald=False)
    b = cell.kbr_builder_tables(s.gs, s.cell, s.pp)
    rp = float(b["rcut"][0])
    rs = 0.8 * rp
    itola = [0, 1, 1, 1]                  # projector l -> channel la (s, p, p, p)
    rcl = np.array([rs, rp, rp, rp])
    off, mesh, vnl = tables.setnlc(dict(b, rcut_l=rcl), b["ityp"], b["satm"])
    chan = {la: tables.setnlc(dict(b, rcut=np.array([rc])), b["ityp"], b["satm"]) for la, rc in ((0, rs), (1, rp))}
    nat = s.cell.natom
    assert chan[0][0][-1] < chan[1][0][-1]          # the s lists are strictly smaller
    for a in range(nat):
        u = slice(off[a], off[a + 1])
        for l in range(4):
            co, cm, cv = chan[itola[l]]
            c = slice(co[a], co[a + 1])
            keep = vnl[u, l] != 0.0
            assert np.array_equal(mesh[u][keep], cm[c][cv[c, l] != 0.0])
            assert np.array_equal(vnl[u, l][keep], cv[c, l][cv[c, l] != 0.0])
    rng = np.random.default_rng(9)
    eigv = rng.standard_normal(s.gs.kfft0)
    scale = b["rdelv"] * b["clalp"]

    def calnlc(lists_of):
        sumr = np.zeros((nat, 4))
        for a in range(nat):
            for l in range(4):
                o, m, v = lists_of(l)
                sumr[a, l] = np.dot(v[o[a]:o[a + 1], l], eigv[m[o[a]:o[a + 1]]])
        sumr *= scale
        rk = np.zeros(s.gs.kfft0)
        for a in range(nat):
            for l in range(4):
                o, m, v = lists_of(l)
                np.add.at(rk, m[o[a]:o[a + 1]], v[o[a]:o[a + 1], l] * sumr[a, l])
        return sumr, rk

    sr, rr = calnlc(lambda l: chan[itola[l]])
    su, ru = calnlc(lambda l: (off, mesh, vnl))
    assert np.max(np.abs(su - sr)) <= 1e-13 * np.max(np.abs(sr))
    assert np.max(np.abs(ru - rr)) <= 1e-13 * np.max(np.abs(rr))
