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
