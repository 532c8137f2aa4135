"""Hellmann-Feynman forces of the oracle (flocal_g nlkbpp.f90:1037-1120,
kbnlpp_frc2 nlkbpp.f90:1878-2130, and the ion-ion Ewald term) against
central differences of the corresponding energies on Si8: each term with the
other variables held fixed, and the sum against the self-consistent total
energy.  Tolerances in Ry/bohr are written at each check."""
import math

import numpy as np
import pytest

import oracle
from oracle import forces as of
from oracle.scf import ScfState
from qxmd_b200 import cell


def moved(s, ia, ax, d):
    pos = s.cell.pos.copy()
    pos[ia, ax] += d
    return cell.Cell(rba=s.cell.rba, pos=pos, zv=s.cell.zv)


def test_ewald_forces_match_energy_derivative(si8):
    f = cell.ewald_forces(si8.cell, si8.gs)
    d = 1e-4
    for ia, ax in [(0, 0), (3, 2), (5, 1)]:
        e1 = cell.ewald_energy(moved(si8, ia, ax, d), si8.gs)
        e2 = cell.ewald_energy(moved(si8, ia, ax, -d), si8.gs)
        assert f[ia, ax] == pytest.approx(-(e1 - e2) / (2 * d), abs=1e-8)
    np.testing.assert_allclose(f.sum(axis=0), 0.0, atol=1e-12)


def test_local_force_matches_energy_derivative(si8, si8_psi):
    """E_loc = (Omega / N) sum_r v_loc(r; R) rho(r) at fixed rho."""
    rho = oracle.Ham(si8, 1).softchg(si8_psi, si8.occ)
    t = cell.force_tables(si8)
    f = of.floc_g(t, rho, si8.gs.grid)
    dv = si8.gs.rvol / si8.gs.kfft0
    d = 1e-4
    for ia, ax in [(0, 0), (6, 1)]:
        e1 = dv * np.dot(cell.vloc_grid(si8.gs, moved(si8, ia, ax, d), si8.pp), rho)
        e2 = dv * np.dot(cell.vloc_grid(si8.gs, moved(si8, ia, ax, -d), si8.pp), rho)
        assert f[ia, ax] == pytest.approx(-(e1 - e2) / (2 * d), abs=1e-8)


def test_kb_force_matches_energy_derivative(si8, si8_psi):
    """E_nl = sum_n occ_n sum_j vclalp_j <beta_j|psi_n>^2 (KB metric) at fixed psi."""
    t = cell.force_tables(si8)
    f = of.fnl_kb(t, si8.kb_g, si8.vclalp, si8_psi, si8.occ)

    def enl(c):
        kb, vcl = cell.kb_tables_g(si8.gs, c, si8.pp)
        p = 2.0 * kb.T @ si8_psi.T - np.outer(kb[0], si8_psi[:, 0]) - 2.0 * np.outer(kb[1], si8_psi[:, 1])
        return float(np.sum(si8.occ[None, :] * vcl[:, None] * p * p))

    d = 1e-4
    for ia, ax in [(1, 2), (4, 0)]:
        fd = -(enl(moved(si8, ia, ax, d)) - enl(moved(si8, ia, ax, -d))) / (2 * d)
        assert f[ia, ax] == pytest.approx(fd, abs=1e-8)


def test_total_force_matches_scf_energy_derivative(si8, si8_psi):
    """F = floc + fnl + fewald against -dE/dR of the converged total energy
    (Pulay mixing, residual < 1e-10).  The FFT grid breaks translation
    invariance slightly, so the tolerance is 2e-5 Ry/bohr (the force-error
    gate of the mixed path is 2e-4 Ry/bohr)."""
    def converge(s):
        st = ScfState(s, si8_psi, nlmode=1, mixbeta=0.8, kerker_q0=0.8, pulay=10)
        for _ in range(30):
            r = st.iteration(noband=16)
        assert r["resid"] < 1e-10
        return st, r

    st, _ = converge(si8)
    t = cell.force_tables(si8)
    rho = st.ham.softchg(st.psi, si8.occ)
    f = (of.floc_g(t, rho, si8.gs.grid) + of.fnl_kb(t, si8.kb_g, si8.vclalp, st.psi, si8.occ)
         + cell.ewald_forces(si8.cell, si8.gs))
    ia, ax, d = 3, 2, 2e-3
    e = []
    for sgn in (1, -1):
        s = cell.build_system(moved(si8, ia, ax, sgn * d), 12.0, 48.0, 16)
        e.append(converge(s)[1]["etot"])
    assert f[ia, ax] == pytest.approx(-(e[0] - e[1]) / (2 * d), abs=2e-5)


def _kbr_energy(s, b, off, mesh, vnl, psir):
    """sum_n occ_n / Omega sum_l clalp_l P_l^2, P_l = rdelv sum vnl_l psi_n(r)."""
    e = 0.0
    for n in range(psir.shape[0]):
        for a in range(off.size - 1):
            sl = slice(off[a], off[a + 1])
            p = b["rdelv"] * (psir[n, mesh[sl]] @ vnl[sl])
            e += s.occ[n] / s.gs.rvol * float(np.sum(b["clalp"] * p * p))
    return e


def test_real_space_kb_force_matches_fixed_point_derivative(si8, si8_psi):
    """fnnlcl2 restated (oracle.forces.fnl_r) against central differences of
    the real-space KB energy over the SAME point set, the projector values
    recomputed at the moved atom (what fnnlcl2 differentiates).  The two differ
    only by the tables' interpolation (derivative table against the
    derivative of the interpolated table) and the h^2 term: 1e-6 of the
    largest component."""
    import dataclasses
    from oracle import tables
    b = cell.kbr_builder_tables(si8.gs, si8.cell, si8.pp)
    off, mesh, vnl, dvnl = tables.setnlc(b, b["ityp"], b["satm"], grad=True)
    psir = np.array([oracle.wvg2r(si8.gs, c) for c in si8_psi])
    f = of.fnl_r(off, mesh, vnl, dvnl, b["clalp"], b["rdelv"], si8.gs.rvol, psir, si8.occ)
    k = np.array(si8.gs.grid)
    h = 1e-4
    for a, ax in [(0, 0), (2, 1), (5, 2), (7, 0)]:
        sl = slice(off[a], off[a + 1])
        m = mesh[sl]
        n = np.stack([m % k[0], (m // k[0]) % k[1], m // (k[0] * k[1])], axis=1)
        e = []
        for sgn in (1, -1):
            satm = b["satm"].copy()
            satm[a] += sgn * h * np.linalg.inv(si8.gs.rba)[:, ax]
            df = n / k - satm[a]
            df -= np.round(df)
            d = df @ si8.gs.rba.T
            r = np.sqrt(np.einsum("ij,ij->i", d, d))
            v2 = vnl.copy()
            for l in range(4):
                v2[sl, l] = tables.setqlm(r, b["dltnl"][0], b["tabnl"][l], tables._poly(l, d[:, 0], d[:, 1], d[:, 2]))
            e.append(_kbr_energy(si8, b, off, mesh, v2, psir))
        fd = -(e[0] - e[1]) / (2 * h)
        assert f[a, ax] == pytest.approx(fd, abs=1e-6 * np.max(np.abs(f)))
    assert np.max(np.abs(f)) > 1e-3
