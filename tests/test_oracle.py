"""The CPU oracle against independent references (numpy pocketfft, direct DFT,
LAPACK) and against its own invariants.  Parity with QXMD itself is unpinned:
the reference ships no test vectors and cannot be built here."""
import numpy as np
import pytest

import oracle
from qxmd_b200 import cell


def direct_dft(x, sign):
    n = x.size
    k = np.arange(n)
    return np.exp(sign * 2j * np.pi * np.outer(k, k) / n) @ x


@pytest.mark.parametrize("n", [2, 3, 4, 5, 7, 12, 20, 21, 24, 27, 45, 54])
def test_fft1_matches_direct_dft(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for sign in (-1, 1):
        y = x.copy()
        oracle.lib().orc_fft1(y, n, sign)
        np.testing.assert_allclose(y, direct_dft(x, sign), atol=1e-12)


def test_fft3_matches_numpy():
    rng = np.random.default_rng(0)
    g = (6, 10, 9)
    a = rng.standard_normal(540) + 1j * rng.standard_normal(540)
    np.testing.assert_allclose(oracle.fft3(a, g, -1), np.fft.fftn(a.reshape(9, 10, 6)).ravel(), atol=1e-11)
    np.testing.assert_allclose(oracle.fft3(a, g, +1), (np.fft.ifftn(a.reshape(9, 10, 6)) * 540).ravel(), atol=1e-11)


def test_wvg2r_real_and_parseval(si8, si8_psi):
    gs = si8.gs
    c = si8_psi[0]
    psir = oracle.wvg2r(gs, c)
    # sum_r psi^2 / N = sum_G |c|^2 (full sphere) = Gamma-metric norm = 1
    assert np.sum(psir ** 2) / gs.kfft0 == pytest.approx(1.0, abs=1e-12)


def test_hcnonloc_matches_numpy_restatement(si8, si8_psi):
    gs = si8.gs
    h = oracle.Ham(si8, 0)
    c = si8_psi[3]
    out = h.hcnonloc(c, np.zeros_like(c))
    # independent: numpy inverse FFT, multiply, forward FFT, pick
    z = np.zeros(gs.kfft0, complex)
    cc = c[0::2] + 1j * c[1::2]
    cc[0] = c[0]
    n = gs.nplw + 1
    z[gs.ijk_pos[:n]] = cc
    z[gs.ijk_neg[1:n]] = np.conj(cc[1:])
    k1, k2, k3 = gs.grid
    psir = np.fft.ifftn(z.reshape(k3, k2, k1)).real * gs.kfft0
    f = np.fft.fftn(psir * si8.vloc.reshape(k3, k2, k1)).ravel() / gs.kfft0
    ref = np.empty_like(c)
    ref[0::2] = f[gs.ijk_pos[:n]].real
    ref[1::2] = f[gs.ijk_pos[:n]].imag
    np.testing.assert_allclose(out, ref, atol=1e-12)


def test_hamiltonian_hermitian_and_nl_modes_agree(si8, si8_psi):
    c = si8_psi
    A = {}
    for mode in (1, 2):
        hc = oracle.Ham(si8, mode).hpsi(c)
        A[mode] = np.array([[oracle.dot(c[i], hc[j]) for j in range(16)] for i in range(16)])
        np.testing.assert_allclose(A[mode], A[mode].T, atol=1e-13)
    # G-space and real-space KB are the same operator up to grid aliasing
    np.testing.assert_allclose(A[1], A[2], atol=1e-5)


def test_cholinv_known_spd():
    rng = np.random.default_rng(3)
    m = rng.standard_normal((12, 12))
    s = m @ m.T + 12 * np.eye(12)
    linv, rc = oracle.cholinv(s)
    assert rc == 0
    L = np.linalg.cholesky(s)
    np.testing.assert_allclose(np.tril(linv), np.linalg.inv(L), atol=1e-12)
    bad = -np.eye(3)
    _, rc = oracle.cholinv(bad)
    assert rc == 1


def test_schmidt_orthonormalises(si8):
    c = cell.random_wavefunctions(si8.gs.nplwex, 16)
    q, _, rc = oracle.schmidt(c)
    assert rc == 0
    S = np.array([[oracle.dot(q[i], q[j]) for j in range(16)] for i in range(16)])
    np.testing.assert_allclose(S, np.eye(16), atol=1e-12)


def test_jacobi_matches_lapack():
    rng = np.random.default_rng(5)
    m = rng.standard_normal((40, 40))
    a = m + m.T
    w, v, sw = oracle.jacobi(a)
    assert sw > 0
    np.testing.assert_allclose(w, np.linalg.eigvalsh(a), atol=1e-12)
    np.testing.assert_allclose(v.T @ a @ v, np.diag(w), atol=1e-11)
    # sign convention: largest-magnitude component positive
    k = np.argmax(np.abs(v), axis=0)
    assert np.all(v[k, np.arange(40)] > 0)


def test_bkl_cg_lowers_band_energies(si8, si8_psi):
    h = oracle.Ham(si8, 1)
    c = si8_psi
    hc = h.hpsi(c)
    e0 = np.array([oracle.dot(c[b], hc[b]) for b in range(16)])
    _, ekib = h.ekinetic(c)
    x, hx, eig, bzan, nri = h.eigen(c, hc, ekib, noband=16)
    assert np.all(eig <= e0 + 1e-12)
    assert np.all((nri >= 1) & (nri <= 4))
    # hx stays H x
    np.testing.assert_allclose(hx, h.hpsi(x), atol=1e-10)
    # each band stays normalised
    for b in range(16):
        assert oracle.dot(x[b], x[b]) == pytest.approx(1.0, abs=1e-12)


def test_softchg_integrates_to_electron_count(si8, si8_psi):
    h = oracle.Ham(si8, 1)
    rho = h.softchg(si8_psi, si8.occ)
    assert rho.sum() * si8.gs.rvol / si8.gs.kfft0 == pytest.approx(si8.cell.nel, rel=1e-12)


def test_xclda_known_values():
    # Perdew-Zunger LDA at rs = 2 (rs >= 1 branch) and rs = 0.5 (rs < 1), Ry
    rho = np.array([3.0 / (4 * np.pi * 8.0), 3.0 / (4 * np.pi * 0.125)])
    v, e, _ = oracle.xclda(rho, 1.0)
    rs = 2.0
    assert e[0] == pytest.approx(2 * (-0.4582 / rs - 0.1423 / (1 + 1.0529 * np.sqrt(rs) + 0.3334 * rs)), rel=1e-6)
    rs = 0.5
    ec = -0.0480 + 0.0311 * np.log(rs) - 0.0116 * rs + 0.0020 * rs * np.log(rs)
    assert e[1] == pytest.approx(2 * (-0.4582 / rs + ec), rel=1e-6)
    assert np.all(v < 0) and np.all(e < 0)
