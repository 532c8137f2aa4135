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


def test_bkl_cg_sequential_order(si8, si8_psi):
    """One rank (eigen.f90:699): band k is projected against the FINAL vectors
    of bands < k.  So band k of a sequential sweep equals band k of a batched
    sweep whose input already holds the sequential finals below k (the batched
    sweep projects against its entry copy), to the last bit."""
    h = oracle.Ham(si8, 1)
    c = si8_psi
    hc = h.hpsi(c)
    _, ekib = h.ekinetic(c)
    xs, hxs, es, _, ns = h.eigen(c, hc, ekib, noband=16, sequential=True)
    xb, _, eb, _, _ = h.eigen(c, hc, ekib, noband=16)
    # band 0 has no lower bands: both orders agree; later bands do not
    np.testing.assert_array_equal(xs[0], xb[0])
    assert np.abs(xs[1:] - xb[1:]).max() > 1e-8
    for k in (1, 5, 15):
        x_in = np.concatenate([xs[:k], c[k:]])
        hx_in = np.concatenate([hxs[:k], hc[k:]])
        xk, hxk, ek, _, nk = h.eigen(x_in, hx_in, ekib, noband=16)
        np.testing.assert_array_equal(xk[k], xs[k])
        np.testing.assert_array_equal(hxk[k], hxs[k])
        assert ek[k] == es[k] and nk[k] == ns[k]
    np.testing.assert_allclose(hxs, h.hpsi(xs), atol=1e-10)


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


def test_pulay_mixing_converges_faster_than_linear(si8, si8_psi):
    """mxchgg_pulay (chgdns.f90:954-1120) with the reference defaults
    (itratn 10, aslh 0.8, bslh 0.64, cmetric 20) against Kerker-filtered
    linear mixing: a far smaller density residual after the same iterations."""
    from oracle.scf import ScfState
    lin = ScfState(si8, si8_psi, nlmode=1, mixbeta=0.3, kerker_q0=1.0)
    pul = ScfState(si8, si8_psi, nlmode=1, mixbeta=0.8, kerker_q0=0.8, pulay=10)
    for _ in range(16):
        rl = lin.iteration(noband=16)
        rp = pul.iteration(noband=16)
    assert rp["resid"] < 0.01 * rl["resid"]


def test_pulay_history_rules():
    """The history bookkeeping of mxchgg_pulay on synthetic residuals: one
    Kerker step first, c sums to 1, a singular metric drops the oldest entry,
    a full history restarts on the next call."""
    from oracle.scf import Pulay
    g2 = np.array([0.0, 1.0, 2.0, 4.0, 8.0, -1.0])
    p = Pulay(g2, 1.0, itratn=3)
    rng = np.random.default_rng(0)
    rin = rng.standard_normal(6) + 0j
    out = rin + rng.standard_normal(6)
    new = p.mix(rin, out)
    m = g2 > 0
    np.testing.assert_allclose(new[m], (rin + p.k * (out - rin))[m])
    assert len(p.u) == 1
    p.mix(rin + 0.1, out + 0.3)
    assert len(p.u) == 2
    # same residual again: singular metric, the oldest entry goes
    p.mix(rin + 0.2, out + 0.3)
    assert len(p.u) == 2
    p.mix(rin + 0.3, out * 1.5)
    assert len(p.u) == 3 and p.reset_next
    p.mix(rin, out)
    assert len(p.u) == 1
