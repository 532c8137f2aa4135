"""Band-space routines through the C ABI against the oracle: schmidt2
(schmidt.f90:117-378), hmatrix2 (engrad.f90:845-956), untryt2/untryhc2
(eigen.f90:1171-1451), eigen_BKL (eigen.f90:199-938), softchg
(chgdns.f90:388-454), gradresnv and rfft3 (fft3.f90:113-232).

FP64 tolerances 1e-10 (eigenvector-dependent quantities 1e-8); mixed 1e-4."""
import numpy as np
import pytest

import oracle
from qxmd_b200 import cell
from qxmd_b200.lib import CgParm, Context, QxError, QX_NL_GSPACE, QX_NL_RSPACE, QX_PREC_FP64, QX_PREC_MIXED

from gpu_util import need_gpu, relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True, params=["size_threshold", "tensor_cores"])
def fp32_contraction_path(request, monkeypatch):
    """Every test here twice: FP32 contractions below QX_TC_MIN_FLOPS on the
    CUDA-core kernel (the default, which sends this module's Si8 shapes
    there), and all of them on the tensor cores (threshold 0)."""
    if request.param == "tensor_cores":
        monkeypatch.setenv("QX_TC_MIN_FLOPS", "0")
    else:
        monkeypatch.delenv("QX_TC_MIN_FLOPS", raising=False)
    return request.param


def raw_psi(s, nb):
    return cell.random_wavefunctions(s.gs.nplwex, nb)


@pytest.mark.parametrize("prec,tol", [(QX_PREC_FP64, 1e-11), (QX_PREC_MIXED, 1e-4)])
def test_schmidt(si8, prec, tol):
    need_gpu()
    c = raw_psi(si8, 16)
    ctx = Context(si8, prec, QX_NL_GSPACE)
    q = ctx.schmidt_host(c)
    ref, _, rc = oracle.schmidt(c)
    assert rc == 0
    assert relerr(q, ref) < tol


def test_schmidt_not_positive_definite(si8):
    need_gpu()
    c = raw_psi(si8, 16)
    # A zero band gives a zero pivot; the reference's test is pivot <= 1e-30
    # (schmidt.f90:256-267), which rounding noise of merely dependent bands
    # does not reach.
    c[5] = 0.0
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    with pytest.raises(QxError) as e:
        ctx.schmidt_host(c)
    assert e.value.code == 3


@pytest.mark.parametrize("prec,tol", [(QX_PREC_FP64, 1e-11), (QX_PREC_MIXED, 5e-5)])
def test_hmatrix_untryt_untryhc(si8, si8_psi, prec, tol):
    need_gpu()
    h = oracle.Ham(si8, 1)
    hc = h.hpsi(si8_psi)
    ctx = Context(si8, prec, QX_NL_GSPACE)
    ctx.put_psi(si8_psi)
    ctx.put_hpsi(hc)
    hm = ctx.hmatrix()
    hm_ref, eig_ref = oracle.hmatrix(si8_psi, hc)
    assert relerr(hm, hm_ref) < tol
    assert relerr(ctx.get_eig(), eig_ref) < tol
    ev = ctx.untryt()
    ctx.untryhc()
    w, u, _ = oracle.jacobi(hm_ref)
    assert relerr(ev, w) < tol
    psi_ref = oracle.rotate(si8_psi, u)
    hc_ref = oracle.rotate(hc, u)
    assert relerr(ctx.get_psi(), psi_ref) < tol * 1e3
    assert relerr(ctx.get_hpsi(), hc_ref) < tol * 1e3


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
@pytest.mark.parametrize("nlmode", [QX_NL_GSPACE, QX_NL_RSPACE])
def test_eigen_bkl(si8, si8_psi, prec, nlmode):
    need_gpu()
    h = oracle.Ham(si8, nlmode)
    hc = h.hpsi(si8_psi)
    _, ekib = h.ekinetic(si8_psi)
    x_ref, hx_ref, eig_ref, _, nri_ref = h.eigen(si8_psi, hc, ekib, noband=16)
    ctx = Context(si8, prec, nlmode)
    p = CgParm.defaults(16)
    x, hx, eig = ctx.eigen_host(si8_psi, hc, ekib, p)
    if prec == QX_PREC_FP64:
        assert relerr(eig, eig_ref) < 1e-10
        assert relerr(x, x_ref) < 1e-8
        assert relerr(hx, hx_ref) < 1e-8
    else:
        assert relerr(eig, eig_ref) < 1e-4
        assert relerr(x, x_ref) < 1e-2


def test_eigen_snapshot_semantics_real4(si8, si8_psi):
    """CCREAL4: the lower-band snapshot is rounded to real*4 (eigen.f90:78-82)."""
    need_gpu()
    h = oracle.Ham(si8, 1)
    hc = h.hpsi(si8_psi)
    _, ekib = h.ekinetic(si8_psi)
    ref = h.eigen(si8_psi, hc, ekib, noband=16, ccreal4=True)
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    x, hx, eig = ctx.eigen_host(si8_psi, hc, ekib, CgParm.defaults(16, ccreal4=1))
    assert relerr(eig, ref[2]) < 1e-10
    assert relerr(x, ref[0]) < 1e-8


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
@pytest.mark.parametrize("nlmode", [QX_NL_GSPACE, QX_NL_RSPACE])
def test_eigen_bkl_sequential(si8, si8_psi, prec, nlmode):
    """One-rank order: bands one after another, each against the final
    vectors of the bands below (one graph launch for the sweep)."""
    need_gpu()
    h = oracle.Ham(si8, nlmode)
    hc = h.hpsi(si8_psi)
    _, ekib = h.ekinetic(si8_psi)
    x_ref, hx_ref, eig_ref, _, nri_ref = h.eigen(si8_psi, hc, ekib, noband=16, sequential=True)
    ctx = Context(si8, prec, nlmode)
    p = CgParm.defaults(16, sequential=1)
    for _ in range(2):   # the second call replays the cached graph
        x, hx, eig = ctx.eigen_host(si8_psi, hc, ekib, p)
        if prec == QX_PREC_FP64:
            assert relerr(eig, eig_ref) < 1e-10
            assert relerr(x, x_ref) < 1e-8
            assert relerr(hx, hx_ref) < 1e-8
        else:
            assert relerr(eig, eig_ref) < 1e-4
            assert relerr(x, x_ref) < 1e-2


def test_eigen_sequential_real4(si8, si8_psi):
    """One-rank order with the real*4 snapshot of the CCREAL4 build."""
    need_gpu()
    h = oracle.Ham(si8, 1)
    hc = h.hpsi(si8_psi)
    _, ekib = h.ekinetic(si8_psi)
    ref = h.eigen(si8_psi, hc, ekib, noband=16, ccreal4=True, sequential=True)
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    x, hx, eig = ctx.eigen_host(si8_psi, hc, ekib, CgParm.defaults(16, ccreal4=1, sequential=1))
    assert relerr(eig, ref[2]) < 1e-10
    assert relerr(x, ref[0]) < 1e-8


@pytest.mark.parametrize("prec,tol", [(QX_PREC_FP64, 1e-12), (QX_PREC_MIXED, 1e-5)])
def test_softchg(si8, si8_psi, prec, tol):
    need_gpu()
    ctx = Context(si8, prec, QX_NL_GSPACE)
    rho = ctx.softchg_host(si8_psi)
    ref = oracle.Ham(si8, 1).softchg(si8_psi, si8.occ)
    assert relerr(rho, ref) < tol
    assert rho.sum() * si8.gs.rvol / si8.gs.kfft0 == pytest.approx(si8.cell.nel, rel=10 * tol)


def test_gradres(si8, si8_psi):
    need_gpu()
    h = oracle.Ham(si8, 1)
    hc = h.hpsi(si8_psi)
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    ctx.put_psi(si8_psi)
    ctx.put_hpsi(hc)
    ctx.hmatrix()
    prod, zmax, zsum = ctx.gradres()
    _, eig = oracle.hmatrix(si8_psi, hc)
    pref, zm, zs = oracle.gradres(si8_psi, hc, eig, si8.occ)
    assert relerr(prod, pref) < 1e-10
    assert zmax == pytest.approx(zm, rel=1e-10)


def test_rfft3(si8):
    need_gpu()
    gs = si8.gs
    rng = np.random.default_rng(2)
    x = rng.standard_normal(gs.kfft0)
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    fx, fy = ctx.rfft3_host(1, x, np.zeros_like(x))
    k1, k2, k3 = gs.grid
    ref = np.fft.fftn(x.reshape(k3, k2, k1)).ravel() / gs.kfft0
    assert relerr(fx + 1j * fy, ref) < 1e-13
    bx, by = ctx.rfft3_host(2, fx, fy)
    assert relerr(bx, x) < 1e-13
    assert np.all(by == 0.0)


def _si8_at(ecutdens):
    return cell.build_system(cell.diamond_si((1, 1, 1), seed=1), ecutdens / 4.0, ecutdens, 4, with_ewald=False)


@pytest.mark.parametrize("make,grid", [
    (lambda: _si8_at(32.5), (20, 20, 20)), (lambda: cell.batch_cell(42), (21, 21, 21)),
    (lambda: cell.batch_cell(14), (24, 25, 25)), (lambda: cell.batch_cell(5), (25, 24, 25)),
    (lambda: cell.batch_cell(1), (25, 27, 27)), (lambda: cell.batch_cell(47), (27, 27, 27)),
    (lambda: _si8_at(75.0), (30, 30, 30)), (lambda: _si8_at(85.0), (32, 32, 32)),
    (lambda: cell.batch_cell(6), (54, 25, 27))])
def test_rfft3_register_lines(monkeypatch, make, grid):
    """The FP64 full-grid transform with its z and y passes one line per
    thread in registers (lengths up to 32) against numpy, both directions,
    and against the shared-memory passes (QX_FULL_LINES=0)."""
    need_gpu()
    s = make()
    assert tuple(s.gs.grid) == grid
    k1, k2, k3 = grid
    x = np.random.default_rng(5).standard_normal(s.gs.kfft0)
    ref = np.fft.fftn(x.reshape(k3, k2, k1)).ravel() / s.gs.kfft0
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("QX_FULL_LINES", mode)
        ctx = Context(s, QX_PREC_FP64, QX_NL_GSPACE, nband=4)
        try:
            fx, fy = ctx.rfft3_host(1, x, np.zeros_like(x))
            bx, by = ctx.rfft3_host(2, fx, fy)
        finally:
            ctx.close()
        assert relerr(fx + 1j * fy, ref) < 1e-13
        assert relerr(bx, x) < 1e-13
        out[mode] = fx + 1j * fy
    assert relerr(out["1"], out["0"]) < 1e-13


@pytest.mark.parametrize("prec,tol", [(QX_PREC_FP64, 1e-12), (QX_PREC_MIXED, 1e-5)])
def test_tddft_overlap(si8, si8_psi, prec, tol):
    """tddft_fssh_cal_matrix (tddft_fssh.f90:1344-1414): aij = <psi_i(t)|psi_j(t+dt)>
    with the Gamma metric, previous-step wavefunctions kept on the device."""
    need_gpu()
    rng = np.random.default_rng(7)
    prev = si8_psi
    cur = si8_psi + 1e-2 * rng.standard_normal(si8_psi.shape)
    cur[:, 1] = 0.0
    ctx = Context(si8, prec, QX_NL_GSPACE)
    ctx.put_psi(prev)
    ctx.tddft_store()
    ctx.put_psi(cur)
    a = ctx.tddft_overlap()
    ref = np.array([[oracle.dot(prev[i], cur[j]) for j in range(16)] for i in range(16)])
    assert relerr(a, ref) < tol
