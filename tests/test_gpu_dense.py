"""Band-space dense algebra at band counts that span several 32-wide blocks:
Gram-Schmidt through the blocked FP64 Cholesky and triangular inverse
(schmidt2 + rsdecmp/rsinvcd, schmidt.f90:117-544) and the subspace
eigen-decomposition + rotation (untryt2/untryhc2, eigen.f90:1171-1451),
against the oracle.  nb = 160 is the Si64 band count (matrix in one CTA's
registers); nb = 200 exceeds one SM and runs on the cooperative kernels that
spread the columns over one CTA per SM; nb = 300 also takes the
back-transformation that keeps 8 eigenvector columns per CTA in shared
memory.

Tolerances: FP64 1e-10 (orthonormalised bands), eigenvalues 1e-10 relative;
mixed precision (FP32 bands, 3xTF32 tensor-core contractions, FP64
Cholesky/eigensolver) 1e-4.
"""
import numpy as np
import pytest

import oracle
from qxmd_b200 import cell
from qxmd_b200.lib import QX_NL_GSPACE, QX_PREC_FP64, QX_PREC_MIXED, Context, QxError

from gpu_util import need_gpu, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nb", [48, 160, 200])
@pytest.mark.parametrize("prec,tol", [(QX_PREC_FP64, 1e-10), (QX_PREC_MIXED, 1e-4)])
def test_schmidt_many_blocks(si8, nb, prec, tol):
    need_gpu()
    c = cell.random_wavefunctions(si8.gs.nplwex, nb)
    ref, _, rc = oracle.schmidt(c)
    assert rc == 0
    ctx = Context(si8, prec, QX_NL_GSPACE, nband=nb)
    try:
        q = ctx.schmidt_host(c)
    finally:
        ctx.close()
    assert relerr(q, ref) < tol
    # orthonormal in the Gamma metric
    s = 2.0 * q @ q.T - np.outer(q[:, 0], q[:, 0])
    assert np.max(np.abs(s - np.eye(nb))) < (1e-10 if prec == QX_PREC_FP64 else 1e-4)


@pytest.mark.parametrize("nb,bad", [(100, 70), (200, 170)])
def test_schmidt_reports_first_bad_pivot_in_later_block(si8, nb, bad):
    """A zero band gives a zero Cholesky pivot at its row and the error names
    it.  nb = 100 runs the one-CTA register kernel, nb = 200 the cooperative
    whole-GPU kernel."""
    need_gpu()
    c = cell.random_wavefunctions(si8.gs.nplwex, nb)
    c[bad] = 0.0
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE, nband=nb)
    try:
        with pytest.raises(QxError) as e:
            ctx.schmidt_host(c)
        assert e.value.code == 3
        assert "band %d" % bad in str(e.value)
    finally:
        ctx.close()


@pytest.mark.parametrize("nb", [48, 160, 200, 300])
@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_untryt_many_blocks(si8, nb, prec):
    need_gpu()
    c = cell.random_wavefunctions(si8.gs.nplwex, nb)
    c, _, rc = oracle.schmidt(c)
    assert rc == 0
    h = oracle.Ham(si8, 1)
    hc = h.hpsi(c)
    hm, _ = oracle.hmatrix(c, hc)
    w_ref, u_ref, sweeps = oracle.jacobi(hm, maxsweep=80)
    assert sweeps >= 0
    ctx = Context(si8, prec, QX_NL_GSPACE, nband=nb)
    try:
        ctx.put_psi(c)
        ctx.put_hpsi(hc)
        ctx.hmatrix()
        ev = ctx.untryt()
        ctx.untryhc()
        psi = ctx.get_psi()
        hpsi = ctx.get_hpsi()
    finally:
        ctx.close()
    etol = 1e-10 if prec == QX_PREC_FP64 else 1e-5
    assert relerr(ev, w_ref) < etol
    # the rotated bands diagonalise the subspace Hamiltonian
    hm2 = 2.0 * psi @ hpsi.T - np.outer(psi[:, 0], hpsi[:, 0])
    off = hm2 - np.diag(np.diag(hm2))
    scale = np.max(np.abs(w_ref))
    assert np.max(np.abs(off)) / scale < (1e-9 if prec == QX_PREC_FP64 else 1e-4)
    assert relerr(np.diag(hm2), w_ref) < etol * 10
    # and match the oracle's rotation where eigenvalues are separated
    ref_psi = oracle.rotate(c, u_ref)
    gaps = np.minimum(np.diff(w_ref, prepend=-np.inf), np.diff(w_ref, append=np.inf))
    sep = gaps > 1e-6 * scale
    assert relerr(psi[sep], ref_psi[sep]) < (1e-8 if prec == QX_PREC_FP64 else 1e-3)


def test_mixed_contractions_with_unaligned_band_stride():
    """nplwex = 5042 is not a multiple of four floats, so the band arrays'
    rows break the 16-byte stride rule of the tensor maps: the tensor-core
    contractions restage their operands (Gram-Schmidt: S = C^T C and C L^-T;
    the KB contractions <beta|psi> and K P read a padded copy of the projector
    table made once), with the FP32 tolerances of the mixed path against the
    oracle."""
    need_gpu()
    s = cell.build_system(cell.diamond_si((1, 1, 1), seed=1), 170.0 / 4.0, 170.0, 48, with_ewald=False)
    assert s.gs.nplwex % 4 == 2
    c = cell.random_wavefunctions(s.gs.nplwex, 48)
    ref, _, rc = oracle.schmidt(c)
    assert rc == 0
    for _ in range(2):
        ctx = Context(s, QX_PREC_MIXED, QX_NL_GSPACE, nband=48)
        try:
            q = ctx.schmidt_host(c)
            ctx.put_psi(q)
            ctx.enonloc()
            hq = ctx.get_hpsi()
            kb = ctx.hckbpp_g_host(q, np.zeros_like(q))
        finally:
            ctx.close()
        assert relerr(q, ref) < 1e-4
        h = oracle.Ham(s, QX_NL_GSPACE)
        assert relerr(hq, h.hpsi(q)) < 2e-5
        kref = np.array([h.hckbpp(q[b], np.zeros_like(q[b]))[0] for b in range(q.shape[0])])
        assert relerr(kb, kref) < 2e-4
