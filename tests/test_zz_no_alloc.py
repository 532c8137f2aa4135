"""qx_hmatrix_static, the allocation-free band matrix, against qx_hmatrix.

Some host programs cannot allocate device memory once their run has started
(every byte comes from a pool sized at start-up, or an allocation inside the
time step could fail or stall it).  qx_hmatrix_static serves them: it takes
device arrays the caller already owns and keeps its split-K partial sums in a
fixed file-scope device array, so it calls no allocator.  Here its output is
checked against the context path qx_hmatrix (engrad.f90:845-956) on the same
device-resident psi and H psi, on two calls in a row with different inputs,
since the second call finds the first call's partials still in the scratch.

This file sorts last so that a run stopping at its first failure has already
run every other test; it also passes alone in a fresh process (the first call
on a device looks up the scratch address itself).
"""
import numpy as np
import pytest

from qxmd_b200 import cell
from qxmd_b200.lib import QX_NL_GSPACE, QX_PREC_FP64, Context, _ck, last_error, lib

from gpu_util import need_gpu, relerr

pytestmark = pytest.mark.gpu

TOL = 1e-11   # FP64, as the other FP64 band-matrix tests


def _static(torch, ctx, c_ptr, hc_ptr):
    nb, ne = ctx.nb, ctx.ne
    out = torch.full((nb, nb), float("nan"), dtype=torch.float64, device="cuda")
    ctx.sync()
    _ck(lib().qx_hmatrix_static(c_ptr, hc_ptr, ne, nb, out.data_ptr(), None), "qx_hmatrix_static")
    torch.cuda.synchronize()
    # out is column-major hsub(j, i) read as a row-major (i, j) array
    return out.cpu().numpy().T.copy()


def _upper(a):
    """Entries j <= i (row j, column i): the triangle qx_hmatrix keeps."""
    return a[np.triu_indices(a.shape[0])]


@pytest.mark.parametrize("which", ["si8", "si64"])
def test_hmatrix_static_matches_context_path(which):
    need_gpu()
    torch = pytest.importorskip("torch")
    s = cell.si8(with_ewald=False) if which == "si8" else cell.si64(with_ewald=False)
    nb = s.nband
    psi = cell.random_wavefunctions(s.gs.nplwex, nb)
    ctx = Context(s, QX_PREC_FP64, QX_NL_GSPACE)
    try:
        ctx.put_psi(psi)
        ctx.enonloc()                       # hpsi = H psi on the device
        ref_h = ctx.hmatrix()               # <psi_j|H|psi_i>, symmetrised
        c_ptr, hc_ptr = ctx.dev_ptr(0), ctx.dev_ptr(1)
        # first call: H_sub
        got_h = _static(torch, ctx, c_ptr, hc_ptr)
        assert np.all(np.isfinite(got_h))
        assert relerr(_upper(got_h), _upper(ref_h)) < TOL
        # second call, different inputs: the overlap S = <psi_j|psi_i>
        ctx.put_hpsi(psi)
        ref_s = ctx.hmatrix()
        got_s = _static(torch, ctx, c_ptr, c_ptr)
        assert relerr(_upper(got_s), _upper(ref_s)) < TOL
    finally:
        ctx.close()


def test_hmatrix_static_at_the_largest_band_count():
    """nb = 1024, the most the scratch takes: its two split-K partials fill
    the 16 MiB exactly.  Small random operands, checked against an FP64
    matmul with the Gamma-point metric 2 sum - c(1) hc(1), twice in a row."""
    need_gpu()
    torch = pytest.importorskip("torch")
    nb, ne = 1024, 2048
    gen = torch.Generator(device="cuda").manual_seed(3)
    for _ in range(2):
        c = torch.randn((nb, ne), dtype=torch.float64, device="cuda", generator=gen)
        hc = torch.randn((nb, ne), dtype=torch.float64, device="cuda", generator=gen)
        out = torch.full((nb, nb), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        _ck(lib().qx_hmatrix_static(c.data_ptr(), hc.data_ptr(), ne, nb, out.data_ptr(), None), "qx_hmatrix_static")
        torch.cuda.synchronize()
        # column-major hsub(j, i) sits at out[i, j] of the row-major tensor:
        # [i, j] = <c_j|hc_i>
        got = out.cpu().numpy()
        ref = (2.0 * hc @ c.t() - torch.outer(hc[:, 0], c[:, 0])).cpu().numpy()
        assert np.all(np.isfinite(got))
        assert relerr(got, ref) < TOL


def test_hmatrix_static_rejects_oversize():
    need_gpu()
    torch = pytest.importorskip("torch")
    nb, ne = 1025, 64
    c = torch.zeros((nb, ne), dtype=torch.float64, device="cuda")
    out = torch.zeros((nb, nb), dtype=torch.float64, device="cuda")
    rc = lib().qx_hmatrix_static(c.data_ptr(), c.data_ptr(), ne, nb, out.data_ptr(), None)
    assert rc == 1
    assert "1024" in last_error()
