"""H|psi> through the C ABI against the oracle (hcnonloc engrad.f90:411-606,
hckbpp_ib_g nlkbpp.f90:1623-1721, calnlc nlkbppr.f90:1773-1900).

Tolerances: FP64 context 1e-11 relative to max|H psi|; mixed (FP32 FFT and
contractions) 2e-5."""
import numpy as np
import pytest

import oracle
from qxmd_b200 import cell
from qxmd_b200.lib import (Context, QX_NL_GSPACE, QX_NL_NONE, QX_NL_RSPACE, QX_PREC_FP64,
                           QX_PREC_MIXED)

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
TOL = {QX_PREC_FP64: 1e-11, QX_PREC_MIXED: 2e-5}


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
@pytest.mark.parametrize("nlmode", [QX_NL_NONE, QX_NL_GSPACE, QX_NL_RSPACE])
def test_enonloc_matches_oracle_si8(si8, si8_psi, prec, nlmode):
    need_gpu()
    ctx = Context(si8, prec, nlmode)
    ctx.put_psi(si8_psi)
    ctx.enonloc()
    hc = ctx.get_hpsi()
    ref = oracle.Ham(si8, nlmode).hpsi(si8_psi)
    assert relerr(hc, ref) < TOL[prec]
    # the imaginary part of the G=0 coefficient stays exactly zero
    assert np.all(hc[:, 1] == 0.0)


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_hcnonloc_shim_accumulates(si8, si8_psi, prec):
    need_gpu()
    ctx = Context(si8, prec, QX_NL_RSPACE)
    rng = np.random.default_rng(7)
    rhcr = rng.standard_normal(si8_psi.shape)
    rhcr[:, 1] = 0.0
    out = ctx.hcnonloc_host(si8_psi, rhcr)
    h = oracle.Ham(si8, 2)
    ref = np.array([h.hcnonloc(si8_psi[b], rhcr[b]) for b in range(si8_psi.shape[0])])
    assert relerr(out, ref) < TOL[prec] * 10


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_hckbpp_shim(si8, si8_psi, prec):
    need_gpu()
    ctx = Context(si8, prec, QX_NL_GSPACE)
    z = np.zeros_like(si8_psi)
    out = ctx.hckbpp_g_host(si8_psi, z)
    h = oracle.Ham(si8, 1)
    ref = np.array([h.hckbpp(si8_psi[b], z[b])[0] for b in range(si8_psi.shape[0])])
    assert relerr(out, ref) < TOL[prec] * 10


def test_odd_band_count(si8, si8_psi):
    need_gpu()
    s = si8
    ctx = Context(s, QX_PREC_FP64, QX_NL_GSPACE, nband=15)
    ctx.put_psi(si8_psi[:15])
    ctx.enonloc()
    ref = oracle.Ham(s, 1).hpsi(si8_psi[:15])
    assert relerr(ctx.get_hpsi(), ref) < 1e-11


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_enonloc_si64_subset(prec):
    """Si64 (54^3 grid, 4657 plane waves): 6 bands against the oracle."""
    need_gpu()
    s = cell.si64(with_ewald=False)
    c = cell.random_wavefunctions(s.gs.nplwex, 6)
    c /= np.sqrt(np.array([oracle.dot(x, x) for x in c]))[:, None]
    for nl in (QX_NL_GSPACE, QX_NL_RSPACE):
        ctx = Context(s, prec, nl, nband=6)
        ctx.put_psi(c)
        ctx.enonloc()
        ref = oracle.Ham(s, nl).hpsi(c)
        assert relerr(ctx.get_hpsi(), ref) < TOL[prec]


def test_hpsi_linearity_full_si64():
    """Full Si64 band count: H(a x + b y) = a H x + b H y (size-independent check)."""
    need_gpu()
    s = cell.si64(with_ewald=False)
    rng = np.random.default_rng(11)
    x = rng.standard_normal((s.nband, s.gs.nplwex))
    y = rng.standard_normal((s.nband, s.gs.nplwex))
    x[:, 1] = y[:, 1] = 0.0
    ctx = Context(s, QX_PREC_FP64, QX_NL_GSPACE)
    out = []
    for v in (x, y, 2.0 * x - 3.0 * y):
        ctx.put_psi(v)
        ctx.enonloc()
        out.append(ctx.get_hpsi())
    assert relerr(out[2], 2.0 * out[0] - 3.0 * out[1]) < 1e-12
    # and Hermitian: <x|Hy> = <y|Hx> band by band
    for b in range(0, s.nband, 37):
        assert oracle.dot(x[b], out[1][b]) == pytest.approx(oracle.dot(y[b], out[0][b]), rel=1e-10)


def _plane_pass_vs_oracle(monkeypatch, s):
    """H|psi> and softchg of 4 random bands of system s on the mixed path
    with the fused plane and column kernels (QX_PLANE=1, QX_ZCOLS=1) and
    with the separate y/x and shared-memory z passes (0), each against the
    oracle and against each other."""
    c = cell.random_wavefunctions(s.gs.nplwex, 4)
    c /= np.sqrt(np.array([oracle.dot(x, x) for x in c]))[:, None]
    h = oracle.Ham(s, QX_NL_GSPACE)
    ref = h.hpsi(c)
    rref = h.softchg(c, s.occ[:4])
    out, rho = {}, {}
    for mode in ("1", "0"):
        monkeypatch.setenv("QX_PLANE", mode)
        monkeypatch.setenv("QX_ZCOLS", mode)
        ctx = Context(s, QX_PREC_MIXED, QX_NL_GSPACE, nband=4)
        try:
            ctx.put_psi(c)
            ctx.enonloc()
            out[mode] = ctx.get_hpsi()
            rho[mode] = ctx.softchg_host(c)
        finally:
            ctx.close()
        assert relerr(out[mode], ref) < TOL[QX_PREC_MIXED]
        assert relerr(rho[mode], rref) < TOL[QX_PREC_MIXED]
    assert relerr(out["1"], out["0"]) < TOL[QX_PREC_MIXED]
    assert relerr(rho["1"], rho["0"]) < TOL[QX_PREC_MIXED]


@pytest.mark.parametrize("ecutdens,n", [(40.0, 21), (55.0, 25), (152.5, 42), (170.0, 45), (200.0, 48),
                                          (217.5, 49), (235.0, 54), (295.0, 60), (760.0, 96)])
def test_plane_pass_lengths(monkeypatch, ecutdens, n):
    """The fused FP32 plane pass on the larger specialised lengths (Si8 cells
    whose density cutoff gives an n^3 grid, wave cutoff ecutdens/4 so the
    sphere spans half the grid) against the oracle and against the separate
    passes, the density pass (softchg) the same way.  96 runs the
    two-threads-a-line kernels (plane, density and inverse z passes)."""
    need_gpu()
    s = cell.build_system(cell.diamond_si((1, 1, 1), seed=1), ecutdens / 4.0, ecutdens, 4, with_ewald=False)
    assert tuple(s.gs.grid) == (n, n, n)
    _plane_pass_vs_oracle(monkeypatch, s)


@pytest.mark.parametrize("index,grid", [(14, (24, 25, 25)), (5, (25, 24, 25)), (1, (25, 27, 27)),
                                        (8, (27, 25, 25)), (2, (42, 21, 21)), (3, (45, 24, 24)),
                                        (32, (45, 42, 21)), (43, (48, 45, 24)), (9, (49, 25, 25)),
                                        (41, (54, 24, 24)), (6, (54, 25, 27)), (10, (54, 27, 27))])
def test_plane_pass_rectangular(monkeypatch, index, grid):
    """The plane kernels on k1 != k2 planes (x and y transforms of different
    lengths; planes of at most 32 rows run both planes' x transforms at
    once): one batch cell of each elongated shape, as above."""
    need_gpu()
    s = cell.batch_cell(index)
    assert tuple(s.gs.grid) == grid
    _plane_pass_vs_oracle(monkeypatch, s)


@pytest.mark.parametrize("plan", ["2x3x4", "3x8", "4x6", "6x4", "8x3", "2x2x2x3", "3x2x2x2"])
def test_fft_radix_plans(si8, si8_psi, monkeypatch, plan):
    """Every stage kernel on a forced radix plan of the 24-point axes
    (QX_FFT_PLAN, the plans the autotuner chooses among): FP64 H|psi> and the
    FP64 full-grid transforms of the density against the oracle, and the
    mixed path's H|psi>."""
    need_gpu()
    monkeypatch.setenv("QX_FFT_PLAN", plan)
    ref = oracle.Ham(si8, QX_NL_GSPACE).hpsi(si8_psi)
    for prec in (QX_PREC_FP64, QX_PREC_MIXED):
        ctx = Context(si8, prec, QX_NL_GSPACE)
        ctx.put_psi(si8_psi)
        ctx.enonloc()
        assert relerr(ctx.get_hpsi(), ref) < TOL[prec]
        ctx.close()
    rng = np.random.default_rng(3)
    x = rng.standard_normal(si8.gs.kfft0)
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    fx, fy = ctx.rfft3_host(1, x, np.zeros_like(x))
    k1, k2, k3 = si8.gs.grid
    z = np.fft.fftn(x.reshape(k3, k2, k1)).ravel() / x.size
    assert relerr(fx + 1j * fy, z) < 1e-13
    ctx.close()


@pytest.mark.parametrize("tile", ["64", "128"])
def test_tensor_core_tile_widths(monkeypatch, tile):
    """The contractions on the other tile widths the autotuner may pick
    (QX_TC_TILE forces one wherever it is valid): Si64 H|psi> with the G-space
    KB contractions, H_sub and Gram-Schmidt, mixed against FP64."""
    need_gpu()
    s = cell.si64(with_ewald=False)
    c = cell.random_wavefunctions(s.gs.nplwex, s.nband)
    c, _, rc = oracle.schmidt(c)
    assert rc == 0
    out = {}
    for prec in (QX_PREC_FP64, QX_PREC_MIXED):
        if prec == QX_PREC_MIXED:
            monkeypatch.setenv("QX_TC_TILE", tile)
        ctx = Context(s, prec, QX_NL_GSPACE)
        ctx.put_psi(c)
        ctx.enonloc()
        hc = ctx.get_hpsi()
        hs = ctx.hmatrix()
        q = ctx.schmidt_host(c + 0.01 * np.roll(c, 1, axis=0))
        out[prec] = (hc, hs, q)
        ctx.close()
    monkeypatch.delenv("QX_TC_TILE")
    for a, b in zip(out[QX_PREC_MIXED], out[QX_PREC_FP64]):
        assert relerr(a, b) < 5e-5
