"""The device path against the committed oracle fixtures (tests/golden/,
written by tests/golden/make_fixtures.py from the CPU FP64 oracle) on the
workloads the benchmark runs:

* Si64 (54^3 grid, 160 bands, 256 G-space KB projectors) at the reference's
  LCG start: Gram-Schmidt (schmidt2), H|psi> of every band (enonloc: four
  bands in full, every band through its norm and two seeded projections),
  H_sub (hmatrix2), its eigenvalues (untryt2), one batched eigen_BKL sweep and
  the density (softchg);
* Si64 iterated in pwlda_md order to self-consistency (Pulay mixing with the
  reference defaults): total energy per atom, eigenvalues and forces, in
  both precisions and both CG band orders, at the gates of 2e-6 Ry/atom and
  2e-4 Ry/bohr for the mixed path;
* three cells of the 48-cell batch (21^3, 42x21x21, 25^3 grids) advanced
  concurrently on their own streams, to self-consistency;
* four bands of H|psi> on Si512 (96^3 grid, 2048 projectors).
"""
import os

import numpy as np
import pytest

import oracle
from qxmd_b200 import cell
from qxmd_b200.lib import CgParm, Context, QX_NL_GSPACE, QX_PREC_FP64, QX_PREC_MIXED

from gpu_util import need_gpu, relerr

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PULAY = dict(mixbeta=0.8, kerker_q0=0.8)
# relative tolerances of single H|psi>-level results (FP64 / mixed)
TOL = {QX_PREC_FP64: 1e-11, QX_PREC_MIXED: 2e-5}
# gates on self-consistent results: Ry/atom, Ry/bohr, Ry (occupied eigenvalues)
GATE = {QX_PREC_FP64: (1e-9, 1e-7, 1e-8), QX_PREC_MIXED: (2e-6, 2e-4, 2e-5)}


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def gamma_dot(a, b):
    return 2.0 * np.sum(a * b, axis=-1) - a[..., 0] * b[..., 0]


def checksum_vectors(nplwex, n=2):
    return np.random.default_rng(2024).standard_normal((n, nplwex))


def low_g(rho, gs, n):
    k1, k2, k3 = gs.grid
    z = np.fft.fftn(rho.reshape(k3, k2, k1)).ravel() / rho.size
    return z[gs.ijk_pos[:n]]


@pytest.fixture(scope="module")
def si64():
    return cell.si64()


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_si64_start_against_fixture(si64, prec):
    need_gpu()
    g = golden("si64_start")
    s = si64
    raw = cell.random_wavefunctions(s.gs.nplwex, s.nband)
    psi, _, rc = oracle.schmidt(raw)            # the oracle's orthonormal start
    assert rc == 0
    ctx = Context(s, prec, QX_NL_GSPACE)
    try:
        # schmidt2 on the raw LCG vectors
        q = ctx.schmidt_host(raw)
        assert relerr(q, psi) < (1e-10 if prec == QX_PREC_FP64 else 2e-4)
        # H|psi> of every band
        ctx.put_psi(psi)
        ctx.enonloc()
        hc = ctx.get_hpsi()
        sel = list(g["sel_bands"])
        assert relerr(hc[sel], g["hpsi_sel"]) < TOL[prec]
        assert relerr(gamma_dot(hc, hc), g["hpsi_norm2"]) < 10 * TOL[prec]
        chk = np.stack([gamma_dot(hc, v[None, :]) for v in checksum_vectors(s.gs.nplwex)])
        assert relerr(chk, g["hpsi_chk"]) < 10 * TOL[prec]
        # H_sub and its eigenvalues
        hs = ctx.hmatrix()
        iu = np.triu_indices(s.nband)
        assert relerr(hs[iu], g["hsub"][iu]) < TOL[prec]
        ev = ctx.untryt()
        assert relerr(ev, g["hsub_eig"]) < (1e-11 if prec == QX_PREC_FP64 else 1e-5)
        # one batched eigen_BKL sweep from the orthonormal start
        ctx.put_psi(psi)
        ctx.enonloc()
        ctx.ekinetic()
        nri, _ = ctx.eigen(CgParm.defaults(int(s.cell.nel // 2)))
        eig = ctx.get_eig()
        if prec == QX_PREC_FP64:
            assert relerr(eig, g["cg_eig"]) < 1e-10
            np.testing.assert_array_equal(nri, g["cg_nriter"])
            x = ctx.get_psi()
            chk = np.stack([gamma_dot(x, v[None, :]) for v in checksum_vectors(s.gs.nplwex)])
            assert relerr(chk, g["cg_psi_chk"]) < 1e-9
        else:
            assert np.max(np.abs(eig - g["cg_eig"])) < 1e-4
        # density of the orthonormal start
        rho = ctx.softchg_host(psi)
        assert rho.sum() * s.gs.rvol / s.gs.kfft0 == pytest.approx(float(g["rho_sum"]), rel=TOL[prec])
        assert relerr(low_g(rho, s.gs, g["rho_lowg"].size), g["rho_lowg"]) < 10 * TOL[prec]
    finally:
        ctx.close()


@pytest.mark.parametrize("prec,sequential", [(QX_PREC_FP64, 0), (QX_PREC_FP64, 1), (QX_PREC_MIXED, 0)])
def test_si64_scf_against_fixture(si64, prec, sequential):
    """40 SCF iterations from the LCG start: the self-consistent total energy,
    occupied eigenvalues and forces (local + G-space KB) against the oracle's
    after the same count; for the FP64 batched path, also the first iterations
    one by one (same algorithm, same order)."""
    need_gpu()
    g = golden("si64_scf")
    s = si64
    psi = cell.random_wavefunctions(s.gs.nplwex, s.nband)
    ctx = Context(s, prec, QX_NL_GSPACE)
    try:
        ctx.put_psi(psi)
        ctx.schmidt()
        ctx.scf_init(**PULAY)
        ctx.scf_mixing(10, 20.0)
        ctx.scf_rho_from_psi()
        p = CgParm.defaults(int(g["noband"]), sequential=sequential)
        outs = [ctx.scf_iteration(p) for _ in range(g["etot"].size)]
        e = np.array([o["etot"] for o in outs])
        if prec == QX_PREC_FP64 and not sequential:
            # same trajectory while the energy still moves by hundreds of Ry
            assert relerr(e[:4], g["etot"][:4]) < 1e-9
        natom = int(g["natom"])
        de, dfc, deig = GATE[prec]
        assert abs(e[-1] - g["etot"][-1]) / natom < de
        nocc = int(g["noband"])
        assert np.max(np.abs(ctx.get_eig()[:nocc] - g["eig"][:nocc])) < deig
        ctx.set_force_tables()
        fl, fn = ctx.forces()
        assert np.max(np.abs(fl - g["floc"])) < dfc
        assert np.max(np.abs(fn - g["fnl"])) < dfc
    finally:
        ctx.close()


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_si64_scf_rspace_against_fixture(si64, prec):
    """The same 40 iterations with real-space KB projectors (calnlc, the
    reference's default for Si): self-consistent energy per atom and
    occupied eigenvalues against the oracle's."""
    need_gpu()
    from qxmd_b200.lib import QX_NL_RSPACE
    g = golden("si64_scf_rspace")
    s = si64
    ctx = Context(s, prec, QX_NL_RSPACE)
    try:
        ctx.put_psi(cell.random_wavefunctions(s.gs.nplwex, s.nband))
        ctx.schmidt()
        ctx.scf_init(**PULAY)
        ctx.scf_mixing(10, 20.0)
        ctx.scf_rho_from_psi()
        p = CgParm.defaults(int(g["noband"]))
        e = [ctx.scf_iteration(p)["etot"] for _ in range(g["etot"].size)]
        if prec == QX_PREC_FP64:
            assert relerr(np.array(e[:4]), g["etot"][:4]) < 1e-9
        de, _, deig = GATE[prec]
        assert abs(e[-1] - g["etot"][-1]) / int(g["natom"]) < de
        nocc = int(g["noband"])
        assert np.max(np.abs(ctx.get_eig()[:nocc] - g["eig"][:nocc])) < deig
    finally:
        ctx.close()


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_batch_cells_against_fixture(prec):
    """Three cells of the batch, each on its own stream and enqueued before any
    is read, iterated to self-consistency."""
    need_gpu()
    torch = pytest.importorskip("torch")
    g = golden("batch_cells")
    ids = [int(i) for i in g["cells"]]
    cells = [cell.batch_cell(i) for i in ids]
    streams = [torch.cuda.Stream() for _ in cells]
    ctxs, parms = [], []
    try:
        for s, st in zip(cells, streams):
            ctx = Context(s, prec, QX_NL_GSPACE, stream=st.cuda_stream)
            ctx.put_psi(cell.random_wavefunctions(s.gs.nplwex, s.nband))
            ctx.schmidt()
            ctx.scf_init(**PULAY)
            ctx.scf_mixing(10, 20.0)
            ctx.scf_rho_from_psi()
            ctxs.append(ctx)
            parms.append(CgParm.defaults(int(s.cell.nel // 2)))
        last = None
        for _ in range(int(g["iters"])):
            for ctx, p in zip(ctxs, parms):
                ctx.scf_launch(p)
            last = [ctx.scf_result() for ctx in ctxs]
        de = GATE[prec][0]
        for i, s, r, ctx in zip(ids, cells, last, ctxs):
            assert abs(r["etot"] - g[f"c{i}_etot"][-1]) / s.cell.natom < de, i
            nocc = int(s.cell.nel // 2)
            assert np.max(np.abs(ctx.get_eig()[:nocc] - g[f"c{i}_eig"][:nocc])) < GATE[prec][2], i
    finally:
        for ctx in ctxs:
            ctx.close()


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_si512_hpsi_against_fixture(prec):
    """H|psi> of four bands on the Si512 cell (96^3 grid, 48490 real
    components, 2048 projectors)."""
    need_gpu()
    g = golden("si512_hpsi")
    s = cell.si512()
    psi = cell.random_wavefunctions(s.gs.nplwex, 4)
    ctx = Context(s, prec, QX_NL_GSPACE, nband=4)
    try:
        ctx.put_psi(psi)
        ctx.enonloc()
        hc = ctx.get_hpsi()
    finally:
        ctx.close()
    hs = psi @ hc.T * 2.0 - np.outer(psi[:, 0], hc[:, 0])
    assert relerr(hs, g["hsub"]) < TOL[prec]
    assert relerr(gamma_dot(hc, hc), g["hpsi_norm2"]) < 10 * TOL[prec]
    chk = np.stack([gamma_dot(hc, v[None, :]) for v in checksum_vectors(s.gs.nplwex)])
    assert relerr(chk, g["hpsi_chk"]) < 10 * TOL[prec]
    assert relerr(hc[:, :1024], g["hpsi_head"]) < TOL[prec]
