"""Whole SCF iterations (pwlda.f90:1628-3700 order) on the device against the
oracle's iteration on the same inputs (Si8, G-space and real-space KB; linear
Kerker and Pulay density mixing; batched and one-rank CG order)."""
import numpy as np
import pytest

import oracle
from oracle.scf import ScfState
from qxmd_b200 import cell
from qxmd_b200.lib import CgParm, Context, QX_NL_GSPACE, QX_NL_RSPACE, QX_PREC_FP64, QX_PREC_MIXED

from gpu_util import need_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nlmode", [QX_NL_GSPACE, QX_NL_RSPACE])
def test_scf_iterations_match_oracle_fp64(si8, si8_psi, nlmode):
    need_gpu()
    st = ScfState(si8, si8_psi, nlmode=nlmode)
    ctx = Context(si8, QX_PREC_FP64, nlmode)
    ctx.put_psi(si8_psi)
    ctx.scf_init()
    ctx.scf_rho_from_psi()
    p = CgParm.defaults(16)
    for it in range(4):
        g = ctx.scf_iteration(p)
        r = st.iteration(noband=16)
        assert g["etot"] == pytest.approx(r["etot"], abs=1e-8 * max(1.0, abs(r["etot"])))
        assert g["ncg_hpsi"] == r["ncg_hpsi"]
        assert g["resid"] == pytest.approx(r["resid"], rel=1e-6)


def test_scf_mixed_tracks_fp64(si8, si8_psi):
    need_gpu()
    p = CgParm.defaults(16)
    e = {}
    for prec in (QX_PREC_FP64, QX_PREC_MIXED):
        ctx = Context(si8, prec, QX_NL_GSPACE)
        ctx.put_psi(si8_psi)
        ctx.scf_init()
        ctx.scf_rho_from_psi()
        e[prec] = [ctx.scf_iteration(p)["etot"] for _ in range(6)]
    # same trajectory to FP32 accuracy over the first iterations
    assert abs(e[QX_PREC_MIXED][0] - e[QX_PREC_FP64][0]) < 1e-3
    assert abs(e[QX_PREC_MIXED][-1] - e[QX_PREC_FP64][-1]) < 5e-2


@pytest.mark.parametrize("sequential", [0, 1])
def test_scf_pulay_matches_oracle_fp64(si8, si8_psi, sequential):
    """Pulay mixing (mxchgg_pulay, chgdns.f90:954-1120) with the reference
    defaults aslh 0.8, bslh 0.64, cmetric 20, here with a 4-entry history so
    that the restart after a full history is crossed too."""
    need_gpu()
    st = ScfState(si8, si8_psi, nlmode=QX_NL_GSPACE, mixbeta=0.8, kerker_q0=0.8, pulay=4)
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    ctx.put_psi(si8_psi)
    ctx.scf_init(mixbeta=0.8, kerker_q0=0.8)
    ctx.scf_mixing(4, 20.0)
    ctx.scf_rho_from_psi()
    p = CgParm.defaults(16, sequential=sequential)
    for it in range(7):
        g = ctx.scf_iteration(p)
        r = st.iteration(noband=16, sequential=bool(sequential))
        assert g["etot"] == pytest.approx(r["etot"], abs=1e-8 * max(1.0, abs(r["etot"])))
        assert g["ncg_hpsi"] == r["ncg_hpsi"]
        assert g["resid"] == pytest.approx(r["resid"], rel=1e-6)


def test_scf_graph_replay_matches_stream_launches(si8, si8_psi, monkeypatch):
    """The iteration captured as a CUDA graph (and replayed for the alternating
    buffer arrangements) gives the same numbers as the same launches issued
    one by one."""
    need_gpu()
    p = CgParm.defaults(16)
    res = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("QX_GRAPH", mode)
        for prec in (QX_PREC_FP64, QX_PREC_MIXED):
            ctx = Context(si8, prec, QX_NL_GSPACE)
            ctx.put_psi(si8_psi)
            ctx.scf_init(mixbeta=0.8, kerker_q0=0.8)
            ctx.scf_mixing(10, 20.0)
            ctx.scf_rho_from_psi()
            outs = [ctx.scf_iteration(p) for _ in range(6)]
            res[mode, prec] = (outs, ctx.get_psi(), ctx.get_rho())
    for prec in (QX_PREC_FP64, QX_PREC_MIXED):
        (oa, pa, ra), (ob, pb, rb) = res["0", prec], res["1", prec]
        for a, b in zip(oa, ob):
            assert a["etot"] == b["etot"] and a["ncg_hpsi"] == b["ncg_hpsi"]
            assert a["eig_clusters"] == b["eig_clusters"] and a["zmax"] == b["zmax"]
        np.testing.assert_array_equal(pa, pb)
        np.testing.assert_array_equal(ra, rb)


@pytest.mark.parametrize("graph", ["1", "0"])
@pytest.mark.parametrize("prec", [QX_PREC_MIXED, QX_PREC_FP64])
def test_scf_iteration_host_matches_separate_calls(si8, si8_psi, prec, graph, monkeypatch):
    """qx_scf_iteration_host (psi in, iteration, psi / rho / eigenvalues read
    back as soon as each is final, on their own stream) against
    qx_put_psi + qx_scf_iteration + qx_get_psi / qx_get_rho / qx_get_eig on a
    twin context from the same state: identical numbers over four iterations,
    graph replay and plain launches, one buffer for psi in and out, pageable
    and page-locked host arrays, outputs left out."""
    need_gpu()
    import torch
    monkeypatch.setenv("QX_GRAPH", graph)
    p = CgParm.defaults(16)
    ctxs = []
    for _ in range(2):
        ctx = Context(si8, prec, QX_NL_GSPACE)
        ctx.put_psi(si8_psi)
        ctx.scf_init(mixbeta=0.8, kerker_q0=0.8)
        ctx.scf_mixing(10, 20.0)
        ctx.scf_rho_from_psi()
        ctxs.append(ctx)
    a, b = ctxs
    try:
        nb, ne, n = a.nb, si8.gs.nplwex, si8.gs.kfft0
        pin = lambda k: torch.empty(k, dtype=torch.float64).pin_memory().numpy()
        for it in range(4):
            start = a.get_psi()
            ra = a.scf_iteration(p)
            pa, rhoa, ea = a.get_psi(), a.get_rho(), a.get_eig()
            if it < 2:   # page-locked, psi in and out in one buffer
                buf, rho, eig = pin(nb * ne), pin(n), pin(nb)
                buf[:] = start.ravel()
                rb = b.scf_iteration_host(p, psi_in=buf, psi_out=buf, rho_out=rho, eig_out=eig)
                pb = buf.reshape(nb, ne)
            elif it == 2:   # pageable, device psi kept (no psi_in)
                pb, rho, eig = np.empty((nb, ne)), np.empty(n), np.empty(nb)
                rb = b.scf_iteration_host(p, psi_out=pb.reshape(-1), rho_out=rho, eig_out=eig)
            else:           # outputs left out
                rb = b.scf_iteration_host(p, psi_in=np.ascontiguousarray(start).reshape(-1))
                pb, rho, eig = b.get_psi(), b.get_rho(), b.get_eig()
            assert ra["etot"] == rb["etot"] and ra["ncg_hpsi"] == rb["ncg_hpsi"]
            np.testing.assert_array_equal(pa, pb)
            np.testing.assert_array_equal(rhoa, rho)
            np.testing.assert_array_equal(ea, eig)
    finally:
        a.close()
        b.close()


def test_autotune_then_refine_to_fp64(si8, si8_psi):
    """The autotuner's choices keep the mixed path's numbers, and the FP64
    refinement sweep (qx_refine_from + 3 FP64 iterations) of a converged
    mixed solution lands on the FP64 solution."""
    need_gpu()
    p = CgParm.defaults(16)

    def setup(prec):
        ctx = Context(si8, prec, QX_NL_GSPACE)
        ctx.put_psi(si8_psi)
        ctx.scf_init(mixbeta=0.8, kerker_q0=0.8)
        ctx.scf_mixing(10, 20.0)
        return ctx

    ref = setup(QX_PREC_FP64)
    ref.scf_rho_from_psi()
    e64 = [ref.scf_iteration(p)["etot"] for _ in range(30)][-1]
    mixed = setup(QX_PREC_MIXED)
    report = mixed.autotune()
    assert "split" in report
    mixed.put_psi(si8_psi)
    mixed.scf_rho_from_psi()
    emx = [mixed.scf_iteration(p)["etot"] for _ in range(30)][-1]
    assert abs(emx - e64) / si8.cell.natom < 2e-6          # Ry/atom, FP32 level
    fine = setup(QX_PREC_FP64)
    fine.refine_from(mixed)
    efine = [fine.scf_iteration(p)["etot"] for _ in range(3)][-1]
    assert abs(efine - e64) / si8.cell.natom < 2e-9        # Ry/atom, FP64 level


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_autotune_plans_keep_results(si8, si8_psi, prec):
    """qx_autotune picks an FFT radix plan per grid length (and, mixed, a
    tile width and K split per contraction shape); afterwards H|psi> still
    matches the oracle and SCF iterations match an untuned context's."""
    need_gpu()
    p = CgParm.defaults(16)
    res = []
    for tune in (False, True):
        ctx = Context(si8, prec, QX_NL_GSPACE)
        ctx.put_psi(si8_psi)
        ctx.scf_init(mixbeta=0.8, kerker_q0=0.8)
        ctx.scf_mixing(10, 20.0)
        if tune:
            report = ctx.autotune()
            assert "FFT length 24" in report
            if prec == QX_PREC_MIXED:
                assert "tile" in report
        ctx.put_psi(si8_psi)
        ctx.enonloc()
        ref = oracle.Ham(si8, QX_NL_GSPACE).hpsi(si8_psi)
        tol = 1e-11 if prec == QX_PREC_FP64 else 2e-5
        assert np.max(np.abs(ctx.get_hpsi() - ref)) / np.max(np.abs(ref)) < tol
        ctx.scf_rho_from_psi()
        res.append([ctx.scf_iteration(p)["etot"] for _ in range(4)])
        ctx.close()
    tol = 1e-9 if prec == QX_PREC_FP64 else 1e-4
    np.testing.assert_allclose(res[1], res[0], rtol=tol)
