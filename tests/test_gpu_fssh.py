"""TDDFT-FSSH surface hopping on the device (qx_fssh_init / qx_fssh_step,
tddft_fssh_dm tddft_fssh.f90:1989-2402) against the oracle's restatement:

* 32 states over 12 MD steps of a strongly coupled synthetic sequence with
  hops: the FP64 density matrices equal the oracle's bit for bit (both use
  plain IEEE double operations in the reference's order), the accumulated
  probabilities to 1e-14, and the hop sequence, occupations and the rnd00
  state exactly;
* the device overlap path: a Si8 band window whose wavefunctions are rotated
  among the bands from step to step, the overlap computed on the device from
  the kept and the current psi (FP64 and the mixed tensor-core path), against
  the oracle fed the overlap of the same host arrays."""
import numpy as np
import pytest
from scipy.linalg import expm

import oracle
from qxmd_b200 import cell
from qxmd_b200.lib import Context, FsshParm, QX_NL_GSPACE, QX_PREC_FP64, QX_PREC_MIXED

from gpu_util import need_gpu

pytestmark = pytest.mark.gpu
DTMD = 20.67          # 1 fs in Rydberg time units
TREQ = 0.0019         # 300 K in Ry


def near_identity(n, rng, scale):
    x = rng.standard_normal((n, n)) * scale
    return expm(x - x.T)


def parm(b0, nst, seed):
    return FsshParm(b0=b0, nstate=nst, dtmd=DTMD, dttddft=0.02, boltzmann=1, treq=TREQ, hop=1, seed=seed)


def test_fssh_matches_oracle_bit_for_bit(si8):
    need_gpu()
    rng = np.random.default_rng(5)
    nst = 32
    occ = np.array([2.0] * 16 + [0.0] * 16)
    eig = np.sort(rng.uniform(-0.3, 0.3, nst))
    ref = oracle.Fssh(occ, seed=12345.0, dtmd=DTMD, treq=TREQ)
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE, nband=nst)
    try:
        ctx.put_psi(cell.random_wavefunctions(si8.gs.nplwex, nst))
        ctx.fssh_init(parm(0, nst, 12345.0), occ)
        hops = 0
        for step in range(12):
            A = near_identity(nst, rng, 0.1)
            t_ref, bkl_ref = ref.step(A, eig)
            t, occ_d, bkl = ctx.fssh_step(A, eig)
            assert t == t_ref, step
            np.testing.assert_array_equal(occ_d, ref.occ)
            assert np.max(np.abs(bkl - bkl_ref)) <= 1e-14 * max(1.0, np.max(np.abs(bkl_ref)))
            hops += t is not None
        dnr, dni, acc, rndx = ctx.fssh_state()
    finally:
        ctx.close()
    assert hops >= 1
    np.testing.assert_array_equal(dnr, ref.dnr)
    np.testing.assert_array_equal(dni, ref.dni)
    assert np.max(np.abs(acc - ref.accum)) <= 1e-14 * np.max(np.abs(ref.accum))
    assert rndx == ref.rndx.value


@pytest.mark.parametrize("prec,tol", [(QX_PREC_FP64, 1e-10), (QX_PREC_MIXED, 2e-4)])
def test_fssh_device_overlap(si8, si8_psi, prec, tol):
    """Window of bands 2..13 of Si8 (6 occupied, 6 empty in the window's
    occupations), three steps; each step rotates all 16 bands by a
    near-identity orthogonal matrix, so A(k, j) = <psi_k(t)|psi_j(t+dt)> is
    that rotation's window block."""
    need_gpu()
    rng = np.random.default_rng(8)
    b0, nst = 2, 12
    occ = np.array([2.0] * 6 + [0.0] * 6)
    eig = np.sort(rng.uniform(-0.2, 0.2, nst))
    ref = oracle.Fssh(occ, seed=4321.0, dtmd=DTMD, treq=TREQ)
    psi = si8_psi.copy()
    ctx = Context(si8, prec, QX_NL_GSPACE)
    try:
        ctx.put_psi(psi)
        ctx.fssh_init(parm(b0, nst, 4321.0), occ)
        for step in range(3):
            R = near_identity(si8.nband, rng, 0.08)
            new = R.T @ psi                       # new_j = sum_k R[k, j] psi_k
            A = 2.0 * psi @ new.T - np.outer(psi[:, 0], new[:, 0])
            ctx.put_psi(new)
            t, occ_d, bkl = ctx.fssh_step(None, eig)
            t_ref, bkl_ref = ref.step(A[b0:b0 + nst, b0:b0 + nst], eig)
            assert t == t_ref
            np.testing.assert_array_equal(occ_d, ref.occ)
            assert np.max(np.abs(bkl - bkl_ref)) <= tol * max(1e-3, np.max(np.abs(bkl_ref)))
            psi = new
        dnr, dni, _, _ = ctx.fssh_state()
    finally:
        ctx.close()
    assert np.max(np.abs(dnr - ref.dnr)) < tol
    assert np.max(np.abs(dni - ref.dni)) < tol


def test_fssh_rejects_bad_windows(si8):
    need_gpu()
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    try:
        with pytest.raises(Exception):
            ctx.fssh_init(parm(10, 8, 1.0), np.zeros(8))        # beyond 16 bands
        with pytest.raises(Exception):
            ctx.fssh_init(parm(0, 8, 0.0), np.zeros(8))         # rnd00 seed must be positive
        with pytest.raises(Exception):
            ctx.fssh_step()                                     # before qx_fssh_init
    finally:
        ctx.close()
