"""Forces on the device (qx_forces: flocal_g nlkbpp.f90:1037-1120 and
kbnlpp_frc2 nlkbpp.f90:1878-2130) against the oracle on the same psi, and
the force-error gate of the mixed path at self-consistency (Si8).
FP64: 1e-10 relative to the largest component; mixed: 1e-4."""
import numpy as np
import pytest

import oracle
from oracle import forces as of
from qxmd_b200 import cell
from qxmd_b200.lib import CgParm, Context, QX_NL_GSPACE, QX_PREC_FP64, QX_PREC_MIXED

from gpu_util import need_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,tol", [(QX_PREC_FP64, 1e-10), (QX_PREC_MIXED, 1e-4)])
def test_forces_match_oracle(si8, si8_psi, prec, tol):
    need_gpu()
    t = cell.force_tables(si8)
    rho = oracle.Ham(si8, 1).softchg(si8_psi, si8.occ)
    fl_ref = of.floc_g(t, rho, si8.gs.grid)
    fn_ref = of.fnl_kb(t, si8.kb_g, si8.vclalp, si8_psi, si8.occ)
    ctx = Context(si8, prec, QX_NL_GSPACE)
    ctx.set_force_tables()
    ctx.put_psi(si8_psi)
    fl, fn = ctx.forces()
    assert np.abs(fl - fl_ref).max() <= tol * np.abs(fl_ref).max()
    assert np.abs(fn - fn_ref).max() <= tol * np.abs(fn_ref).max()
    # drop-in shim adds into the caller's array
    base = np.full((si8.cell.natom, 3), 0.25)
    out = base + ctx.kbnlpp_frc2_host(si8_psi)
    assert np.abs(out - base - fn_ref).max() <= tol * np.abs(fn_ref).max()


def test_mixed_force_error_gate(si8, si8_psi):
    """At self-consistency (Pulay, 30 iterations) the mixed-precision forces
    are within 1e-4 Ha/bohr of the FP64 ones."""
    need_gpu()
    p = CgParm.defaults(16)
    f = {}
    for prec in (QX_PREC_FP64, QX_PREC_MIXED):
        ctx = Context(si8, prec, QX_NL_GSPACE)
        ctx.put_psi(si8_psi)
        ctx.scf_init(mixbeta=0.8, kerker_q0=0.8)
        ctx.scf_mixing(10, 20.0)
        ctx.scf_rho_from_psi()
        for _ in range(30):
            ctx.scf_iteration(p)
        ctx.set_force_tables()
        fl, fn = ctx.forces()
        f[prec] = fl + fn
    err_ha = 0.5 * np.abs(f[QX_PREC_MIXED] - f[QX_PREC_FP64]).max()
    assert err_ha < 1e-4
