"""Independent cells advanced together: each context on its own stream, every
cell's SCF iteration enqueued (qx_scf_launch, a CUDA graph replay) before any
result is read (qx_scf_result).  The results equal those of the same cells
iterated one after another, bit for bit."""
import numpy as np
import pytest
import torch

from qxmd_b200 import cell
from qxmd_b200.lib import CgParm, Context, QX_NL_GSPACE, QX_PREC_MIXED

from gpu_util import need_gpu

pytestmark = pytest.mark.gpu


def make(s, stream=0):
    ctx = Context(s, QX_PREC_MIXED, QX_NL_GSPACE, stream=stream)
    ctx.put_psi(cell.random_wavefunctions(s.gs.nplwex, s.nband))
    ctx.schmidt()
    ctx.scf_init(mixbeta=0.8, kerker_q0=0.8)
    ctx.scf_mixing(10, 20.0)
    ctx.scf_rho_from_psi()
    return ctx


def test_concurrent_cells_match_sequential():
    need_gpu()
    cells = [cell.batch_cell(i) for i in (12, 2, 7)]   # 21^3, 42x21x21, 25^3 grids
    parms = [CgParm.defaults(int(s.cell.nel // 2)) for s in cells]
    seq = []
    for s, p in zip(cells, parms):
        ctx = make(s)
        seq.append([ctx.scf_iteration(p)["etot"] for _ in range(5)])
        ctx.close()
    streams = [torch.cuda.Stream() for _ in cells]
    ctxs = [make(s, st.cuda_stream) for s, st in zip(cells, streams)]
    conc = [[] for _ in cells]
    for _ in range(5):
        for ctx, p in zip(ctxs, parms):
            ctx.scf_launch(p)
        for k, ctx in enumerate(ctxs):
            conc[k].append(ctx.scf_result()["etot"])
    for a, b in zip(seq, conc):
        assert a == b


def test_small_cell_first_in_a_fresh_process():
    """A batch cell's Gram-Schmidt and SCF iteration as the first dense calls
    of a process (the shared-memory opt-in of the register Cholesky must not
    depend on a larger cell having run before)."""
    need_gpu()
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from qxmd_b200 import cell\n"
            "from qxmd_b200.lib import CgParm, Context, QX_NL_GSPACE, QX_PREC_MIXED\n"
            "s = cell.batch_cell(0)\n"
            "ctx = Context(s, QX_PREC_MIXED, QX_NL_GSPACE)\n"
            "ctx.put_psi(cell.random_wavefunctions(s.gs.nplwex, s.nband))\n"
            "ctx.schmidt()\n"
            "ctx.scf_init(mixbeta=0.8, kerker_q0=0.8)\n"
            "ctx.scf_rho_from_psi()\n"
            "print(ctx.scf_iteration(CgParm.defaults(int(s.cell.nel // 2)))['etot'])\n") % root
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
