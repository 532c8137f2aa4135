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
