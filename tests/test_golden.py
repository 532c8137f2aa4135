"""The committed oracle fixtures (tests/golden/) are reproduced by the oracle
as it is built now (CPU only): the pieces that take seconds are recomputed and
compared, so a fixture can never drift from the oracle the GPU tests trust."""
import os

import numpy as np
import pytest

import oracle
from oracle.scf import ScfState
from qxmd_b200 import cell

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def si64():
    return cell.si64()


def test_si64_start_fixture(si64):
    g = golden("si64_start")
    raw = cell.random_wavefunctions(si64.gs.nplwex, si64.nband)
    psi, linv, rc = oracle.schmidt(raw)
    assert rc == 0
    assert rel(np.tril(linv), np.tril(g["linv"])) < 1e-13
    sel = list(g["sel_bands"])
    hc = oracle.Ham(si64, 1).hpsi(psi[sel])
    assert rel(hc, g["hpsi_sel"]) < 1e-13
    # the selected bands' entries of H_sub and of the checksums
    hs = 2.0 * psi[sel] @ hc.T - np.outer(psi[sel, 0], hc[:, 0])
    assert rel(hs, g["hsub"][np.ix_(sel, sel)]) < 1e-12
    n2 = 2.0 * np.sum(hc * hc, axis=1) - hc[:, 0] ** 2
    assert rel(n2, g["hpsi_norm2"][sel]) < 1e-12
    # H_sub is symmetric and its eigenvalues are those of the stored matrix
    assert rel(g["hsub"], g["hsub"].T) < 1e-12
    assert rel(np.linalg.eigvalsh(g["hsub"]), g["hsub_eig"]) < 1e-11


def test_si64_scf_fixture_is_self_consistent():
    g = golden("si64_scf")
    assert g["etot"].size == 40
    assert g["resid"][-1] < 1e-14
    assert abs(g["etot"][-1] - g["etot"][-2]) < 1e-10
    # forces of a relaxed-looking model cell: the three terms nearly cancel
    # in sum, each is finite and of the expected size
    f = g["floc"] + g["fnl"] + g["fewald"]
    assert np.all(np.isfinite(f)) and np.max(np.abs(f)) < 1.0


def test_batch_cell_fixture_first_iterations():
    g = golden("batch_cells")
    i = int(g["cells"][0])
    s = cell.batch_cell(i)
    psi, _, rc = oracle.schmidt(cell.random_wavefunctions(s.gs.nplwex, s.nband))
    assert rc == 0
    st = ScfState(s, psi, nlmode=1, mixbeta=0.8, kerker_q0=0.8, pulay=10, cmetric=20.0)
    e = [st.iteration(noband=int(s.cell.nel // 2))["etot"] for _ in range(3)]
    assert rel(np.array(e), g[f"c{i}_etot"][:3]) < 1e-12
