"""Caller-side set-up: G half sphere, chkftm, index maps (reclat.f90, modules.f90)."""
import numpy as np
import pytest

from qxmd_b200 import cell


def test_chkftm_rounds_to_fftw3_sizes():
    # reclat.f90:1007-1084 with the FFTW3 size list
    assert cell.chkftm(23, 23, 23) == (24, 24, 24)
    assert cell.chkftm(53, 53, 53) == (54, 54, 54)
    assert cell.chkftm(45, 23, 23) == (45, 24, 24)
    assert cell.chkftm(11, 13, 17) == (12, 14, 18)
    assert cell.chkftm(97, 97, 97) == (98, 98, 98)


@pytest.mark.parametrize("reps,ecut,ecutd,nplw,grid", [
    ((1, 1, 1), 12.0, 48.0, 369, (24, 24, 24)),      # Si8
    ((2, 2, 2), 16.0, 64.0, 4657, (54, 54, 54)),     # Si64, NCPP ecutdens = 4 ecut
    ((2, 2, 2), 16.0, 50.0, 4657, (48, 48, 48)),     # Si64 at the 48^3 grid
    ((2, 1, 1), 12.0, 48.0, 747, (45, 24, 24)),      # Si16
    ((2, 2, 1), 12.0, 48.0, 1509, (45, 45, 24)),     # Si32
])
def test_sphere_sizes_match_scope_table(reps, ecut, ecutd, nplw, grid):
    c = cell.diamond_si(reps, seed=2)
    gs = cell.strvec(c.rba, ecut, ecutd)
    assert gs.nplw == nplw
    assert gs.grid == grid
    assert gs.nplwex == 2 * (nplw + 1)


def test_half_sphere_properties(si8):
    gs = si8.gs
    t = np.stack([gs.nga, gs.ngb, gs.ngc], axis=1)[1:]
    s = set(map(tuple, t))
    # one member of each +-G pair, no G = 0
    assert len(s) == t.shape[0]
    assert not any((-a, -b, -c) in s for a, b, c in s)
    assert (0, 0, 0) not in s
    # sorted by |G|^2
    assert np.all(np.diff(gs.recnrm) >= -1e-12)
    # the wave sphere is a prefix of the density sphere
    assert np.all(gs.recnrm[: gs.nplw + 1] <= gs.ecut + 1e-12)
    assert np.all(gs.recnrm[gs.nplw + 1:] > gs.ecut)
    # -G index is the grid mirror of +G
    k1, k2, k3 = gs.grid
    p, m = gs.ijk_pos, gs.ijk_neg
    assert np.all(m % k1 == (k1 - p % k1) % k1)
    assert np.all((m // k1) % k2 == (k2 - (p // k1) % k2) % k2)
    assert np.all(m // (k1 * k2) == (k3 - p // (k1 * k2)) % k3)
    # all grid positions distinct
    allidx = np.concatenate([p, m[1:]])
    assert np.unique(allidx).size == allidx.size


def test_enumeration_is_stable_sorted():
    # equal |G|^2 keep the enumeration order (stable radix + odd-even sort, funcs.f90:1211-1380)
    c = cell.diamond_si((1, 1, 1), seed=1, disp=0.0)
    gs = cell.strvec(c.rba, 12.0, 48.0)
    # first shell of a cubic cell: the 3 half-space members of |n| = 1
    t = np.stack([gs.nga, gs.ngb, gs.ngc], axis=1)
    assert [tuple(x) for x in t[1:4]] == [(1, 0, 0), (0, 1, 0), (0, 0, 1)]


def test_random_wavefunctions_lcg():
    # rnd00 (funcs.f90:1673-1689), seed 25: x1 = 16807*25 mod (2^31-1)
    x = cell.random_wavefunctions(10, 2)
    assert x[0, 0] == pytest.approx(16807 * 25 / 2147483647.0 - 0.5, abs=0)
    assert np.all(x[:, 1] == 0.0)
    assert np.all(np.abs(x) < 0.5)


def test_lcg_minimal_standard_known_answer():
    # rnd00 is the Park-Miller minimal standard generator (a = 16807,
    # m = 2^31 - 1); its published check value: from seed 1 the 10000th
    # state is 1043618065 (Park & Miller, CACM 31 (1988) 1192).
    v = cell.random_wavefunctions(10000, 1, seed=1.0)[0, 9999]
    assert round((v + 0.5) * 2147483647.0) == 1043618065


def test_kb_tables_consistent_between_g_and_r(si8):
    # G-space table = Fourier transform of the real-space projector (same operator)
    s = si8
    assert s.kb_g.shape == (s.gs.nplwex, 4 * s.cell.natom)
    assert s.kb_r.off[-1] == s.kb_r.mesh.size
    assert np.all(s.kb_g[1, :] == 0.0)   # Im beta(G=0) = 0 for every projector


def test_vloc_is_real_and_finite(si8):
    assert np.all(np.isfinite(si8.vloc))
    assert si8.vloc.shape == (si8.gs.kfft0,)
