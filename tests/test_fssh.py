"""The oracle's tddft_fssh_dm (tddft_fssh.f90:1989-2402) on the CPU: its RK4
integration against the exact propagator of the same equations, and the
trivial cases.  The equations of the reference are
d rho/dt = -i [E + i d, rho] with d(k, j) = -(A(k, j) - A(j, k)) / (2 dtmd)
real antisymmetric, so over the MD step rho(T) = U rho(0) U^+ with
U = exp(-i (E + i d) T), T = int(dtmd/dttddft) dttddft."""
import numpy as np
import pytest
from scipy.linalg import expm

import oracle

DTMD = 20.67          # 1 fs in Rydberg time units


def near_identity(n, rng, scale):
    x = rng.standard_normal((n, n)) * scale
    return expm(x - x.T)


def test_rk4_matches_exact_propagator():
    rng = np.random.default_rng(1)
    nst = 12
    occ = np.array([2.0] * 6 + [0.0] * 6)
    eig = np.sort(rng.uniform(-0.3, 0.3, nst))
    A = near_identity(nst, rng, 0.1)
    f = oracle.Fssh(occ, seed=99.0, dtmd=DTMD)
    f.step(A, eig)
    d = -(A - A.T) / 2.0 / DTMD
    T = int(DTMD / 0.02) * 0.02
    for s in range(nst):
        active = occ[s] > 0.5 and any(0 <= s + u < nst and u != 0 and occ[s + u] <= 1.5 for u in range(-3, 4))
        if not active:
            np.testing.assert_array_equal(f.dnr[s, 3, 3], 1.0)
            continue
        w = [s + u for u in range(-3, 4) if 0 <= s + u < nst]
        o = w[0] - s + 3
        H = np.diag(eig[w]) + 1j * d[np.ix_(w, w)]
        U = expm(-1j * H * T)
        rho0 = np.zeros((len(w), len(w)), dtype=complex)
        rho0[s - w[0], s - w[0]] = 1.0
        rho = U @ rho0 @ U.conj().T
        got = f.dnr[s, o:o + len(w), o:o + len(w)] + 1j * f.dni[s, o:o + len(w), o:o + len(w)]
        assert np.max(np.abs(got - rho)) < 1e-9, s
        assert abs(np.trace(got).real - 1.0) < 1e-12


def test_no_coupling_leaves_the_state_and_draws_once_per_step():
    nst = 8
    occ = np.array([2.0] * 4 + [0.0] * 4)
    eig = np.linspace(-0.2, 0.2, nst)
    f = oracle.Fssh(occ, seed=25.0, dtmd=DTMD)
    for _ in range(3):
        t, bkl = f.step(np.eye(nst), eig)
        assert t is None
        assert np.all(bkl == 0.0)
    assert np.all(f.dnr[:, 3, 3] == 1.0)
    assert np.count_nonzero(f.dnr) == nst and np.count_nonzero(f.dni) == 0
    np.testing.assert_array_equal(f.occ, occ)
    # three Park-Miller draws from 25: the state after them
    x = 25.0
    for _ in range(3):
        x = (16807.0 * x) % 2147483647.0
    assert f.rndx.value == x


def test_hops_conserve_electrons_and_follow_the_draws():
    """A strongly coupled sequence with hops: every accepted transition moves
    one electron to a state that was not full, and it is the pair whose
    probability interval holds that step's draw."""
    rng = np.random.default_rng(5)
    nst = 32
    occ = np.array([2.0] * 16 + [0.0] * 16)
    eig = np.sort(rng.uniform(-0.3, 0.3, nst))
    f = oracle.Fssh(occ, seed=12345.0, dtmd=DTMD, treq=0.0019)
    draws = oracle.rnd00(12345.0, 12)
    nhop = 0
    for step in range(12):
        A = near_identity(nst, rng, 0.1)
        before = f.occ.copy()
        t, bkl = f.step(A, eig)
        assert f.occ.sum() == before.sum()
        # the interval of the running sum of positive probabilities, in the
        # reference's order (states, then neighbours -3..3)
        cum, hit = 0.0, None
        for s in range(nst):
            if not before[s] > 0.5:
                continue
            for u in range(-3, 4):
                ns = s + u
                if ns < 0 or ns >= nst or ns == s or before[ns] > 1.5:
                    continue
                p = max(bkl[s, u + 3], 0.0)
                if cum <= draws[step] < cum + p:
                    hit = (s, ns)
                cum += p
        assert t == hit
        if t:
            nhop += 1
            s, ns = t
            assert f.occ[s] == before[s] - 1 and f.occ[ns] == before[ns] + 1
    assert nhop >= 1
