#!/usr/bin/env python
"""Generator of the golden fixtures in this directory (test infrastructure).

Runs the CPU oracle (oracle/qxmd_oracle.c through oracle/, oracle/scf.py,
oracle/forces.py) on the seeded workloads and writes compressed .npz files
that the GPU parity tests and bench.py's accuracy block compare against:

* si64_start.npz  -- Si64 (2x2x2 diamond, 54^3 grid, 160 bands, G-space KB)
  at the reference's LCG start psi (rdwfns, seed 25): the overlap's L^-1 of
  schmidt2, H_sub = <psi|H|psi> of the orthonormalised psi and its
  eigenvalues, H|psi> of four bands in full plus size-independent checksums of
  every band (Gamma-metric norm and two seeded random projections), the
  density's low-G components, and one batched eigen_BKL sweep (eigenvalues and
  CG iterations per band).
* si64_scf.npz    -- the same cell iterated in pwlda_md order (batched CG,
  Pulay mixing with the reference defaults itratn 10, aslh 0.8, bslh 0.64,
  cmetric 20) to self-consistency: total energy, residual and CG work per
  iteration, the final eigenvalues and the Hellmann-Feynman forces (local
  flocal_g + G-space KB kbnlpp_frc2 + Ewald).
* si64_scf_rspace.npz -- the same iteration with real-space KB projectors
  (calnlc, the reference's default for Si) to self-consistency.
* batch_cells.npz -- three cells of the 48-cell batch with different grids
  (21^3, 42x21x21, 25^3) iterated the same way to self-consistency.
* si512_hpsi.npz  -- H|psi> of four LCG bands of Si512 (96^3 grid, 2048
  projectors): <psi_i|H|psi_j>, norms, checksums and the first 1024
  components of every band.

Usage: python tests/golden/make_fixtures.py [--only NAME ...] [--threads N]
The oracle's results do not depend on the thread count.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import forces as oforces  # noqa: E402
from oracle.scf import ScfState  # noqa: E402
from qxmd_b200 import cell  # noqa: E402

# Pulay mixing with the reference defaults (modules.f90:136-142)
ASLH, Q0, ITRATN, CMETRIC = 0.8, 0.8, 10, 20.0
SI64_ITERS = 40
BATCH_CELLS = (12, 2, 7)
BATCH_ITERS = 30
SEL_BANDS = (0, 57, 127, 159)
NLOWG = 300


def gamma_dot(a, b):
    """2 sum a b - a(1) b(1) over the last axis (eigen.f90:382-386)."""
    return 2.0 * np.sum(a * b, axis=-1) - a[..., 0] * b[..., 0]


def checksum_vectors(nplwex: int, n: int = 2) -> np.ndarray:
    """Seeded random vectors the checksums project on (same seed everywhere)."""
    return np.random.default_rng(2024).standard_normal((n, nplwex))


def low_g(rho: np.ndarray, gs, n: int = NLOWG) -> np.ndarray:
    """rho(G) = (1/N) sum_r rho(r) e^{-iG.r} at the first n G of the density
    half sphere (sorted by |G|^2, G = 0 first)."""
    k1, k2, k3 = gs.grid
    z = np.fft.fftn(rho.reshape(k3, k2, k1)).ravel() / rho.size
    return z[gs.ijk_pos[:n]]


def scf_to_convergence(s, iters: int, noband: int, nlmode: int = 1):
    psi = cell.random_wavefunctions(s.gs.nplwex, s.nband)
    psi, _, rc = oracle.schmidt(psi)
    assert rc == 0
    st = ScfState(s, psi, nlmode=nlmode, mixbeta=ASLH, kerker_q0=Q0, pulay=ITRATN, cmetric=CMETRIC)
    out = []
    for it in range(iters):
        r = st.iteration(noband=noband)
        out.append(r)
        print(f"  iter {it + 1:3d} etot {r['etot']:.12f} resid {r['resid']:.3e} ncg {r['ncg_hpsi']}", flush=True)
    return st, out


def make_si64_start():
    s = cell.si64()
    raw = cell.random_wavefunctions(s.gs.nplwex, s.nband)
    psi, linv, rc = oracle.schmidt(raw)
    assert rc == 0
    ham = oracle.Ham(s, 1)
    hc = ham.hpsi(psi)
    hsub, _ = oracle.hmatrix(psi, hc)
    w, _, _ = oracle.jacobi(hsub)
    _, ekib = ham.ekinetic(psi)
    x, _, eig, _, nri = ham.eigen(psi, hc, ekib, noband=int(s.cell.nel // 2))
    rho = ham.softchg(psi, s.occ)
    v = checksum_vectors(s.gs.nplwex)
    return dict(linv=linv, hsub=hsub, hsub_eig=w, sel_bands=np.array(SEL_BANDS),
                hpsi_sel=hc[list(SEL_BANDS)], hpsi_norm2=gamma_dot(hc, hc),
                hpsi_chk=np.stack([gamma_dot(hc, vv[None, :]) for vv in v]),
                rho_lowg=low_g(rho, s.gs), rho_sum=rho.sum() * s.gs.rvol / s.gs.kfft0,
                cg_eig=eig, cg_nriter=nri.astype(np.int32),
                cg_psi_chk=np.stack([gamma_dot(x, vv[None, :]) for vv in v]))


def make_si64_scf():
    s = cell.si64()
    noband = int(s.cell.nel // 2)
    st, out = scf_to_convergence(s, SI64_ITERS, noband)
    t = cell.force_tables(s)
    floc = oforces.floc_g(t, st.ham.softchg(st.psi, s.occ), s.gs.grid)
    fnl = oforces.fnl_kb(t, s.kb_g, s.vclalp, st.psi, s.occ)
    few = cell.ewald_forces(s.cell, s.gs)
    return dict(etot=np.array([r["etot"] for r in out]), resid=np.array([r["resid"] for r in out]),
                ncg_hpsi=np.array([r["ncg_hpsi"] for r in out], dtype=np.int32),
                eig=out[-1]["eig"], floc=floc, fnl=fnl, fewald=few, natom=s.cell.natom, noband=noband,
                eewald=s.eewald)


def make_si64_scf_rspace():
    """The Si64 iteration with real-space KB projectors (calnlc, QXMD's
    default for Si) to self-consistency: energies per iteration and the final
    eigenvalues."""
    s = cell.si64()
    noband = int(s.cell.nel // 2)
    st, out = scf_to_convergence(s, SI64_ITERS, noband, nlmode=2)
    return dict(etot=np.array([r["etot"] for r in out]), resid=np.array([r["resid"] for r in out]),
                ncg_hpsi=np.array([r["ncg_hpsi"] for r in out], dtype=np.int32), eig=out[-1]["eig"],
                natom=s.cell.natom, noband=noband)


def make_batch_cells():
    d = {"cells": np.array(BATCH_CELLS, dtype=np.int32), "iters": BATCH_ITERS}
    for i in BATCH_CELLS:
        s = cell.batch_cell(i)
        print(f" cell {i}: grid {s.gs.grid}, {s.nband} bands", flush=True)
        st, out = scf_to_convergence(s, BATCH_ITERS, int(s.cell.nel // 2))
        d[f"c{i}_etot"] = np.array([r["etot"] for r in out])
        d[f"c{i}_resid"] = np.array([r["resid"] for r in out])
        d[f"c{i}_eig"] = out[-1]["eig"]
        d[f"c{i}_natom"] = s.cell.natom
    return d


def make_si512_hpsi():
    s = cell.si512()
    psi = cell.random_wavefunctions(s.gs.nplwex, 4)
    hc = oracle.Ham(s, 1).hpsi(psi)
    v = checksum_vectors(s.gs.nplwex)
    return dict(hsub=psi @ hc.T * 2.0 - np.outer(psi[:, 0], hc[:, 0]), hpsi_norm2=gamma_dot(hc, hc),
                hpsi_chk=np.stack([gamma_dot(hc, vv[None, :]) for vv in v]), hpsi_head=hc[:, :1024])


MAKERS = {"si64_start": make_si64_start, "si64_scf": make_si64_scf, "si64_scf_rspace": make_si64_scf_rspace,
          "batch_cells": make_batch_cells,
          "si512_hpsi": make_si512_hpsi}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=list(MAKERS))
    ap.add_argument("--threads", type=int, default=len(os.sched_getaffinity(0)))
    a = ap.parse_args()
    oracle.set_threads(a.threads)
    for name in a.only:
        t = time.time()
        print(f"{name} ...", flush=True)
        d = MAKERS[name]()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print(f"{name}: {time.time() - t:.1f} s", flush=True)


if __name__ == "__main__":
    main()
