"""KB tables built on the device against the oracle's restatement, and
H|psi> after MD-like moves of the atoms that rebuild the tables in place:
G space (qx_set_kb_builder once per cell, qx_build_kb_g once per geometry:
setqlm nlkbpp.f90:2196-2247, setbgq nlkbpp.f90:2135-2187, phases of
stscfn_pw pwlda.f90:5711-5850) and real space (qx_set_kb_r_builder,
qx_build_kb_r: setnlc nlkbppr.f90:1010-1560, the points, values and x-line
index that calnlc's kernels read).

Tolerances: the FP64 table 1e-13 of its largest entry (the device cos/sin
and fused multiply-adds against numpy); the FP32 table 2e-7 (one rounding);
H|psi> as in the H|psi> parity tests (FP64 1e-11, mixed 2e-5)."""
import dataclasses

import numpy as np
import pytest

import oracle
from oracle import forces as oforces
from oracle import tables
from qxmd_b200 import cell
from qxmd_b200.lib import QX_NL_GSPACE, QX_NL_RSPACE, QX_PREC_FP64, QX_PREC_MIXED, Context

from gpu_util import device_array, need_gpu, relerr

pytestmark = pytest.mark.gpu
TAB_TOL = {QX_PREC_FP64: 1e-13, QX_PREC_MIXED: 2e-7}
H_TOL = {QX_PREC_FP64: 1e-11, QX_PREC_MIXED: 2e-5}


def _moved(satm, step):
    rng = np.random.default_rng(40 + step)
    return satm + rng.uniform(-0.01, 0.01, satm.shape)


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_build_kb_g_matches_oracle_and_rebuilds_in_place(si8, si8_psi, prec):
    need_gpu()
    b = cell.kb_builder_tables(si8.gs, si8.cell, si8.pp)
    ctx = Context(si8, prec, QX_NL_GSPACE)
    try:
        ctx.set_kb_builder(b)
        satm = b["satm"]
        for step in range(3):
            ctx.build_kb_g(b["ityp"], satm)
            ref, vref = tables.setbgq(b, b["ityp"], satm)
            tab, vcl = ctx.get_kb_g(ref.shape[1])
            assert np.max(np.abs(tab - ref)) / np.max(np.abs(ref)) < TAB_TOL[prec]
            assert relerr(vcl, vref) < TAB_TOL[prec]
            ctx.put_psi(si8_psi)
            ctx.enonloc()
            hc = ctx.get_hpsi()
            h = oracle.Ham(dataclasses.replace(si8, kb_g=ref, vclalp=vref), QX_NL_GSPACE)
            assert relerr(hc, h.hpsi(si8_psi)) < H_TOL[prec]
            satm = _moved(satm, step)
    finally:
        ctx.close()


def test_build_kb_g_unaligned_band_stride():
    """nplwex % 4 = 2 (Si8 at 170 Ry): the builder also fills the padded FP32
    copy the tensor-core contractions read (qx_get_kb_g fails if a row of
    that copy differs), and H|psi> matches the oracle."""
    need_gpu()
    s = cell.build_system(cell.diamond_si((1, 1, 1), seed=1), 170.0 / 4.0, 170.0, 48, with_ewald=False)
    assert s.gs.nplwex % 4 == 2
    b = cell.kb_builder_tables(s.gs, s.cell, s.pp)
    c = cell.random_wavefunctions(s.gs.nplwex, 48)
    c, _, rc = oracle.schmidt(c)
    assert rc == 0
    ctx = Context(s, QX_PREC_MIXED, QX_NL_GSPACE, nband=48)
    try:
        ctx.set_kb_builder(b)
        satm = _moved(b["satm"], 7)
        ctx.build_kb_g(b["ityp"], satm)
        ref, vref = tables.setbgq(b, b["ityp"], satm)
        tab, _ = ctx.get_kb_g(ref.shape[1])
        assert np.max(np.abs(tab - ref)) / np.max(np.abs(ref)) < TAB_TOL[QX_PREC_MIXED]
        ctx.put_psi(c)
        ctx.enonloc()
        hc = ctx.get_hpsi()
    finally:
        ctx.close()
    h = oracle.Ham(dataclasses.replace(s, kb_g=ref, vclalp=vref), QX_NL_GSPACE)
    assert relerr(hc, h.hpsi(c)) < H_TOL[QX_PREC_MIXED]


def test_build_kb_g_rejects_short_radial_table(si8):
    need_gpu()
    b = dict(cell.kb_builder_tables(si8.gs, si8.cell, si8.pp))
    b["mxqlm"] = 8
    b["tbqlm"] = np.ascontiguousarray(b["tbqlm"][:, :9])
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    try:
        with pytest.raises(Exception) as e:
            ctx.set_kb_builder(b)
        assert "radial table too short" in str(e.value)
    finally:
        ctx.close()


def _kbr_system(s, off, mesh, vnl, b):
    kr = cell.KBReal(off=off, mesh=mesh, vnl=vnl, clalp=b["clalp"], rdelv=b["rdelv"])
    return dataclasses.replace(s, kb_r=kr)


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_build_kb_r_matches_oracle_and_rebuilds_in_place(si8, si8_psi, prec):
    """Points in the oracle's box order exactly, values within the table
    tolerance, and real-space-KB H|psi> over three geometries."""
    need_gpu()
    b = cell.kbr_builder_tables(si8.gs, si8.cell, si8.pp)
    nat = si8.cell.natom
    ctx = Context(si8, prec, QX_NL_RSPACE)
    try:
        ctx.set_kb_r_builder(b)
        satm = b["satm"]
        for step in range(3):
            ctx.build_kb_r(b["ityp"], satm)
            roff, rmesh, rvnl = tables.setnlc(b, b["ityp"], satm)
            off, mesh, vnl = ctx.get_kb_r(nat)
            assert np.array_equal(off, roff)
            assert np.array_equal(mesh, rmesh)
            assert np.max(np.abs(vnl - rvnl)) / np.max(np.abs(rvnl)) < TAB_TOL[prec]
            ctx.put_psi(si8_psi)
            ctx.enonloc()
            hc = ctx.get_hpsi()
            h = oracle.Ham(_kbr_system(si8, roff, rmesh, rvnl, b), QX_NL_RSPACE)
            assert relerr(hc, h.hpsi(si8_psi)) < H_TOL[prec]
            satm = _moved(satm, 20 + step)
    finally:
        ctx.close()


@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_build_kb_r_channel_radii_match_oracle(si8, si8_psi, prec):
    """Per-channel projector radii (qx_set_kb_r_channel_radii; setnlc's
    rmxnlc(la), nlkbppr.f90:1405-1431): an s channel at 0.8 of the p radius.
    The points are the species sphere's, the s projector is zero beyond its
    own radius (and nonzero somewhere inside it), the values match the
    oracle's setnlc, and real-space H|psi> and the real-space KB forces match
    the oracle (restated calnlc and fnnlcl2 on those tables)."""
    need_gpu()
    b = cell.kbr_builder_tables(si8.gs, si8.cell, si8.pp)
    rp = float(b["rcut"][0])
    b = dict(b, rcut_l=np.array([0.8 * rp, rp, rp, rp]))
    nat = si8.cell.natom
    satm = _moved(b["satm"], 7)
    roff, rmesh, rvnl, rdvnl = tables.setnlc(b, b["ityp"], satm, grad=True)
    ctx = Context(si8, prec, QX_NL_RSPACE)
    try:
        ctx.set_kb_r_builder(b)
        ctx.build_kb_r(b["ityp"], satm)
        off, mesh, vnl = ctx.get_kb_r(nat)
        assert np.array_equal(off, roff)
        assert np.array_equal(mesh, rmesh)
        assert np.max(np.abs(vnl - rvnl)) / np.max(np.abs(rvnl)) < TAB_TOL[prec]
        zero_s = rvnl[:, 0] == 0.0
        assert zero_s.any() and not zero_s.all()
        assert np.all(vnl[zero_s, 0] == 0.0)
        ctx.put_psi(si8_psi)
        ctx.enonloc()
        hc = ctx.get_hpsi()
        h = oracle.Ham(_kbr_system(si8, roff, rmesh, rvnl, b), QX_NL_RSPACE)
        assert relerr(hc, h.hpsi(si8_psi)) < H_TOL[prec]
        f = ctx.forces_nl_r()
    finally:
        ctx.close()
    psir = np.array([oracle.wvg2r(si8.gs, c) for c in si8_psi])
    ref = oforces.fnl_r(roff, rmesh, rvnl, rdvnl, b["clalp"], b["rdelv"], si8.gs.rvol, psir, si8.occ[:si8_psi.shape[0]])
    assert np.max(np.abs(f - ref)) / np.max(np.abs(ref)) < (1e-10 if prec == QX_PREC_FP64 else 1e-4)


def _with_channels(b, lmx):
    """The model's builder tables with lmx projectors per atom: s only
    (lmx 1) or s, three p and five d (lmx 9; the d radial part a Gaussian
    like the others, times the d polynomials 4-8 of kbr_poly, KB energy
    0.1 Ry), with channel radii 0.8 (s), 1.0 (p) and 0.9 (d) of the species
    radius."""
    rc = float(b["rcut"][0])
    tab, dtab = b["tabnl"], b["dtabnl"]
    if lmx == 1:
        return dict(b, lmx=1, tabnl=tab[:1].copy(), dtabnl=dtab[:1].copy(), poly=np.zeros(1, dtype=np.int32),
                    clalp=b["clalp"][:1].copy(), rcut_l=np.array([0.8 * rc]))
    d = 0.6 * tab[1]
    return dict(b, lmx=9, tabnl=np.ascontiguousarray(np.vstack([tab] + [d] * 5)),
                dtabnl=np.ascontiguousarray(np.vstack([dtab] + [0.6 * dtab[1]] * 5)),
                poly=np.arange(9, dtype=np.int32), clalp=np.concatenate([b["clalp"], [0.1] * 5]),
                rcut_l=np.array([0.8 * rc] + [rc] * 3 + [0.9 * rc] * 5))


@pytest.mark.parametrize("lmx", [1, 9])
@pytest.mark.parametrize("prec", [QX_PREC_FP64, QX_PREC_MIXED])
def test_build_kb_r_s_or_spd_channels_match_oracle(si8, si8_psi, prec, lmx):
    """lmx other than 4 (the reference's lmx(it): 1 for s only, 9 for s, p,
    d): the device tables against the oracle's setnlc, real-space H|psi>
    against the oracle's calnlc through the builder and through host tables
    (qx_set_kb_r), and the real-space KB forces against the restated
    fnnlcl2."""
    need_gpu()
    b = _with_channels(cell.kbr_builder_tables(si8.gs, si8.cell, si8.pp), lmx)
    nat = si8.cell.natom
    satm = _moved(b["satm"], 11)
    roff, rmesh, rvnl, rdvnl = tables.setnlc(b, b["ityp"], satm, grad=True)
    assert rvnl.shape[1] == lmx
    sr = _kbr_system(si8, roff, rmesh, rvnl, b)
    href = oracle.Ham(sr, QX_NL_RSPACE).hpsi(si8_psi)
    ctx = Context(si8, prec, QX_NL_RSPACE)
    try:
        ctx.set_kb_r_builder(b)
        ctx.build_kb_r(b["ityp"], satm)
        off, mesh, vnl = ctx.get_kb_r(nat)
        assert np.array_equal(off, roff) and np.array_equal(mesh, rmesh)
        assert np.max(np.abs(vnl - rvnl)) / np.max(np.abs(rvnl)) < TAB_TOL[prec]
        ctx.put_psi(si8_psi)
        ctx.enonloc()
        assert relerr(ctx.get_hpsi(), href) < H_TOL[prec]
        f = ctx.forces_nl_r()
    finally:
        ctx.close()
    psir = np.array([oracle.wvg2r(si8.gs, c) for c in si8_psi])
    ref = oforces.fnl_r(roff, rmesh, rvnl, rdvnl, b["clalp"], b["rdelv"], si8.gs.rvol, psir, si8.occ[:si8_psi.shape[0]])
    assert np.max(np.abs(f - ref)) / np.max(np.abs(ref)) < (1e-10 if prec == QX_PREC_FP64 else 1e-4)
    ctx = Context(sr, prec, QX_NL_RSPACE)   # the same tables uploaded from the host
    try:
        ctx.put_psi(si8_psi)
        ctx.enonloc()
        assert relerr(ctx.get_hpsi(), href) < H_TOL[prec]
    finally:
        ctx.close()


def test_channel_radii_rejected_beyond_species_radius(si8):
    need_gpu()
    b = cell.kbr_builder_tables(si8.gs, si8.cell, si8.pp)
    rp = float(b["rcut"][0])
    ctx = Context(si8, QX_PREC_FP64, QX_NL_RSPACE)
    try:
        with pytest.raises(Exception) as e:
            ctx.set_kb_r_channel_radii(np.array([rp, rp, rp, rp]))
        assert "qx_set_kb_r_builder first" in str(e.value)
        ctx.set_kb_r_builder(b)
        with pytest.raises(Exception) as e:
            ctx.set_kb_r_channel_radii(np.array([rp, 1.1 * rp, rp, rp]))
        assert "outside" in str(e.value)
    finally:
        ctx.close()


def test_build_kb_r_grows_its_buffers(si8, si8_psi):
    """A larger projector radius (4.0 -> 4.4 bohr, 33 % more points) outgrows
    the first build's 25 % headroom: the buffers are reallocated and H|psi>
    still matches the oracle."""
    need_gpu()
    ctx = Context(si8, QX_PREC_FP64, QX_NL_RSPACE)
    try:
        npts = []
        for rc in (4.0, 4.4):
            b = cell.kbr_builder_tables(si8.gs, si8.cell, dataclasses.replace(si8.pp, rcut=rc))
            ctx.set_kb_r_builder(b)
            ctx.build_kb_r(b["ityp"], b["satm"])
            roff, rmesh, rvnl = tables.setnlc(b, b["ityp"], b["satm"])
            off, mesh, vnl = ctx.get_kb_r(si8.cell.natom)
            assert np.array_equal(mesh, rmesh)
            npts.append(mesh.size)
            ctx.put_psi(si8_psi)
            ctx.enonloc()
            hc = ctx.get_hpsi()
            h = oracle.Ham(_kbr_system(si8, roff, rmesh, rvnl, b), QX_NL_RSPACE)
            assert relerr(hc, h.hpsi(si8_psi)) < H_TOL[QX_PREC_FP64]
        assert npts[1] > 1.25 * npts[0]
    finally:
        ctx.close()


def test_build_kb_r_rejects_sphere_wider_than_half_cell(si8):
    need_gpu()
    b = cell.kbr_builder_tables(si8.gs, si8.cell, dataclasses.replace(si8.pp, rcut=5.5))
    ctx = Context(si8, QX_PREC_FP64, QX_NL_RSPACE)
    try:
        with pytest.raises(Exception) as e:
            ctx.set_kb_r_builder(b)
        assert "wider than half the cell" in str(e.value)
    finally:
        ctx.close()


def _e_nl_r(s, b, satm, psi):
    """sum_n occ_n <psi_n|V_NL psi_n> with the oracle's real-space tables
    (setnlc restated) at the fractional coordinates satm."""
    off, mesh, vnl = tables.setnlc(b, b["ityp"], satm)
    sr = _kbr_system(s, off, mesh, vnl, b)
    dh = oracle.Ham(sr, QX_NL_RSPACE).hpsi(psi) - oracle.Ham(sr, 0).hpsi(psi)
    return sum(s.occ[n] * oracle.dot(psi[n], dh[n]) for n in range(min(s.occ.size, psi.shape[0])))


@pytest.mark.parametrize("prec,tol", [(QX_PREC_FP64, 1e-4), (QX_PREC_MIXED, 1e-4)])
def test_real_space_kb_forces_match_energy_differences(si8, si8_psi, prec, tol):
    """fnnlcl2 on the device (qx_forces_nl_r) against central differences
    (h = 1e-3 bohr) of the oracle's real-space KB energy with the tables
    rebuilt at each displaced geometry; tolerance relative to the largest
    force component.  The force, like fnnlcl2's, differentiates over a fixed
    point set; the energy differences also see grid points crossing the
    projector radius, a term proportional to the projector's size there
    (3e-4 of the force at 4.0 bohr, measured), so the test uses a 4.4 bohr
    radius where the Gaussian projectors are 13 times smaller at the edge."""
    need_gpu()
    b = cell.kbr_builder_tables(si8.gs, si8.cell, dataclasses.replace(si8.pp, rcut=4.4))
    satm = _moved(b["satm"], 3)
    ctx = Context(si8, prec, QX_NL_RSPACE)
    try:
        ctx.set_kb_r_builder(b)
        ctx.build_kb_r(b["ityp"], satm)
        ctx.put_psi(si8_psi)
        f = ctx.forces_nl_r()
    finally:
        ctx.close()
    h = 1e-3
    ainv = np.linalg.inv(si8.gs.rba)
    fd = np.zeros((2, 3))
    for k, a in enumerate((0, 5)):
        for d in range(3):
            ds = ainv[:, d] * h
            sp, sm = satm.copy(), satm.copy()
            sp[a] += ds
            sm[a] -= ds
            fd[k, d] = -(_e_nl_r(si8, b, sp, si8_psi) - _e_nl_r(si8, b, sm, si8_psi)) / (2 * h)
    scale = np.max(np.abs(f))
    assert scale > 1e-3
    assert np.max(np.abs(f[[0, 5]] - fd)) / scale < tol


@pytest.mark.parametrize("prec,tol", [(QX_PREC_FP64, 1e-10), (QX_PREC_MIXED, 1e-4)])
@pytest.mark.parametrize("nb", [16, 15])
def test_real_space_kb_forces_match_restated_fnnlcl2(si8, si8_psi, prec, tol, nb):
    """qx_forces_nl_r against the oracle's restatement of fnnlcl2
    (oracle.forces.fnl_r) on the same point set and gradient tables, every
    atom and component, relative to the largest component; 15 bands take the
    odd-band path of the pair kernels (the last pair has one band)."""
    need_gpu()
    b = cell.kbr_builder_tables(si8.gs, si8.cell, si8.pp)
    satm = _moved(b["satm"], 5)
    off, mesh, vnl, dvnl = tables.setnlc(b, b["ityp"], satm, grad=True)
    psi = si8_psi[:nb]
    occ = si8.occ[:nb]
    psir = np.array([oracle.wvg2r(si8.gs, c) for c in psi])
    ref = oforces.fnl_r(off, mesh, vnl, dvnl, b["clalp"], b["rdelv"], si8.gs.rvol, psir, occ)
    ctx = Context(si8, prec, QX_NL_RSPACE, nband=nb)
    try:
        ctx.set_kb_r_builder(b)
        ctx.build_kb_r(b["ityp"], satm)
        ctx.put_psi(psi)
        f = ctx.forces_nl_r()
    finally:
        ctx.close()
    assert np.max(np.abs(f - ref)) / np.max(np.abs(ref)) < tol


def test_build_kb_g_moves_the_force_tables(si8, si8_psi):
    """After qx_set_force_tables at one geometry, qx_build_kb_g at another
    carries the force path along (species, phases, KB derivative tables):
    qx_forces then equals a context set up from scratch at the new geometry
    with the analytic tables (1e-6 of the largest component: the tables
    differ by the interpolation, 5e-9 of their largest entry)."""
    need_gpu()
    b = cell.kb_builder_tables(si8.gs, si8.cell, si8.pp)
    satm = _moved(b["satm"], 30)
    pos = satm @ si8.gs.rba.T
    cb = dataclasses.replace(si8.cell, pos=pos)
    kb, vcl = cell.kb_tables_g(si8.gs, cb, si8.pp)
    sb = dataclasses.replace(si8, cell=cb, kb_g=kb, vclalp=vcl)
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    try:
        ctx.set_force_tables()
        ctx.set_kb_builder(b)
        ctx.build_kb_g(b["ityp"], satm)
        ctx.put_psi(si8_psi)
        fl, fn = ctx.forces()
    finally:
        ctx.close()
    ref = Context(sb, QX_PREC_FP64, QX_NL_GSPACE)
    try:
        ref.set_force_tables()
        ref.put_psi(si8_psi)
        rl, rn = ref.forces()
    finally:
        ref.close()
    assert np.max(np.abs(fl - rl)) / np.max(np.abs(rl)) < 1e-10
    assert np.max(np.abs(fn - rn)) / np.max(np.abs(rn)) < 1e-6


def test_build_vloc_matches_host_potential_after_moves(si8):
    """qx_build_vloc (vlocal_g, nlkbpp.f90:862-1036) at the set-up geometry
    and after qx_build_kb_g moved the atoms: the device potential against
    the host's v(r) = sum_G V(G) e^{iG.r} of the same geometry (1e-12 of its
    largest value: recurrence phases against direct cosines)."""
    need_gpu()
    torch = pytest.importorskip("torch")
    b = cell.kb_builder_tables(si8.gs, si8.cell, si8.pp)
    ctx = Context(si8, QX_PREC_FP64, QX_NL_GSPACE)
    try:
        ctx.scf_init()
        ctx.set_force_tables()
        ctx.set_kb_builder(b)
        satm = b["satm"]
        for step in range(3):
            if step:
                satm = _moved(satm, 60 + step)
                ctx.build_kb_g(b["ityp"], satm)
            ctx.build_vloc()
            ctx.sync()
            got = device_array(torch, ctx.dev_ptr(5), si8.gs.kfft0)
            moved = dataclasses.replace(si8.cell, pos=satm @ si8.gs.rba.T)
            ref = cell.vloc_grid(si8.gs, moved, si8.pp)
            assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-12
    finally:
        ctx.close()
