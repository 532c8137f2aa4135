#!/usr/bin/env python
"""Benchmark of the Kohn-Sham hot path: SCF iterations per second on Si64.

Workload: Si64 2x2x2 diamond supercell, a = 20.52 bohr, seeded +-0.05 bohr
displacements, Gamma point, Ecut 16 Ry with the norm-conserving density cutoff
4*Ecut (54^3 FFT grid by the reference's chkftm rule), 160 bands (128
occupied), G-space KB projectors (256), model pseudopotential, reference LCG
initial wavefunctions.  One step = one SCF iteration in the reference's order
(potential, H|psi> for all bands, H_sub, subspace rotation, BKL CG, Gram-
Schmidt, density, mixing), mixed precision (FP32 FFTs and band contractions,
FP64 Cholesky/eigen/density).  The FP64 drop-in path is timed beside it.

Arms:
  --impl ours       the CUDA library through its C ABI (default)
  --impl reference  the CPU restatement of the reference algorithm (the
                    oracle; QXMD itself needs gfortran+FFTW+MPI, absent on
                    this image), all host cores, same metric.
Multi-GPU: the single-cell path does not shard, so N ranks run N independent
replicas ("replicas only"); value = all iterations / max time over ranks.  The
48-cell batch (key batch48) is split over the ranks by cell, with no exchange
on the data path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SCF iter/s"
# Pulay density mixing with the reference defaults (modules.f90:136-142:
# imxchg 1, aslh 0.8, bslh 0.64 = 0.8^2, itratn 10, cmetric 20)
PULAY_ASLH, PULAY_Q0, PULAY_ITRATN, PULAY_CMETRIC = 0.8, 0.8, 10, 20.0
# dram__bytes_read.sum + dram__bytes_write.sum over the four launches of one
# FP32 H|psi> pass of this workload (ncu, --profile-hpsi; the capture command
# is listed with the figures in the profiles directory)
HPSI_PASS_DRAM_BYTES = 69974016
# What limits the pipeline (ncu on the plane pass, the largest of its
# kernels): its DRAM traffic is a fraction of the algorithmic bytes because
# the z-transformed planes stay in L2, so it is not HBM-bound; it is bound by
# latency at low occupancy.
PIPELINE_LIMITER = ("latency, not HBM: DRAM traffic is 0.17x the algorithmic bytes (the pruned transforms keep "
                    "only the z-transformed planes); plane pass k_plane (two z planes a CTA) at 22.7% achieved "
                    "occupancy (128 registers), 41.4% issue active, FMA pipe 36%, stalls led by long scoreboard, "
                    "instruction fetch and wait")
# FP64 SCF iterations of the refinement sweep after the mixed solution converged
REFINE_ITERS = 3
# iteration caps of the Si512 run to self-consistency and of its FP64 sweep
SI512_MAX_ITERS, SI512_REFINE_MAX = 80, 12
UNIT = "iter/s"
WORKLOAD = "Si64 diamond 2x2x2, Gamma, Ecut 16 Ry / 64 Ry, 54^3 grid, 160 bands, G-space KB"
DATA = "synthetic (seeded Si64 cell, model pseudopotential)"
# SCF iterations of the CPU oracle in the cpu_baseline sample (after as many
# untimed ones): about 10 s on 16 host threads
CPU_SAMPLE_WARMUP, CPU_SAMPLE_ITERS = 2, 3
GOLDEN = os.path.join(ROOT, "tests", "golden")
# TDDFT-FSSH workload: 32 adiabatic states, 1 fs MD steps, 100 steps
FSSH_STATES, FSSH_DT_FS, FSSH_MD_STEPS, FSSH_SCF_PER_STEP, FSSH_SEED = 32, 1.0, 100, 4, 20240.0


def workload_config(sys_, ws):
    """The workload as both arms name it."""
    return {"workload": WORKLOAD, "bands": sys_.nband, "nplwex": sys_.gs.nplwex, "grid": list(sys_.gs.grid),
            "parallelism": "replicas" if ws > 1 else "single",
            "l2": "256 MB buffer written between timed iterations (device arm)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile-hpsi", action="store_true",
                    help="only the FP32 H|psi> FFT pipeline over all bands (warm-up, then --steps passes): "
                         "the launches whose DRAM traffic ncu measures for the roofline")
    ap.add_argument("--profile-step", action="store_true",
                    help="only the mixed-precision SCF iterations (warm-up, then --steps), no L2 flush, "
                         "no extra arms: the launch sequence profiled under ncu")
    ap.add_argument("--profile-batch", action="store_true",
                    help="W + K steps of the 48-cell batch and nothing else, printing launch counts for an ncu "
                         "launch list")
    ap.add_argument("--si512", action="store_true",
                    help="only H|psi> band applications/s on the Si512 cell (1100 bands, 96^3 grid), mixed and FP64")
    ap.add_argument("--sequential", action="store_true",
                    help="with --profile-step: the plain FP64 path (one-rank band order) instead of mixed")
    ap.add_argument("--accuracy-iters", type=int, default=40,
                    help="SCF iterations (from the same start) after which the paths' energies are compared")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# FP64 peak of a B200 at its maximum SM clock: 148 SMs x 64 FP64 FMA lanes a
# clock x 2 flops (no FP64 figure is measured alongside the HBM and bf16 peaks)
FP64_FLOPS_PER_CLOCK = 148 * 64 * 2
SM_MAX_MHZ = 1965.0


def band_matrix_timing(ctx, sys_, R, flush, sm_max_mhz=None):
    """The band matrix <psi_j|H psi_i> of an FP64 context alone (qx_hmatrix
    with no host copy: one FP64 GEMM of nband x nband x nplwex, split over K,
    the reduction of its partial sums and the symmetrisation), device-timed
    over R calls with L2 flushed between them; throughput against the FP64
    peak at the maximum SM clock."""
    import torch
    _hm(ctx)
    t = 0.0
    for _ in range(R):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _hm(ctx)
        e1.record()
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1)
    ms = t / R
    nb, ne = sys_.nband, sys_.gs.nplwex
    flops = 2.0 * nb * nb * ne
    peak = FP64_FLOPS_PER_CLOCK * (sm_max_mhz or SM_MAX_MHZ) * 1e6 / 1e12
    tf = flops / (ms * 1e-3) / 1e12
    return {"kernels": "k_dgemm (FP64 DMMA tensor cores, split-K) + k_gemm_reduce + k_symmetrize", "shape_mnk": [nb, nb, ne],
            "ms": ms, "tflops": tf, "peak_tflops": peak, "frac": tf / peak,
            "peak_kind": "nominal FP64 at max SM clock (148 SMs x 64 FMA/clock x 2)"}


def _hm(ctx):
    rc = ctx.L.qx_hmatrix(ctx.h, None)
    if rc:
        raise RuntimeError(f"qx_hmatrix failed ({rc})")


class Clocks:
    """SM clock and clock-event-reason sampler for the timed region: an NVML
    thread every 5 ms (the timed regions here are tens of milliseconds), else
    nvidia-smi every 200 ms.  Reads only."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, index):
        self.index = index
        self.p = None
        self.thread = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            self.mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.sm, self.bits, self.stop_flag = [], 0, threading.Event()

            def run():
                while not self.stop_flag.is_set():
                    try:
                        self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                        self.bits |= int(get_reasons(h))
                    except Exception:
                        pass
                    self.stop_flag.wait(0.005)
            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            reasons = sorted(nm for nm, bit in self.REASONS.items() if self.bits & bit)
            sm = self.sm
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.mx,
                    "reasons": reasons, "samples": len(sm), "sampler": "nvml 5 ms"}
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "sampler": "nvidia-smi 200 ms"}


def dist_setup(args):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    import torch
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def run_profile_step(args):
    """W + K mixed-precision SCF iterations of the workload (the Si512 cell
    with --si512) and nothing else, printing the library's launch counts so
    that an ncu capture can skip the set-up and warm-up launches (-s) and
    take exactly the timed ones (-c)."""
    import torch

    from qxmd_b200 import cell
    from qxmd_b200.lib import CgParm, Context, QX_NL_GSPACE, QX_PREC_FP64, QX_PREC_MIXED, launch_count
    torch.cuda.set_device(0)
    sys_ = cell.si512() if args.si512 else cell.si64()
    ctx = Context(sys_, QX_PREC_FP64 if args.sequential else QX_PREC_MIXED, QX_NL_GSPACE)
    ctx.put_psi(cell.random_wavefunctions(sys_.gs.nplwex, sys_.nband))
    ctx.schmidt()
    ctx.scf_init(mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0)
    ctx.scf_mixing(PULAY_ITRATN, PULAY_CMETRIC)
    ctx.scf_rho_from_psi()
    parm = CgParm.defaults(int(sys_.cell.nel // 2), sequential=int(args.sequential))
    for _ in range(args.warmup):
        ctx.scf_iteration(parm)
    ctx.sync()
    n0 = launch_count()
    t = time.perf_counter()
    for _ in range(args.steps):
        out = ctx.scf_iteration(parm)
    ctx.sync()
    dt = time.perf_counter() - t
    print(json.dumps({"profile_step": True, "launches_before": n0, "launches_per_step": (launch_count() - n0) / max(1, args.steps),
                      "wall_ms_per_step": 1e3 * dt / max(1, args.steps), "etot": out["etot"]}), flush=True)
    ctx.close()


def run_profile_batch(args):
    """W + K steps of the 48-cell batch of run_batch (mixed precision, one
    context and stream per cell, every cell's iteration enqueued before any is
    read) and nothing else, printing the library's launch counts so that an
    ncu launch list can skip the set-up and warm-up (-s) and take exactly the
    timed steps (-c)."""
    import torch

    from qxmd_b200 import cell
    from qxmd_b200.lib import CgParm, Context, QX_NL_GSPACE, QX_PREC_MIXED, launch_count
    torch.cuda.set_device(0)
    cells = [cell.batch_cell(i) for i in range(48)]
    streams = [torch.cuda.Stream() for _ in cells]
    ctxs, parms = [], []
    for s, st in zip(cells, streams):
        ctx = Context(s, QX_PREC_MIXED, QX_NL_GSPACE, stream=st.cuda_stream)
        ctx.put_psi(cell.random_wavefunctions(s.gs.nplwex, s.nband))
        ctx.schmidt()
        ctx.scf_init(mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0)
        ctx.scf_mixing(PULAY_ITRATN, PULAY_CMETRIC)
        ctx.scf_rho_from_psi()
        ctxs.append(ctx)
        parms.append(CgParm.defaults(int(s.cell.nel // 2)))

    def step():
        for ctx, p in zip(ctxs, parms):
            ctx.scf_launch(p)
        return [ctx.scf_result() for ctx in ctxs]

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    n0 = launch_count()
    t = time.perf_counter()
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t
    print(json.dumps({"profile_batch": True, "launches_before": n0,
                      "launches_per_step": (launch_count() - n0) / max(1, args.steps),
                      "wall_ms_per_step": 1e3 * dt / max(1, args.steps)}), flush=True)
    for ctx in ctxs:
        ctx.close()


def run_profile_hpsi(args):
    """W + K passes of the FP32 H|psi> pipeline (local potential and kinetic
    term, all 160 bands) on the workload, printing the launch counts."""
    import torch

    from qxmd_b200 import cell
    from qxmd_b200.lib import Context, QX_HPSI_KINETIC, QX_NL_GSPACE, QX_PREC_MIXED, launch_count
    torch.cuda.set_device(0)
    sys_ = cell.si64()
    ctx = Context(sys_, QX_PREC_MIXED, QX_NL_GSPACE)
    ctx.put_psi(cell.random_wavefunctions(sys_.gs.nplwex, sys_.nband))
    p_psi, p_h = ctx.dev_ptr(0), ctx.dev_ptr(1)
    for _ in range(args.warmup):
        ctx.hpsi_dev(p_psi, p_h, sys_.nband, QX_HPSI_KINETIC)
    ctx.sync()
    n0 = launch_count()
    for _ in range(args.steps):
        ctx.hpsi_dev(p_psi, p_h, sys_.nband, QX_HPSI_KINETIC)
    ctx.sync()
    print(json.dumps({"profile_hpsi": True, "launches_before": n0,
                      "launches_per_pass": (launch_count() - n0) / max(1, args.steps)}), flush=True)
    ctx.close()


def accuracy(acc, natom, iters):
    """Total energy, eigenvalues and forces of every path after at least
    `iters` SCF iterations from the same start (each path's count is given),
    against the CPU FP64 oracle run to self-consistency in `iters` iterations
    on the same inputs (the
    fixture tests/golden/si64_scf.npz, made by tests/golden/make_fixtures.py).
    Energies Ha/atom, eigenvalues Ha, forces Ha/bohr (local + KB terms; the
    Ewald term is geometry only and the same everywhere)."""
    g = np.load(os.path.join(GOLDEN, "si64_scf.npz"))
    e_or, eig_or, f_or = float(g["etot"][-1]), g["eig"], g["floc"] + g["fnl"]
    nocc = int(g["noband"])
    out = {"reference": f"CPU FP64 oracle after {g['etot'].size} iterations (self-consistent: residual "
                        f"{float(g['resid'][-1]):.1e}, last energy change "
                        f"{abs(float(g['etot'][-1] - g['etot'][-2])):.1e} Ry)",
           "iterations": iters, "etot_oracle_ry": e_or}
    for name in ("mixed", "fp64", "fp64_batched", "mixed_refined"):
        a = acc[name]
        out[name] = {"iterations": a["iterations"], "etot_ry": a["etot"], "resid": a["resid"],
                     "detot_last_ry": a["detot_last"],
                     "err_ha_per_atom": 0.5 * abs(a["etot"] - e_or) / natom,
                     "eig_occ_max_abs_err_ha": 0.5 * float(np.max(np.abs(a["eig"][:nocc] - eig_or[:nocc]))),
                     "eig_max_abs_err_ha": 0.5 * float(np.max(np.abs(a["eig"] - eig_or))),
                     "force_max_abs_err_ha_per_bohr": 0.5 * float(np.max(np.abs(a["force"] - f_or)))}
    out["mixed_refined"]["fp64_iterations"] = REFINE_ITERS
    out["mixed_refined"]["ms"] = acc["mixed_refined"]["ms"]
    out["err_ha_per_atom"] = out["mixed"]["err_ha_per_atom"]
    out["force_err_ha_per_bohr"] = out["mixed"]["force_max_abs_err_ha_per_bohr"]
    out["force_max_abs_oracle_ha_per_bohr"] = 0.5 * float(np.max(np.abs(f_or)))
    out["gates"] = {"err_ha_per_atom": 1e-6, "force_err_ha_per_bohr": 1e-4}
    out["force_terms"] = "local pseudopotential (flocal_g) + G-space KB (kbnlpp_frc2)"
    return out


def kb_build_timing(sys_, ctx, R, W, flush):
    """Per-geometry rebuild of the G-space KB projector tables on the device
    (qx_build_kb_g: phases, setbgq into the context's table, as an MD step
    needs), the atoms moved a little every call; CUDA-event time per build
    and the table bytes written (FP32 table, plus its padded copy when
    nplwex % 4 != 0)."""
    import torch

    from qxmd_b200 import cell
    b = cell.kb_builder_tables(sys_.gs, sys_.cell, sys_.pp)
    ctx.set_kb_builder(b)
    rng = np.random.default_rng(11)
    geoms = [b["satm"] + rng.uniform(-0.005, 0.005, b["satm"].shape) for _ in range(R + W)]
    for g in geoms[:W]:
        ctx.build_kb_g(b["ityp"], g)
    ctx.sync()
    t = 0.0
    for g in geoms[W:]:
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.build_kb_g(b["ityp"], g)
        e1.record()
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1)
    nproj, ne = b["lmx"] * sys_.cell.natom, sys_.gs.nplwex
    nbytes = 4 * nproj * ne * (2 if ne % 4 else 1)
    ms = t / R
    out = {"ms_per_geometry": ms, "table_bytes_written": nbytes, "gb_per_s": nbytes / (ms * 1e-3) / 1e9,
           "builds_timed": R}
    # real-space tables (setnlc): point search, values, x-line index; one
    # host read of the point count per build (buffer capacity check)
    br = cell.kbr_builder_tables(sys_.gs, sys_.cell, sys_.pp)
    ctx.set_kb_r_builder(br)
    for g in geoms[:W]:
        ctx.build_kb_r(br["ityp"], g)
    ctx.sync()
    t = 0.0
    for g in geoms[W:]:
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.build_kb_r(br["ityp"], g)
        e1.record()
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1)
    npts = ctx.get_kb_r(sys_.cell.natom)[1].size
    out["real_space"] = {"ms_per_geometry": t / R, "points": int(npts)}
    # real-space KB forces (fnnlcl2) of all bands on these tables: psi(r) by
    # the inverse passes, then the projector and gradient sums per atom
    ctx.put_psi(cell.random_wavefunctions(sys_.gs.nplwex, ctx.nb))
    ctx.forces_nl_r()
    t = 0.0
    for _ in range(R):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.forces_nl_r()
        e1.record()
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1)
    out["real_space"]["forces_ms"] = t / R
    return out


def run_si512(args):
    """H|psi> band applications per second (kinetic + local + G-space KB, all
    1100 bands: qx_enonloc) on the Si512 cell, 96^3 grid, mixed and FP64;
    then whole mixed-precision SCF iterations (the FP64 Cholesky and
    tridiagonalisation on the cooperative whole-GPU kernels)."""
    import torch

    from qxmd_b200 import cell
    from qxmd_b200.lib import Context, QX_NL_GSPACE, QX_PREC_FP64, QX_PREC_MIXED
    t0 = time.perf_counter()
    sys_ = cell.si512(with_ewald=True)
    setup_s = time.perf_counter() - t0
    psi = cell.random_wavefunctions(sys_.gs.nplwex, sys_.nband)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    out = {"metric": "H|psi> band-apps/s", "config": {"workload": "Si512 diamond 4x4x4, Gamma, Ecut 12 Ry / 48 Ry, "
                                                                  "96^3 grid, 1100 bands, G-space KB",
                                                      "nplwex": sys_.gs.nplwex, "nproj": int(sys_.kb_g.shape[1])},
           "host_setup_s": setup_s}
    for name, prec in (("mixed", QX_PREC_MIXED), ("fp64", QX_PREC_FP64)):
        ctx = Context(sys_, prec, QX_NL_GSPACE)
        ctx.put_psi(psi)
        for _ in range(max(1, args.warmup)):
            ctx.enonloc()
        ctx.sync()
        t = 0.0
        R = max(2, args.steps)
        for _ in range(R):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ctx.enonloc()
            e1.record()
            torch.cuda.synchronize()
            t += e0.elapsed_time(e1)
        out[name] = {"value": sys_.nband * R / (t / 1e3), "ms_per_pass": t / R}
        if name == "fp64":
            out[name]["band_matrix_gemm"] = band_matrix_timing(ctx, sys_, R, flush)
        ctx.close()
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    # whole SCF iterations of the mixed path from the random start (Pulay
    # mixing, batched CG); the CG work per iteration varies as it converges
    from qxmd_b200.lib import CgParm
    ctx = Context(sys_, QX_PREC_MIXED, QX_NL_GSPACE)
    ctx.put_psi(psi)
    ctx.schmidt()
    ctx.scf_init(mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0)
    ctx.scf_mixing(PULAY_ITRATN, PULAY_CMETRIC)
    ctx.scf_rho_from_psi()
    parm = CgParm.defaults(int(sys_.cell.nel // 2))
    for _ in range(max(1, args.warmup)):
        ctx.scf_iteration(parm)
    ctx.sync()
    t, nh = 0.0, 0
    R = max(2, args.steps)
    for _ in range(R):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = ctx.scf_iteration(parm)
        e1.record()
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1)
        nh += r["ncg_hpsi"]
    out["scf_mixed"] = {"value": R / (t / 1e3), "unit": "iter/s", "ms_per_iter": t / R,
                        "cg_bapps_per_iter": nh / R, "etot_last_ry": r["etot"],
                        "iterations_before": max(1, args.warmup)}
    # on to self-consistency (|dE| < 1e-8 Ry between iterations), then the
    # FP64 refinement sweep of the converged mixed state, both timed
    done = max(1, args.warmup) + R
    # the mixed path's energy settles to within its FP32 noise (about 2e-8
    # Ry/atom here), so its stopping rule is per atom: |dE| / natom < 1e-8 Ry
    # over two successive iterations; the FP64 sweep then runs until |dE| <
    # 1e-8 Ry for the whole cell
    hist, t_conv, e_prev, quiet = [], 0.0, r["etot"], 0
    nat = sys_.cell.natom
    for _ in range(SI512_MAX_ITERS - done):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = ctx.scf_iteration(parm)
        e1.record()
        torch.cuda.synchronize()
        t_conv += e0.elapsed_time(e1)
        done += 1
        hist.append((r["etot"], r["resid"]))
        quiet = quiet + 1 if abs(r["etot"] - e_prev) / nat < 1e-8 else 0
        e_prev = r["etot"]
        if quiet >= 2:
            break
    dlast = abs(hist[-1][0] - hist[-2][0]) if len(hist) > 1 else None
    conv = {"iterations": done, "converged_mixed": quiet >= 2, "rule_mixed": "|dE|/natom < 1e-8 Ry twice",
            "etot_ry": r["etot"], "etot_ry_per_atom": r["etot"] / nat, "resid": r["resid"],
            "detot_last_ry": dlast, "ms_after_timed": t_conv,
            "etot_history_ry": [h[0] for h in hist[-6:]], "resid_history": [h[1] for h in hist[-6:]]}
    ref = Context(sys_, QX_PREC_FP64, QX_NL_GSPACE)
    ref.scf_init(mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0)
    ref.scf_mixing(PULAY_ITRATN, PULAY_CMETRIC)
    ref.refine_from(ctx)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    routs = []
    for _ in range(SI512_REFINE_MAX):
        routs.append(ref.scf_iteration(CgParm.defaults(int(sys_.cell.nel // 2))))
        if len(routs) >= REFINE_ITERS and abs(routs[-1]["etot"] - routs[-2]["etot"]) < 1e-8:
            break
    e1.record()
    torch.cuda.synchronize()
    conv["fp64_refinement"] = {"iterations": len(routs), "ms": e0.elapsed_time(e1),
                               "rule": "|dE| < 1e-8 Ry, at least 3 iterations",
                               "converged": abs(routs[-1]["etot"] - routs[-2]["etot"]) < 1e-8,
                               "etot_ry": routs[-1]["etot"], "resid": routs[-1]["resid"],
                               "mixed_minus_fp64_ha_per_atom": 0.5 * (r["etot"] - routs[-1]["etot"]) / nat,
                               "detot_last_ry": abs(routs[-1]["etot"] - routs[-2]["etot"]),
                               "etot_history_ry": [o["etot"] for o in routs]}
    ref.close()
    # the same cutoffs (12/48 Ry) on the smaller cells: the energy per atom
    # approaches the Si512 value as the Gamma-point sampling of the larger
    # cells improves
    trend = {}
    for name, s in (("si8", cell.si8()), ("si64_12ry", cell.build_system(cell.diamond_si((2, 2, 2), seed=2),
                                                                         12.0, 48.0, 160))):
        c = Context(s, QX_PREC_MIXED, QX_NL_GSPACE)
        c.put_psi(cell.random_wavefunctions(s.gs.nplwex, s.nband))
        c.schmidt()
        c.scf_init(mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0)
        c.scf_mixing(PULAY_ITRATN, PULAY_CMETRIC)
        c.scf_rho_from_psi()
        p = CgParm.defaults(int(s.cell.nel // 2))
        e = [c.scf_iteration(p)["etot"] for _ in range(40)]
        trend[name] = {"etot_ry_per_atom": e[-1] / s.cell.natom, "detot_last_ry": abs(e[-1] - e[-2])}
        c.close()
    trend["si512"] = {"etot_ry_per_atom": r["etot"] / sys_.cell.natom}
    conv["energy_per_atom_12ry"] = trend
    out["scf_to_convergence"] = conv
    out["kb_tables"] = kb_build_timing(sys_, ctx, max(3, args.steps), max(3, args.warmup), flush)
    ctx.close()
    print(json.dumps(out), flush=True)


def run_batch(K, W, ws=1, rank=0):
    """The batch of 48 independent cells (Si8/Si16/Si32, strained, Ecut 10-16
    Ry, 21^3 to 54x54x27 grids, 16-78 bands), mixed precision: one context and
    stream per cell, every cell's SCF iteration enqueued as a graph replay
    before any result is read.  Device time from an event before the first
    launch to one after the last cell finished.  With ws ranks the cells are
    split by cost (qxmd_b200.batch.partition) and each rank advances its own
    (no exchange); the time is the max over ranks, the results are gathered."""
    import torch

    from qxmd_b200 import batch as qb
    from qxmd_b200 import cell
    from qxmd_b200.lib import CgParm, Context, QX_NL_GSPACE, QX_PREC_MIXED
    cells = [cell.batch_cell(i) for i in range(48)]
    mine = qb.partition([qb.cell_cost(s.nband, s.gs.grid, s.gs.nplwex) for s in cells], ws)[rank]
    streams = [torch.cuda.Stream() for _ in mine]
    ctxs, parms = [], []
    for i, st in zip(mine, streams):
        s = cells[i]
        ctx = Context(s, QX_PREC_MIXED, QX_NL_GSPACE, stream=st.cuda_stream)
        ctx.put_psi(cell.random_wavefunctions(s.gs.nplwex, s.nband))
        ctx.schmidt()
        ctx.scf_init(mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0)
        ctx.scf_mixing(PULAY_ITRATN, PULAY_CMETRIC)
        ctx.scf_rho_from_psi()
        ctxs.append(ctx)
        parms.append(CgParm.defaults(int(s.cell.nel // 2)))

    def step():
        for ctx, p in zip(ctxs, parms):
            ctx.scf_launch(p)
        return [ctx.scf_result() for ctx in ctxs]

    for _ in range(W):
        step()
    barrier(ws)
    main = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(main)
    for st in streams:
        st.wait_event(e0)
    for _ in range(K):
        for ctx, p in zip(ctxs, parms):
            ctx.scf_launch(p)
    for st in streams:
        ev = torch.cuda.Event()
        ev.record(st)
        main.wait_event(ev)
    e1.record(main)
    torch.cuda.synchronize()
    outs = {i: ctx.scf_result() for i, ctx in zip(mine, ctxs)}
    ms = max_over_ranks(e0.elapsed_time(e1), ws)
    for ctx in ctxs:
        ctx.close()
    res = qb.gather_results({i: (o["etot"], o["resid"]) for i, o in outs.items()}, ws)
    return {"value": 48 * K / (ms / 1e3), "unit": "cell-iter/s", "cells": 48, "ms_per_step": ms / K,
            "ranks": ws, "cells_per_rank": [len(p) for p in qb.partition(
                [qb.cell_cost(s.nband, s.gs.grid, s.gs.nplwex) for s in cells], ws)],
            "scaling": "strong (the same 48 cells over the ranks)" if ws > 1 else None,
            "grids": sorted({"x".join(map(str, s.gs.grid)) for s in cells}),
            "bands": [min(s.nband for s in cells), max(s.nband for s in cells)],
            "precision": "mixed", "resid_max_last": max(r[1] for r in res.values()),
            "cells_reported": len(res),
            "launch": "one stream and one captured SCF-iteration graph per cell, all enqueued before any is read; "
                      "cells split over ranks by cost, no exchange"}


def run_rspace(sys_, psi0, K, W, iters, flush):
    """The same SCF iteration with real-space KB projectors (calnlc, the
    reference's default for Si), mixed precision: K timed iterations after W,
    then on to `iters` in all, the self-consistent energy and occupied
    eigenvalues against the oracle's (tests/golden/si64_scf_rspace.npz)."""
    import torch

    from qxmd_b200.lib import CgParm, Context, QX_NL_RSPACE, QX_PREC_MIXED
    ctx = Context(sys_, QX_PREC_MIXED, QX_NL_RSPACE)
    ctx.put_psi(psi0)
    ctx.schmidt()
    ctx.scf_init(mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0)
    ctx.scf_mixing(PULAY_ITRATN, PULAY_CMETRIC)
    ctx.scf_rho_from_psi()
    parm = CgParm.defaults(int(sys_.cell.nel // 2))
    for _ in range(W):
        ctx.scf_iteration(parm)
    t = 0.0
    for _ in range(K):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.scf_iteration(parm)
        e1.record()
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1)
    outs = [ctx.scf_iteration(parm) for _ in range(max(2, iters - W - K))]
    eig = ctx.get_eig()
    ctx.close()
    g = np.load(os.path.join(GOLDEN, "si64_scf_rspace.npz"))
    nocc = int(g["noband"])
    return {"path": "mixed, real-space KB (calnlc), projector points from setnlc's rule",
            "value": K / (t * 1e-3), "unit": UNIT, "ms_per_step": t / K,
            "accuracy": {"iterations": W + K + len(outs), "etot_ry": outs[-1]["etot"],
                         "etot_oracle_ry": float(g["etot"][-1]),
                         "err_ha_per_atom": 0.5 * abs(outs[-1]["etot"] - float(g["etot"][-1])) / sys_.cell.natom,
                         "eig_occ_max_abs_err_ha": 0.5 * float(np.max(np.abs(eig[:nocc] - g["eig"][:nocc])))}}


def run_fssh_md(nmd=FSSH_MD_STEPS, nscf=FSSH_SCF_PER_STEP):
    """TDDFT-FSSH on Si64 (32 adiabatic states around the gap, 1 fs MD
    steps): after the ground state is converged, every MD step moves the
    atoms by seeded 300 K Maxwell-Boltzmann velocities (constant: the MD
    integrator is the host's), rebuilds the KB projector table and the local
    potential on the device (qx_build_kb_g, qx_build_vloc), runs nscf SCF
    iterations from the previous step's state, then one surface-hopping step
    (qx_fssh_step: overlap of the two steps' wavefunctions on the tensor cores,
    couplings, FP64 RK4 density matrices over 1033 substeps, hop).  Device
    time per MD step and of the FSSH part alone."""
    import torch

    from qxmd_b200 import cell
    from qxmd_b200.lib import CgParm, Context, FsshParm, QX_NL_GSPACE, QX_PREC_MIXED
    sys_ = cell.si64()
    noband = int(sys_.cell.nel // 2)
    b = cell.kb_builder_tables(sys_.gs, sys_.cell, sys_.pp)
    ctx = Context(sys_, QX_PREC_MIXED, QX_NL_GSPACE)
    ctx.put_psi(cell.random_wavefunctions(sys_.gs.nplwex, sys_.nband))
    ctx.schmidt()
    ctx.scf_init(mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0)
    ctx.scf_mixing(PULAY_ITRATN, PULAY_CMETRIC)
    ctx.set_force_tables()
    ctx.set_kb_builder(b)
    ctx.scf_rho_from_psi()
    parm = CgParm.defaults(noband)
    for _ in range(30):
        ctx.scf_iteration(parm)
    # 300 K Maxwell-Boltzmann velocities in Rydberg units (hbar = 1, mass unit
    # 2 m_e, energy Ry), constant over the run
    rng = np.random.default_rng(7)
    kt = 300.0 * 6.333623e-6                                    # Ry
    mass = 28.0855 * 1822.888486 / 2.0                          # Si mass in units of 2 m_e
    vel = rng.standard_normal((sys_.cell.natom, 3)) * math.sqrt(kt / mass)
    vel -= vel.mean(axis=0)
    dtmd = FSSH_DT_FS * 20.670687                                # fs -> Rydberg time (hbar / Ry)
    b0, nst = noband - FSSH_STATES // 2, FSSH_STATES
    occ = np.array([2.0] * (FSSH_STATES // 2) + [0.0] * (FSSH_STATES // 2))
    ctx.fssh_init(FsshParm(b0=b0, nstate=nst, dtmd=dtmd, dttddft=0.02, boltzmann=1, treq=kt, hop=1,
                           seed=FSSH_SEED), occ)
    pos = sys_.cell.pos.copy()
    ainv = np.linalg.inv(sys_.gs.rba)
    tot = fs = 0.0
    hops = 0
    occ_last = occ
    for step in range(nmd):
        pos = pos + vel * dtmd
        satm = pos @ ainv.T
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        ctx.build_kb_g(b["ityp"], satm)
        ctx.build_vloc()
        ctx.scf_rho_from_psi()          # the new step's SCF starts from rho(psi), mixing history restarted
        for _ in range(nscf):
            ctx.scf_launch(parm)
        e1.record()
        tr, occ_last, _ = ctx.fssh_step()
        e2.record()
        torch.cuda.synchronize()
        r = ctx.scf_result()
        tot += e0.elapsed_time(e2)
        fs += e1.elapsed_time(e2)
        hops += tr is not None
    dnr, _, _, _ = ctx.fssh_state()
    ctx.close()
    trace_dev = float(np.max(np.abs(np.trace(dnr, axis1=1, axis2=2) - 1.0)))
    return {"metric": "TDDFT-FSSH MD steps/s", "value": nmd / (tot * 1e-3), "unit": "MD step/s",
            "workload": f"Si64, {nst} adiabatic states (bands {b0}-{b0 + nst - 1}), dt {FSSH_DT_FS} fs, "
                        f"{nmd} MD steps, {nscf} SCF iterations per step, 300 K velocities",
            "ms_per_md_step": tot / nmd, "fssh_ms_per_step": fs / nmd,
            "substeps_per_md_step": int(dtmd / 0.02), "hops": hops,
            "electrons_in_window": float(occ_last.sum()), "etot_last_ry": r["etot"], "resid_last": r["resid"],
            "max_trace_dev": trace_dev,
            "precision": "mixed SCF and overlap (3xTF32); FP64 density-matrix propagation and hops"}


def run_ours(args):
    import torch

    from qxmd_b200 import cell
    from qxmd_b200.lib import (CgParm, Context, QX_HPSI_KINETIC, QX_NL_GSPACE, QX_PREC_FP64,
                               QX_PREC_MIXED, gemm_fallbacks, launch_count)
    ws, rank, local = dist_setup(args)
    sys_ = cell.si64()
    psi0 = cell.random_wavefunctions(sys_.gs.nplwex, sys_.nband)
    noband = int(sys_.cell.nel // 2)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    K, W = args.steps, args.warmup
    res = {}
    clocks = Clocks(local)
    # mixed: FP32 FFT/H|psi> + 3xTF32 tensor-core contractions, CG over all
    # bands at once; fp64: the plain drop-in (FP64, bands one after another as
    # on one rank of the reference); fp64_batched: FP64 with the batched CG
    variants = (("mixed", QX_PREC_MIXED, 0), ("fp64", QX_PREC_FP64, 1), ("fp64_batched", QX_PREC_FP64, 0))
    ctxs = {}
    for name, prec, seq in variants:
        parm = CgParm.defaults(noband, sequential=seq)
        ctx = Context(sys_, prec, QX_NL_GSPACE)
        ctx.put_psi(psi0)
        if name == "mixed":
            tune_report = ctx.autotune()
        ctx.schmidt()
        ctx.scf_init(mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0)
        ctx.scf_mixing(PULAY_ITRATN, PULAY_CMETRIC)
        ctx.scf_rho_from_psi()
        for _ in range(W):
            ctx.scf_iteration(parm)
        barrier(ws)
        if name == "mixed":
            clocks.start()
        n0, f0 = launch_count(), gemm_fallbacks()
        tot_ms, outs = 0.0, []
        for _ in range(K):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            outs.append(ctx.scf_iteration(parm))
            e1.record()
            torch.cuda.synchronize()
            tot_ms += e0.elapsed_time(e1)
        launches = launch_count() - n0
        fallbacks = gemm_fallbacks() - f0
        if name == "mixed":
            clk = clocks.stop()
        barrier(ws)
        tmax = max_over_ranks(tot_ms, ws)
        r = {"ms_per_step": tmax / K, "value": ws * K / (tmax / 1e3), "launches": launches,
             "fp32_gemm_fallbacks_per_step": fallbacks / K,
             "etot_last": outs[-1]["etot"], "cg_bapps_per_iter": float(np.mean([o["ncg_hpsi"] for o in outs])),
             "eig_clusters": float(np.mean([o["eig_clusters"] for o in outs]))}
        r["iters_done"] = W + K
        res[name] = r
        ctxs[name] = (ctx, parm)
        if name == "fp64_batched":
            continue
        # H|psi> band applications per second (enonloc: kinetic + local + KB, all bands)
        R = max(3, K)
        ctx.enonloc()
        t = 0.0
        for _ in range(R):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ctx.enonloc()
            e1.record()
            torch.cuda.synchronize()
            t += e0.elapsed_time(e1)
        r["hpsi_band_apps_per_s"] = ws * sys_.nband * R / (max_over_ranks(t, ws) / 1e3)
        # FFT pipeline alone (kinetic + local potential): roofline unit
        p_psi, p_h = ctx.dev_ptr(0), ctx.dev_ptr(1)
        t = 0.0
        for _ in range(R):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ctx.hpsi_dev(p_psi, p_h, sys_.nband, QX_HPSI_KINETIC)
            e1.record()
            torch.cuda.synchronize()
            t += e0.elapsed_time(e1)
        r["fft_pipeline_ms"] = t / R
        if name == "fp64":
            r["band_matrix"] = band_matrix_timing(ctx, sys_, R, flush)
        if name == "mixed":
            # end to end through the host-array API (qx_scf_iteration_host):
            # H2D psi (pinned), one iteration, D2H psi, rho, eigenvalues
            hpsi = torch.empty((sys_.nband, sys_.gs.nplwex), dtype=torch.float64).pin_memory()
            hrho = torch.empty(sys_.gs.kfft0, dtype=torch.float64).pin_memory()
            heig = torch.empty(sys_.nband, dtype=torch.float64).pin_memory()
            npsi, nrho, neig = hpsi.numpy(), hrho.numpy(), heig.numpy()
            npsi[:] = ctx.get_psi()
            npsi_flat = npsi.reshape(-1)
            for _ in range(W):
                ctx.scf_iteration_host(parm, psi_in=npsi_flat, psi_out=npsi_flat, rho_out=nrho, eig_out=neig)
            t = 0.0
            for _ in range(K):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                # psi in, the iteration, psi / rho / eigenvalues out, each
                # read back as soon as the iteration has made it final
                ctx.scf_iteration_host(parm, psi_in=npsi_flat, psi_out=npsi_flat, rho_out=nrho, eig_out=neig)
                e1.record()
                torch.cuda.synchronize()
                t += e0.elapsed_time(e1)
            tm = max_over_ranks(t, ws)
            r["e2e"] = {"value": ws * K / (tm / 1e3), "unit": UNIT,
                        "h2d_bytes_per_step": int(npsi.nbytes),
                        "d2h_bytes_per_step": int(npsi.nbytes + nrho.nbytes + neig.nbytes)}
            r["clocks"] = clk
            r["iters_done"] += W + K
    # accuracy: every variant continues from its timed iterations to the
    # same total count, then the final total energies and eigenvalues are
    # compared with the plain FP64 path's
    acc = {}
    for name, _, _ in variants:
        ctx, parm = ctxs[name]
        # at least accuracy_iters iterations, two of them here so that the
        # last energy change is known
        nmore = max(2, args.accuracy_iters - res[name]["iters_done"])
        outs = [ctx.scf_iteration(parm) for _ in range(nmore)]
        ctx.sync()
        last = outs[-1] if outs else None
        ctx.set_force_tables()
        fl, fn = ctx.forces()
        acc[name] = {"force": fl + fn, "iterations": res[name]["iters_done"] + nmore,
                     "etot": last["etot"] if last else res[name]["etot_last"],
                     "resid": last["resid"] if last else None,
                     "detot_last": abs(outs[-1]["etot"] - outs[-2]["etot"]) if len(outs) > 1 else None,
                     "eig": ctx.get_eig()}
        if name == "mixed":
            # FP64 refinement sweep of the converged mixed-precision state
            ref_ctx = Context(sys_, QX_PREC_FP64, QX_NL_GSPACE)
            ref_ctx.scf_init(mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0)
            ref_ctx.scf_mixing(PULAY_ITRATN, PULAY_CMETRIC)
            ref_ctx.refine_from(ctx)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            routs = [ref_ctx.scf_iteration(CgParm.defaults(noband)) for _ in range(REFINE_ITERS)]
            e1.record()
            torch.cuda.synchronize()
            ref_ctx.set_force_tables()
            rl, rn = ref_ctx.forces()
            acc["mixed_refined"] = {"force": rl + rn, "iterations": acc["mixed"]["iterations"] + REFINE_ITERS,
                                    "etot": routs[-1]["etot"], "resid": routs[-1]["resid"],
                                    "detot_last": abs(routs[-1]["etot"] - routs[-2]["etot"]),
                                    "eig": ref_ctx.get_eig(), "ms": e0.elapsed_time(e1)}
            ref_ctx.close()
        ctx.close()
    kb_ctx = Context(sys_, QX_PREC_MIXED, QX_NL_GSPACE)
    kb_tables = kb_build_timing(sys_, kb_ctx, max(3, K), max(3, W), flush)
    kb_ctx.close()
    mixed, fp64, fp64b = res["mixed"], res["fp64"], res["fp64_batched"]
    batch = run_batch(K, W, ws, rank)
    fssh = run_fssh_md() if ws == 1 else None
    rspace = run_rspace(sys_, psi0, K, W, args.accuracy_iters, flush)
    hbm, peak_kind = peaks()
    N, ne = sys_.gs.kfft0, sys_.gs.nplwex
    bytes_per_bapp = 4 * N * 4 + 2 * ne * 4
    achieved = bytes_per_bapp * sys_.nband / (mixed["fft_pipeline_ms"] * 1e-3) / 1e9
    fft_flops_pass = 5.0 * N * math.log2(N) * sys_.nband     # two complex transforms per band pair
    line = {
        "metric": METRIC, "value": mixed["value"], "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": mixed["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": DATA,
        "config": workload_config(sys_, ws),
        "precision": "mixed: FP32 FFTs and H|psi>, 3xTF32 tensor-core contractions, FP64 Cholesky/eigen/density",
        "autotune": tune_report,
        "hpsi_band_apps_per_s": mixed["hpsi_band_apps_per_s"],
        "fp64": {"path": "plain FP64 drop-in, one-rank band order (sequential CG, one graph launch per sweep)",
                 "value": fp64["value"], "ms_per_step": fp64["ms_per_step"],
                 "hpsi_band_apps_per_s": fp64["hpsi_band_apps_per_s"],
                 "cg_bapps_per_iter": fp64["cg_bapps_per_iter"], "gpu_launches": fp64["launches"],
                 "band_matrix_gemm": fp64["band_matrix"]},
        "fp64_batched": {"path": "FP64, all bands at once (one band per rank order)",
                         "value": fp64b["value"], "ms_per_step": fp64b["ms_per_step"],
                         "cg_bapps_per_iter": fp64b["cg_bapps_per_iter"]},
        "batch48": batch,
        "fssh_md": fssh,
        "mixed_rspace": rspace,
        "kb_tables": kb_tables,
        "mixed_over_fp64": mixed["value"] / fp64["value"],
        "mixed_over_fp64_batched": mixed["value"] / fp64b["value"],
        "accuracy": accuracy(acc, sys_.cell.natom, args.accuracy_iters),
        "cg_bapps_per_iter": mixed["cg_bapps_per_iter"],
        "eig_clusters": mixed["eig_clusters"],
        "e2e": mixed["e2e"],
        "gpu_launches": mixed["launches"],
        "fp32_gemm_fallbacks_per_step": mixed["fp32_gemm_fallbacks_per_step"],
        "roofline": {"kernel": "H|psi> FFT pipeline (z inverse, plane pass, z forward), FP32",
                     "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_band_app": bytes_per_bapp,
                     # DRAM read + write of one all-band pass, from the ncu
                     # capture of this workload
                     "traffic": HPSI_PASS_DRAM_BYTES, "traffic_unit": "bytes per 160-band pass",
                     "algorithmic_bytes_per_pass": bytes_per_bapp * sys_.nband,
                     "fft_pipeline_ms": mixed["fft_pipeline_ms"],
                     "dram_gbs": HPSI_PASS_DRAM_BYTES / (mixed["fft_pipeline_ms"] * 1e-3) / 1e9,
                     "fp32_tflops": fft_flops_pass / (mixed["fft_pipeline_ms"] * 1e-3) / 1e12,
                     "limiter": PIPELINE_LIMITER},
        "clocks": mixed["clocks"],
    }
    if ws == 1 and rank == 0:
        times, ncg = oracle_scf_timing(sys_, psi0, CPU_SAMPLE_WARMUP, CPU_SAMPLE_ITERS, host_cores())
        v = 1.0 / float(np.mean(times))
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": host_cores(), "kind": "port",
                                "sample": f"SCF iterations {CPU_SAMPLE_WARMUP + 1}-"
                                          f"{CPU_SAMPLE_WARMUP + CPU_SAMPLE_ITERS} of this workload from the "
                                          f"same start on the FP64 CPU oracle (whole iterations, "
                                          f"{np.mean(ncg):.0f} CG band applications each), "
                                          f"{host_cores()} host threads"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def oracle_scf_timing(sys_, psi0, W, K, threads):
    """W untimed then K timed SCF iterations of the FP64 CPU oracle (the
    restatement of pwlda_md's iteration: potential, H|psi> of all bands,
    H_sub, Jacobi diagonalisation and rotation, batched eigen_BKL, schmidt2,
    softchg, Pulay mixing) from the same start as the device path, on
    `threads` host threads.  Returns the per-iteration wall times (s) and the
    CG band applications of the timed iterations."""
    import oracle
    from oracle.scf import ScfState
    oracle.set_threads(threads)
    psi, _, rc = oracle.schmidt(psi0)
    if rc:
        raise RuntimeError("oracle schmidt failed on the start wavefunctions")
    st = ScfState(sys_, psi, nlmode=1, mixbeta=PULAY_ASLH, kerker_q0=PULAY_Q0, pulay=PULAY_ITRATN,
                  cmetric=PULAY_CMETRIC)
    noband = int(sys_.cell.nel // 2)
    for _ in range(W):
        st.iteration(noband=noband)
    times, ncg = [], []
    for _ in range(K):
        t = time.perf_counter()
        r = st.iteration(noband=noband)
        times.append(time.perf_counter() - t)
        ncg.append(r["ncg_hpsi"])
    return times, ncg


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args):
    """The reference arm: QXMD's own CPU build cannot be compiled on this image
    (Fortran, FFTW and MPI are absent), so this times the CPU restatement of
    the same iteration (the oracle) on all host threads, one SCF iteration per
    step, on this workload from the same start."""
    rank = int(os.environ.get("RANK", "0"))
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from qxmd_b200 import cell
    sys_ = cell.si64()
    psi0 = cell.random_wavefunctions(sys_.gs.nplwex, sys_.nband)
    ncores = host_cores()
    times, ncg = oracle_scf_timing(sys_, psi0, args.warmup, args.steps, ncores)
    ms = 1e3 * float(np.mean(times))
    v = 1e3 / ms
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
            "config": workload_config(sys_, ws),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": ncores, "kind": "port",
                             "sample": f"timed SCF iterations {args.warmup + 1}-{args.warmup + args.steps} of this "
                                       f"workload on the FP64 CPU oracle (restatement of the reference "
                                       f"iteration, batched CG, {np.mean(ncg):.0f} CG band applications per "
                                       f"iteration), {ncores} host threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.profile_step:
        run_profile_step(args)
    elif args.profile_hpsi:
        run_profile_hpsi(args)
    elif args.profile_batch:
        run_profile_batch(args)
    elif args.si512:
        run_si512(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
