#!/usr/bin/env python
"""chi0(q, omega) throughput on one or more B200s: (k,E)-points per second.

Workload (default): the 2D square monolayer with 2 spd atoms per cell
(dimH = 36, chi dimension 648), seeded Slater-Koster model, 200 x 200 k mesh
(40 401 points after boundary folding), 128 imaginary-axis energies
(5 171 328 (E,k) points) plus 64 real-axis energies x the 40 401-point BZ for
every omega != 0, 32 frequencies in [0, 0.5] eV at q = 0.  One step is one
call of the public batched entry point (tg_chi0_batch) over --omegas-per-step
frequencies; steps walk through the 32 frequencies.  A unit is one (k, E)
quadrature point for one (q, omega): n_imag + n_real(omega) * nk per omega.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision split|fp64]
    python bench.py --impl reference ...     # CPU oracle on a bounded sample

With N > 1 (torchrun) every rank computes its own frequencies (the
reference's frequency-group split, no collective on the data path): weak
scaling, value = all ranks' units / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np

METRIC = "χ⁰(q,ω) (k,E)-points/s: split-precision vs FP64 on 1 B200 at rel err ≤1e-9"
UNIT = "(k,E)-points/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="split", choices=["split", "fp64"])
    ap.add_argument("--config", default="sq2")
    ap.add_argument("--omegas-per-step", type=int, default=0,
                    help="frequencies per step (0: 4, or 1 for slab16 and slab5, whose frequency costs tens of seconds)")
    ap.add_argument("--qs-per-step", type=int, default=0,
                    help="wave vectors per step along Gamma-X (tg_chi0_qbatch; 0: 2 for slab5, else 1 at q = 0)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="cost-model split counts only (no trial launches; for profiler launch lists)")
    ap.add_argument("--chi-orbitals", default="auto", choices=["auto", "all", "d"],
                    help="orbitals that enter chi (auto: d for slab16, the d-only chi of dimension 1600, else all)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-compare-fp64", action="store_true",
                    help="skip the FP64 arm (one step of the FP64 path on the same frequencies, untimed for value)")
    ap.add_argument("--no-check", action="store_true",
                    help="skip the untimed split-vs-FP64 accuracy check of the chi0 workload")
    ap.add_argument("--green", default="auto", choices=["auto", "gauss-jordan", "spectral"],
                    help="Green-function method (tg_set_green_method)")
    ap.add_argument("--workload", default="chi0", choices=["chi0", "she", "ldos", "scf", "lsoc", "jij", "newton"],
                    help="chi0: the susceptibility integral (headline); she: the disturbance integral "
                         "(eintshe) of the same mesh, one frequency per step; ldos: the real-axis LDOS; "
                         "scf: occupations + Jacobian of one Newton step; lsoc: the linear-SOC chi0; "
                         "jij: the exchange coupling; newton: Newton self-consistency to max|f| <= 1e-10 "
                         "with the (V, B) adjoint checked by central differences at the fixed point")
    ap.add_argument("--small", action="store_true",
                    help="30 x 30 k mesh, 64 + 16 energies: a few-second case for profiler captures")
    return ap.parse_args()


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------- workload
def workload(config: str, small: bool = False):
    from titan_b200.host import synthetic
    from titan_b200.host.system import initial_state
    deck = synthetic.make_deck(config, nk=(30, 30, 30), n1gl=32, parts=2, n3gl=16) if small else \
        synthetic.make_deck(config)
    s = deck.system
    h0 = s.h0(initial_state(s))
    omegas = deck.frequencies()
    reals = [deck.real_points(e, s.Ef) for e in omegas]
    return deck, h0, omegas, reals


def units_of(deck, omegas_idx, reals):
    nimag = deck.ek.n_points
    nk = deck.real_kp.shape[0]
    return sum(nimag + len(reals[i][0]) * nk for i in omegas_idx)


def inversions_of(deck, per, reals, first, nq=1, shared=False, real_per_q=False):
    """Green functions formed in one step: G2 once per imaginary point (shared by the step's
    frequencies, and by its wave vectors when shared), G1 per imaginary point, frequency and
    wave vector (G1 = G2 at e = 0, q = 0 on a single-q call), two per real-axis point (G2 of a
    real-axis point shared by the wave vectors when shared, unless the real axis is spectral
    (real_per_q), where every wave vector forms its own G2)."""
    n_om = len(reals)
    idx = [(first + j) % n_om for j in range(per)]
    nimag = deck.ek.n_points
    nk = deck.real_kp.shape[0]
    if shared:
        inv = nimag
        for i in idx:
            inv += nq * nimag
            if len(reals[i][0]):
                inv += (2 * nq if real_per_q else 1 + nq) * len(reals[i][0]) * nk
        return inv
    inv = nimag
    for i in idx:
        if len(reals[i][0]) == 0 and i == idx[0]:
            continue
        inv += nimag + 2 * len(reals[i][0]) * nk
    return nq * inv


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def cpu_baseline(deck, h0, reals, omegas, seconds_target=15.0, sel=None):
    """The oracle (numpy/LAPACK, all host threads) on a bounded sample of the workload.

    A 200-point calibration run sizes the sample so that it takes about
    seconds_target: two thirds imaginary-axis points (in mesh order), one
    third real-axis points (all real energies of omega_1 x the first k points).
    """
    from oracle import titan_oracle as O
    from titan_b200.host.mesh import EKMesh
    s = deck.system
    m = O.Model(s, h0)
    w_idx = 1 if len(omegas) > 1 else 0
    e = float(omegas[w_idx])
    x2, p2 = reals[w_idx]
    ek = deck.ek

    def run(n_imag_s, nk_s):
        sub = EKMesh(ek.y, ek.wght, ek.energy_index[:n_imag_s], ek.kp[:n_imag_s], ek.weight[:n_imag_s])
        rk = (deck.real_kp[:max(nk_s, 1)], deck.real_w[:max(nk_s, 1)])
        t0 = time.perf_counter()
        O.eintshechi(m, sub, rk, np.zeros(3), e, s.Ef, s.eta, s.etap, x2 if nk_s else None, p2 if nk_s else None,
                     sel=sel)
        return time.perf_counter() - t0

    cal = min(200 if s.dimH <= 90 else 20, ek.n_points)
    rate = cal / max(run(cal, 0), 1e-6)
    n_imag_s = int(min(ek.n_points, max(cal, rate * seconds_target * 2 / 3)))
    nk_s = int(min(deck.real_kp.shape[0], max(1, rate * seconds_target / 3 / max(len(x2), 1)))) if len(x2) else 0
    dt = run(n_imag_s, nk_s)
    units = n_imag_s + len(x2) * nk_s
    cores = os.cpu_count()
    return {"value": units / dt, "unit": UNIT, "cores": cores, "kind": "port", "seconds": dt,
            "sample": f"oracle eintshechi (numpy/LAPACK, {cores} threads) on {n_imag_s} imaginary-axis points + "
                      f"{len(x2)} real-axis energies x {nk_s} k of the {deck.system.name} workload at omega={e:.4g} "
                      f"({units} units, {dt:.1f} s)"}


# --------------------------------------------------------------------------- reference arm
def chi_selection(args, system):
    """Per-site orbitals of chi: every orbital, or the d orbitals (the d-only chi of the 16-layer slab)."""
    mode = args.chi_orbitals
    if mode == "auto":
        mode = "d" if args.config == "slab16" else "all"
    return [list(d) for d in system.dorbs] if mode == "d" else None


def chi_dim(system, sel):
    return system.dimens if sel is None else 4 * sum(len(x) ** 2 for x in sel)


def chi0_workload_desc(args, deck, omegas, reals):
    """The headline workload's name, the same on both arms."""
    s = deck.system
    sel = chi_selection(args, s)
    return (f"{args.config}: dimH={s.dimH}, chi dim={chi_dim(s, sel)}{' (d orbitals)' if sel else ''}, "
            f"{deck.ek.n_points} imag (E,k) points, {deck.real_kp.shape[0]} real-axis k x {len(reals[-1][0])} "
            f"energies, {len(omegas)} omega in [0,{max(omegas):.2g}], q=0")


def qs_per_step(args):
    if args.qs_per_step > 0:
        return args.qs_per_step
    return 2 if args.config == "slab5" else 1


def q_grid(system, nq=16):
    """nq wave vectors uniform along Gamma-X (X = b1 / 2): q_i = (i / nq) b1 / 2, i = 0 .. nq - 1."""
    b1 = np.asarray(system.reciprocal()[0], float)
    return [0.5 * i / nq * b1 for i in range(nq)]


def step_qs(args, system, step):
    """The wave vectors of one step: [0] when a step has one, else consecutive Gamma-X points."""
    nq = qs_per_step(args)
    if nq == 1 and args.config != "slab5":
        return [np.zeros(3)]
    grid = q_grid(system)
    return [grid[(step * nq + j) % len(grid)] for j in range(nq)]


def omegas_per_step(args):
    if args.omegas_per_step > 0:
        return args.omegas_per_step
    return 1 if args.config in ("slab16", "slab5") else 4


def run_reference(args, rank, world):
    if rank != 0:
        return
    deck, h0, omegas, reals = workload(args.config, args.small)
    cb = None
    vals, secs = [], []
    # every warm-up step runs (on a shorter sample), then the timed steps on ~8 s samples, so
    # that the driver's --steps 20 --warmup 5 ends within a few minutes
    sel = chi_selection(args, deck.system)
    for _ in range(args.warmup):
        cpu_baseline(deck, h0, reals, omegas, seconds_target=2.0, sel=sel)
    for _ in range(args.steps):
        cb = cpu_baseline(deck, h0, reals, omegas, seconds_target=8.0, sel=sel)
        vals.append(cb["value"])
        secs.append(cb["seconds"])
    v = statistics.median(vals)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(secs), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Slater-Koster model, no external data)", "impl": "reference",
            "config": {"workload": chi0_workload_desc(args, deck, omegas, reals),
                       "step": "a bounded sample of the workload through the CPU restatement of eintshechi "
                               "(the reference is Fortran; no Fortran compiler in this image)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cb["cores"], "kind": "port", "sample": cb["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- our arm
def timed_steps(gpu, deck, h0, omegas, reals, steps, start, per, precision, prof=True, args=None, step0=0):
    """Run `steps` chi0 calls (tg_chi0_batch at q = 0, or tg_chi0_qbatch over the step's wave
    vectors); returns (device ms list, units, launches, last timing)."""
    s = deck.system
    n_om = len(omegas)
    ms, units, launches = [], 0, 0
    for st in range(steps):
        idx = [(start + st * per + j) % n_om for j in range(per)]
        es = [float(omegas[i]) for i in idx]
        qs = step_qs(args, s, step0 + st) if args is not None else [np.zeros(3)]
        if len(qs) == 1 and not np.any(qs[0]):
            gpu.chi0_batch(np.zeros(3), es, s.Ef, s.eta, s.etap, [reals[i][0] for i in idx],
                           [reals[i][1] for i in idx], precision)
        else:
            gpu.chi0_qbatch(np.array(qs), es, s.Ef, s.eta, s.etap, [reals[i][0] for i in idx],
                            [reals[i][1] for i in idx], precision)
        t = gpu.last_timing()
        ms.append(t[3])
        launches += int(t[10])
        units += len(qs) * units_of(deck, idx, reals)
    return ms, units, launches, t


def split_accuracy(gpu, deck, omegas, reals, per):
    """Split chi0 against the FP64 path on the full workload, untimed: the frequencies of one
    step (the largest ones, which carry the real-axis part too), worst one.  Normwise per 4 x 4
    spin block, max over blocks, and over the whole matrix."""
    from titan_b200.host.accuracy import spin_block_errors, spin_block_table
    s = deck.system
    idx = list(range(len(omegas) - per, len(omegas)))
    es = [float(omegas[i]) for i in idx]
    x2s, p2s = [reals[i][0] for i in idx], [reals[i][1] for i in idx]
    sp = gpu.chi0_batch(np.zeros(3), es, s.Ef, s.eta, s.etap, x2s, p2s, "split").copy()
    bound = gpu.error_bound(len(es))
    fp = gpu.chi0_batch(np.zeros(3), es, s.Ef, s.eta, s.etap, x2s, p2s, "fp64")
    per_w = [spin_block_errors(sp[w], fp[w], significant=1e-8) for w in range(len(idx))]
    tables = [spin_block_table(sp[w], fp[w]) for w in range(len(idx))]
    by_threshold = {t: [tables[0][t][0], max(tb[t][1] for tb in tables)] for t in tables[0]}
    return {"max": max(e[1] for e in per_w),
            "max_by_block_size": by_threshold,
            "frobenius": max(e[2] for e in per_w),
            "max_incl_roundoff_zero_blocks": max(e[0] for e in per_w),
            "per_omega_max": [e[1] for e in per_w], "omegas": es, "nonzero_blocks": per_w[0][3],
            "error_bound": {"per_omega": [float(b) for b in bound],
                            "basis": "tg_chi0_error_bound: worst-case normwise bound of the split format "
                                     "(46-bit rounding per chunk scale + dropped digit products), relative "
                                     "to ||chi||_F; compare with frobenius"},
            "measure": "max over 4x4 spin blocks b holding >= 1e-8 of the largest block norm of "
                       "||chi_split_b - chi_fp64_b||_F / ||chi_fp64_b||_F (the smaller blocks are zero by "
                       "symmetry up to FP64 roundoff; max_incl_roundoff_zero_blocks includes them); "
                       "max_by_block_size: {threshold: [blocks holding >= threshold of the largest, max error]}; "
                       "frobenius: whole matrix; same calls, full mesh"}


def run_ours(args, rank, world, local_rank):
    import torch
    from titan_b200.native import GreenGPU
    torch.cuda.set_device(local_rank)
    deck, h0, omegas, reals = workload(args.config, args.small)
    s = deck.system
    gpu = GreenGPU(local_rank)
    gpu.setup(deck, h0)
    sel = chi_selection(args, s)
    gpu.set_chi_orbitals(sel)
    D = chi_dim(s, sel)
    gpu.set_green_method(args.green)
    gpu.set_autotune(not args.no_autotune)
    gpu.profile(True)
    per = omegas_per_step(args)
    start = rank * per * (args.steps + args.warmup)     # ranks take different frequencies
    # warm-up (untimed)
    timed_steps(gpu, deck, h0, omegas, reals, args.warmup, start, per, args.precision, args=args, step0=0)
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(local_rank)
    clk.start()
    ms, units, launches, last = timed_steps(gpu, deck, h0, omegas, reals, args.steps, start + args.warmup * per, per,
                                            args.precision, args=args, step0=args.warmup)
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier(world)
    total_ms = sum(ms)
    total_ms_max = allreduce_max(total_ms, world)
    units_all = allreduce_sum(units, world)
    value = units_all / (total_ms_max / 1e3)
    # roofline of the chi0 contraction kernel (kind 1: the tcgen05 kernel alone on the split
    # path, the FP64 GEMM on the fp64 path): algorithmic 8 * dimens^2 flops per unit
    con_ms, con_n = last[6], last[7]
    grn_ms, grn_n = last[4], last[5]
    q_ms, q_n = last[11], last[12]
    nq = len(step_qs(args, s, args.warmup + args.steps - 1))
    last_units = nq * units_of(deck, [(start + args.warmup * per + (args.steps - 1) * per + j) % len(omegas)
                                      for j in range(per)], reals)
    pk, pk_kind = peaks()
    flops_con = 8.0 * D ** 2 * last_units
    achieved = flops_con / (con_ms / 1e3) / 1e12 if con_ms > 0 else None
    # the contraction runs inside a seconds-long step: the sustained (power-capped) GEMM peak
    peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
    # DRAM traffic per contraction launch from the ncu capture in
    # profiles/split_contract_sq2_small.md (2.188 GB over 1984 K-steps of 32 points),
    # scaled by the K-steps one launch of this run processes
    kstep_bytes = 2.188e9 / 1984
    traffic = kstep_bytes * (last_units / 32.0) / con_n if (con_n and args.precision == "split") else None
    roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": (achieved / peak) if achieved else None, "traffic": traffic,
            "kernel": "chi0 contraction (" + ("tcgen05 int8-sliced split_contract_kernel" if args.precision == "split"
                                              else "fp64 SIMT gemm64_kernel") + ")",
            "peak_source": ("of measured bf16 dense sustained (MEASURED_PEAKS.json)" if pk_kind == "measured"
                            else "of fallback 1.4 PF sustained"),
            "flops_per_unit": 8.0 * D ** 2,
            "launches_in_last_step": int(con_n), "avg_launch_ms": (con_ms / con_n) if con_n else None,
            "quantize_ms_last_step": q_ms if args.precision == "split" else None}
    if args.precision == "split" and con_n:
        # what the tensor pipe executes: 21 int8 MMAs of 128 x 80 x 32 per 64 x 40 complex tile
        # and K-step of 32 points (tiles: ceil(M/64) x ceil(M/40) per site pair, M = 4 n_i n_j)
        nc = s.norbs if sel is None else [len(x) for x in sel]
        tiles = sum(-(-4 * a * b // 64) * -(-4 * a * b // 40) for a in nc for b in nc)
        ops = tiles * (last_units / 32.0) / con_n * 21 * 2 * 128 * 80 * 32
        tops = ops / (con_ms / con_n / 1e3) / 1e12
        roof["executed_int8"] = {"tops": tops, "nominal_dense_tops": 4500.0, "frac_of_nominal": tops / 4500.0,
                                 "frac_of_2x_measured_bf16": tops / (2.0 * peak),
                                 "basis": "int8 MMA ops issued per launch (K-step padding not counted) / "
                                          "launch time, against the nominal dense int8 rate (4.5 POPS); that "
                                          "fraction is the one to set beside ncu's sm__pipe_tensor_cycles_active "
                                          "of the kernel (profiles/split_contract_sq2_small.md). Twice the "
                                          "measured bf16 rate is below the nominal int8 rate because the bf16 "
                                          "GEMM it comes from runs at the power cap"}
    from titan_b200.native import fp64_peak
    dfma, dmma = fp64_peak()
    native_n = s.dimH in (4, 8, 16, 18, 20, 36, 40, 54, 72, 90)
    tabulated = len(set(np.bincount(deck.ek.energy_index).tolist())) == 1   # every energy on the same k list
    # chi0's Green functions on meshes whose energies share a k list: spectral from the unpacked
    # Jacobi kernel (even dimH <= 72), else under AUTO from a Householder tridiagonalisation per k
    # (G over the rows chi needs: 8 |S|^2 n flops per point, a DMMA GEMM); adaptive imaginary axes
    # (shared G2 across q) keep Gauss-Jordan there and use these on the real axis only
    eig_fast = args.green != "gauss-jordan" and s.dimH % 2 == 0 and s.dimH <= 72
    tri_ok = args.green == "auto" and not eig_fast
    shared = nq > 1 and not tabulated
    spectral = eig_fast and tabulated
    spectral_real = eig_fast and shared
    tri_all = tri_ok and tabulated
    tri_real = tri_ok and shared
    # the spectral real axis forms G2 again per wave vector; the tridiagonalised one shares it
    n_inv = inversions_of(deck, per, reals, start + args.warmup * per + (args.steps - 1) * per, nq, shared,
                          spectral_real and shared)
    ns = sum(2 * len(o) for o in sel) if sel is not None else s.dimH
    tri_name = ("hh_tridiag_kernel + tri_green_kernel (Householder tridiagonalisation per k, G over the %d rows "
                "of chi per point: tridiagonal solves + FP64 DMMA GEMM) + gather_kernel" % ns)
    gj_name = ("green_w1_kernel / green_team_kernel (fused H(k) + Gauss-Jordan)" if native_n else
               "green_cluster_kernel (thread-block-cluster Gauss-Jordan) + gather_kernel")
    kname = ("eig_jacobi_kernel + spec_green_kernel (spectral G, FP64 DMMA)" if spectral else
             gj_name + " on the imaginary axis; eig_jacobi_kernel + spec_green_kernel (spectral) on the real axis"
             if spectral_real else
             tri_name if tri_all else
             gj_name + " on the imaginary axis; " + tri_name + " on the real axis" if tri_real else gj_name)
    dmma_path = spectral or spectral_real or tri_all or tri_real
    peak64 = dmma if dmma_path else dfma
    # algorithmic flops per Green function: 8 n^3 (an inversion or a full spectral G), 8 |S|^2 n where
    # the tridiagonalised path forms G over the rows S only (mixed paths: the n^3 figure)
    flops_g = 8.0 * ns * ns * s.dimH if tri_all else 8.0 * s.dimH ** 3
    roof_inv = {"bound": "fp64", "achieved": (flops_g * n_inv) / (grn_ms / 1e3) / 1e12 if grn_ms else None,
                "peak": peak64, "unit": "TFLOP/s",
                "peak_source": ("of measured FP64 DMMA (tg_fp64_peak, this run)" if dmma_path
                                else "of measured FP64 DFMA (tg_fp64_peak, this run)"),
                "kernel": kname, "flops_per_inversion": flops_g, "inversions_last_step": n_inv,
                "ms_last_step": grn_ms, "launches_in_last_step": int(grn_n)}
    roof_inv["frac"] = roof_inv["achieved"] / peak64 if roof_inv["achieved"] else None
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "s8 tensor-core slices + f64" if args.precision == "split" else "f64",
            "data": "synthetic (seeded Slater-Koster model, no external data)",
            "config": {"workload": chi0_workload_desc(args, deck, omegas, reals),
                       "omegas_per_step": per, "precision": args.precision, "green": args.green,
                       "l2": "inputs larger than L2 (mesh 200+ MB, operands GBs per pass)"},
            "roofline": roof, "roofline_inversion": roof_inv, "gpu_launches": launches, "clocks": clocks,
            "schedule": {"nsplit_autotuned": gpu.tuning()[1 if args.precision == "split" else 0],
                         "split_chunk_points": 1024, "wave_vectors_per_step": nq,
                         "g2_shared_across_q": bool(shared)}}
    if not args.no_compare_fp64 and args.precision != "fp64":
        # the FP64 arm of the metric: the same step (same frequencies as the last timed step) on the
        # plain FP64 path, device-timed the same way
        f0 = start + args.warmup * per + (args.steps - 1) * per
        ms64, u64, _, _ = timed_steps(gpu, deck, h0, omegas, reals, 1, f0, per, "fp64", args=args,
                                      step0=args.warmup + args.steps - 1)
        line["fp64_path"] = {"value": u64 / (sum(ms64) / 1e3), "unit": UNIT, "ms_per_step": sum(ms64),
                             "step": "one chi0 call over the frequencies and wave vectors of the last timed step, "
                                     "TG_PREC_FP64 (FP64 SIMT contraction), same Green functions"}
        line["split_over_fp64"] = (value / world) / line["fp64_path"]["value"]
    if args.precision == "split" and not args.no_check:
        line["split_rel_err"] = split_accuracy(gpu, deck, omegas, reals, per)
    # end to end: public API from pinned host buffers, full set-up + call + read-back every step
    if not args.no_e2e:
        e2e = run_e2e(gpu, deck, h0, omegas, reals, args, start + args.warmup * per, per, world)
        line["e2e"] = e2e
    if rank == 0 and not args.no_cpu and world == 1:
        line["cpu_baseline"] = cpu_baseline(deck, h0, reals, omegas, sel=sel)
    gpu.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_e2e(gpu, deck, h0, omegas, reals, args, start, per, world):
    import torch
    s = deck.system
    ek = deck.ek

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()

    y = pinned(np.ascontiguousarray(ek.point_energy(), np.float64))
    kp = pinned(np.ascontiguousarray(ek.kp, np.float64))
    w = pinned(np.ascontiguousarray(ek.weight, np.float64))
    rk = pinned(np.ascontiguousarray(deck.real_kp, np.float64))
    rw = pinned(np.ascontiguousarray(deck.real_w, np.float64))
    h0p = pinned(np.ascontiguousarray(h0, np.complex128).view(np.float64))
    sel = chi_selection(args, s)
    D = chi_dim(s, sel)
    out = torch.empty((per, D, D * 2), dtype=torch.float64, pin_memory=True).numpy().view(np.complex128)
    gpu.profile(False)
    h2d = y.nbytes + kp.nbytes + w.nbytes + rk.nbytes + rw.nbytes + h0p.nbytes
    units = 0
    barrier(world)
    t0 = time.perf_counter()
    for st in range(args.steps):
        idx = [(start + st * per + j) % len(omegas) for j in range(per)]
        gpu.set_system(s)
        gpu.set_chi_orbitals(sel)
        gpu.set_h0(h0p.view(np.complex128).reshape(s.dimH, s.dimH))
        gpu.set_imag_mesh_arrays(y, kp.reshape(-1, 3), w)
        gpu.set_real_mesh(rk.reshape(-1, 3), rw)
        gpu.chi0_batch(np.zeros(3), [float(omegas[i]) for i in idx], s.Ef, s.eta, s.etap,
                       [reals[i][0] for i in idx], [reals[i][1] for i in idx], args.precision, out=out)
        units += units_of(deck, idx, reals)
    dt = time.perf_counter() - t0
    dt_max = allreduce_max(dt, world)
    units_all = allreduce_sum(units, world)
    return {"value": units_all / dt_max, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(out.nbytes), "timer": "host wall clock around the public API calls"}


# --------------------------------------------------------------------------- disturbance integral
SHE_METRIC = "eintshe disturbance integral (k,E)-points/s on 1 B200 (FP64)"
SHE_UE = (1.0, 0.0, 0.0)


def she_vertex_flops(s, real_axis):
    """Algorithmic FP64 flops of the vertex sandwiches of one point: per term Y^b = L V
    (2 n no^2 complex FMA) and the 4 dimens output entries (no complex FMA each); two terms
    on the imaginary axis, one on the real axis; 8 flops per complex FMA."""
    n, no = s.dimH, s.dimH // 2
    per_term = 8.0 * (2 * n * no * no + 4 * s.dimens * no)
    return per_term * (1 if real_axis else 2)


def she_cpu_baseline(deck, h0, reals, omegas, seconds_target=15.0):
    """The oracle's eintshe (numpy, all host threads) on a bounded sample of the workload."""
    from oracle import titan_oracle as O
    from titan_b200.host.mesh import EKMesh
    s = deck.system
    m = O.Model(s, h0)
    w_idx = 1 if len(omegas) > 1 else 0
    e = float(omegas[w_idx])
    x2, p2 = reals[w_idx]
    ek = deck.ek

    def run(n_imag_s, nk_s):
        sub = EKMesh(ek.y, ek.wght, ek.energy_index[:n_imag_s], ek.kp[:n_imag_s], ek.weight[:n_imag_s])
        rk = (deck.real_kp[:max(nk_s, 1)], deck.real_w[:max(nk_s, 1)])
        t0 = time.perf_counter()
        O.eintshe(m, sub, rk, np.zeros(3), e, s.Ef, s.eta, s.etap, x2 if nk_s else None, p2 if nk_s else None,
                  SHE_UE)
        return time.perf_counter() - t0

    cal = min(100, ek.n_points)
    rate = cal / max(run(cal, 0), 1e-6)
    n_imag_s = int(min(ek.n_points, max(200, rate * seconds_target * 2 / 3)))
    nk_s = int(min(deck.real_kp.shape[0], max(1, rate * seconds_target / 3 / max(len(x2), 1)))) if len(x2) else 0
    dt = run(n_imag_s, nk_s)
    units = n_imag_s + len(x2) * nk_s
    cores = os.cpu_count()
    return {"value": units / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"oracle eintshe (numpy, {cores} threads) on {n_imag_s} imaginary-axis points + "
                      f"{len(x2)} real-axis energies x {nk_s} k of the {deck.system.name} workload at omega={e:.4g} "
                      f"({units} units, {dt:.1f} s)"}


def run_she(args, rank, world, local_rank):
    """One tg_she call per step (one frequency, q = 0, E along x), frequencies walked per rank."""
    import torch
    from titan_b200.native import GreenGPU
    torch.cuda.set_device(local_rank)
    deck, h0, omegas, reals = workload(args.config, args.small)
    s = deck.system
    gpu = GreenGPU(local_rank)
    gpu.setup(deck, h0)
    gpu.set_green_method(args.green)
    gpu.profile(True)
    n_om = len(omegas)
    start = 1 + rank * (args.steps + args.warmup)   # omega_0 = 0 has no real axis; start at omega_1

    def steps(k, first):
        ms, units, launches, vert = [], 0, 0, 0.0
        flops = 0.0
        for st in range(k):
            i = (first + st) % n_om
            if i == 0:
                i = 1
            x2, p2 = reals[i]
            gpu.she(np.zeros(3), float(omegas[i]), s.Ef, s.eta, s.etap, x2, p2, SHE_UE)
            t = gpu.last_timing()
            ms.append(t[3])
            launches += int(t[10])
            vert = (t[6], t[7])
            nreal = len(x2) * deck.real_kp.shape[0]
            units += deck.ek.n_points + nreal
            flops = she_vertex_flops(s, False) * deck.ek.n_points + she_vertex_flops(s, True) * nreal
        return ms, units, launches, vert, flops, t

    steps(args.warmup, start)
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(local_rank)
    clk.start()
    ms, units, launches, vert, flops_last, last = steps(args.steps, start + args.warmup)
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier(world)
    total_ms_max = allreduce_max(sum(ms), world)
    value = allreduce_sum(units, world) / (total_ms_max / 1e3)
    v_ms, v_n = vert
    fp64_nominal = 37.0
    achieved = flops_last / (v_ms / 1e3) / 1e12 if v_ms else None
    roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_nominal, "unit": "TFLOP/s",
            "frac": achieved / fp64_nominal if achieved else None, "traffic": None,
            "peak_source": "nominal B200 FP64 (not measured)", "kernel": "she_kernel (vertex sandwiches)",
            "flops_per_unit": {"imag": she_vertex_flops(s, False), "real": she_vertex_flops(s, True)},
            "launches_in_last_step": int(v_n), "ms_last_step": v_ms,
            "inversion_ms_last_step": last[4], "reduce_prefactor_ms_last_step": last[8]}
    line = {"metric": SHE_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Slater-Koster model, no external data)",
            "config": {"workload": f"{args.config}: dimH={s.dimH}, dimens={s.dimens}, {deck.ek.n_points} imag (E,k) "
                                   f"points + {deck.real_kp.shape[0]} real-axis k x 64 energies per omega, q=0, "
                                   f"E along x, one omega per step", "green": args.green,
                       "l2": "inputs larger than L2 (G1/G2 buffers GBs per pass)"},
            "roofline": roof, "gpu_launches": launches, "clocks": clocks}
    if rank == 0 and not args.no_cpu and world == 1:
        line["cpu_baseline"] = she_cpu_baseline(deck, h0, reals, omegas)
    gpu.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- local density of states
LDOS_METRIC = "real-axis LDOS (k,E)-points/s on 1 B200 (FP64)"
LDOS_ENERGIES = 1001


def ldos_energies(deck):
    s = deck.system
    return s.Ef + np.linspace(-2.0, 1.0, LDOS_ENERGIES)


def ldos_cpu_baseline(deck, h0, seconds_target=15.0):
    """The oracle's ldos (numpy, all host threads) on a bounded sample: all k, the first energies."""
    from oracle import titan_oracle as O
    s = deck.system
    m = O.Model(s, h0)
    es = ldos_energies(deck)
    t0 = time.perf_counter()
    O.ldos(m, (deck.real_kp, deck.real_w), es[:1], s.eta)
    rate = deck.real_kp.shape[0] / max(time.perf_counter() - t0, 1e-6)
    ne = int(min(len(es), max(1, rate * seconds_target / deck.real_kp.shape[0])))
    t0 = time.perf_counter()
    O.ldos(m, (deck.real_kp, deck.real_w), es[:ne], s.eta)
    dt = time.perf_counter() - t0
    units = ne * deck.real_kp.shape[0]
    cores = os.cpu_count()
    return {"value": units / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"oracle ldos (numpy/LAPACK, {cores} threads) on {ne} energies x {deck.real_kp.shape[0]} k of the "
                      f"{s.name} real-axis BZ ({units} units, {dt:.1f} s)"}


def run_ldos(args, rank, world, local_rank):
    """One tg_ldos call per step: 1001 energies over the real-axis BZ (weak scaling over ranks)."""
    import torch
    from titan_b200.native import GreenGPU
    torch.cuda.set_device(local_rank)
    deck, h0, _, _ = workload(args.config, args.small)
    s = deck.system
    gpu = GreenGPU(local_rank)
    gpu.setup(deck, h0)
    gpu.set_green_method(args.green)
    es = ldos_energies(deck)
    nk = deck.real_kp.shape[0]
    for _ in range(args.warmup):
        gpu.ldos(es, s.eta)
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(local_rank)
    clk.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        gpu.ldos(es, s.eta)
    stop.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier(world)
    ms = allreduce_max(start.elapsed_time(stop), world)
    units = allreduce_sum(len(es) * nk * args.steps, world)
    line = {"metric": LDOS_METRIC, "value": units / (ms / 1e3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Slater-Koster model, no external data)",
            "config": {"workload": f"{args.config}: dimH={s.dimH}, {nk} real-axis k x {len(es)} energies per step",
                       "green": args.green,
                       "timer": "CUDA events on the current stream around the blocking tg_ldos calls"},
            "clocks": clocks}
    if rank == 0 and not args.no_cpu and world == 1:
        line["cpu_baseline"] = ldos_cpu_baseline(deck, h0)
    gpu.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


SCF_METRIC = "self-consistency Newton step: occupations + Jacobian (k,E)-points/s on 1 B200 (FP64)"


def scf_cpu_baseline(deck, h0, seconds_target=15.0):
    """The oracle's expectation + jacobian (numpy, all host threads) on a bounded sample: the
    first imaginary-axis points in mesh order and the first real-axis k (Fermi column)."""
    from oracle import titan_oracle as O
    from titan_b200.host.mesh import EKMesh
    s = deck.system
    m = O.Model(s, h0)
    ek = deck.ek

    def run(npts):
        sub = EKMesh(ek.y, ek.wght, ek.energy_index[:npts], ek.kp[:npts], ek.weight[:npts])
        nk = max(1, min(deck.real_kp.shape[0], npts // 64))
        rk = (deck.real_kp[:nk], deck.real_w[:nk])
        t0 = time.perf_counter()
        O.expectation(m, sub, s.Ef, s.eta)
        O.jacobian(m, sub, rk, s.Ef, s.eta, False)
        return time.perf_counter() - t0

    cal = min(256, ek.n_points)
    dt = run(cal)
    npts = int(min(ek.n_points, max(cal, cal * seconds_target / max(dt, 1e-6))))
    dt = run(npts)
    cores = os.cpu_count()
    return {"value": npts / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"oracle expectation + jacobian (numpy/LAPACK, {cores} threads) on the first {npts} "
                      f"imaginary-axis points of the {s.name} mesh and {max(1, npts // 64)} real-axis k "
                      f"({dt:.1f} s)"}


def run_scf(args, rank, world, local_rank):
    """One self-consistency step's Green-function work per step: tg_expectation (occupations
    and moments) and tg_jacobian (GG tensors over the imaginary axis + the Fermi column over the
    real-axis BZ) at the same state; a unit is one imaginary-axis (E, k) point through both."""
    import torch
    from titan_b200.native import GreenGPU
    torch.cuda.set_device(local_rank)
    deck, h0, _, _ = workload(args.config, args.small)
    s = deck.system
    gpu = GreenGPU(local_rank)
    gpu.setup(deck, h0)
    gpu.set_green_method(args.green)

    def step():
        gpu.expectation(s.Ef, s.eta)
        gpu.jacobian(s.Ef, s.eta, False)

    for _ in range(args.warmup):
        step()
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(local_rank)
    clk.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        step()
    stop.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier(world)
    ms = allreduce_max(start.elapsed_time(stop), world)
    units = allreduce_sum(deck.ek.n_points * args.steps, world)
    line = {"metric": SCF_METRIC, "value": units / (ms / 1e3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Slater-Koster model, no external data)",
            "config": {"workload": f"{args.config}: dimH={s.dimH}, {deck.ek.n_points} imag (E,k) points through "
                                   f"tg_expectation and tg_jacobian, Fermi column over {deck.real_kp.shape[0]} k",
                       "green": args.green,
                       "timer": "CUDA events on the current stream around the blocking calls"},
            "clocks": clocks}
    if rank == 0 and not args.no_cpu and world == 1:
        line["cpu_baseline"] = scf_cpu_baseline(deck, h0)
    gpu.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


NEWTON_METRIC = "Newton self-consistency (k,E)-points/s (one point through one iteration: residual + Jacobian)"


def run_newton(args, rank, world, local_rank):
    """Newton self-consistency on the full mesh of the configuration (default bcc4: dimH 72,
    48^3 k, 96 imaginary energies) to max |f| <= 1e-10, from the seeded initial state: first
    converged to 1e-8 on a 12^3 mesh (untimed warm start), then on the full mesh (timed: every
    residual and Jacobian evaluation, line searches included).  At the fixed point the (V, B)
    adjoint (tg_adjoint_vb) is timed and one of its columns checked by central differences
    (h = 1e-5 eV).  One process: the fixed point is a single-GPU computation."""
    import torch
    from titan_b200.host import scf, synthetic
    from titan_b200.host.system import initial_state
    from titan_b200.host.vb import site_observables, vb_perturbation
    from titan_b200.native import GreenGPU
    torch.cuda.set_device(local_rank)
    deck, h0, _, _ = workload(args.config, args.small)
    s = deck.system
    coarse = synthetic.make_deck(args.config, nk=(12, 12, 12) if s.sysdim == 3 else (48, 48, 1))
    gpu = GreenGPU(local_rank)
    st0 = initial_state(s)
    gpu.setup(coarse, s.h0(st0))
    t0 = time.perf_counter()
    warm = scf.newton(gpu, s, st0, max_step=0.5, ftol=1e-8, maxit=80)
    t_warm = time.perf_counter() - t0
    gpu.setup(deck, s.h0(warm.state))
    torch.cuda.synchronize()
    clk = ClockSampler(local_rank)
    clk.start()
    t0 = time.perf_counter()
    res = scf.newton(gpu, s, warm.state, max_step=0.5, ftol=1e-10, maxit=60)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    clocks = clk.stop()
    # the adjoint at the fixed point, and one column by central differences
    st = scf.state_from_unknowns(s, res.x, warm.state)
    h_fix = s.h0(st)
    gpu.set_h0(h_fix)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    A = gpu.adjoint_vb(st.Ef, s.eta)
    torch.cuda.synchronize()
    t_adj = time.perf_counter() - t1
    hstep = 1e-5

    def x_of(V, B):
        gpu.set_h0(h_fix + vb_perturbation(s, V, B))
        rho, mx, my, mz, _ = gpu.expectation(st.Ef, s.eta)
        return site_observables(s, rho, mx, my, mz).reshape(-1)

    B0 = np.zeros((s.n_atoms, 3))
    cols = {}
    for b in (0, 3):   # V and Bz of site 0
        dV = np.zeros(s.n_atoms)
        dB = np.zeros((s.n_atoms, 3))
        if b == 0:
            dV[0] = hstep
        else:
            dB[0, 2] = hstep
        fd = (x_of(dV, B0 + dB) - x_of(-dV, B0 - dB)) / (2 * hstep)
        nm = "V0" if b == 0 else "Bz0"
        cols[nm] = float(np.max(np.abs(fd - A[:, b])))
        cols[nm + "_relative"] = float(np.max(np.abs(fd - A[:, b])) / np.max(np.abs(A[:, b])))
    # one iteration evaluates the residual (plus line-search residuals) and the Jacobian
    evals = res.iterations
    units = deck.ek.n_points * max(evals, 1)
    line = {"metric": NEWTON_METRIC, "value": units / dt, "unit": UNIT, "n_gpus": 1, "steps": res.iterations,
            "warmup": warm.iterations, "ms_per_step": 1e3 * dt / max(res.iterations, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Slater-Koster model, no external data)",
            "config": {"workload": f"{args.config}: dimH={s.dimH}, {deck.ek.n_points} imag (E,k) points, "
                                   f"Fermi column over {deck.real_kp.shape[0]} k, {len(res.x)} unknowns",
                       "start": f"seeded initial state iterated on a coarse mesh ({coarse.ek.n_points} points, "
                                f"{warm.iterations} iterations to max|f| = {np.max(np.abs(warm.residual)):.1e}, "
                                f"{t_warm:.1f} s, untimed)",
                       "timer": "host wall clock around the blocking Newton iteration (GPU work + N x N solves)"},
            "newton": {"converged": bool(res.converged), "iterations": res.iterations,
                       "max_abs_residual": float(np.max(np.abs(res.residual))), "seconds": dt},
            "adjoint": {"seconds": t_adj, "fd_h": hstep, "max_abs_adjoint": float(np.max(np.abs(A))),
                        "fd_minus_adjoint": cols},
            "clocks": clocks}
    gpu.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_row(args, rank, world, local_rank):
    """The linear-SOC susceptibility (--workload lsoc: one tg_chi0_linear_soc call at the
    second frequency, q = 0, per step; units as chi0) and the exchange coupling (--workload
    jij: one tg_jij call at q = 0 with all moments along z, per step; a unit is one
    imaginary-axis point), each with the oracle on a bounded slice of the same mesh."""
    import torch
    from oracle import titan_oracle as O
    from titan_b200.host.mesh import EKMesh
    from titan_b200.host.system import initial_state
    from titan_b200.native import GreenGPU
    torch.cuda.set_device(local_rank)
    deck, h0, omegas, reals = workload(args.config, args.small)
    s = deck.system
    ek = deck.ek
    gpu = GreenGPU(local_rank)
    q = np.zeros(3)
    e = float(omegas[1])
    x2, p2 = reals[1]
    nk = deck.real_kp.shape[0]
    if args.workload == "lsoc":
        h00, V = s.linear_soc_split(initial_state(s))
        gpu.setup(deck, h00)
        metric = "linear-SOC chi0 (eintshechilinearsoc) (k,E)-points/s on 1 B200 (FP64)"
        step_units = ek.n_points + len(x2) * nk
        desc = f"{ek.n_points} imag (E,k) points + {len(x2)} real-axis energies x {nk} k at omega={e:.5f}, q=0"

        def step():
            gpu.chi0_linear_soc(q, e, s.Ef, s.eta, s.etap, x2, p2, V)

        def cpu(npts):
            sub = EKMesh(ek.y, ek.wght, ek.energy_index[:npts], ek.kp[:npts], ek.weight[:npts])
            t0 = time.perf_counter()
            O.eintshechi_linear_soc(O.Model(s, h00), V, sub, (deck.real_kp[:1], deck.real_w[:1]), q, e, s.Ef, s.eta,
                                    s.etap, x2, p2)
            return time.perf_counter() - t0, npts + len(x2)
        what = "oracle eintshechi_linear_soc"
    else:
        gpu.setup(deck, h0)
        evec = np.tile([0.0, 0.0, 1.0], (s.n_atoms, 1))
        metric = "exchange coupling J_ij(q) (jij_energy) (k,E)-points/s on 1 B200 (FP64)"
        step_units = ek.n_points
        desc = f"{ek.n_points} imag (E,k) points, q=0, moments along z"

        def step():
            gpu.jij(q, s.Ef, s.eta, evec, s.Um())

        def cpu(npts):
            sub = EKMesh(ek.y, ek.wght, ek.energy_index[:npts], ek.kp[:npts], ek.weight[:npts])
            t0 = time.perf_counter()
            O.jij(O.Model(s, h0), sub, q, s.Ef, s.eta, evec, s.Um(), s.dorbs)
            return time.perf_counter() - t0, npts
        what = "oracle jij"
    gpu.set_green_method(args.green)
    for _ in range(args.warmup):
        step()
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(local_rank)
    clk.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        step()
    stop.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier(world)
    ms = allreduce_max(start.elapsed_time(stop), world)
    units = allreduce_sum(step_units * args.steps, world)
    line = {"metric": metric, "value": units / (ms / 1e3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Slater-Koster model, no external data)",
            "config": {"workload": f"{args.config}: dimH={s.dimH}, {desc}", "green": args.green,
                       "timer": "CUDA events on the current stream around the blocking calls"},
            "clocks": clocks}
    if rank == 0 and not args.no_cpu and world == 1:
        cal = min(256, ek.n_points)
        dt, _ = cpu(cal)
        npts = int(min(ek.n_points, max(cal, cal * 15.0 / max(dt, 1e-6))))
        dt, u = cpu(npts)
        cores = os.cpu_count()
        line["cpu_baseline"] = {"value": u / dt, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"{what} (numpy/LAPACK, {cores} threads) on the first {npts} "
                                          f"imaginary-axis points ({dt:.1f} s)"}
    gpu.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- distributed helpers
def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device="cuda" if dist.get_backend() == "nccl" else "cpu", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device="cuda" if dist.get_backend() == "nccl" else "cpu", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # the CPU reference arm: rank 0 alone works; no process group, no GPU
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.workload == "she":
            run_she(args, rank, world, local_rank)
        elif args.workload == "ldos":
            run_ldos(args, rank, world, local_rank)
        elif args.workload == "scf":
            run_scf(args, rank, world, local_rank)
        elif args.workload == "newton":
            run_newton(args, rank, world, local_rank)
        elif args.workload in ("lsoc", "jij"):
            run_row(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
