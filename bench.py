#!/usr/bin/env python
"""Benchmark of the J/K engine on the (H2O)16 DF-JK workload.

Workload: (H2O)16 water cluster (seeded, 9 A cube), RHF/cc-pVDZ (n = 384)
with the VDZ-JKFIT fitting basis (naux = 1856), nocc = 80: the density-fitted
J/K build molecular2 runs every SCF iteration (Fock::formJKdf,
src/fockbuild.cpp:171-174, 585-660).  A step is one J/K build for the
converged occupied orbitals; `value` is builds/s with everything resident in
HBM, `e2e` the same through the host-pointer C entry point (C uploaded, J and
K downloaded every step).  The whole RHF SCF is timed once per precision
mode and reported under "scf" (mixed = split-BF16 tensor-core builds, then
FP64 builds to convergence), with |dE| between the two.  Two more
workloads are timed once and reported beside the line: the FP64 analytic
gradient of (H2O)8/cc-pVDZ ("gradient") and one FP64 integral-direct J/K
build of C20H42/6-311G** ("direct_jk"); --no-extras skips them.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision mixed|fp64] [--profile]

--impl reference times molecular2's own algorithm on the host cores: the
oracle's restatement of compute_2body_fock_df's naive loops (molecular2
itself needs libint2/Eigen and cannot be built here), on a bounded sample of
the fitting functions, extrapolated linearly in naux.
--profile runs only the timed builds (no SCF, e2e or CPU leg) for ncu.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DF-JK Fock builds/s, (H2O)16 RHF/cc-pVDZ + VDZ-JKFIT"
UNIT = "builds/s"
SEED = 16


_WORKLOAD = None


def workload():
    global _WORKLOAD
    if _WORKLOAD is None:
        from molecular2_b200 import geometry
        from molecular2_b200.basis import BasisSet
        mol = geometry.water16(SEED)
        _WORKLOAD = (mol, BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit"))
    return _WORKLOAD


def traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu capture (None if absent)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    k = json.load(open(p)).get("kernels", {}).get(kernel)
    return k["dram_bytes_read"] + k["dram_bytes_write"] if k else None


def config(mol, obs, aux, prec, world=1):
    return {"workload": f"(H2O)16 RHF/cc-pVDZ + VDZ-JKFIT DF-JK build (n={obs.nbf}, naux={aux.nbf}, "
                        f"nocc={mol.nocc}), seed {SEED}",
            "precision": prec,
            "l2": "inputs larger than L2 (B tensor %.2f GB FP64 / %.2f GB split BF16)"
                  % (obs.nbf ** 2 * aux.nbf * 8 / 1e9, obs.nbf ** 2 * aux.nbf * 4 / 1e9),
            "parallelism": ("single GPU" if world == 1 else
                            f"aux-sharded x{world}: fitted-index slices per rank, one NCCL all-reduce of J and K "
                            "per build")}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


# ---------------------------------------------------------------- CPU leg
def cpu_sample(nthreads, target_s=12.0):
    """Time the naive per-iteration loops of compute_2body_fock_df on a
    contiguous block of fitting functions, doubling the block until one run
    takes target_s / 3 (the whole sample stays within about target_s);
    returns (builds/s extrapolated to all fitting functions, sample text, s)."""
    import oracle
    mol, obs, aux = workload()
    n, naux, nocc = obs.nbf, aux.nbf, mol.nocc
    rng = np.random.default_rng(0)
    npair = n * (n + 1) // 2
    C = np.asfortranarray(rng.normal(size=(n, nocc)))
    Bfull = None

    def run(nk):
        B = np.asfortranarray(Bfull[:, :nk])
        t = time.perf_counter()
        oracle.df_jk(B, C, (0, nk), nthreads=nthreads)
        return time.perf_counter() - t

    nk, prev, total = 2, None, 0.0
    Bfull = np.asfortranarray(rng.normal(size=(npair, 2)))
    while True:
        if Bfull.shape[1] < nk:
            Bfull = np.asfortranarray(rng.normal(size=(npair, nk)))
        t = run(nk)
        total += t
        if t >= target_s / 3 or nk >= naux:
            break
        prev = (nk, t)
        nk = min(naux, 2 * nk)
    if prev is not None and t > prev[1]:
        per_k = (t - prev[1]) / (nk - prev[0])          # slope, per fitting function
        t_full = max(t + per_k * (naux - nk), t)
    else:
        t_full = t * naux / nk
    sample = (f"naive X/K/gamma/J loops of compute_2body_fock_df over {nk} of {naux} fitting functions "
              f"(synthetic B values), {nthreads} thread(s), last run {t:.2f} s of {total:.1f} s sampled, "
              f"extrapolated linearly to {naux}")
    return 1.0 / t_full, sample, total


def run_reference(args, rank, world):
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    # each step a bounded sample, sized so that warm-up + steps take about 2-3 minutes
    per_step = min(3.0, max(0.3, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_sample(nthreads, target_s=per_step)
    vals = []
    t0 = time.perf_counter()
    sample = ""
    for _ in range(args.steps):
        v, sample, _ = cpu_sample(nthreads, target_s=per_step)
        vals.append(v)
    wall = time.perf_counter() - t0
    v = statistics.median(vals)
    mol, obs, aux = workload()
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(mol, obs, aux, "fp64"),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- clocks
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, path):
        self.path = path
        self.p = None
        try:
            self.f = open(path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(index), "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.close()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def roofline_fp64(n, naux, nocc, stages):
    names = ["X=B.C (cuBLAS DGEMM)", "K=X.X^T (cuBLAS DGEMM)", "gamma (k_gamma)", "J=B.gamma (k_df_J_lower)"]
    hbm, bf16, src = peaks()
    B_bytes = (n * (n + 1) // 2) * naux * 8   # k_df_J_lower reads the lower half of B
    own = 3
    ach = B_bytes / (stages[own] * 1e-3) / 1e9 if len(stages) > own else None
    return {"kernel": names[own], "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
            "frac": ach / hbm if ach else None, "traffic": None, "peak_source": src,
            "algorithmic_bytes_per_launch": B_bytes,
            "stage_ms": {names[i]: round(float(stages[i]), 5) for i in range(len(stages))}}


def roofline_mixed(n, naux, nocc, stages):
    """Dominant kernel of the mixed build and the per-stage bounds.
    GEMM1 (k_gemm1): reads Bhi+Blo, writes Xhi+Xlo -> HBM-bound;
    GEMM2 (k_gemm2): 3 split products over the lower-triangle tiles -> tensor;
    J (k_J_mixed): reads the lower half of Bhi+Blo -> HBM-bound."""
    hbm, bf16, src = peaks()
    ldb = ((n + 63) // 64) * 64
    NP = ((nocc + 15) // 16) * 16
    nt = (n + 127) // 128
    b_bytes = 2 * n * naux * ldb * 2
    x_bytes = 2 * n * naux * NP * 2
    g1_bytes = b_bytes + x_bytes
    g1_flops = 3 * 2 * (n * naux) * NP * ldb
    g2_flops = 3 * 2 * (128 * 128) * (naux * NP) * (nt * (nt + 1) // 2)
    j_bytes = b_bytes * (n + 1) / (2 * n)
    names = ["split C + GEMM1 X=B.C (k_gemm1, tcgen05)", "GEMM2 K=X.X^T (k_gemm2, tcgen05)",
             "J=B.gamma (k_J_mixed)", "finalize (k_finalize_mixed)"]
    per = []
    if len(stages) >= 3:
        per = [{"stage": names[0], "ms": stages[0], "bound": "hbm", "achieved_GBs": g1_bytes / stages[0] / 1e6,
                "frac_hbm": g1_bytes / stages[0] / 1e6 / hbm, "tflops": g1_flops / stages[0] / 1e9},
               {"stage": names[1], "ms": stages[1], "bound": "tensor", "tflops": g2_flops / stages[1] / 1e9,
                "frac_tensor": g2_flops / stages[1] / 1e9 / bf16},
               {"stage": names[2], "ms": stages[2], "bound": "hbm", "achieved_GBs": j_bytes / stages[2] / 1e6,
                "frac_hbm": j_bytes / stages[2] / 1e6 / hbm}]
    dom = int(np.argmax(stages[:3])) if len(stages) >= 3 else 0
    if dom == 1:
        ach = g2_flops / stages[1] / 1e9
        rl = {"kernel": names[1], "bound": "tensor", "achieved": ach, "peak": bf16, "unit": "TFLOP/s",
              "frac": ach / bf16, "algorithmic_flops_per_launch": g2_flops}
    else:
        byts = g1_bytes if dom == 0 else j_bytes
        ach = byts / stages[dom] / 1e6 if stages else None
        rl = {"kernel": names[dom], "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
              "frac": ach / hbm if ach else None, "algorithmic_bytes_per_launch": byts}
    kern = "k_gemm2" if dom == 1 else ("k_gemm1" if dom == 0 else "k_J_mixed")
    rl.update({"traffic": traffic(kern), "traffic_source": "profiles/ncu_traffic.json (ncu dram bytes per launch)",
               "peak_source": src, "stages": per,
               "stage_ms": {names[i]: round(float(stages[i]), 5) for i in range(len(stages))}})
    return rl


# ---------------------------------------------------------------- other workloads
def measure_gradient(local):
    """RHF analytic gradient of (H2O)8/cc-pVDZ (n=192), FP64, after a direct
    SCF from the SOAD guess: Fock::compute_forces (src/rhfgrad.cpp:15-89)."""
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water8()
    eng = IntegralEngine(BasisSet(mol, "cc-pvdz"), device=local)
    t = time.perf_counter()
    r, ex = eng.scf_rhf(mol.nocc, mol.enuc(), guess="soad", want=True, densconverge=1e-8, enconverge=1e-10,
                        maxiter=60)
    scf_s = time.perf_counter() - t
    C = ex["C"][:, :mol.nocc]
    W = C @ np.diag(ex["eps"][:mol.nocc]) @ C.T
    eng.compute_forces(ex["D"], W)
    ts = []
    for _ in range(3):
        t = time.perf_counter()
        g, _ = eng.compute_forces(ex["D"], W)
        ts.append(time.perf_counter() - t)
    eng.close()
    out = {"workload": f"(H2O)8 RHF/cc-pVDZ analytic nuclear gradient, FP64 direct (n=192, {mol.natom} atoms), "
                       "seed 8, SOAD guess",
           "scf_s": scf_s, "scf_iterations": r.iterations, "energy": r.energy,
           "gradient_ms": 1e3 * statistics.median(ts), "timing": "host wall clock around jk_grad_rhf",
           "max_abs_sum_g": float(np.abs(g.sum(axis=0)).max())}
    # the same molecule with VDZ-JKFIT: mixed-precision DF SCF, then the DF gradient
    eng = IntegralEngine(BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit"), device=local)
    eng.df_setup()
    kw = dict(df=True, guess="soad", want=True, densconverge=1e-8, enconverge=1e-10, maxiter=60)
    eng.scf_rhf(mol.nocc, mol.enuc(), df=True, maxiter=2)
    eng.scf_rhf(mol.nocc, mol.enuc(), df=True, prec_mode=1, maxiter=2)   # split B once, untimed
    t = time.perf_counter()
    r64, _ = eng.scf_rhf(mol.nocc, mol.enuc(), **kw)
    s64 = time.perf_counter() - t
    t = time.perf_counter()
    rmx, ex = eng.scf_rhf(mol.nocc, mol.enuc(), prec_mode=1, **kw)
    smx = time.perf_counter() - t
    o = mol.nocc
    eng.compute_forces_df(ex["C"][:, :o], ex["eps"][:o])
    ts = []
    for _ in range(3):
        t = time.perf_counter()
        gdf, _ = eng.compute_forces_df(ex["C"][:, :o], ex["eps"][:o])
        ts.append(time.perf_counter() - t)
    eng.close()
    out["df"] = {"workload": "(H2O)8 RHF/cc-pVDZ + VDZ-JKFIT (naux=928): DF SCF fp64 and mixed, DF gradient at the "
                             "mixed-SCF orbitals",
                 "scf_fp64_s": s64, "scf_mixed_s": smx, "iterations_fp64": r64.iterations,
                 "iterations_mixed": rmx.iterations, "abs_dE_mixed_vs_fp64": abs(rmx.energy - r64.energy),
                 "gradient_ms": 1e3 * statistics.median(ts), "timing": "host wall clock around jk_grad_df",
                 "max_abs_df_minus_direct_gradient": float(np.abs(gdf - g).max())}
    return out


def measure_direct(local):
    """One FP64 integral-direct J/K build of C20H42/6-311G** (n=612) for the
    SOAD-guess density: Fock::formJKdirect (src/fockbuild.cpp:64-164)."""
    import scipy.linalg as sl
    import torch
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.c20h42()
    b = BasisSet(mol, "6-311g**")
    eng = IntegralEngine(b, device=local)
    S, _, _ = eng.one_body()
    _, C = sl.eigh(eng.soad_fock(), S)
    D = 2.0 * C[:, :mol.nocc] @ C[:, :mol.nocc].T
    n = b.nbf
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        dD = torch.from_numpy(np.ascontiguousarray(D)).cuda()
        dJ = torch.empty_like(dD)
        dK = torch.empty_like(dD)
    torch.cuda.synchronize()
    build = lambda: eng.jk_direct_device(dD.data_ptr(), dJ.data_ptr(), dK.data_ptr(), 1e-12,
                                         stream=stream.cuda_stream)
    build()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nb = 3
    ev0.record(stream)
    for _ in range(nb):
        build()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / nb
    q = eng.last_quartets()
    eng.close()
    return {"workload": f"C20H42 RHF/6-311G** FP64 integral-direct J/K build (n={n}), seed 20, SOAD-guess density, "
                        "Schwarz x density screen 1e-12",
            "ms_per_build": ms, "quartets": q, "quartets_per_s": q / (ms * 1e-3)}


def profile_direct(local):
    """Two FP64 direct J/K builds of (H2O)8/cc-pVDZ at the density of one
    diagonalisation of the SOAD Fock matrix (the ncu workload of the direct
    classes)."""
    import scipy.linalg as sl
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water8()
    eng = IntegralEngine(BasisSet(mol, "cc-pvdz"), device=local)
    S, _, _ = eng.one_body()
    _, C = sl.eigh(eng.soad_fock(), S)
    D = 2.0 * C[:, :mol.nocc] @ C[:, :mol.nocc].T
    for _ in range(2):
        t = time.perf_counter()
        eng.jk_direct(D, 1e-12)
        print(json.dumps({"profile_direct": True, "build_s": time.perf_counter() - t,
                          "quartets": eng.last_quartets()}), flush=True)
    eng.close()


# ---------------------------------------------------------------- GPU leg
def run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist
    from molecular2_b200.engine import IntegralEngine
    torch.cuda.set_device(local)
    mol, obs, aux = workload()
    n, naux, nocc = obs.nbf, aux.nbf, mol.nocc
    eng = IntegralEngine(obs, aux, device=local)
    t = time.perf_counter()
    eng.df_setup()
    setup_s = time.perf_counter() - t
    prec_mode = {"fp64": 0, "mixed": 1}[args.precision]
    scf = {}
    if args.profile:
        rng = np.random.default_rng(0)
        C, _ = np.linalg.qr(rng.normal(size=(n, nocc)))
    else:
        # SCF in both modes (not part of the timed builds); the FP64 orbitals feed the builds.
        # One short untimed SCF first, so neither timed run pays the library's first-call setup.
        eng.scf_rhf(nocc, mol.enuc(), df=True, maxiter=2)
        eng.scf_rhf(nocc, mol.enuc(), df=True, prec_mode=1, maxiter=2)
        t = time.perf_counter()
        r64, ex = eng.scf_rhf(nocc, mol.enuc(), df=True, densconverge=1e-6, enconverge=1e-8, want=True)
        s64 = time.perf_counter() - t
        t = time.perf_counter()
        rmx, _ = eng.scf_rhf(nocc, mol.enuc(), df=True, prec_mode=1, densconverge=1e-6, enconverge=1e-8)
        smx = time.perf_counter() - t
        scf = {"fp64": {"energy": r64.energy, "iterations": r64.iterations, "converged": r64.converged,
                        "time_s": s64, "jk_ms_total": r64.jk_ms},
               "mixed": {"energy": rmx.energy, "iterations": rmx.iterations, "converged": rmx.converged,
                         "time_s": smx, "jk_ms_total": rmx.jk_ms, "mixed_builds": rmx.mixed_builds},
               "abs_dE_mixed_vs_fp64": abs(rmx.energy - r64.energy),
               "speedup_time": s64 / smx if smx > 0 else None,
               "convergence": "||dD||_F < 1e-6 and |dE| < 1e-8 Eh, core-Hamiltonian guess"}
        C = np.ascontiguousarray(ex["C"][:, :nocc])
    if world > 1:
        # aux-sharded build: this rank keeps only its slice of the fitted index
        from molecular2_b200.sharding import aux_ranges
        eng.close()
        eng = IntegralEngine(obs, aux, device=local)
        eng.set_df_range(*aux_ranges(naux, world)[rank])
        t = time.perf_counter()
        if eng.df_range[0] < eng.df_range[1]:
            eng.df_setup()
        setup_s = time.perf_counter() - t
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    with torch.cuda.stream(stream):
        dC = torch.from_numpy(np.ascontiguousarray(C.T)).cuda()   # column-major n x nocc
        dJ = torch.empty((n, n), dtype=torch.float64, device="cuda")
        dK = torch.empty((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    def step():
        if world > 1:
            from molecular2_b200.sharding import df_jk_sharded
            df_jk_sharded(eng, dC, nocc, dJ, dK, prec_mode, stream=stream)
        else:
            eng.jk_df_device(dC.data_ptr(), nocc, dJ.data_ptr(), dK.data_ptr(), prec_mode, stream=sh)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = None
    if rank == 0 and not args.profile:
        clocks = Clocks(local, os.path.join(args.clock_dir or tempfile.gettempdir(), f"clocks_rank{rank}.csv"))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
        dist.barrier()
    clk = clocks.stop() if clocks else None
    # N = 1: builds/s of one GPU; N > 1: each step is one build of the whole job
    value = args.steps / (ms / 1e3)
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "ms_per_step": ms / args.steps, "value": value}), flush=True)
        eng.close()
        return

    # per-stage durations of the same builds (events recorded by the library on `stream`)
    eng.set_profiling(True)
    acc = None
    for _ in range(args.steps):
        step()
        s = np.array(eng.stage_ms()) if eng.df_range[0] < eng.df_range[1] else np.zeros(4)
        acc = s if acc is None else acc + s
    eng.set_profiling(False)
    stages = list(acc / args.steps)
    roofline = roofline_mixed(n, naux, nocc, stages) if prec_mode == 1 else roofline_fp64(n, naux, nocc, stages)
    if prec_mode == 1:
        J64 = torch.empty_like(dJ)
        K64 = torch.empty_like(dK)
        if world > 1:
            from molecular2_b200.sharding import df_jk_sharded
            df_jk_sharded(eng, dC, nocc, J64, K64, 0, stream=stream)
        else:
            eng.jk_df_device(dC.data_ptr(), nocc, J64.data_ptr(), K64.data_ptr(), 0, stream=sh)
        step()
        torch.cuda.synchronize()
        roofline["max_rel_err_vs_fp64"] = {
            "J": float((dJ - J64).abs().max() / J64.abs().max()),
            "K": float((dK - K64).abs().max() / K64.abs().max())}

    # e2e: host C in (pinned), host J/K out, through the public host-pointer call
    hC = torch.from_numpy(np.asfortranarray(C)).pin_memory()
    hJ = torch.empty((n, n), dtype=torch.float64).pin_memory()
    hK = torch.empty((n, n), dtype=torch.float64).pin_memory()

    def e2e_step():
        if world > 1:   # host C in, sharded build + all-reduce, host J/K out
            with torch.cuda.stream(stream):
                dC.copy_(hC.t(), non_blocking=True)
            step()
            with torch.cuda.stream(stream):
                hJ.copy_(dJ, non_blocking=True)
                hK.copy_(dK, non_blocking=True)
            stream.synchronize()
            return
        rc = eng.lib.jk_df(eng.h, ctypes.c_void_p(hC.data_ptr()), nocc, prec_mode, ctypes.c_void_p(hJ.data_ptr()),
                           ctypes.c_void_p(hK.data_ptr()))
        if rc:
            eng._check(rc)

    for _ in range(3):
        e2e_step()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = time.perf_counter() - t
    if world > 1:
        tt = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e = {"value": args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": n * nocc * 8,
           "d2h_bytes_per_step": 2 * n * n * 8, "timing": "host wall clock around synchronous calls"}

    other = {}
    if rank == 0 and not args.no_extras:
        other["gradient"] = measure_gradient(local)
        other["direct_jk"] = measure_direct(local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sample, _ = cpu_sample(1)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample}

    if rank == 0:
        launches = 5 if prec_mode == 1 else 3
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak" if world == 1 else "strong", "vs_baseline": None,
                "dtype": "f64" if prec_mode == 0 else "bf16x3->f32",
                "data": "synthetic (seeded geometry; basis data from molecular2's library)",
                "config": config(mol, obs, aux, args.precision, world), "e2e": e2e, "roofline": roofline,
                "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches * args.steps, "scf": scf,
                "df_setup_s": setup_s, **other}
        print(json.dumps(line), flush=True)
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--clock-dir", default=None, help="where the nvidia-smi clock samples go (default: a temp dir)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the gradient and direct J/K measurements")
    ap.add_argument("--profile-direct", action="store_true",
                    help="only two FP64 direct J/K builds of (H2O)8/cc-pVDZ at the SOAD-guess density (for ncu)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.profile_direct:
        profile_direct(local)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
