#!/usr/bin/env python
"""Benchmark of the J/K engine on (H2O)64 / aug-cc-pVDZ + AVDZ-JKFIT.

Workload: 64 rigid water monomers placed by seeded
random rotation and translation in a 14 A cube (O-O >= 2.7 A), RHF with the
aug-cc-pVDZ orbital basis (n = 2624) and the AVDZ-JKFIT fitting basis
(naux = 9600), nocc = 320: the density-fitted J/K build molecular2 runs every
SCF iteration (Fock::formJKdf, src/fockbuild.cpp:171-174, 585-660).  The
fitted tensor is kept in the tiled split-BF16 layout (145 GB); the FP64 path
recomputes the three-index integrals per build.

A step is one mixed-precision (split-BF16 tcgen05) J/K build for the
converged occupied orbitals; `value` is builds/s with everything resident in
HBM (inputs are larger than L2: 145 GB of B per build), `e2e` the same through
the host-pointer entry point jk_df (C uploaded, J and K downloaded every step).
Reported beside it, each timed once:
  * "scf": the FP64 SCF and the mixed SCF (split-BF16 builds, then FP64
    anchor builds with split-BF16 builds of the density change since the
    anchor) from the SOAD guess, both with canonical orthogonalisation
    (overlap eigenvalues below 1e-4 dropped), their wall times, iterations,
    J/K time and |dE|;
  * "jk_builds_per_s": mixed (the timed steps) and FP64 (from the FP64 SCF's
    builds), and the mixed build's J/K error against an FP64 build;
  * "gradient": one DF nuclear gradient at the mixed-SCF orbitals;
  * "df_setup_s": metric factorisation and tiled fitted tensor;
  * "extras": the smaller workloads ((H2O)16 DF builds, C20H42 direct build,
    (H2O)8 FP64 and DF gradients); --no-extras skips them.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload water64|water16] [--profile]

--impl reference times molecular2's own algorithm on the host cores: the
oracle's restatement of compute_2body_fock_df's naive loops (molecular2
itself needs libint2/Eigen and cannot be built here; its packed FP64 B for
this system would be 264 GB), on a bounded sample of the fitting functions,
extrapolated linearly in naux.
--profile runs only the set-up and the timed builds (for ncu launch lists);
--profile-direct water8|c20h42 runs only two direct J/K builds;
--precision fp64 times FP64 builds instead of mixed ones; --workload water16aug
is the small case of the tiled kernels used for ncu captures.
With --gpus N > 1 every rank runs its own replica of the workload (the
headline measurement is single-GPU).
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

METRIC = "SCF time & J/K builds/s, mixed vs FP64 GPU at |dE|<=1e-6 Eh; gradient time"
UNIT = "builds/s"
WORKLOADS = {
    "water64": dict(label="(H2O)64 RHF/aug-cc-pVDZ + AVDZ-JKFIT", k=64, box=14.0, seed=64,
                    obs="aug-cc-pvdz", aux="avdz-jkfit", storage="tiled"),
    "water16": dict(label="(H2O)16 RHF/cc-pVDZ + VDZ-JKFIT", k=16, box=9.0, seed=16,
                    obs="cc-pvdz", aux="vdz-jkfit", storage="unpacked"),
    # the small case of the tiled kernels for ncu captures (3.3 GB of split B)
    "water16aug": dict(label="(H2O)16 RHF/aug-cc-pVDZ + AVDZ-JKFIT", k=16, box=9.0, seed=16,
                       obs="aug-cc-pvdz", aux="avdz-jkfit", storage="tiled"),
}
_CACHE = {}


def workload(name):
    if name not in _CACHE:
        from molecular2_b200 import geometry
        from molecular2_b200.basis import BasisSet
        w = WORKLOADS[name]
        mol = geometry.water_cluster(w["k"], w["box"], w["seed"])
        _CACHE[name] = (mol, BasisSet(mol, w["obs"]), BasisSet(mol, w["aux"]))
    return _CACHE[name]


def config(name, mol, obs, aux, world=1, stored_bytes=None):
    w = WORKLOADS[name]
    gb = obs.nbf * obs.nbf * aux.nbf
    return {"workload": f"{w['label']} DF-JK build (n={obs.nbf}, naux={aux.nbf}, nocc={mol.nocc}), "
                        f"{w['k']} waters in a {w['box']:.0f} A cube, seed {w['seed']}",
            "precision": "mixed split-BF16 (hi*hi + hi*lo + lo*hi, FP32 accumulate) build; FP64 SCF and "
                         "corrections",
            "storage": w["storage"],
            "l2": "inputs larger than L2 (fitted tensor %.1f GB split BF16 per build)"
                  % ((stored_bytes if stored_bytes else (gb / 2 if w["storage"] == "tiled" else gb) * 4) / 1e9),
            "parallelism": "single GPU" if world == 1 else f"{world} independent replicas, one per GPU"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


def traffic(kernel):
    """DRAM bytes per launch of `kernel` at the benchmark size, from the committed ncu summary (None if absent)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    k = json.load(open(p)).get("kernels", {}).get(kernel)
    return k.get("dram_bytes_per_launch_full_size") if k else None


# ---------------------------------------------------------------- CPU leg
def cpu_sample(name, nthreads, target_s=12.0):
    """Time the naive per-iteration loops of compute_2body_fock_df (the
    oracle's restatement) on a block of fitting functions of workload `name`,
    doubling the block until one run takes target_s / 3; returns (builds/s
    extrapolated to all fitting functions, sample text, seconds spent)."""
    import oracle
    mol, obs, aux = workload(name)
    n, naux, nocc = obs.nbf, aux.nbf, mol.nocc
    rng = np.random.default_rng(0)
    npair = n * (n + 1) // 2
    C = np.asfortranarray(rng.normal(size=(n, nocc)))
    nk, prev, total = 1, None, 0.0
    while True:
        B = np.asfortranarray(rng.normal(size=(npair, nk)))
        t = time.perf_counter()
        oracle.df_jk(B, C, (0, nk), nthreads=nthreads)
        t = time.perf_counter() - t
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
              f"(synthetic B values, n={n}, nocc={nocc}), {nthreads} thread(s), last run {t:.2f} s of "
              f"{total:.1f} s sampled, extrapolated linearly to {naux}")
    return 1.0 / t_full, sample, total


def run_reference(args, rank, world):
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    per_step = min(6.0, max(0.5, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_sample(args.workload, nthreads, target_s=per_step)
    vals = []
    t0 = time.perf_counter()
    sample = ""
    for _ in range(args.steps):
        v, sample, _ = cpu_sample(args.workload, nthreads, target_s=per_step)
        vals.append(v)
    wall = time.perf_counter() - t0
    v = statistics.median(vals)
    mol, obs, aux = workload(args.workload)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(args.workload, mol, obs, aux),
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


# ---------------------------------------------------------------- roofline
def roofline_tiled(n, naux, nocc, st, stored_bytes):
    """Tiled mixed build.  st = [GEMM1 total ms, GEMM2 total ms, J ms,
    finalize ms, blocks].  Algorithmic work (B counted unpacked): GEMM1
    X = B C is 2 n^2 o naux flops, GEMM2 K = X X^T n(n+1) o naux flops; J
    reads the stored tiles (split BF16, stored_bytes) once."""
    hbm, bf16, src = peaks()
    nt = (n + 127) // 128
    g1_flops = 2.0 * n * n * nocc * naux
    g2_flops = 1.0 * n * (n + 1) * nocc * naux
    j_bytes = float(stored_bytes)
    nhalf = (nocc + 159) // 160
    g1_exec = 3 * 2.0 * (nt * 128) ** 2 * (nhalf * 160) * naux      # split products over padded tiles
    g1, g2, jm, fm, blocks = st[:5]
    blocks = max(1, int(round(blocks)))
    stages = [{"kernel": "k_gemm1_sym (X = B C, tcgen05, symmetric tiles)", "ms_total": g1, "launches": blocks,
               "ms_per_launch": g1 / blocks, "bound": "tensor", "algorithmic_tflops": g1_flops / g1 / 1e9,
               "frac_of_bf16_peak": g1_flops / g1 / 1e9 / bf16,
               "executed_tflops": g1_exec / g1 / 1e9, "frac_executed": g1_exec / g1 / 1e9 / bf16},
              {"kernel": "k_gemm2 (K = X X^T, tcgen05)", "ms_total": g2, "launches": blocks, "bound": "tensor",
               "algorithmic_tflops": g2_flops / g2 / 1e9, "frac_of_bf16_peak": g2_flops / g2 / 1e9 / bf16},
              {"kernel": "k_J_tiles (J = sum_K gamma_K B_K)", "ms": jm, "bound": "hbm",
               "achieved_GBs": j_bytes / jm / 1e6, "frac_of_hbm": j_bytes / jm / 1e6 / hbm},
              {"kernel": "k_finalize_mixed", "ms": fm}]
    ach = g1_flops / g1 / 1e9
    return {"kernel": "k_gemm1_sym", "bound": "tensor", "achieved": ach, "peak": bf16, "unit": "TFLOP/s",
            "frac": ach / bf16, "traffic": traffic("k_gemm1_sym"),
            "algorithmic_flops_per_launch": g1_flops / blocks,
            "work_model": "2 n^2 nocc w flops per launch of w fitted functions (B counted unpacked); the three "
                          "split-BF16 products and tile padding are overhead (executed_tflops)",
            "peak_source": src, "timing": "CUDA events on the launch stream around every launch, averaged "
                                          "over profiled steps", "stages": stages}


def roofline_unpacked(n, naux, nocc, st):
    """Unpacked mixed build: st = [GEMM1, GEMM2, J, finalize] ms."""
    hbm, bf16, src = peaks()
    ldb = ((n + 63) // 64) * 64
    NP = ((nocc + 15) // 16) * 16
    g1_bytes = 2 * n * naux * ldb * 2 + 2 * n * naux * NP * 2
    ach = g1_bytes / st[0] / 1e6
    return {"kernel": "k_gemm1", "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
            "traffic": traffic("k_gemm1"), "peak_source": src, "algorithmic_bytes_per_launch": g1_bytes,
            "stages_ms": {"gemm1": st[0], "gemm2": st[1], "J": st[2], "finalize": st[3]}}


# ---------------------------------------------------------------- other workloads
def measure_gradient(local):
    """RHF analytic gradient of (H2O)8/cc-pVDZ (n=192): FP64 direct
    (Fock::compute_forces, src/rhfgrad.cpp:15-89) and DF."""
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
    t = time.perf_counter()
    g, _ = eng.compute_forces(ex["D"], W)
    gms = 1e3 * (time.perf_counter() - t)
    eng.close()
    out = {"workload": f"(H2O)8 RHF/cc-pVDZ analytic nuclear gradient, FP64 direct (n=192, {mol.natom} atoms), "
                       "seed 8, SOAD guess",
           "scf_s": scf_s, "scf_iterations": r.iterations, "energy": r.energy, "gradient_ms": gms,
           "timing": "host wall clock around jk_grad_rhf", "max_abs_sum_g": float(np.abs(g.sum(axis=0)).max())}
    eng = IntegralEngine(BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit"), device=local)
    import torch
    torch.cuda.synchronize()
    t = time.perf_counter()
    eng.df_setup()
    torch.cuda.synchronize()
    out["df_setup_s"] = time.perf_counter() - t
    _, ex = eng.scf_rhf(mol.nocc, mol.enuc(), df=True, guess="soad", want=True, densconverge=1e-8,
                        enconverge=1e-10, maxiter=60)
    o = mol.nocc
    eng.compute_forces_df(ex["C"][:, :o], ex["eps"][:o])
    t = time.perf_counter()
    gdf, _ = eng.compute_forces_df(ex["C"][:, :o], ex["eps"][:o])
    out["df"] = {"gradient_ms": 1e3 * (time.perf_counter() - t), "timing": "host wall clock around jk_grad_df",
                 "max_abs_df_minus_direct_gradient": float(np.abs(gdf - g).max())}
    eng.close()
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
    work = eng.last_class_work()
    eng.close()
    # FP64 work of the build from the frozen per-class table (flops per bra
    # primitive pair, per primitive quartet, per quartet of digestion)
    table = json.load(open(os.path.join(ROOT, "molecular2_b200", "data", "flop_table.json")))["table"]
    flops = 0.0
    for A in range(6):
        for B in range(A + 1):
            t = table[f"{A},{B}"]
            nq, wb, wq = (float(x) for x in work[A, B])
            flops += t["bra"] * wb + t["quartet"] * wq + t["digest"] * nq
    fp64_peak = 40.0   # TFLOP/s, nominal B200 FP64 (no measured FP64 figure is available)
    roof = {"kernel": "k_jk_direct (all classes)", "bound": "fp64", "flops_per_build": flops,
            "achieved_tflops": flops / (ms * 1e-3) / 1e12, "peak_tflops": fp64_peak, "peak_source": "nominal",
            "frac": flops / (ms * 1e-3) / 1e12 / fp64_peak,
            "work_model": "molecular2_b200/data/flop_table.json x jk_last_class_work counts"}
    return {"workload": f"C20H42 RHF/6-311G** FP64 integral-direct J/K build (n={n}), seed 20, SOAD-guess density, "
                        "Schwarz x density screen 1e-12",
            "ms_per_build": ms, "quartets": q, "quartets_per_s": q / (ms * 1e-3), "roofline": roof}


def measure_scf_h2o(local):
    """H2O/cc-pVDZ direct FP64 SCF from the SOAD guess (the smallest
    configuration) on the GPU."""
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water()
    eng = IntegralEngine(BasisSet(mol, "cc-pvdz"), device=local)
    kw = dict(guess="soad", densconverge=1e-8, enconverge=1e-10, maxiter=60)
    eng.scf_rhf(mol.nocc, mol.enuc(), **kw)
    t = time.perf_counter()
    r, ex = eng.scf_rhf(mol.nocc, mol.enuc(), want=True, **kw)
    s = time.perf_counter() - t
    C = ex["C"][:, :mol.nocc]
    W = C @ np.diag(ex["eps"][:mol.nocc]) @ C.T
    eng.compute_forces(ex["D"], W)
    t = time.perf_counter()
    eng.compute_forces(ex["D"], W)
    gs = time.perf_counter() - t
    eng.close()
    return {"workload": "H2O RHF/cc-pVDZ direct FP64 SCF, SOAD guess, and its analytic gradient", "scf_s": s,
            "iterations": r.iterations, "energy": r.energy, "gradient_s": gs}


def cpu_baselines(extra):
    """The oracle's restatement of the reference's loops on one host core
    beside the GPU figures of `extra` (each bounded to ~10-20 s): direct J/K
    (C20H42, every 41st shell row, scaled by the quartet count), DF set-up
    ((H2O)8 three- and two-index integrals and B = (mn|P) L^-T, whole), SCF
    (H2O, whole) and the two-electron gradient ((H2O)8, every 8th shell row,
    scaled by 8)."""
    import scipy.linalg as sl
    import oracle
    from oracle import scf as oscf
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    out = {"cores": 1, "kind": "port"}
    # direct J/K, C20H42/6-311G**, the GPU measurement's SOAD-guess density
    mol = geometry.c20h42()
    b = BasisSet(mol, "6-311g**")
    rhf = oscf.RHF(b, minbasis=BasisSet(mol, "sto-3g"), nthreads=1)
    _, C = sl.eigh(rhf.soad_fock(), rhf.S)
    D = 2.0 * C[:, :mol.nocc] @ C[:, :mol.nocc].T
    Q = oracle.schwarz(b)
    t, q = time.perf_counter(), 0
    for s1 in range(0, Q.shape[0], 41):
        q += oracle.jk_direct_rows(b, D, Q, 1e-12, s1, s1 + 1)[2]
    t = time.perf_counter() - t
    d = extra.get("direct_jk_c20h42", {})
    q_all = d.get("quartets") or q * 41
    cpu_s = t * q_all / max(1, q)
    out["direct_jk_c20h42"] = {"cpu_s_per_build": cpu_s, "gpu_s_per_build": d.get("ms_per_build", float("nan")) / 1e3,
                               "sample": f"every 41st shell row: {q} of {q_all} quartets in {t:.1f} s, scaled"}
    # DF set-up, (H2O)8 cc-pVDZ + VDZ-JKFIT
    mol = geometry.water8()
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    t = time.perf_counter()
    oracle.df_B(oracle.eri3(obs, aux), oracle.eri2(aux), nthreads=1)
    g = extra.get("gradient_water8", {})
    out["df_setup_water8"] = {"cpu_s": time.perf_counter() - t, "gpu_s": g.get("df_setup_s"),
                              "sample": "whole: (P|mn), (P|Q), Cholesky and B"}
    # SCF, H2O cc-pVDZ direct
    h2o = geometry.water()
    t = time.perf_counter()
    oscf.RHF(BasisSet(h2o, "cc-pvdz"), guess="soad", minbasis=BasisSet(h2o, "sto-3g"), densconverge=1e-8,
             enconverge=1e-10, maxiter=60, nthreads=1).run()
    sc = extra.get("scf_h2o", {})
    out["scf_h2o"] = {"cpu_s": time.perf_counter() - t, "gpu_s": sc.get("scf_s"), "sample": "whole"}
    # two-electron gradient of H2O cc-pVDZ (the (H2O)8 one takes ~25 min on one core)
    bh = BasisSet(h2o, "cc-pvdz")
    rng = np.random.default_rng(8)
    Cr = np.linalg.qr(rng.normal(size=(bh.nbf, h2o.nocc)))[0]
    t = time.perf_counter()
    oracle.grad2e(bh, 2.0 * Cr @ Cr.T, oracle.schwarz(bh), 1e-12, nthreads=1)
    out["gradient_2e_h2o"] = {"cpu_s": time.perf_counter() - t, "gpu_s": sc.get("gradient_s"),
                              "sample": "whole two-electron term (random orthonormal orbitals); the GPU figure "
                                        "is the whole gradient at the SCF density"}
    return out


def measure_water16(local):
    """(H2O)16 / cc-pVDZ + VDZ-JKFIT (unpacked storage): mixed and FP64 DF
    build times and SCF times."""
    import torch
    from molecular2_b200.engine import IntegralEngine
    mol, obs, aux = workload("water16")
    n, o = obs.nbf, mol.nocc
    eng = IntegralEngine(obs, aux, device=local)
    eng.set_df_storage("unpacked")
    eng.df_setup()
    kw = dict(df=True, densconverge=1e-6, enconverge=1e-8, guess="soad")
    eng.scf_rhf(o, mol.enuc(), df=True, maxiter=2)
    eng.scf_rhf(o, mol.enuc(), df=True, prec_mode=2, maxiter=2)
    t = time.perf_counter()
    r64, ex = eng.scf_rhf(o, mol.enuc(), want=True, **kw)
    s64 = time.perf_counter() - t
    t = time.perf_counter()
    rmx, _ = eng.scf_rhf(o, mol.enuc(), prec_mode=2, **kw)
    smx = time.perf_counter() - t
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        dC = torch.from_numpy(np.ascontiguousarray(ex["C"][:, :o].T)).cuda()
        dJ = torch.empty((n, n), dtype=torch.float64, device="cuda")
        dK = torch.empty_like(dJ)
    torch.cuda.synchronize()
    out = {"workload": f"(H2O)16 RHF/cc-pVDZ + VDZ-JKFIT (n={n}, naux={aux.nbf}), unpacked storage, SOAD guess",
           "scf_fp64_s": s64, "scf_mixed_s": smx, "iterations_fp64": r64.iterations,
           "iterations_mixed": rmx.iterations, "fp64_anchor_builds": rmx.jk_builds - rmx.mixed_builds,
           "abs_dE_mixed_vs_fp64": abs(rmx.energy - r64.energy)}
    for mode, name in ((0, "fp64"), (1, "mixed")):
        for _ in range(3):
            eng.jk_df_device(dC.data_ptr(), o, dJ.data_ptr(), dK.data_ptr(), mode, stream=stream.cuda_stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(20):
            eng.jk_df_device(dC.data_ptr(), o, dJ.data_ptr(), dK.data_ptr(), mode, stream=stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        out[f"{name}_ms_per_build"] = ev0.elapsed_time(ev1) / 20
    eng.close()
    return out


# ---------------------------------------------------------------- GPU leg
def run_ours(args, rank, world, local):
    import torch
    from molecular2_b200.engine import IntegralEngine
    torch.cuda.set_device(local)
    name = args.workload
    mol, obs, aux = workload(name)
    n, naux, nocc = obs.nbf, aux.nbf, mol.nocc
    eng = IntegralEngine(obs, aux, device=local)
    eng.set_df_storage(WORKLOADS[name]["storage"])
    scf, extra, fp64_build_ms = {}, {}, None
    conv = dict(densconverge=1e-5, enconverge=1e-8, maxiter=60, lindep=1e-4)
    if args.profile:
        rng = np.random.default_rng(0)
        C, _ = np.linalg.qr(rng.normal(size=(n, nocc)))
        t = time.perf_counter()
        eng.df_setup()
        setup_s = time.perf_counter() - t
    else:
        t = time.perf_counter()
        Fs = eng.soad_fock(1e-12)
        soad_s = time.perf_counter() - t
        # FP64 SCF first: on tiled storage it needs only the metric (the
        # three-index integrals are recomputed per build)
        t = time.perf_counter()
        r64, ex = eng.scf_rhf(nocc, mol.enuc(), df=True, prec_mode=0, guess_fock=Fs, want=True, **conv)
        s64 = time.perf_counter() - t
        fp64_build_ms = r64.jk_ms / max(1, r64.jk_builds)
        t = time.perf_counter()
        eng.df_setup()
        setup_s = time.perf_counter() - t
        t = time.perf_counter()
        rmx, exm = eng.scf_rhf(nocc, mol.enuc(), df=True, prec_mode=2, guess_fock=Fs, want=True, **conv)
        smx = time.perf_counter() - t
        scf = {"fp64": {"energy": r64.energy, "iterations": r64.iterations, "converged": r64.converged,
                        "time_s": s64, "jk_ms_total": r64.jk_ms, "jk_builds": r64.jk_builds,
                        "diag_ms_total": r64.diag_ms},
               "mixed": {"energy": rmx.energy, "iterations": rmx.iterations, "converged": rmx.converged,
                         "time_s": smx, "jk_ms_total": rmx.jk_ms, "jk_builds": rmx.jk_builds,
                         "mixed_builds": rmx.mixed_builds, "fp64_builds": rmx.jk_builds - rmx.mixed_builds,
                         "diag_ms_total": rmx.diag_ms},
               "abs_dE_mixed_vs_fp64": abs(rmx.energy - r64.energy),
               "speedup_time": s64 / smx if smx > 0 else None,
               "speedup_time_with_fitted_tensor_setup": s64 / (smx + setup_s) if smx > 0 else None,
               "guess": f"SOAD ({soad_s:.1f} s, not in either SCF time)",
               "convergence": "||dD||_F < 1e-5 and |dE| < 1e-8 Eh; canonical orthogonalisation, overlap "
                              f"eigenvalues below 1e-4 dropped ({r64.lindep_dropped} of {n})",
               "mixed_schedule": "split-BF16 builds while ||dD|| falls, then FP64 anchor builds G64(D_ref) with "
                                 "split-BF16 builds of the rank-2nocc change D - D_ref in between; a new anchor "
                                 "where ||dD|| stalls at the noise of those builds; converged only with "
                                 "||D - D_ref|| < 1e-3",
               "fitted_tensor_setup_s": setup_s}
        C = np.ascontiguousarray(ex["C"][:, :nocc])
        Cm, epsm = exm["C"][:, :nocc], exm["eps"][:nocc]
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    with torch.cuda.stream(stream):
        dC = torch.from_numpy(np.ascontiguousarray(C.T)).cuda()   # column-major n x nocc
        dJ = torch.empty((n, n), dtype=torch.float64, device="cuda")
        dK = torch.empty((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    mode = 0 if args.precision == "fp64" else 1

    def step():
        eng.jk_df_device(dC.data_ptr(), nocc, dJ.data_ptr(), dK.data_ptr(), mode, stream=sh)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
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
    clk = clocks.stop() if clocks else None
    if world > 1:   # independent replicas: the slowest rank's time, all ranks' builds
        import torch.distributed as dist
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * args.steps / (ms / 1e3)
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "ms_per_step": ms / args.steps, "value": value,
                              "df_setup_s": setup_s}), flush=True)
        eng.close()
        return

    # per-kernel durations of the same builds (events recorded by the library on `stream`)
    eng.set_profiling(True)
    acc = None
    nprof = max(3, min(args.steps, 5))
    for _ in range(nprof):
        step()
        s = np.array(eng.stage_ms(8), dtype=float)
        acc = s if acc is None else acc + s
    eng.set_profiling(False)
    st = list(acc / nprof)
    tiled = eng.df_storage == "tiled"
    stored = eng.df_tensor_bytes if tiled else None
    roofline = (roofline_tiled(n, naux, nocc, st, stored) if tiled
                else roofline_unpacked(n, naux, nocc, st))
    # mixed J/K error against an FP64 build at the same orbitals
    Jm, Km = dJ.clone(), dK.clone()
    t = time.perf_counter()
    eng.jk_df_device(dC.data_ptr(), nocc, dJ.data_ptr(), dK.data_ptr(), 0, stream=sh)
    torch.cuda.synchronize()
    fp64_with_b_s = time.perf_counter() - t
    err = {"J": float((Jm - dJ).abs().max() / dJ.abs().max()), "K": float((Km - dK).abs().max() / dK.abs().max()),
           "definition": "max |mixed - FP64| over the largest |FP64| element, at the FP64-SCF orbitals"}
    jk_rates = {"mixed": value / world, "fp64": 1e3 / fp64_build_ms if fp64_build_ms else None,
                "fp64_source": "mean J/K build time of the FP64 SCF (metric-only storage, one integral pass per "
                               "occupied slice plus the J pass)",
                "fp64_build_with_tiled_B_resident_s": fp64_with_b_s, "mixed_vs_fp64_rel_err": err}

    # e2e: host C in (pinned), host J/K out, through the public host-pointer call
    hC = torch.from_numpy(np.asfortranarray(C)).pin_memory()
    hJ = torch.empty((n, n), dtype=torch.float64).pin_memory()
    hK = torch.empty((n, n), dtype=torch.float64).pin_memory()

    def e2e_step():
        rc = eng.lib.jk_df(eng.h, ctypes.c_void_p(hC.data_ptr()), nocc, 1, ctypes.c_void_p(hJ.data_ptr()),
                           ctypes.c_void_p(hK.data_ptr()))
        if rc:
            eng._check(rc)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = time.perf_counter() - t
    e2e = {"value": world * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": n * nocc * 8,
           "d2h_bytes_per_step": 2 * n * n * 8, "timing": "host wall clock around synchronous jk_df calls"}
    eng.close()

    # one DF nuclear gradient at the mixed-SCF orbitals (fresh engine: metric only)
    gradient = None
    if rank == 0:
        eng2 = IntegralEngine(obs, aux, device=local)
        eng2.set_df_storage(WORKLOADS[name]["storage"])
        t = time.perf_counter()
        g, g2 = eng2.compute_forces_df(Cm, epsm)
        gs = time.perf_counter() - t
        eng2.close()
        gradient = {"time_s": gs, "timing": "host wall clock around jk_grad_df (includes the metric "
                                            "factorisation of the fresh engine)",
                    "max_abs_sum_g": float(np.abs(g.sum(axis=0)).max()),
                    "max_abs_g": float(np.abs(g).max()), "kind": "DF (AVDZ-JKFIT) RHF nuclear gradient, FP64"}
        if not args.no_extras:
            extra["water16"] = measure_water16(local)
            extra["gradient_water8"] = measure_gradient(local)
            extra["direct_jk_c20h42"] = measure_direct(local)
            extra["scf_h2o"] = measure_scf_h2o(local)
            if rank == 0 and world == 1 and not args.no_cpu_baseline:
                extra["cpu_baselines"] = cpu_baselines(extra)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sample, _ = cpu_sample(name, 1)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample}

    if rank == 0:
        blocks = int(round(st[4])) if tiled else 1
        launches = 2 * blocks + 3   # GEMM1 and GEMM2 per block, split C, J, finalize
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3->f32",
                "data": "synthetic (seeded geometry; basis data from molecular2's library)",
                "config": config(name, mol, obs, aux, world, stored), "e2e": e2e, "roofline": roofline,
                "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches * args.steps, "scf": scf,
                "jk_builds_per_s": jk_rates, "gradient": gradient, "df_setup_s": setup_s, "extras": extra}
        print(json.dumps(line), flush=True)


def profile_direct(local, name):
    """Driver for ncu launch lists of the direct J/K kernels: engine, SOAD
    Fock, one diagonalisation, two jk_direct builds of (H2O)8/cc-pVDZ
    ("water8") or C20H42/6-311G** ("c20h42")."""
    import scipy.linalg as sl
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    from molecular2_b200.engine import IntegralEngine
    mol, basis = (geometry.water8(), "cc-pvdz") if name == "water8" else (geometry.c20h42(), "6-311g**")
    eng = IntegralEngine(BasisSet(mol, basis), device=local)
    S, _, _ = eng.one_body()
    _, C = sl.eigh(eng.soad_fock(), S)
    D = 2.0 * C[:, :mol.nocc] @ C[:, :mol.nocc].T
    for _ in range(2):
        t = time.perf_counter()
        eng.jk_direct(D, 1e-12)
        print(json.dumps({"profile_direct": name, "ms": 1e3 * (time.perf_counter() - t),
                          "quartets": eng.last_quartets()}), flush=True)
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="water64", choices=sorted(WORKLOADS))
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="precision of the timed builds (the SCF comparison runs both)")
    ap.add_argument("--clock-dir", default=None, help="where the nvidia-smi clock samples go (default: a temp dir)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the smaller workloads")
    ap.add_argument("--profile-direct", default=None, choices=["water8", "c20h42"],
                    help="only run two direct J/K builds (driver for ncu launch lists)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.profile_direct:
        profile_direct(local, args.profile_direct)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
