#!/usr/bin/env python3
"""Benchmark of the integral-direct Cholesky ERI + AO->MO path on B200.

One step = one complete job on a seeded synthetic molecule: the two-step
Cholesky decomposition of (pq|rs) (diagonal, pivot search, pivot block,
Inv_L) and the AO->MO transformation of the Cholesky vectors into the
occupied x virtual block, through the library's C ABI (libgci.so).

``value`` is the algorithmic GFLOP/s of the job (flops.py: GEMM formulas +
per-class ERI arithmetic) with the inputs resident on the device, timed with
CUDA events on the library's stream; ``e2e`` is the same job through the
host API (TAOBasis + MO coefficients in pinned host memory, Rkab read back).
``--impl reference`` times the CPU restatement of the reference algorithm
(oracle/, all host threads) on a bounded sample of the same workload.

Multi-GPU: the path runs as independent replicas (one job per rank); value is
the flops of all ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Cholesky-ERI wall time & GFLOP/s, mixed vs FP64 on B200 at ≤1e-8 max ERI err"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--buffer-mb", type=int, default=16384)
    ap.add_argument("--tune-pairs", type=int, default=40, help="shell pairs per class sampled by the ERI autotuner")
    ap.add_argument("--eri-kernels", default="hermite", choices=["hermite", "class"],
                    help="product stages on the Hermite-matrix tensor-core kernels or the per-class kernels")
    ap.add_argument("--dump-work", nargs="?", const=str(ROOT / "oracle" / "job_work.json"), default=None,
                    metavar="PATH", help="record the job's per-class work counts (reference-arm input) in PATH, "
                                         "by default oracle/job_work.json")
    ap.add_argument("--hm-profile", action="store_true",
                    help="diagnostic: time every Hermite-matrix class launch (serialised) and print the table")
    ap.add_argument("--streams", type=int, default=32, help="c3: workers (CUDA streams) of gci_rkpq_batch")
    ap.add_argument("--dense", action="store_true",
                    help="time the library's FP64 dense kernels (gci_dgemm, gci_cholesky_inverse, gci_trsm_rlt) "
                         "and the split-precision GEMM against torch/cuBLAS/cuSOLVER at fixed shapes")
    ap.add_argument("--decode-storage", action="store_true",
                    help="decode diagonal-shell-pair pivots in storage order (GCI_FLAG_PIVOT_DECODE_STORAGE)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(seconds: float, world: int, device) -> float:
    """The slowest rank's time: every rank takes part in the same all-reduce
    (MAX) whenever more than one rank runs."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(work_per_step: float, steps: int, world: int, t_max: float) -> float:
    """Whole-job rate of independent replicas: the work of all ranks over the slowest rank's time."""
    return work_per_step * steps * world / t_max


def measured_fp64_peak(torch):
    """FP64 reference rate for the roofline (MEASURED_PEAKS.json has no FP64
    figure): cuBLAS DGEMM 8192^3, best of 5, CUDA events."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


WORK_FIXTURE = ROOT / "oracle" / "job_work.json"


def job_work(config: str):
    """Per-class work of the library's job on `config` (gci_stats layout), recorded by
    ``bench.py --config <cfg> --dump-work`` on a B200 and committed in oracle/job_work.json:
    the counts the oracle's time is extrapolated over.  None if not recorded."""
    if not WORK_FIXTURE.exists():
        return None
    d = json.loads(WORK_FIXTURE.read_text())
    w = d.get(config)
    return None if w is None else np.asarray(w["stats"], dtype=np.float64)


def oracle_job_seconds(config: str, work, budget_s: float, rates=None, nthreads: int = 0, seed: int = 0):
    """Time of the complete `config` job on the oracle (FP64 C restatement of the
    reference algorithm, scheme 0 = W-matrix + HRR, all host threads), extrapolated
    from a bounded sample: every ERI class of the job is timed on a seeded sample of
    its shell quartets from the same molecule, and the job's count of primitive
    quartets of that class (all of them, as the reference evaluates) is multiplied by
    the measured seconds per primitive quartet; the GEMM work of the job is timed as
    numpy DGEMM (OpenBLAS) flops.  `rates` (s per primitive quartet per class, from a
    previous call) sizes the sample to about `budget_s` seconds.
    Returns (seconds, rates, sample description)."""
    from gammcor_integrals_b200 import flops, molecules
    from oracle import oracle as O
    m = molecules.config(config)
    ob = O.make_basis(m.atoms, m.shells)
    O.set_eri_scheme(0)
    Ls = np.array([sh[1] for sh in m.shells])
    nprim = np.array([len(sh[2]) for sh in m.shells])
    byl = {l: np.flatnonzero(Ls == l) for l in range(4)}
    types = flops.pair_types(3)
    ntypes, nc = flops.LAYOUTS["lib"]
    rng = np.random.default_rng(1000 + seed)
    classes = []
    for tb in range(ntypes):
        for tk in range(tb + 1):
            cnt = work[8 + nc * (tb * ntypes + tk) + 3]
            if cnt > 0:
                classes.append((tb, tk, cnt))
    new_rates, t_eri, n_q = {}, 0.0, 0
    for tb, tk, cnt in classes:
        (la, lb), (lc, ld) = types[tb], types[tk]
        if rates is None:
            nq = 2
        else:
            # this class's share of the budget, in quartets of its mean primitive count
            share = cnt * rates[(tb, tk)] / sum(c * rates[(b, k)] for b, k, c in classes)
            mean_pq = np.mean(nprim[byl[la]]) * np.mean(nprim[byl[lb]]) * np.mean(nprim[byl[lc]]) * \
                np.mean(nprim[byl[ld]])
            nq = int(np.clip(budget_s * share / (rates[(tb, tk)] * mean_pq), 2, 20000))
        q = np.stack([rng.choice(byl[la], nq), rng.choice(byl[lb], nq), rng.choice(byl[lc], nq),
                      rng.choice(byl[ld], nq)], axis=1).astype(np.int32)
        pq = float(np.sum(np.prod(nprim[q], axis=1)))
        t0 = time.perf_counter()
        O.eri_quartets_batch(ob, q, 0.0, nthreads)
        dt = time.perf_counter() - t0
        new_rates[(tb, tk)] = dt / pq
        t_eri += cnt * dt / pq
        n_q += nq
    O.set_eri_scheme(1)
    gemm = float(np.sum(work[:5]))
    n = 2048
    a = np.random.default_rng(7).standard_normal((n, n))
    a @ a
    t0 = time.perf_counter()
    a @ a
    gemm_rate = 2.0 * n ** 3 / (time.perf_counter() - t0)
    total = t_eri + gemm / gemm_rate
    desc = (f"{n_q} shell quartets over {len(classes)} ERI classes of the {config} molecule timed on the oracle "
            f"(W-matrix + HRR route, {os.cpu_count()} threads), extrapolated over the job's primitive-quartet "
            f"counts per class; GEMM work {gemm / 1e12:.1f} TFLOP at the host DGEMM rate {gemm_rate / 1e9:.0f} GFLOP/s")
    return total, new_rates, desc


def cpu_baseline(config: str, budget_s: float = 20.0):
    """Reported CPU baseline of our line: the oracle's extrapolated time of the whole
    job (c1: the full job, measured)."""
    from gammcor_integrals_b200 import molecules
    if config == "c1":
        t, desc = oracle_full_c1()
    else:
        work = job_work(config)
        if work is None:
            return None
        _, rates, _ = oracle_job_seconds(config, work, budget_s)
        t, _, desc = oracle_job_seconds(config, work, budget_s, rates)
    return {"value": t, "unit": "s", "cores": os.cpu_count(), "kind": "port", "sample": desc}


def oracle_full_c1():
    """The full c1 job on the oracle (decomposition + AO->MO), measured."""
    from gammcor_integrals_b200 import molecules
    from oracle import oracle as O
    m = molecules.config("c1")
    b = O.make_basis(m.atoms, m.shells)
    nocc, nvirt, seed = molecules.MO_SPLIT["c1"]
    Cm = molecules.mo_coefficients(b.nao, seed)
    t0 = time.perf_counter()
    ch = O.cholesky(b, m.tau)
    O.mo_transf(ch, b, Cm, 0, nocc - 1, Cm, nocc, nocc + nvirt - 1)
    dt = time.perf_counter() - t0
    nv = ch.nvecs
    O.free(ch)
    return dt, (f"full c1 job (NAO={b.nao}, {nv} vectors, MO {nocc}x{nvirt}) on the oracle "
                f"(FP64 C restatement, OpenMP {os.cpu_count()} threads), measured")


def run_reference(args, rank):
    """--impl reference: the CPU restatement of the reference algorithm (oracle/) on
    the same workload as our arm; each step times a bounded sample (c1: the whole
    job) and reports the job's seconds."""
    if rank != 0:
        return
    import gammcor_pkg
    gammcor_pkg.load()
    if args.config in ("c3", "c4"):
        print(json.dumps({"impl": "reference", "unavailable": f"the reference arm times the Cholesky job configs "
                                                              f"(c1, c2, c2s, c5); {args.config} has its own bench"}))
        return
    work = job_work(args.config) if args.config != "c1" else None
    if args.config != "c1" and work is None:
        print(json.dumps({"impl": "reference", "unavailable": f"no recorded work counts for {args.config} "
                                                              f"in oracle/job_work.json"}))
        return
    budget = 5.0
    rates = None
    desc = ""

    def step():
        nonlocal rates, desc
        if args.config == "c1":
            t, desc = oracle_full_c1()
            return t
        t, rates, desc = oracle_job_seconds(args.config, work, budget, rates)
        return t

    step() if args.config != "c1" else None   # sizes the per-class samples
    for _ in range(args.warmup):
        step()
    vals = [step() for _ in range(args.steps)]
    v = float(np.mean(vals))
    cores = os.cpu_count()
    line = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload_name(args.config), "precision": "fp64"},
            "cpu_baseline": {"value": v, "unit": "s", "cores": cores, "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "step_values_s": vals}
    print(json.dumps(line), flush=True)


def mixed_vs_fp64(L, bstruct, c_dev, nao, a0, a1, b0, b1, buffer_mb, state, torch) -> dict:
    """Largest difference of the MO Cholesky vectors (and of the MO integrals they
    reconstruct, sampled) between the split-precision and the FP64 path of one job."""
    import ctypes as C
    from gammcor_integrals_b200 import _capi
    from gammcor_integrals_b200 import cholesky_gammcor as cg
    out = {}
    h = C.c_void_p()
    _capi.check(L.gci_rkpq(C.byref(bstruct), cg.CHOL_ACCURACY_TIGHT, 0.0, 0, C.byref(h)))
    nv = C.c_int64()
    _capi.check(L.gci_query(h, C.byref(nv), None, None, None, None, None))
    res = {}
    for name, prec in (("fp64", _capi.GCI_PREC_FP64), ("mixed", _capi.GCI_PREC_MIXED)):
        r = torch.empty(nv.value * (a1 - a0 + 1) * (b1 - b0 + 1), dtype=torch.float64, device="cuda")
        _capi.check(L.gci_rkab_device(h, C.c_void_p(c_dev.data_ptr()), nao, a0, a1, C.c_void_p(c_dev.data_ptr()),
                                      nao, b0, b1, buffer_mb, prec, C.c_void_p(r.data_ptr())))
        res[name] = r.view(-1, nv.value)   # (NA*NB, NVecs): column k of vector k
    L.gci_free(h)
    d = (res["mixed"] - res["fp64"]).abs().max().item()
    g = torch.Generator(device="cpu").manual_seed(5)
    idx = torch.randint(0, res["fp64"].shape[0], (512,), generator=g).cuda()
    A, B = res["fp64"][idx], res["mixed"][idx]
    mo = (A @ A.T - B @ B.T).abs().max().item()
    out["rkab_mixed_vs_fp64"] = d
    out["mo_integrals_mixed_vs_fp64_sampled"] = mo
    return out


def virtual_ranges(nvecs: int, na: int, b0: int, b1: int, free_bytes: float, frac: float = 0.55):
    """Split the virtual orbitals b0..b1 (1-based, inclusive) into the fewest equal ranges
    whose Rkab block (nvecs x na x range, FP64) fits in `frac` of the free device memory."""
    nb = b1 - b0 + 1
    nparts = 1
    while nparts < nb and 8.0 * nvecs * na * -(-nb // nparts) > frac * free_bytes:
        nparts += 1
    width = -(-nb // nparts)
    return [(q0, min(b1, q0 + width - 1)) for q0 in range(b0, b1 + 1, width)]


def workload_name(config: str) -> str:
    from gammcor_integrals_b200 import molecules
    m = molecules.config(config)
    nocc, nvirt, _ = molecules.MO_SPLIT.get(config, (20, 60, 101))
    return (f"{config}: {len(m.atoms)} atoms, NAO={m.nao}, tau={m.tau}, two-step Cholesky of (pq|rs) + "
            f"AO->MO {nocc}x{nvirt}")


def run_grad(args, rank, world, local):
    """c4: Coulomb energy and nuclear gradient of D = X X^T (X ~ N(0, 0.1^2), 280 x 30, seed 104)
    through the adjoint kernels (gci_coulomb_grad_device; e2e through gci_coulomb_grad)."""
    import torch
    import gammcor_pkg
    gammcor_pkg.load()
    from gammcor_integrals_b200 import _capi, basis, flops, molecules
    L = _capi.lib()
    L.gci_eri_hm(1 if args.eri_kernels == "hermite" else 0)
    _capi.check(L.gci_init())
    mol = molecules.config("c4")
    tb = basis.from_molecule(mol)
    nao = tb.NAO
    X = np.random.default_rng(104).normal(0.0, 0.1, (nao, 30))
    Dm = X @ X.T
    Dd = torch.from_numpy(Dm).cuda()
    sptr = C.c_void_p()
    _capi.check(L.gci_get_stream(C.byref(sptr)))
    lib_stream = torch.cuda.ExternalStream(sptr.value)
    s = tb.c_struct()
    e = C.c_double()
    g = np.zeros((tb.NAtoms, 3))

    def step():
        _capi.check(L.gci_coulomb_grad_device(C.byref(s), 0.0, C.c_void_p(Dd.data_ptr()), nao, C.byref(e),
                                              _capi.ptr(g), None, nao))

    for _ in range(args.warmup):
        step()
    n0 = C.c_int64()
    _capi.check(L.gci_kernel_launches(C.byref(n0)))
    flush = torch.empty(64 << 20, dtype=torch.float64, device="cuda")
    t = 0.0
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for _ in range(args.steps):
            with torch.cuda.stream(lib_stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(lib_stream)
            step()
            e1.record(lib_stream)
            e1.synchronize()
            t += e0.elapsed_time(e1) * 1e-3
        torch.cuda.synchronize()
    n1 = C.c_int64()
    _capi.check(L.gci_kernel_launches(C.byref(n1)))
    work = np.zeros(49)
    _capi.check(L.gci_coulomb_grad_work(_capi.ptr(work), 49))
    fl = flops.grad_flops(work)
    # end to end: density from pinned host memory, gradient and energy back to the host
    pin = torch.from_numpy(Dm).pin_memory()
    te0, te1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    te0.record(lib_stream)
    for _ in range(max(1, args.e2e_steps)):
        _capi.check(L.gci_coulomb_grad(C.byref(s), 0.0, _capi.ptr(pin.numpy()), nao, C.byref(e), _capi.ptr(g),
                                       None, nao))
    te1.record(lib_stream)
    te1.synchronize()
    te = te0.elapsed_time(te1) * 1e-3 / max(1, args.e2e_steps)
    peak64 = measured_fp64_peak(torch)
    rate = fl / (t / args.steps) / 1e12
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        sub = molecules.Molecule(atoms=mol.atoms[:3], shells=[sh for sh in mol.shells if sh[0] < 3])
        ob = O.make_basis(sub.atoms, sub.shells)
        Xs = X[:ob.nao]
        t0 = time.perf_counter()
        O.coulomb_energy_grad(ob, Xs @ Xs.T)
        dt = time.perf_counter() - t0
        scale = (len(mol.shells) / len(sub.shells)) ** 4     # the oracle loops over every ordered shell quartet
        cpu = {"value": 1.0 / (dt * scale), "unit": "gradients/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"oracle (orc_coulomb_energy_grad, OpenMP) on the first 3 atoms of c4 "
                         f"({len(sub.shells)} shells) in {dt:.2f} s, extrapolated by (120/{len(sub.shells)})^4 "
                         f"shell quartets"}
    line = {"metric": "c4 Coulomb energy + nuclear gradient (adjoint kernels)", "value": args.steps / t,
            "unit": "gradients/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"c4: 20 atoms, NAO={nao}, D = X X^T (X 280 x 30)",
                       "l2": "flushed before every timed step (512 MB write outside the timed events)"},
            "energy": e.value, "gflop_per_step": fl / 1e9, "primitive_quartets": float(work.sum()),
            "gpu_launches": int(n1.value - n0.value),
            "roofline": {"bound": "fp64", "kernel": "k_grad_potential (all level classes) + set-up",
                         "achieved": rate, "peak": peak64, "unit": "TFLOP/s", "frac": rate / peak64,
                         "traffic": None, "peak_source": "cuBLAS DGEMM 8192^3 measured in this run"},
            "e2e": {"value": 1.0 / te, "unit": "gradients/s", "h2d_bytes_per_step": int(Dm.nbytes),
                    "d2h_bytes_per_step": int(g.nbytes + 8)},
            "clocks": clk.summary(), "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def run_batch(args, local):
    """c3: the 64 c3 molecules (3-30 atoms, c1 recipe, tau = 1e-5) decomposed by one
    gci_rkpq_batch call (one CUDA stream per worker), against one gci_rkpq call per molecule."""
    import torch
    import gammcor_pkg
    gammcor_pkg.load()
    from gammcor_integrals_b200 import _capi, basis, flops, molecules
    L = _capi.lib()
    L.gci_eri_hm(1 if args.eri_kernels == "hermite" else 0)
    _capi.check(L.gci_init())
    mols = [molecules.config("c3", i) for i in range(64)]
    tbs = [basis.from_molecule(m) for m in mols]
    views = [tb.c_struct() for tb in tbs]
    arr = (_capi.gci_basis * 64)(*views)
    tune = np.zeros(400)
    _capi.check(L.gci_autotune_eri(C.byref(views[int(np.argmax([tb.NAO for tb in tbs]))]), args.tune_pairs,
                                   _capi.ptr(tune)))
    nstreams = args.streams

    def batch():
        hs = (C.c_void_p * 64)()
        _capi.check(L.gci_rkpq_batch(64, arr, _capi.GCI_ACCURACY_DEFAULT, 0.0, 0, nstreams, hs))
        return hs

    phase_names = ("vdiag", "step1_eri", "subtract_r", "pivots", "compress", "vjj_eri", "potrf_trtri")
    phase_sum = dict.fromkeys(phase_names, 0.0)
    extra = {"rkpq_host_s": 0.0, "macro_iterations": 0.0}

    def stats_of(hs, record=False):
        tot = 0.0
        nv = []
        for h in hs:
            st = np.zeros(8 + 600)
            _capi.check(L.gci_stats(C.c_void_p(h), _capi.ptr(st), st.size))
            tot += flops.job_flops(st, "lib")["total"]
            q = C.c_int64()
            _capi.check(L.gci_query(C.c_void_p(h), C.byref(q), None, None, None, None, None))
            nv.append(q.value)
            if record:
                tm = np.zeros(13)
                _capi.check(L.gci_timings(C.c_void_p(h), _capi.ptr(tm), 13))
                for i, nme in enumerate(phase_names):
                    phase_sum[nme] += float(tm[i])
                extra["macro_iterations"] += float(tm[10])
                extra["rkpq_host_s"] += float(tm[11])
            L.gci_free(C.c_void_p(h))
        return tot, nv

    for _ in range(args.warmup):
        stats_of(batch())
    n0 = C.c_int64()
    _capi.check(L.gci_kernel_launches(C.byref(n0)))
    flush = torch.empty(64 << 20, dtype=torch.float64, device="cuda")
    t = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            hs = batch()
            torch.cuda.synchronize()
            t += time.perf_counter() - t0
            fl, nv = stats_of(hs, record=True)
    n1 = C.c_int64()
    _capi.check(L.gci_kernel_launches(C.byref(n1)))
    # the same molecules one gci_rkpq call after another (one stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for v in views:
        h = C.c_void_p()
        _capi.check(L.gci_rkpq(C.byref(v), _capi.GCI_ACCURACY_DEFAULT, 0.0, 0, C.byref(h)))
        L.gci_free(h)
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    line = {"metric": "c3 batched Cholesky-ERI GFLOP/s (64 molecules)", "value": fl * args.steps / t / 1e9,
            "unit": "GFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"c3: 64 molecules, {min(tb.NAO for tb in tbs)}-{max(tb.NAO for tb in tbs)} AOs, "
                                   f"tau=1e-5, gci_rkpq_batch with {nstreams} streams",
                       "timing": "host clock between device-wide synchronisations (the batch spans "
                                 f"{nstreams} CUDA streams)",
                       "l2": "flushed before every timed step"},
            "molecules_per_s": 64 * args.steps / t, "sequential_s": t_seq, "batch_s": t / args.steps,
            "speedup_vs_sequential": t_seq / (t / args.steps), "nvecs_total": int(sum(nv)),
            "gpu_launches": int(n1.value - n0.value), "clocks": clk.summary(),
            "per_molecule_sums": {"device_phase_s": {k: v / args.steps for k, v in phase_sum.items()},
                                  "macro_iterations": extra["macro_iterations"] / args.steps,
                                  "gci_rkpq_wall_s": extra["rkpq_host_s"] / args.steps,
                                  "definition": "sums over the 64 molecules of each handle's phase timers "
                                                "(CUDA events on its worker's stream) and call wall time"}}
    print(json.dumps(line), flush=True)


def run_dense(args):
    """The dense kernels of the decomposition alone, on one GPU: each shape timed with CUDA
    events (best of 3 after one warm-up) next to the vendor library doing the same job
    (torch.matmul = cuBLAS DGEMM; torch.linalg.cholesky + solve_triangular = cuSOLVER), and
    the largest difference of the results."""
    import ctypes as C
    import torch
    import gammcor_pkg
    gammcor_pkg.load()
    from gammcor_integrals_b200 import _capi
    L = _capi.lib()
    _capi.check(L.gci_init())
    vp = lambda t: C.c_void_p(t.data_ptr())

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(3):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            best = min(best, time.perf_counter() - t0)
        return best

    out = {}
    g = torch.Generator(device="cuda").manual_seed(11)
    for m, n, k in ((8192, 8192, 8192), (200000, 1000, 1024), (16285, 2000, 16285)):
        At = torch.randn(k, m, dtype=torch.float64, device="cuda", generator=g)
        Bt = torch.randn(k, n, dtype=torch.float64, device="cuda", generator=g)
        Ct = torch.empty(n, m, dtype=torch.float64, device="cuda")
        t_ours = timed(lambda: _capi.check(L.gci_dgemm(m, n, k, 1.0, vp(At), m, vp(Bt), n, 0.0, vp(Ct), m)))
        t_lib = timed(lambda: torch.matmul(At.T, Bt))
        err = float((Ct.T - At.T @ Bt).abs().max())
        t_split = timed(lambda: _capi.check(L.gci_dgemm_split(m, n, k, 1.0, vp(At), m, vp(Bt), n, 0.0, vp(Ct),
                                                              m)))
        err_split = float((Ct.T - At.T @ Bt).abs().max())
        f = 2.0 * m * n * k / 1e12
        out[f"gemm_nt {m}x{n}x{k}"] = {"k_dgemm_tflops": f / t_ours, "cublas_dgemm_tflops": f / t_lib,
                                       "k_dgemm_max_abs_diff": err, "split_int8_tflops_fp64_equivalent": f / t_split,
                                       "split_max_abs_diff": err_split}
        del At, Bt, Ct
        torch.cuda.empty_cache()
    for nn in (4096, 16285):
        X0 = torch.randn(nn, nn, dtype=torch.float64, device="cuda", generator=g)
        S = X0 @ X0.T / nn + torch.eye(nn, dtype=torch.float64, device="cuda")
        del X0
        A, X = torch.empty_like(S), torch.empty_like(S)
        eye = torch.eye(nn, dtype=torch.float64, device="cuda")

        def ours():
            A.copy_(S)
            torch.cuda.synchronize()
            _capi.check(L.gci_cholesky_inverse(nn, vp(A), nn, vp(X)))

        t_ours = timed(ours) - timed(lambda: A.copy_(S))
        t_lib = timed(lambda: torch.linalg.solve_triangular(torch.linalg.cholesky(S), eye, upper=False))
        Xr = torch.linalg.solve_triangular(torch.linalg.cholesky(S), eye, upper=False)
        out[f"cholesky_inverse {nn}"] = {"ours_s": t_ours, "cusolver_potrf_plus_trsm_s": t_lib,
                                         "max_rel_diff": float((X.T - Xr).abs().max() / Xr.abs().max())}
        del S, A, X, eye, Xr
        torch.cuda.empty_cache()
    rows, w = 600000, 400
    Z = torch.randn(w, w, dtype=torch.float64, device="cuda", generator=g)
    Lp = torch.linalg.cholesky(Z @ Z.T / w + torch.eye(w, dtype=torch.float64, device="cuda"))
    B0 = torch.randn(w, rows, dtype=torch.float64, device="cuda", generator=g)
    B, Lt = B0.clone(), Lp.T.contiguous()

    def ours_trsm():
        B.copy_(B0)
        torch.cuda.synchronize()
        _capi.check(L.gci_trsm_rlt(rows, w, vp(B), rows, vp(Lt), w))

    t_ours = timed(ours_trsm) - timed(lambda: B.copy_(B0))
    t_lib = timed(lambda: torch.linalg.solve_triangular(Lp, B0, upper=False))
    ref = torch.linalg.solve_triangular(Lp, B0, upper=False)
    ours_trsm()   # the timing of the copy above left B = B0
    out[f"trsm_rlt {rows}x{w}"] = {"ours_s": t_ours, "cublas_trsm_s": t_lib, "max_abs_diff": float((B - ref).abs().max())}
    print(json.dumps({"dense_kernels": out, "note": "wall time around each call with a device synchronisation; "
                      "the library calls include their argument checks and stream synchronisation"}), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.dense:
        if rank == 0:
            run_dense(args)
        return
    if args.config == "c3":
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            run_batch(args, local)
        return
    if args.config == "c4":
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            run_grad(args, rank, world, local)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=torch.device("cuda", local))
    import gammcor_pkg
    gammcor_pkg.load()
    from gammcor_integrals_b200 import _capi, basis, flops, molecules
    from gammcor_integrals_b200 import cholesky_gammcor as cg
    L = _capi.lib()
    L.gci_eri_hm((2 if args.hm_profile else 1) if args.eri_kernels == "hermite" else 0)
    _capi.check(L.gci_init())

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    mol = molecules.config(args.config)
    tb = basis.from_molecule(mol)
    nao = tb.NAO
    nocc, nvirt, seed = molecules.MO_SPLIT.get(args.config, (20, 60, 101))
    Cm = molecules.mo_coefficients(nao, seed)
    a0, a1, b0, b1 = 1, nocc, nocc + 1, nocc + nvirt
    NA, NB = nocc, nvirt
    prec = {"fp64": _capi.GCI_PREC_FP64, "mixed": _capi.GCI_PREC_MIXED}[args.precision]
    c_dev = torch.from_numpy(np.ascontiguousarray(Cm.T)).cuda()    # column-major C on the device
    sptr = C.c_void_p()
    _capi.check(L.gci_get_stream(C.byref(sptr)))
    lib_stream = torch.cuda.ExternalStream(sptr.value)
    bstruct = tb.c_struct()
    state = {"rkab": None, "nvecs": None, "parts": None}
    # per-class kernel choice (team vs ket-first) by the library's autotuner, untimed set-up
    tune = np.zeros(400)
    t_tune = time.perf_counter()
    _capi.check(L.gci_autotune_eri(C.byref(bstruct), args.tune_pairs, _capi.ptr(tune)))
    t_tune = time.perf_counter() - t_tune
    chosen = [L.gci_eri_variant(tb_, tk_, -1) for tb_ in range(10) for tk_ in range(tb_ + 1)]
    kf_classes = {w: sum(1 for v in chosen if v == w) for w in range(4)}

    def job():
        h = C.c_void_p()
        flags = _capi.GCI_FLAG_PIVOT_DECODE_STORAGE if args.decode_storage else 0
        if args.precision == "mixed":
            flags |= _capi.GCI_FLAG_MIXED_STEP1
        _capi.check(L.gci_rkpq(C.byref(bstruct), cg.CHOL_ACCURACY_TIGHT, 0.0, flags, C.byref(h)))
        nv = C.c_int64()
        _capi.check(L.gci_query(h, C.byref(nv), None, None, None, None, None))
        if state["rkab"] is None or state["nvecs"] != nv.value:
            state["rkab"] = None
            # Rkab on the device, in one piece when it fits beside the library's own buffers
            # (Inv_L, the integral chunks); otherwise in ranges of virtual orbitals, one
            # gci_rkab_device call each into the same buffer (c5: 48k vectors x 150 x 2700 =
            # 156 GB, more than the HBM and than 80% of the host memory of the box)
            state["parts"] = virtual_ranges(nv.value, NA, b0, b1, torch.cuda.mem_get_info()[0])
            nbp = max(q1 - q0 + 1 for q0, q1 in state["parts"])
            state["rkab"] = torch.empty(nv.value * NA * nbp, dtype=torch.float64, device="cuda")
            state["nvecs"] = nv.value
        for pb0, pb1 in state["parts"]:
            _capi.check(L.gci_rkab_device(h, C.c_void_p(c_dev.data_ptr()), nao, a0, a1, C.c_void_p(c_dev.data_ptr()),
                                          nao, pb0, pb1, args.buffer_mb, prec, C.c_void_p(state["rkab"].data_ptr())))
        st = np.zeros(8 + 600 + 1)
        _capi.check(L.gci_stats(h, _capi.ptr(st), st.size))
        tm = np.zeros(13)
        _capi.check(L.gci_timings(h, _capi.ptr(tm), 13))
        hs = np.zeros(7 * 7 * 7 * 3)
        _capi.check(L.gci_eri_hm_stats(h, _capi.ptr(hs), hs.size))
        state["hm"] = hs.reshape(7, 7, 7, 3)
        L.gci_free(h)
        return st, tm

    for _ in range(args.warmup):
        job()
    barrier()
    n0 = C.c_int64()
    _capi.check(L.gci_kernel_launches(C.byref(n0)))
    # L2 (126 MB) is flushed before every timed step by writing a 512 MB buffer
    # on the library's stream, outside the events that bracket the step
    flush = torch.empty(64 << 20, dtype=torch.float64, device="cuda")
    t_dev = 0.0
    with ClockSampler(local) as clk:
        barrier()
        stats, times, step_s = [], [], []
        for _ in range(args.steps):
            with torch.cuda.stream(lib_stream):
                flush.fill_(1.0)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(lib_stream)
            st, tm = job()
            ev1.record(lib_stream)
            ev1.synchronize()
            t_dev += ev0.elapsed_time(ev1) * 1e-3
            step_s.append(ev0.elapsed_time(ev1) * 1e-3)
            stats.append(st)
            times.append(tm)
        barrier()
    del flush
    n1 = C.c_int64()
    _capi.check(L.gci_kernel_launches(C.byref(n1)))
    t_max = max_over_ranks(t_dev, world, "cuda")
    if args.hm_profile and rank == 0:
        hs = state["hm"]
        tot = hs[..., 1].sum()
        rows = sorted(((hs[a, b, c, 1], a, b, c + 1, hs[a, b, c, 0], hs[a, b, c, 2])
                       for a in range(7) for b in range(7) for c in range(7) if hs[a, b, c, 0] > 0), reverse=True)
        print(f"# Hermite-matrix classes: {tot:.2f} s, {hs[..., 2].sum() / 1e12:.1f} TFLOP issued", file=sys.stderr)
        for t, a, b, c, n, f in rows:
            print(f"#  L1={a} L2={b} NT={c}  launches {int(n):5d}  {t:8.3f} s  {100 * t / max(tot, 1e-30):5.1f}%  "
                  f"{f / 1e12:8.2f} TF  {f / max(t, 1e-30) / 1e12:6.2f} TF/s", file=sys.stderr)
    if args.dump_work and rank == 0:
        dump = Path(args.dump_work)
        d = json.loads(dump.read_text()) if dump.exists() else {}
        d[args.config] = {"how": f"python bench.py --config {args.config} --dump-work on one B200 "
                                 f"(gci_stats of one job: GEMM flops and per-class ERI counters)",
                          "nvecs": int(state["nvecs"]), "stats": [float(x) for x in stats[-1]]}
        dump.write_text(json.dumps(d, indent=1) + "\n")
    fl = flops.job_flops(stats[-1], "lib")
    flops_step = fl["total"]
    sec = t_max / args.steps
    # accuracy of this job's results: the FP64 path is checked against the oracle by the
    # parity tests (tests/test_gpu_parity.py); a split-precision run is compared here
    # with the FP64 path on the same molecule
    err = {"fp64_path": "parity with the FP64 oracle: tests/test_gpu_parity.py"}
    if args.precision != "fp64" and len(state["parts"]) > 1:
        err["mixed_vs_fp64"] = "not measured: the two outputs do not fit on the device together"
    elif args.precision != "fp64":
        err.update(mixed_vs_fp64(L, bstruct, c_dev, nao, a0, a1, b0, b1, args.buffer_mb, state, torch))

    # ---- end to end through the public host API (pinned host buffers)
    e2e = None
    if args.e2e_steps > 0 and len(state["parts"]) == 1:   # host output of the whole Rkab
        nv = state["nvecs"]
        pin_c = torch.from_numpy(np.ascontiguousarray(Cm.T)).pin_memory()
        pin_out = torch.empty(nv * NA * NB, dtype=torch.float64).pin_memory()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record(lib_stream)
        for _ in range(args.e2e_steps):
            res = cg.chol_gammcor_Rkpq(tb, cg.CHOL_ACCURACY_TIGHT, materialize=False,
                                       decode_storage=args.decode_storage, mixed_step1=args.precision == "mixed")
            _capi.check(L.gci_rkab(res.handle.ptr, _capi.ptr(pin_c.numpy()), nao, a0, a1, _capi.ptr(pin_c.numpy()),
                                   nao, b0, b1, args.buffer_mb, prec, _capi.ptr(pin_out.numpy())))
            checksum = float(pin_out[:16].sum())
            del res
        e1.record(lib_stream)
        e1.synchronize()
        te = max_over_ranks(e0.elapsed_time(e1) * 1e-3, world, "cuda")
        h2d = int(Cm.nbytes) + int(tb.CntrCoeffs.nbytes + tb.Exponents.nbytes + tb.AtomCoords.nbytes)
        d2h = nv * NA * NB * 8
        e2e = {"value": te / args.e2e_steps, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "gflops": aggregate_rate(flops_step, args.e2e_steps, world, te) / 1e9, "checksum": checksum}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    tm = times[-1]
    phases = {"vdiag": tm[0], "step1_eri": tm[1], "subtract_r": tm[2], "pivots": tm[3], "compress": tm[4],
              "vjj_eri": tm[5], "potrf_trtri": tm[6], "fulldim_eri": tm[7], "invl_gemm": tm[8], "mo_gemm": tm[9]}
    eri_t = tm[0] + tm[1] + tm[5] + tm[7]
    gemm_t = tm[2] + tm[8] + tm[9]
    peak64 = measured_fp64_peak(torch)
    eri_alg = flops.eri_flops(stats[-1], "lib", unscreened=False)
    hm_issued = float(stats[-1][608])
    roof = {"bound": "fp64", "kernel": "k_eri_hm (Hermite-matrix ERI kernels, FP64 tensor cores) + the diagonal "
                                       "stage's class kernels: all ERI stages",
            "achieved": eri_alg / eri_t / 1e12 if eri_t > 0 else 0.0, "peak": peak64, "unit": "TFLOP/s",
            "frac": (eri_alg / eri_t / 1e12) / peak64 if (peak64 and eri_t > 0) else None, "traffic": None,
            "achieved_definition": "reference-algorithm ERI flops of the evaluated primitive quartets (flops.py "
                                   "class_flops) / device seconds of the ERI stages",
            "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 (FP64; MEASURED_PEAKS.json has no FP64 figure)",
            "issued_tflops_per_s": hm_issued / eri_t / 1e12 if eri_t > 0 else 0.0,
            "issued_definition": "tensor-core flops the Hermite-matrix kernels issued (padding included)",
            "eri_seconds": eri_t, "gemm_seconds": gemm_t}
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cpu = cpu_baseline(args.config)
    line = {"metric": METRIC, "value": sec, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(args.config), "precision": args.precision,
                       "nvecs": state["nvecs"], "parallelism": f"replicas x{world}",
                       "rkab_output": ("device (gci_rkab_device)" if len(state["parts"]) == 1 else
                                       f"device, in {len(state['parts'])} ranges of virtual orbitals (one "
                                       f"gci_rkab_device call each; the whole Rkab exceeds the HBM)"),
                       "l2": "flushed before every timed step (512 MB write outside the timed events)"},
            "value_definition": "device seconds of one complete job (decomposition + AO->MO) on each GPU, "
                                "CUDA events on the library stream, max over ranks",
            "gflops": aggregate_rate(flops_step, args.steps, world, t_max) / 1e9,
            "gflops_definition": "reference-algorithm work of the job (GEMM formulas + W-matrix ERI arithmetic "
                                 "over every primitive quartet, flops.py) per second, all ranks",
            "gflop_per_step": flops_step / 1e9, "gflop_executed_per_step": fl["executed"] / 1e9,
            "eri_per_s": fl["integrals"] * args.steps * world / t_max, "phases_s": phases,
            "step_seconds": [round(x, 3) for x in step_s],
            "gpu_launches": int(n1.value - n0.value), "roofline": roof, "e2e": e2e,
            "clocks": clk.summary(), "cpu_baseline": cpu}
    line["max_abs_err"] = err
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
