"""Benchmark of the ChainAMPS DMRG hot path on B200.

Workload: iDMRG on four coupled spin-1/2 Heisenberg
chains treated as one vertex (local dimension 16, intrachain J = 1, rung
J_perp = 0.5, total-Sz charge, reference-padded MPO of bond dimension 110),
complex double, bond dimension chi = 512.  One step = one H_eff matvec
(``TwoVertexMPOMPSMultiply``, the operation the Arnoldi solver repeats) at
the chi = 512 sector structure of that run: environments are seeded
synthetic blocks with a Gaussian total-Sz sector profile, the MPO is the
real one.  Inputs (~0.15 GB vector, ~3 GB intermediate) exceed L2, so no L2
flush is needed between steps.

* value: canonical algorithmic TFLOP/s of the device matvec with the vector
  already resident in HBM (CUDA events, max over ranks), for the faster of
  the two split-precision forms (split-TF32, split-BF16; `headline_form`);
  `split_forms` and `fp64_form` give every form;
* e2e: the same through the C ABI with host buffers
  (``cmps_heff_apply``: H2D, matvec, D2H inside the timed region);
* roofline: the two grouped GEMM stages' canonical flops over their CUDA-event
  time against the measured dense bf16 peak (MEASURED_PEAKS.json), with the
  DRAM traffic per matvec from the committed ncu summary;
* idmrg: the iDMRG growth step itself on the same model (real MPO, real
  environments grown from the dummy blocks up to chi = 512; Arnoldi
  tolerance 1e-10): device time per step at full chi in FP64 and in mixed
  precision (split-TF32 and split-BF16 matvecs, FP64 Krylov/SVD/energies),
  the per-phase profile, and the largest relative energy difference between
  the runs;
* idmrg_coupled_ising: the same FP64-vs-mixed iDMRG step on the
  coupled transverse-field Ising chain config (each vertex a periodic
  12-site chain at g = 1.2 cut by exact diagonalisation to its 64 lowest
  states with Z2 parity, interchain J_perp = 0.05 sum_i X_i X_i, MPO D = 26)
  at chi = 64 and 128 (the config's chi = 2048 needs a 137 GB wavefunction),
  plus the FP64 step in the reference's folded contraction order at chi = 64;
* cpu_baseline: the oracle's block-sparse numpy port of the same matvec on
  the host cores (one full matvec);
* --impl reference: the CPU port timed as the reference arm.

Multi-GPU (N > 1): one matvec per step split across the ranks by output
charge sector (``chainamps_b200.sharded``): every rank holds the
environments and the MPO, receives the input sectors its outputs read by one
all-to-all and computes the output sectors it owns, balanced by their flops;
`value` is the whole matvec's canonical TFLOP/s over the max-over-ranks step
time ("strong" scaling: the work per step is the same for every N).  The
iDMRG step figures run on every rank as replicas.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "iDMRG step time & H_eff matvec TFLOP/s, mixed vs FP64 GPU at |dE/E|<1e-9"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--chi", type=int, default=512)
    p.add_argument("--precision", default="all", choices=["all", "both", "fp64", "split_tf32", "split_bf16"],
                   help="all: FP64 and both split forms; both: FP64 and split-TF32")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--idmrg-steps", type=int, default=4, help="timed iDMRG steps at full chi (0: skip)")
    p.add_argument("--ising-steps", type=int, default=2, help="timed coupled-Ising iDMRG steps (0: skip)")
    p.add_argument("--ising-chi", default="64,128", help="bond dimensions of the coupled-Ising steps")
    p.add_argument("--ising-folded-chi", type=int, default=64,
                   help="bond dimension at which the folded-order FP64 step is also timed (0: skip)")
    p.add_argument("--ising-forms", default="fp64,mixed,mixed_bf16",
                   help="forms of the coupled-Ising step: fp64, mixed (split TF32), mixed_bf16 (split BF16)")
    p.add_argument("--ising-matvec-chi", default="128",
                   help="bond dimensions of the coupled-Ising matvec timing per form ('': skip)")
    return p.parse_args()


def workload(chi, seed=20261203):
    from chainamps_b200 import models  # numpy only: does not load the CUDA library
    return models.ladder_workload(chi, seed)


def native_libraries_mapped():
    """This repository's shared libraries mapped into this process."""
    try:
        with open("/proc/self/maps") as f:
            maps = f.read().splitlines()
    except OSError:
        return []
    return sorted({ln.split()[-1] for ln in maps if ln.split() and ln.split()[-1].startswith(ROOT)
                   and ".so" in ln.split()[-1]})


def measured_peaks():
    """Driver-measured peaks of this GPU pool (HBM copy GB/s, cuBLAS bf16
    TFLOP/s burst and sustained), or None."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def profiled_traffic(name):
    """DRAM bytes per matvec of the split-TF32 stages, from the committed ncu
    summary (a line `traffic_bytes_per_matvec: <bytes>`), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for ln in f:
                if ln.strip().startswith("traffic_bytes_per_matvec:"):
                    return float(ln.split(":", 1)[1].split()[0])
    except (OSError, ValueError, IndexError):
        return None
    return None


def clocks_sampler(stop, out):
    cmd = ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits"]
    idx = os.environ.get("LOCAL_RANK", "0")
    while not stop.is_set():
        try:
            r = subprocess.run(cmd + ["-i", idx], capture_output=True, text=True, timeout=5)
            if r.returncode == 0 and r.stdout.strip():
                out.append(r.stdout.strip().splitlines()[0])
        except Exception:
            pass
        stop.wait(0.2)


def summarize_clocks(lines):
    sm, mx, reasons = [], 0.0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in lines:
        f = [x.strip() for x in ln.split(",")]
        try:
            sm.append(float(f[1]))
            mx = max(mx, float(f[2]))
        except (ValueError, IndexError):
            continue
        for n, v in zip(names, f[4:8]):
            if v.lower().startswith("active"):
                reasons.add(n)
    return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
            "reasons": sorted(reasons), "samples": len(sm)}


def cpu_port(wl, reps=1):
    """Block-sparse numpy port of the reference matvec (oracle) on the host."""
    from oracle import blocks as ob
    chi = wl["bond"].shape[0]
    D = wl["bq"].shape[0]

    def mats(t, right):
        return ob.env_matrices(chi, D, t.colptr, t.rowind, t.values)
    t0 = time.perf_counter()
    bh = ob.BlockHeff(wl["rules"], wl["ch"], wl["bond"], wl["bond"], wl["bq"], wl["W"],
                      mats(wl["L"], False), mats(wl["R"], True))
    setup = time.perf_counter() - t0
    x = np.random.default_rng(1).standard_normal(bh.n) + 0j
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        bh.matvec(x)
        ts.append(time.perf_counter() - t0)
    try:
        from threadpoolctl import threadpool_info
        cores = max([i.get("num_threads", 1) for i in threadpool_info()] or [1])
    except Exception:
        cores = os.cpu_count()
    return float(np.mean(ts)), setup, cores, bh.n


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cfg = {"workload": f"iDMRG H_eff matvec, 4-leg Heisenberg ladder vertex (d=16, MPO D=110 reference-padded), "
                       f"chi={a.chi}, complex double, synthetic environments (seed 20261203)",
           "chi": a.chi, "local_dim": 16, "mpo_dim": 110, "l2": "inputs larger than L2 (no flush)",
           "parallelism": "single GPU" if a.gpus == 1 else f"matvec sharded by output sector over {a.gpus} GPUs"}

    if a.impl == "reference":
        if rank != 0:
            return 0
        # the workload is built by numpy-only modules (chainamps_b200.models
        # and .tensors never load the CUDA library) and timed with the oracle
        wl = workload(a.chi)
        steps, warm = a.steps, max(3, a.warmup)
        for _ in range(warm):
            cpu_port(wl, 1)
        mapped = native_libraries_mapped()
        if mapped:
            raise SystemExit(f"reference arm: this repository's native library is mapped: {mapped}")
        t, setup, cores, n = cpu_port(wl, steps)
        flops = canonical_flops_cpu(wl)
        v = flops / t / 1e12
        line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "TFLOP/s", "n_gpus": a.gpus,
                "steps": steps, "warmup": warm, "ms_per_step": t * 1e3, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "complex128", "data": "synthetic", "config": cfg,
                "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": cores, "kind": "port",
                                 "sample": f"one full matvec per step (n={n}), {steps} steps after {warm} warm-up, "
                                           "numpy restatement of the reference's block contraction on the host "
                                           "cores; the reference C++ is not built here (needs CXSparse, ARPACK, "
                                           "LAPACKE)"},
                "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "native_so_loaded": mapped}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from chainamps_b200 import Context, TwoVertexComponents, CMPS_FP64, CMPS_SPLIT_TF32, CMPS_SPLIT_BF16
    wl = workload(a.chi)
    ctx = Context(local)
    # a dedicated (non-default) stream: the library launches on exactly this
    # stream, so the CUDA events below bracket the kernels themselves
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0

    def measure(h, steps, warm):
        n = h.n
        x = torch.randn(n, dtype=torch.complex128, device="cuda")
        y = torch.empty_like(x)
        for _ in range(max(3, warm)):
            h.multiply_device(x.data_ptr(), y.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        h.status()
        stop = threading.Event()
        clk = []
        th = threading.Thread(target=clocks_sampler, args=(stop, clk), daemon=True)
        th.start()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            h.multiply_device(x.data_ptr(), y.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        if dist:
            dist.barrier()
        stop.set()
        th.join(timeout=5)
        h.status()
        st = h.time_stages(x.data_ptr(), y.data_ptr(), stream.cuda_stream, reps=3)
        ms_t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        if dist:
            dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
        return float(ms_t.item()), st, summarize_clocks(clk)

    def measure_sharded(h, steps, warm):
        """N > 1: one matvec split over the ranks by output sector (each rank
        receives the input sectors its owned outputs read by an all-to-all,
        then computes its owned sectors); returns (ms per step, [exchange ms,
        owned-sector matvec ms, 0, 0], clocks, owned executed flops, operator)."""
        from chainamps_b200.sharded import ShardedTwoVertex
        off, fl = h.sector_table()
        sh = ShardedTwoVertex(h)
        op, lay = sh.op, sh.layout
        x = torch.randn(2, lay.n_local, dtype=torch.float64, device="cuda")
        for _ in range(max(3, warm)):
            op(x)
        torch.cuda.synchronize()
        h.status()
        stop = threading.Event()
        clk = []
        th = threading.Thread(target=clocks_sampler, args=(stop, clk), daemon=True)
        th.start()
        dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            op(x)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        dist.barrier()
        stop.set()
        th.join(timeout=5)
        h.status()
        # the two parts alone, on this rank
        parts = []
        for f in (lambda: op.exchange(x), lambda: op.apply_window(op.xwin, op.yloc)):
            g0 = torch.cuda.Event(enable_timing=True)
            g1 = torch.cuda.Event(enable_timing=True)
            g0.record(stream)
            for _ in range(3):
                f()
            g1.record(stream)
            torch.cuda.synchronize()
            parts.append(g0.elapsed_time(g1) / 3)
        ms_t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
        return float(ms_t.item()), [parts[0], parts[1], 0.0, 0.0], summarize_clocks(clk), float(fl[lay.owned].sum()), op

    def e2e_sharded(op, steps):
        """N > 1, end to end: each step copies this rank's input slice from
        pinned host memory, runs the sharded matvec and copies its output
        slice back."""
        lay = op.layout
        xh = torch.randn(2, lay.n_local, dtype=torch.float64).pin_memory()
        yh = torch.empty(2, lay.n_local, dtype=torch.float64).pin_memory()
        op(xh.to("cuda", non_blocking=True))
        torch.cuda.synchronize()
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            yh.copy_(op(xh.to("cuda", non_blocking=True)), non_blocking=True)
            torch.cuda.current_stream().synchronize()
        t = torch.tensor([(time.perf_counter() - t0) / steps], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def e2e(h, steps):
        n = h.n
        xh = torch.randn(n, dtype=torch.complex128).pin_memory().numpy()
        yh = torch.empty(n, dtype=torch.complex128).pin_memory().numpy()
        h.multiply(xh, out=yh)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            h.multiply(xh, out=yh)
        return (time.perf_counter() - t0) / steps

    def gemm_peak(dtype, nn=8192, reps=5):
        A = torch.randn(nn, nn, dtype=dtype, device="cuda")
        B = torch.randn(nn, nn, dtype=dtype, device="cuda")
        for _ in range(2):
            A @ B
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record()
        for _ in range(reps):
            A @ B
        g1.record()
        torch.cuda.synchronize()
        f = (8 if dtype.is_complex else 2) * nn ** 3 * reps
        return f / (g0.elapsed_time(g1) * 1e-3) / 1e12

    want = {"all": ["fp64", "split_tf32", "split_bf16"], "both": ["fp64", "split_tf32"]}.get(a.precision,
                                                                                            [a.precision])
    res = {}
    canonical = executed = n = None
    for p in want:
        prec = {"fp64": CMPS_FP64, "split_tf32": CMPS_SPLIT_TF32, "split_bf16": CMPS_SPLIT_BF16}[p]
        h = TwoVertexComponents(ctx, wl["rules"], wl["L"], wl["Wt"], wl["R"], precision=prec)
        canonical, executed = h.flops()
        n = h.n
        if world == 1:
            ms, st, clk = measure(h, a.steps, a.warmup)
            e2e_s = e2e(h, max(3, a.steps // 2))
            res[p] = dict(ms=ms, st=st, clk=clk, e2e_s=e2e_s, owned=executed, n_io=n)
        else:
            ms, st, clk, owned, op = measure_sharded(h, a.steps, a.warmup)
            e2e_s = e2e_sharded(op, max(3, a.steps // 2))
            res[p] = dict(ms=ms, st=st, clk=clk, e2e_s=e2e_s, owned=owned, n_io=op.layout.n_local,
                          window=op.layout.in_len)
            del op
        del h
        torch.cuda.empty_cache()
    zgemm = gemm_peak(torch.complex128, 4096)
    torch.backends.cuda.matmul.allow_tf32 = True
    tf32 = gemm_peak(torch.float32, 8192)
    # the headline is the fastest split form measured (both meet the metric's
    # energy tolerance through the FP64-refined solver), else the FP64 form
    splits = [p for p in ("split_tf32", "split_bf16") if p in res]
    head = min(splits, key=lambda p: res[p]["ms"]) if splits else "fp64"
    r = res[head]
    gemm_ms = r["st"][1] + r["st"][2]
    # Roofline of the dominant kernels (the two grouped GEMM stages): the
    # algorithmic (canonical four-stage) flops they deliver per matvec over
    # their CUDA-event time.  Split-TF32 is credited the canonical flops, not
    # the 3x emulation work.  The denominator is the driver-measured dense bf16
    # burst peak of this pool (MEASURED_PEAKS.json): the stages are timed
    # alone.  The live cuBLAS ceilings of the pipes the stages actually use
    # (TF32 for split, DMMA FP64 for the FP64 form) are reported beside it.
    pk = measured_peaks()
    peak, peak_src = (pk["bf16_tflops"], "MEASURED_PEAKS.json bf16_tflops (burst), of measured") if pk else \
        (1590.0, "fallback 1.59 PFLOP/s bf16 (MEASURED_PEAKS.json absent), of fallback")
    pipe_ceiling = {"fp64": zgemm, "split_tf32": tf32, "split_bf16": peak}[head]
    if world > 1:
        # this rank's owned-sector matvec against the canonical flops of its share
        share = r["owned"] / executed if executed else 0.0
        ach = share * canonical / (gemm_ms * 1e-3) / 1e12
        kern = "owned-sector matvec of rank 0 (both grouped GEMM stages)"
    else:
        ach = canonical / (gemm_ms * 1e-3) / 1e12
        kern = {"fp64": "zgemm_grouped_fp64 (stage 1 + stage 2)",
                "split_tf32": "tc_split_gemm<1> + tc_split_gemm<2> (tcgen05 kind::tf32, 3-term split)",
                "split_bf16": "tc_split_gemm<3> + tc_split_gemm<4> (tcgen05 kind::f16 with BF16, 3-term split)"}[head]
    prof_file = {"split_tf32": "heff_matvec_split_tf32_ladder4_chi512.md",
                 "split_bf16": "heff_matvec_split_bf16_ladder4_chi512.md"}.get(head)
    traffic = profiled_traffic(prof_file) if prof_file and world == 1 and a.chi == 512 else None
    roof = {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
            "traffic": traffic, "kernel": kern, "peak_source": peak_src,
            "achieved_is": "canonical four-stage complex flops per matvec (8 per complex MAC, non-zero MPO "
                           "entries only) / CUDA-event time of the two GEMM stages",
            "pipe_ceiling_live": pipe_ceiling,
            "pipe_ceiling_is": {"fp64": "live cuBLAS complex128 4096^3 GEMM",
                                "split_tf32": "live cuBLAS TF32 8192^3 GEMM",
                                "split_bf16": "the measured bf16 peak itself"}[head],
            "frac_of_pipe_ceiling": ach / pipe_ceiling,
            "traffic_is": f"DRAM bytes (read + write) of both stages per matvec from the committed ncu summary "
                          f"profiles/{prof_file}: a chi=384 capture scaled to chi=512 by "
                          f"the vector length (T and the environments grow with it)" if traffic else None,
            "algorithmic_bytes": 32.0 * n}
    if head == "split_tf32":
        roof["tf32_issued_tflops"] = 3.0 * executed / (gemm_ms * 1e-3) / 1e12
    if head == "split_bf16":
        roof["bf16_issued_tflops"] = 3.0 * executed / (gemm_ms * 1e-3) / 1e12
    if world > 1:
        roof["stage_ms"] = {"exchange": r["st"][0], "owned_matvec": r["st"][1]}
    else:
        roof["stage_ms"] = {"gather": r["st"][0], "stage1": r["st"][1], "stage2": r["st"][2], "scatter": r["st"][3]}
    roof["flops_canonical"] = canonical
    roof["flops_executed_complex"] = executed
    # one whole matvec per step on every N: over N ranks it is split by output sector
    value = canonical / (r["ms"] * 1e-3) / 1e12
    line = {"metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": a.steps,
            "warmup": max(3, a.warmup), "ms_per_step": r["ms"], "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": {"fp64": "complex128", "split_tf32": "split-tf32 x3, fp32 accumulate",
                                           "split_bf16": "split-bf16 x3, fp32 accumulate"}[head],
            "data": "synthetic", "config": cfg,
            "e2e": {"value": canonical / r["e2e_s"] / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": 16 * r["n_io"],
                    "d2h_bytes_per_step": 16 * r["n_io"], "ms_per_step": r["e2e_s"] * 1e3},
            # ours per matvec: gather, split (split-TF32 only), two GEMM stages,
            # scatter; sharded (N > 1): no gather/scatter (theta layout)
            "gpu_launches": ((5 if head != "fp64" else 4) - (2 if world > 1 else 0)) * a.steps,
            "roofline": roof, "n_allowed": n, "clocks": r["clk"],
            "peaks_measured_live": {"cublas_zgemm_tflops": zgemm, "cublas_tf32_tflops": tf32}}
    if "fp64" in res and head != "fp64":
        f = res["fp64"]
        line["fp64_form"] = {"value": canonical / (f["ms"] * 1e-3) / 1e12, "ms_per_step": f["ms"],
                             "e2e_ms_per_step": f["e2e_s"] * 1e3,
                             "stage_ms": {"gather": f["st"][0], "stage1": f["st"][1], "stage2": f["st"][2],
                                          "scatter": f["st"][3]},
                             "roofline_frac_vs_zgemm": canonical / ((f["st"][1] + f["st"][2]) * 1e-3) / 1e12 / zgemm}
        line["speedup_mixed_vs_fp64"] = f["ms"] / r["ms"]
    line["split_forms"] = {p: {"value": canonical / (res[p]["ms"] * 1e-3) / 1e12, "ms_per_step": res[p]["ms"],
                               "e2e_ms_per_step": res[p]["e2e_s"] * 1e3,
                               "stage_ms": {"gather": res[p]["st"][0], "stage1": res[p]["st"][1],
                                            "stage2": res[p]["st"][2], "scatter": res[p]["st"][3]}}
                           for p in splits}
    line["headline_form"] = head
    if a.idmrg_steps > 0:
        line["idmrg"] = idmrg_bench(ctx, wl, a.chi, a.idmrg_steps, dist)
    if a.ising_steps > 0:
        from chainamps_b200 import (models, CMPS_FP64, CMPS_SPLIT_TF32, CMPS_SPLIT_BF16, CMPS_ORDER_AUTO,
                                    CMPS_ORDER_FOLDED)
        rules, ch, W, bq = models.coupled_ising_model(12, 1.2, 64, 0.05)
        iw = dict(rules=rules, Wt=models.mpo_tensor(ch, W, bq))
        ising = {"model": "coupled TFIM chains: 12-site periodic chain vertex, g=1.2, 64 lowest states (Z2), "
                          "J_perp=0.05 sum X_i X_i, MPO D=26",
                 "forms": {"fp64": "FP64, contraction order chosen by flops (canonical for this vertex)",
                           "mixed": "split TF32 precision (the canonical order in FP32 FMA for this vertex), FP64 "
                                    "Krylov, Rayleigh quotients and SVD",
                           "mixed_bf16": "split BF16 precision (the canonical order as four tcgen05 split-BF16 "
                                         "stages for this vertex), FP64 Krylov, Rayleigh quotients and SVD",
                           "fp64_folded": "FP64 in the reference's folded order (LeftPart . V . RightPart)"}}
        for chi in [int(c) for c in str(a.ising_chi).split(",") if c.strip()]:
            allf = {"fp64": CMPS_FP64, "mixed": CMPS_SPLIT_TF32, "mixed_bf16": CMPS_SPLIT_BF16}
            want = [f.strip() for f in str(a.ising_forms).split(",") if f.strip()]
            forms = [(f, allf[f], CMPS_ORDER_AUTO) for f in want if f in allf]
            if chi == a.ising_folded_chi:
                forms.append(("fp64_folded", CMPS_FP64, CMPS_ORDER_FOLDED))
            ising[f"chi_{chi}"] = idmrg_bench(ctx, iw, chi, a.ising_steps, dist, warm=2, forms=forms,
                                              unit_cell=False)
        line["idmrg_coupled_ising"] = ising
    if a.ising_matvec_chi:
        line["ising_matvec"] = ising_matvec_bench(
            ctx, [int(c) for c in str(a.ising_matvec_chi).split(",") if c.strip()], dist, stream)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        t, setup, cores, _ = cpu_port(wl, 1)
        line["cpu_baseline"] = {"value": canonical / t / 1e12, "unit": "TFLOP/s", "cores": cores, "kind": "port",
                                "sample": "one full matvec of the same workload (oracle block-sparse numpy port)",
                                "seconds": t}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


def ising_matvec_bench(ctx, chis, dist, stream, reps=5):
    """The coupled-Ising H_eff matvec alone, on synthetic Z2 environments
    (``models.ising_workload``, seed 20261203), in each form: FP64 (canonical
    order), split TF32 (canonical order in FP32 FMA) and split BF16
    (canonical order as four tcgen05 stages).  ms per matvec is the sum of
    the library's stage events (gather, first half, second half, scatter;
    mean of ``reps``), max over ranks; canonical TFLOP/s; and the largest
    deviation from the FP64 matvec relative to its largest entry."""
    import torch
    from chainamps_b200 import models, TwoVertexComponents, CMPS_FP64, CMPS_SPLIT_TF32, CMPS_SPLIT_BF16
    out = {}
    for chi in chis:
        wl = models.ising_workload(chi)
        res, ref = {}, None
        for name, prec in (("fp64", CMPS_FP64), ("split_tf32", CMPS_SPLIT_TF32), ("split_bf16", CMPS_SPLIT_BF16)):
            h = TwoVertexComponents(ctx, wl["rules"], wl["L"], wl["Wt"], wl["R"], precision=prec)
            x = torch.randn(h.n, dtype=torch.complex128, device="cuda", generator=torch.Generator("cuda").manual_seed(7))
            y = torch.empty_like(x)
            st = h.time_stages(x.data_ptr(), y.data_ptr(), stream.cuda_stream, reps=reps)
            torch.cuda.synchronize()
            h.status()
            ms_t = torch.tensor([float(np.sum(st))], device="cuda", dtype=torch.float64)
            if dist:
                dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
            can, exe = h.flops()
            r = {"ms_per_matvec": float(ms_t.item()), "canonical_tflops": can / (float(ms_t.item()) * 1e-3) / 1e12,
                 "stage_ms": [float(v) for v in st], "split_form": h.split_form()}
            if ref is None:
                ref = y.clone()
            else:
                r["max_dev_vs_fp64"] = float((y - ref).abs().max() / ref.abs().max())
            res[name] = r
            del h
        res["n_allowed"] = int(ref.numel())
        res["speedup_bf16_vs_fp64"] = res["fp64"]["ms_per_matvec"] / res["split_bf16"]["ms_per_matvec"]
        out[f"chi_{chi}"] = res
    return out


def idmrg_bench(ctx, wl, chi, steps, dist, warm=3, tol=1e-10, unit_cell=True, forms=None):
    """iDMRG growth on the ladder MPO in FP64 and in mixed precision: `warm`
    untimed steps bring the bond dimension to chi, then `steps` timed ones.
    Step time is the library's device time of the whole step (environment
    update, H_eff build, prediction, eigensolve, SVD; CUDA events), the
    median over the timed steps, max over ranks.  unit_cell: after the FP64 run, the unit cell of its last step
    (energy per vertex, entropy, time)."""
    import torch
    from chainamps_b200 import iDMRG, CMPS_FP64, CMPS_SPLIT_TF32, CMPS_SPLIT_BF16, CMPS_ORDER_AUTO
    out = {"chi": chi, "warmup_steps": warm, "timed_steps": steps, "arnoldi_tol": tol, "krylov_dim": 24}
    energies = {}
    if forms is None:
        forms = [("fp64", CMPS_FP64, CMPS_ORDER_AUTO), ("mixed", CMPS_SPLIT_TF32, CMPS_ORDER_AUTO),
                 ("mixed_bf16", CMPS_SPLIT_BF16, CMPS_ORDER_AUTO)]
    for name, prec, order in forms:
        # map most of the free device memory into the library's pool before
        # the run (setup, untimed), so that steps whose buffers outgrow the
        # previous ones do not pay for mapping memory; returned after the run
        torch.cuda.empty_cache()
        ctx.reserve(int(0.6 * torch.cuda.mem_get_info()[0]))
        run = iDMRG(ctx, wl["rules"], wl["Wt"], precision=prec, tol=tol, krylov_dim=24, order=order)
        e, prof, wall = [], [], []
        for i in range(warm + steps):
            t0 = time.perf_counter()
            r = run.grow(chi, 1e-16)
            dt = time.perf_counter() - t0
            e.append(r["energy"])
            if i >= warm:
                prof.append(run.profile())
                wall.append(dt)
        if name == "fp64" and unit_cell:
            # Orthogonalise + iTwoVertexEnergy of the last step (iDMRG_DRV's
            # per-step measurement), timed on the host (it synchronises)
            t0 = time.perf_counter()
            uc = run.unit_cell(tol=1e-12, krylov_dim=30)
            out["unit_cell"] = dict(uc, ms=1e3 * (time.perf_counter() - t0))
        run.close()
        ctx.reserve(0)
        torch.cuda.empty_cache()
        # median over the timed steps: a host-side stall in one step (allocator
        # growth, a busy host) would otherwise dominate a mean over few steps
        ms = float(np.median([p["total_ms"] for p in prof]))
        ms_t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        if dist:
            dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
        keys = [k for k in prof[0] if k != "total_ms"]
        out[name] = {"ms_per_step": float(ms_t.item()), "ms_per_step_mean": float(np.mean([p["total_ms"] for p in prof])),
                     "host_ms_per_step": 1e3 * float(np.mean(wall)),
                     "chi": r["chi"], "energy_last": e[-1],
                     "profile_median": {k: float(np.median([p[k] for p in prof])) for k in keys},
                     "profile_mean": {k: float(np.mean([p[k] for p in prof])) for k in keys}}
        energies[name] = np.array(e)
    if "mixed" in out and "fp64" in out:
        rel = np.abs(energies["mixed"] - energies["fp64"]) / np.abs(energies["fp64"])
        out["max_rel_dE_mixed_vs_fp64"] = float(rel.max())
        out["speedup_mixed_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    if "mixed_bf16" in out and "fp64" in out:
        rel = np.abs(energies["mixed_bf16"] - energies["fp64"]) / np.abs(energies["fp64"])
        out["max_rel_dE_mixed_bf16_vs_fp64"] = float(rel.max())
        out["speedup_mixed_bf16_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed_bf16"]["ms_per_step"]
    if "fp64_folded" in out:
        rel = np.abs(energies["fp64_folded"] - energies["fp64"]) / np.abs(energies["fp64"])
        out["max_rel_dE_folded_vs_fp64"] = float(rel.max())
        for f in ("mixed", "mixed_bf16"):
            if f in out:
                out[f"speedup_{f}_vs_fp64_folded"] = out["fp64_folded"]["ms_per_step"] / out[f]["ms_per_step"]
        out["speedup_fp64_vs_fp64_folded"] = out["fp64_folded"]["ms_per_step"] / out["fp64"]["ms_per_step"]
    return out


def canonical_flops_cpu(wl):
    """Canonical four-stage flop count of the workload, computed on the host
    from the same sector structure the library uses (no GPU needed)."""
    from oracle import blocks as ob
    chi = wl["bond"].shape[0]
    bh = ob.BondSectors(wl["bond"])
    rules = wl["rules"]
    sig = [tuple(int(x) for x in q) for q in wl["ch"]]
    d = len(sig)
    W = wl["W"]
    bq = [tuple(int(x) for x in q) for q in wl["bq"]]
    add = lambda p, q: tuple(x + y for x, y in zip(p, q))
    sub = lambda p, q: tuple(x - y for x, y in zip(p, q))
    dims = {k: bh.dim(k) for k in bh.keys}
    ms = sorted({add(s, k) for s in sig for k in bh.keys} & {sub(k, s) for s in sig for k in bh.keys})
    nrows = {m: sum(dims.get(sub(m, s), 0) for s in sig) for m in ms}
    ncols = {m: sum(dims.get(add(m, s), 0) for s in sig) for m in ms}
    nz = np.argwhere(W != 0)
    bl_used = sorted({int(b) for b in nz[:, 1]})
    br_used = sorted({int(b) for b in nz[:, 3]})
    f = 0.0
    for m in ms:
        for s1 in range(d):
            k = sub(m, sig[s1])
            if k not in dims:
                continue
            for b0 in bl_used:
                kp = add(k, bq[b0])
                if kp in dims:
                    f += 8.0 * dims[kp] * dims[k] * ncols[m]
            for sp, b0, s, b1 in nz:
                if s != s1:
                    continue
                kp = add(k, bq[b0])
                if kp in dims:
                    f += 8.0 * dims[kp] * ncols[m]
        for s2 in range(d):
            t = add(m, sig[s2])
            if t not in dims:
                continue
            for sp, b1, s, b2 in nz:
                if s != s2:
                    continue
                mp = add(m, bq[b1])
                if mp in nrows:
                    f += 8.0 * nrows[mp] * dims[t]
            for b2 in br_used:
                tp = add(t, bq[b2])
                if tp in dims:
                    f += 8.0 * nrows[m] * dims[t] * dims[tp]
    return f


if __name__ == "__main__":
    sys.exit(main())
