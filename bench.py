"""Benchmark of the fem25 hot path on B200.

Headline workload (one step): the batched assembly of 512 complex128 CSR
systems (8 frequencies 0.2-1.6 Hz x 64 ky) of the 400x120 degree-4 mesh of a
layered model into a ring of 32 slots (--nslots) -- the "CSR assemblies/s"
half of the metric.  With N ranks every rank assembles 512 systems of its
own (its frequencies offset by r * 0.2 / N Hz): weak scaling, no data-path
collective (the (omega, py) systems are independent).  Inputs (the per-mesh
basis, 2.6 GB) and outputs (3.98 GB per system) are larger than L2, so no
flush is needed.

Also reported on the same line:
  * plain_fp64: the per-(omega, py) FP64 element + gather kernels (systems/s)
  * e2e: ASMBLE_DRIVER through the C ABI with host buffers (model upload from
    pinned memory, COMPLEX*8 CDIST read back to pinned memory) -- systems/s
  * model_update_step: fem25_update_model + one batch that rebuilds the basis
  * gradient: exact adjoint gradient, elem.rhs/s, 400x120 layered mesh, 32
    sources x 2 pairs of seeded smooth fields: FP64; split precision in the
    covariance form (one-shot call, and its accumulation and contraction
    kernels apart, with an HBM roofline of the accumulation) and in the
    pointwise form (tensor roofline); per-parameter error against FP64
  * sparse_solve: the GPU multifrontal direct solve of one 400x120 system
    (the MUMPS hop of the reference): factorisation time and flop rate,
    solves with A and A^H for 1 and 32 right-hand sides, residual
  * split_precision: the 300x150 jittered workload, 128 sources, 2 of its
    1152 pairs: elem.rhs/s of the three gradient kernels and the per-
    parameter error of both split-precision forms against FP64
  * pipeline: the uneven-batch workload (600x200 jittered mesh with
    topography, 24 frequencies 0.1-2.4 Hz x ceil(16 f / 0.1) ky = 4800 systems,
    64 sources): batched assembly + split-precision covariance accumulation per
    two pairs + one contraction, measured in one CUDA graph over all 4800 pairs,
    against the plain per-(omega, py) FP64 assembly (reference arithmetic and
    FMA build) + FP64 gradient per pair (sampled, scaled); sharded over ranks
    with one NCCL all-reduce when N > 1
  * roofline of the streaming kernel and the CPU baseline (the oracle).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CSR assemblies/s & gradient elem·rhs/s, batched-TF32x3 vs plain FP64 at 1e-6 rel"
# streaming-kernel variant index (fem25_tuning) -> kernel
STREAM_KERNELS = {0: "k_stream<1>", 1: "k_stream<2>", 2: "k_stream<4>", 3: "k_stream_pipe",
                  4: "k_stream_tma<64>", 5: "k_stream_tma<128>", 6: "k_stream_ring<256, 4>",
                  7: "k_stream_ring<512, 4>", 8: "k_stream_big<512, 4>", 9: "k_stream_big<256, 4>"}
UNIT = "assemblies/s"
# DRAM traffic of k_stream_big<512, 4> from one ncu capture of the 100x40
# layout of the same 400x120 layered mesh (NNZ 20 418 489), 16 systems per
# launch: 329.8 MB read (the entry basis and block terms, once per launch)
# and 5.168 GB written (the values; the last ~60 MB still in L2 at kernel end)
STREAM_BIG_READ_PER_ENTRY = 329.8e6 / 20418489           # bytes per CSR entry and launch
STREAM_BIG_WRITE_PER_ENTRY = 5.168e9 / (16 * 20418489)   # bytes per CSR entry and system


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def bf16_peak():
    """Dense bf16 tensor peak (TFLOP/s, burst) of this pool's B200s."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, dev):
        self.dev = dev
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(dev), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for k, n in enumerate(names):
                if "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(rows)}


def headline_config(nelem, ndof, nz, nsys):
    """The workload of the headline step, identical in both arms."""
    return {"workload": f"batched assembly, 400x120 deg-4 layered-model mesh ({nelem} elements, "
                        f"NDOF {ndof}, NNZ {nz}), 8 f x 64 ky = {nsys} complex128 CSR systems "
                        f"per step",
            "systems_per_step": nsys, "nelem": nelem, "ndof": ndof, "nnz": nz,
            "l2": "inputs (basis 2.6 GB) and outputs (4 GB per system) larger than L2; no flush"}


class CpuSampler:
    """The oracle's ASMBLE_DRIVER restatement (COMPLEX*8 CDIST with the
    reference's FP64 element matrices and FP32 accumulation, the output
    ASMBLE_DRIVER produces) on all host cores.  A persistent spawn pool: each
    worker builds the mesh and the oracle's own graph once, then every sample
    has each worker assemble a contiguous slice of elements of a different
    (omega, py) system into its preallocated CDIST; the rate is scaled to
    whole systems by elements."""

    def __init__(self, cfg_idx, workers=None):
        import multiprocessing as mp
        self.cfg = cfg_idx
        self.workers = workers or os.cpu_count()
        self.pool = mp.get_context("spawn").Pool(self.workers)
        r = self.pool.map(_cpu_worker, [(cfg_idx, w, 64) for w in range(self.workers)])
        self.nelem, self.ndof, self.nz = r[0][1:4]
        self.t_elem = max(sum(x[0] for x in r) / (64.0 * self.workers), 1e-9)
        # whether any worker process had this library's libfem25gpu.so mapped
        self.product_loaded = any(x[4] for x in r)

    def sample(self, seconds):
        per = int(max(16, min(self.nelem, seconds / self.t_elem)))
        t0 = time.perf_counter()
        r = self.pool.map(_cpu_worker, [(self.cfg, w, per) for w in range(self.workers)])
        wall = time.perf_counter() - t0
        self.product_loaded = self.product_loaded or any(x[4] for x in r)
        done = per * self.workers
        return {"value": done / self.nelem / wall, "unit": UNIT, "cores": self.workers,
                "kind": "port", "wall_s": wall,
                "sample": f"{done} of {self.nelem} elements per sample (one slice per core, each "
                          f"of a different (omega, py) system of the 400x120 mesh), oracle "
                          f"ASMBLE_DRIVER restatement (COMPLEX*8 CDIST), {wall:.1f} s wall, "
                          f"scaled to whole systems by elements"}

    def close(self):
        self.pool.close()
        self.pool.join()


_CPU_CACHE = {}


def _cpu_worker(arg):
    cfg_idx, w, per = arg
    import numpy as np
    import oracle
    from fem25_b200 import synth
    if cfg_idx not in _CPU_CACHE:
        mesh, pairs, _ = synth.make_config(cfg_idx)
        g = oracle.graph_build(mesh)
        _CPU_CACHE[cfg_idx] = (mesh, pairs, g, np.zeros(g.nzero, np.complex64))
    mesh, pairs, g, cdist = _CPU_CACHE[cfg_idx]
    f, py = pairs[(w * 37) % len(pairs)]
    lo = (w * 997) % max(1, mesh.nelem - per)
    t0 = time.perf_counter()
    oracle.asmble(mesh, g, "B", f, py, elo=lo, ehi=min(mesh.nelem, lo + per), out=(None, cdist))
    return time.perf_counter() - t0, mesh.nelem, g.ndof, g.nzero, _product_mapped()


def _product_mapped():
    """True if this process has libfem25gpu.so mapped (Linux /proc)."""
    try:
        with open("/proc/self/maps") as f:
            return "libfem25gpu" in f.read()
    except OSError:
        return False


def run_reference(args, rank):
    """The reference's own CPU path for the headline workload: the oracle's
    restatement of ASMBLE_DRIVER (the Fortran reference cannot be compiled in
    this image) on every host core of rank 0; each step is a bounded sample."""
    if rank != 0:
        return
    smp = CpuSampler(1)
    for _ in range(max(1, args.warmup)):
        smp.sample(1.0)
    vals, walls, base = [], [], None
    for _ in range(args.steps):
        base = smp.sample(4.0)
        vals.append(base["value"])
        walls.append(base["wall_s"])
    smp.close()
    product_loaded = smp.product_loaded or _product_mapped()
    v = statistics.mean(vals)
    base["value"] = v
    nsys = 512
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": max(1, args.warmup),
           "ms_per_step": statistics.mean(walls) * 1e3,
           "ms_per_step_note": "wall time of one bounded sample step (a slice of elements of one "
                               "system per core); value scales the sample to whole systems by "
                               f"elements; a whole {nsys}-system step would take "
                               f"{nsys / v:.0f} s",
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded layered model; no public dataset exists for this path)",
           "config": headline_config(smp.nelem, smp.ndof, smp.nz, nsys),
           "parallelism": f"{smp.workers} host processes on rank 0",
           "cpu_baseline": base,
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "product_library_loaded": product_loaded}
    print(json.dumps(out))


def _timer(torch, stream):
    """fn -> best device seconds of ``reps`` runs, CUDA events on ``stream``."""
    def timed(fn, reps=1):
        best = None
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        return best / 1e3
    return timed


def _per_param(torch, got, ref):
    """relative 2-norm error per parameter (lambda, mu, rho)."""
    return [float(torch.linalg.norm(got[m] - ref[m]) / torch.linalg.norm(ref[m])) for m in range(3)]


def pipeline_uneven(local, dev, rank=0, world=1, max_over_ranks=None):
    """The target comparison on the uneven-batch workload (600x200 jittered
    mesh with +-200 m topography, 4-element strip, 24 frequencies 0.1-2.4 Hz,
    nky = ceil(16 f / 0.1): 4800 (omega, py) systems, 64 sources).

    Batched split-precision side, measured end to end: one CUDA graph holds
    the batched assembly of every system of this rank (ring of 8 complex128
    slots), one covariance accumulation (fem25_gradient_accumulate_dev) per
    two pairs with their 64 source fields each (two pairs' solutions held at
    a time; a pool of 2 field sets of the adjoint-gradient kind, reused: the
    operator and the kernels do not depend on the values), and the
    contraction (fem25_gradient_finalize_dev); the
    graph is replayed once under CUDA events.  With several ranks the pairs
    are sharded longest-processing-time first and the FP64 gradients summed
    by one NCCL all-reduce, timed apart.
    Plain side (sampled): the per-(omega, py) FP64 assembly of the middle ky
    of each frequency, in the reference arithmetic (-fmad=false) and with the
    FMA build of the same kernels, plus the FP64 gradient of one pair with 64
    sources; per-system and per-pair costs do not depend on the pair and are
    scaled to the 4800 pairs.
    Accuracy: per-parameter error of both split-precision forms against the
    FP64 kernel on one pair; sampled rows (every DOF class, free surface) of
    the last batched system against the plain FP64 assembly."""
    import torch
    from fem25_b200 import (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE,
                            Context, graph_build, synth)
    from fem25_b200.parallel import pair_costs, shard_lpt
    mesh, pairs, cfg = synth.make_config(4)
    nsrc = cfg["nsrc"]
    npairs = len(pairs)
    freqs = [p[0] for p in pairs]
    pys = [p[1] for p in pairs]
    mine = shard_lpt(pair_costs(freqs, nsrc), world)[rank]
    stream = torch.cuda.current_stream(dev)
    timed = _timer(torch, stream)
    t0 = time.perf_counter()
    g = graph_build(mesh)
    # a pool of 2 field sets [pair][64 sources][NDOF] (u and lambda)
    pool_pairs = [pairs[npairs // 3], pairs[(2 * npairs) // 3]]
    pool_u = synth.smooth_fields(mesh, g, pool_pairs, nsrc, seed=4041, device=dev)
    pool_l = synth.smooth_fields(mesh, g, pool_pairs, nsrc, seed=4042, device=dev)
    rows = None
    if rank == 0:
        import numpy as np
        rng = np.random.default_rng(4)
        cnp = np.asarray(g.cnp)
        rows = [1, g.ndof]
        for c in b"AEIB":
            cand = np.nonzero(cnp == c)[0] + 1
            rows += [int(r) for r in rng.choice(cand, min(12, len(cand)), replace=False)]
        rows = np.array(sorted(set(rows)), np.int64)
        lens = g.irptr[rows] - g.irptr[rows - 1]
        ridx = torch.from_numpy(np.concatenate(
            [np.arange(a - 1, a - 1 + n) for a, n in zip(g.irptr[rows - 1], lens)])).to(dev)

    # ---------------- plain side (sampled) and the accuracy reference
    ctx = Context(mesh, g, device=local)
    setup_s = time.perf_counter() - t0
    nz, ndof = ctx.nzero, ctx.ndof
    plain = torch.empty(nz, dtype=torch.complex128, device=dev)
    sel = []
    for f in cfg["freqs"]:
        idx = [i for i, p in enumerate(pairs) if p[0] == f]
        sel.append(idx[len(idx) // 2])
    ctx.assemble("B", freqs[sel[0]], pys[sel[0]], plain, None, stream=stream)
    torch.cuda.synchronize()
    t_pasm = timed(lambda: [ctx.assemble("B", freqs[i], pys[i], plain, None, stream=stream)
                            for i in sel]) / len(sel)
    ctx.plain_fma(True)
    ctx.assemble("B", freqs[sel[0]], pys[sel[0]], plain, None, stream=stream)
    torch.cuda.synchronize()
    t_pasm_fma = timed(lambda: [ctx.assemble("B", freqs[i], pys[i], plain, None, stream=stream)
                                for i in sel]) / len(sel)
    ctx.plain_fma(False)
    klast = mine[-1] if mine else npairs - 1
    plain_rows = None
    if rank == 0:
        ctx.assemble("B", freqs[klast], pys[klast], plain, None, stream=stream)
        plain_rows = plain[ridx].clone()
    del plain
    torch.cuda.empty_cache()
    gp = pool_pairs[0]
    u1, l1 = pool_u[:1], pool_l[:1]
    g64 = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=dev)
    gcv = torch.zeros_like(g64)
    gpw = torch.zeros_like(g64)
    ctx.gradient([gp[0]], [gp[1]], nsrc, u1, l1, g64, FEM25_PREC_FP64, stream=stream)
    ctx.gradient([gp[0]], [gp[1]], nsrc, u1, l1, gpw, FEM25_PREC_TF32X3_POINTWISE, stream=stream)
    torch.cuda.synchronize()

    def run_grad(out, prec):
        out.zero_()
        ctx.gradient([gp[0]], [gp[1]], nsrc, u1, l1, out, prec, stream=stream)
    t_g64 = timed(lambda: run_grad(g64, FEM25_PREC_FP64), reps=2)
    t_gpw = timed(lambda: run_grad(gpw, FEM25_PREC_TF32X3_POINTWISE), reps=2)
    run_grad(gcv, FEM25_PREC_TF32X3)
    ctx.sync_status(stream)
    err_cov = _per_param(torch, gcv, g64)
    err_pw = _per_param(torch, gpw, g64)
    del g64, gcv, gpw
    tuned_plain = ctx.tuning()
    ctx.close()
    torch.cuda.empty_cache()

    # ---------------- batched side: one CUDA graph, replayed once
    ctx = Context(mesh, g, device=local)
    nslots = 8
    sst = (2 * nz + 15) // 16 * 16  # 128-byte aligned ring slots
    ring = torch.empty(nslots * sst, dtype=torch.float64, device=dev)
    gsum = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=dev)
    # set-up calls outside the graph: basis, variant timing, the PML deltas
    # of every frequency, accumulators
    one_per_f = sorted({freqs[k]: k for k in (mine or [0])}.values())
    ctx.assemble_batch("B", [freqs[k] for k in one_per_f], [pys[k] for k in one_per_f], ring, sst,
                       nslots, stream=stream)
    ctx.gradient_accumulate([gp[0]], [gp[1]], nsrc, u1, l1, stream=stream)
    ctx.gradient_finalize(gsum, stream=stream)
    torch.cuda.synchronize()
    # the accumulation (per pair, in the graph's grouping) and the
    # contraction, eager, for the record
    acc_group = 2
    gf = [p[0] for p in pool_pairs[:acc_group]]
    gy = [p[1] for p in pool_pairs[:acc_group]]
    t_acc1 = timed(lambda: ctx.gradient_accumulate([gp[0]], [gp[1]], nsrc, u1, l1, stream=stream),
                   reps=3)
    t_acc = timed(lambda: ctx.gradient_accumulate(gf, gy, nsrc, pool_u[:acc_group],
                                                  pool_l[:acc_group], stream=stream),
                  reps=3) / acc_group
    t_fin = timed(lambda: ctx.gradient_finalize(gsum, stream=stream))
    ctx.sync_status(stream)
    gsum.zero_()
    mine_f = [freqs[k] for k in mine]
    mine_p = [pys[k] for k in mine]
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(stream)
    nlaunch = 0
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            cur = torch.cuda.current_stream(dev)
            if mine:
                ctx.assemble_batch("B", mine_f, mine_p, ring, sst, nslots, stream=cur)
            # the pairs' fields two at a time (two pairs' solutions held), so
            # each element's FP64 accumulators are read and written once per
            # two pairs
            for j in range(0, len(mine), acc_group):
                ks = mine[j:j + acc_group]
                ctx.gradient_accumulate([freqs[k] for k in ks], [pys[k] for k in ks], nsrc,
                                        pool_u[:len(ks)], pool_l[:len(ks)], stream=cur)
            ctx.gradient_finalize(gsum, stream=cur)
    stream.wait_stream(side)
    torch.cuda.synchronize()
    t_graph = timed(graph.replay)
    ctx.sync_status(stream)
    tuned = ctx.tuning()
    t_allreduce = 0.0
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        t_allreduce = timed(lambda: dist.all_reduce(gsum, op=dist.ReduceOp.SUM))
    t_job = t_graph + t_allreduce
    if max_over_ranks is not None:
        t_job = max_over_ranks(t_job)
    csr_rel = None
    if rank == 0 and mine:
        import numpy as np
        k = len(mine) - 1
        slot = ring[(k % nslots) * sst:(k % nslots) * sst + 2 * nz].view(-1, 2)[ridx]
        b = torch.complex(slot[:, 0], slot[:, 1])
        d = (b - plain_rows).abs().cpu().numpy()
        r = plain_rows.abs().cpu().numpy()
        lens = (g.irptr[rows] - g.irptr[rows - 1]).astype(np.int64)
        st = np.concatenate([[0], np.cumsum(lens)[:-1]])
        csr_rel = float((np.maximum.reduceat(d, st) / np.maximum.reduceat(r, st)).max())
    del graph, ring, pool_u, pool_l
    ctx.close()
    torch.cuda.empty_cache()
    # kernel nodes: PML deltas (2 per frequency), streaming launches (one per
    # ring of systems), per accumulation call the field-scale and covariance
    # kernels, the contraction
    n_launch = (len(set(mine_f)) * 2 + -(-len(mine) // nslots) + 2 * -(-len(mine) // acc_group)
                + 1)
    units = mesh.nelem * nsrc
    out = {"workload": f"uneven batch: 600x200 jittered deg-4 mesh with topography, strip 4 "
                       f"({mesh.nelem} elements, NDOF {ndof}, NNZ {nz}), "
                       f"24 f x ceil(16 f/0.1) ky = {npairs} systems, {nsrc} sources",
           "batched_measured_s": t_job, "batched_graph_s": t_graph,
           "batched_form": "one CUDA graph: batched assembly of every system + one covariance "
                           "accumulation per two (omega, py) pairs (64 sources each) + one "
                           "contraction",
           "pairs_this_rank": len(mine), "allreduce_s": t_allreduce,
           "gradient_tf32x3_s_per_pair": t_acc, "gradient_tf32x3_pairs_per_call": acc_group,
           "gradient_tf32x3_s_one_pair_per_call": t_acc1, "gradient_tf32x3_contraction_s": t_fin,
           "gradient_tf32x3_elem_rhs_per_s": units / t_acc,
           "plain_assembly_s_per_system": t_pasm, "plain_assembly_fma_s_per_system": t_pasm_fma,
           "gradient_fp64_s_per_pair": t_g64, "gradient_tf32x3_pointwise_s_per_pair": t_gpw,
           "gradient_fp64_elem_rhs_per_s": units / t_g64,
           "gradient_rel_err_vs_fp64": {"covariance (lambda, mu, rho)": err_cov,
                                        "pointwise (lambda, mu, rho)": err_pw},
           "csr_rel_err_batched_vs_plain_rows": csr_rel,
           "graph_kernel_launches": n_launch,
           "setup_s": round(setup_s, 1), "autotuned": tuned, "autotuned_plain": tuned_plain}
    if world == 1:
        plain_total = (t_pasm + t_g64) * npairs
        plain_total_fma = (t_pasm_fma + t_g64) * npairs
        out.update({"plain_fp64_s": plain_total, "plain_fp64_fma_s": plain_total_fma,
                    "speedup_measured": plain_total / t_job,
                    "speedup_measured_vs_fma_plain": plain_total_fma / t_job,
                    # the pointwise form keeps <= 1e-6 in lambda on solved fields too
                    "speedup_pointwise_estimate": plain_total / max(
                        t_job - npairs * t_acc - t_fin + npairs * t_gpw, 1e-9),
                    "speedup_pointwise_note": "the measured graph with each pair's covariance "
                                              "accumulation (and the contraction) replaced by "
                                              "the pointwise kernel's measured time per pair",
                    "sample": f"batched: all {npairs} systems and pairs measured in one graph; "
                              f"plain: assembly of 1 system per frequency ({len(sel)}) and the "
                              f"FP64 gradient of 1 pair x {nsrc} sources, scaled to {npairs} "
                              f"pairs"})
    return out


def split_precision_leg(local, dev):
    """The split-precision contraction workload (300x150 jittered mesh,
    128 sources, a sample of its 96 ky x 12 f pairs): elem.rhs/s of the FP64
    kernel and of both split-precision forms, and their relative error
    against FP64 per parameter, on seeded smooth fields of the adjoint-
    gradient kind (unit RMS, lognormal amplitude, 5 km-correlated phase)."""
    import torch
    from fem25_b200 import (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE,
                            Context, graph_build, synth)
    mesh, pairs, cfg = synth.make_config(3)
    nsrc = cfg["nsrc"]
    g = graph_build(mesh)
    ctx = Context(mesh, g, device=local)
    stream = torch.cuda.current_stream(dev)
    timed = _timer(torch, stream)
    use = [pairs[96 * 2 + 80], pairs[96 * 9 + 30]]  # (0.6 Hz, high ky), (2.0 Hz, low ky)
    u = synth.smooth_fields(mesh, g, use, nsrc, seed=3031, device=dev)
    lam = synth.smooth_fields(mesh, g, use, nsrc, seed=3032, device=dev)
    fr, py = [p[0] for p in use], [p[1] for p in use]
    res = {}
    outs = {}
    for name, prec in (("fp64", FEM25_PREC_FP64), ("tf32x3_covariance", FEM25_PREC_TF32X3),
                       ("tf32x3_pointwise", FEM25_PREC_TF32X3_POINTWISE)):
        out = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=dev)
        ctx.gradient(fr, py, nsrc, u, lam, out, prec, stream=stream)  # set-up / tuning

        def run():
            out.zero_()
            ctx.gradient(fr, py, nsrc, u, lam, out, prec, stream=stream)
        t = timed(run, reps=2)
        ctx.sync_status(stream)
        outs[name] = out
        res[name] = {"s": t, "elem_rhs_per_s": mesh.nelem * nsrc * len(use) / t}
    for name in ("tf32x3_covariance", "tf32x3_pointwise"):
        res[name]["rel_err_vs_fp64"] = dict(zip(("lambda", "mu", "rho"),
                                                _per_param(torch, outs[name], outs["fp64"])))
    # the covariance form's two kernels: accumulation per pair, contraction once
    acc = timed(lambda: ctx.gradient_accumulate(fr, py, nsrc, u, lam, stream=stream), reps=2)
    tmp = torch.zeros_like(outs["fp64"])
    fin = timed(lambda: ctx.gradient_finalize(tmp, stream=stream))
    ctx.sync_status(stream)
    res["tf32x3_covariance"]["accumulate_s_per_pair"] = acc / len(use)
    res["tf32x3_covariance"]["contraction_s"] = fin
    res["tf32x3_covariance"]["full_workload_s_estimate"] = acc / len(use) * len(pairs) + fin
    res["fp64"]["full_workload_s_estimate"] = res["fp64"]["s"] / len(use) * len(pairs)
    del u, lam, outs, tmp
    ctx.close()
    torch.cuda.empty_cache()
    return {"workload": f"split-precision contraction: 300x150 jittered deg-4 mesh "
                        f"({mesh.nelem} elements, NDOF {g.ndof}), {nsrc} sources, "
                        f"{len(pairs)} (omega, py) pairs (12 f x 96 ky)",
            "sample": f"{len(use)} pairs x {nsrc} sources measured (f = {use[0][0]:.1f} and "
                      f"{use[1][0]:.1f} Hz); full-workload times scale per pair",
            "fields": "seeded smooth fields: unit RMS per (pair, source), lognormal(0, 0.1) "
                      "amplitude, exp(i (omega x / 2500 m/s + phi)), phi 5 km-correlated",
            "units": "elem.rhs = element x source x (omega, py) pair", **res}


def sparse_solve_leg(local, dev):
    """The GPU sparse direct solve on one system of the 400x120 layered mesh
    (the solver hop the reference hands to MUMPS): analysis, factorisation
    (time and FP64 flop rate from the fronts' sizes), solves with A and A^H
    for 1 and 32 right-hand sides, and the residual ||op(A) x - b|| / ||b||
    (A x by a cuSPARSE product of the same CSR)."""
    import numpy as np
    import torch
    from fem25_b200 import Context, graph_build, synth
    mesh, pairs, _ = synth.make_config(1)
    g = graph_build(mesh)
    ctx = Context(mesh, g, device=local)
    stream = torch.cuda.current_stream(dev)
    a = torch.zeros(g.nzero, dtype=torch.complex128, device=dev)
    f, py = pairs[len(pairs) // 2]
    ctx.assemble("B", f, py, a, stream=stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.sparse_factor(a, stream=stream)  # analysis (host) + first factorisation
    first = time.perf_counter() - t0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    # the second factorisation and the first solve form the profiler range
    # (ncu --profile-from-start off)
    torch.cuda.profiler.start()
    ev[0].record(stream)
    ctx.sparse_factor(a, stream=stream)
    ev[1].record(stream)
    torch.cuda.synchronize()
    fac = ev[0].elapsed_time(ev[1]) / 1e3
    fronts, levels, fbytes, wbytes, kmax, nmax, flops = ctx.sparse_info()
    crow = torch.from_numpy(g.irptr.astype(np.int64) - 1).to(dev)
    col = torch.from_numpy(g.jcptr.astype(np.int64) - 1).to(dev)
    A = torch.sparse_csr_tensor(crow, col, a, (g.ndof, g.ndof))
    gen = torch.Generator(device=dev)
    gen.manual_seed(7)
    solves = {}
    for nrhs in (1, 32):
        b = torch.randn((nrhs, g.ndof), dtype=torch.complex128, device=dev, generator=gen)
        for trans, name in ((0, "A"), (2, "A^H")):
            x = b.clone()
            ev[0].record(stream)
            ctx.sparse_solve(x, trans, stream=stream)
            ev[1].record(stream)
            torch.cuda.synchronize()
            torch.cuda.profiler.stop()
            entry = {"ms": ev[0].elapsed_time(ev[1])}
            if trans == 0:  # residual of A (A^H x checked in the tests)
                r = (A @ x.T).T - b
                entry["rel_residual"] = float(torch.linalg.norm(r) / torch.linalg.norm(b))
            solves[f"{name}, {nrhs} rhs"] = entry
    del A, crow, col
    # split-precision gradient error on solved fields: 32 vertical point
    # forces at seeded surface positions, the adjoint of random residuals at
    # 20 surface receivers (3 components), both solved with this factorisation
    from fem25_b200 import FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE
    x, z = synth.dof_coords(mesh, g)
    top = np.flatnonzero((z >= z.max() - 1e-6) & (np.arange(g.ndof) % 3 == 2))  # z DOFs
    rng = np.random.default_rng(2027)
    nsrc = 32
    src_dofs = rng.choice(top, nsrc, replace=False)
    rec = top[np.linspace(0, len(top) - 1, 20).round().astype(int)]
    rec = np.concatenate([rec - 2, rec - 1, rec])  # x, y, z components of each receiver node
    u = torch.zeros((nsrc, g.ndof), dtype=torch.complex128, device=dev)
    u[torch.arange(nsrc), torch.from_numpy(src_dofs).to(dev)] = 1.0
    ctx.sparse_solve(u, 0, stream=stream)
    rdofs = torch.from_numpy(rec).to(dev)
    obs = torch.complex(torch.randn((nsrc, len(rec)), dtype=torch.float64, generator=gen, device=dev),
                        torch.randn((nsrc, len(rec)), dtype=torch.float64, generator=gen, device=dev))
    lam = torch.zeros_like(u)
    lam[:, rdofs] = obs * 1e-10 - u[:, rdofs]
    ctx.sparse_solve(lam, 2, stream=stream)
    grads = {}
    for name, prec in (("fp64", FEM25_PREC_FP64), ("covariance", FEM25_PREC_TF32X3),
                       ("pointwise", FEM25_PREC_TF32X3_POINTWISE)):
        out = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=dev)
        ctx.gradient([f], [py], nsrc, u.view(1, nsrc, -1), lam.view(1, nsrc, -1), out, prec,
                     stream=stream)
        grads[name] = out
    torch.cuda.synchronize()
    solved_err = {name: dict(zip(("lambda", "mu", "rho"), _per_param(torch, grads[name], grads["fp64"])))
                  for name in ("covariance", "pointwise")}
    del u, lam, grads, a
    ctx.close()
    torch.cuda.empty_cache()
    return {"workload": f"one system (f = {f:.2f} Hz) of the 400x120 layered mesh, NDOF {g.ndof}, "
                        f"NNZ {g.nzero}, complex128",
            "method": "multifrontal LU, nested dissection of the elements, partial pivoting "
                      "within each front's fully summed rows",
            "analysis_s": first - fac, "factor_s": fac, "factor_flops": flops,
            "factor_tflops": flops / fac / 1e12, "factor_gb": fbytes / 1e9,
            "work_gb": wbytes / 1e9, "fronts": fronts, "levels": levels,
            "largest_front": nmax, "solves": solves,
            "split_precision_err_on_solved_fields": {
                "what": "per-parameter 2-norm error against the FP64 gradient, 32 surface point "
                        "forces and their adjoint fields from 20 surface receivers, both solved "
                        "with this factorisation (1 pair)",
                **solved_err}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nslots", type=int, default=32,
                    help="ring slots (complex128 systems kept in HBM; 32 x 4 GB at 400x120)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-grad", action="store_true")
    ap.add_argument("--small", action="store_true", help="small mesh (profiling captures)")
    ap.add_argument("--sparse-only", action="store_true",
                    help="only the sparse direct-solve leg (its JSON on one line)")
    ap.add_argument("--no-pipeline", action="store_true",
                    help="skip the uneven-batch pipeline comparison")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from fem25_b200 import (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE,
                            Context, synth)

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.sparse_only:
        print(json.dumps({"sparse_solve": sparse_solve_leg(local, dev)}))
        return
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---------------- setup (untimed)
    t_setup = time.perf_counter()
    if args.small:
        mesh, pairs, cfg = synth.make_config(1, nx=100, nz=40)
    else:
        mesh, pairs, cfg = synth.make_config(1)
    if world > 1:
        # weak scaling over distinct systems: rank r's 8 frequencies sit
        # r * 0.2 / world Hz above the single-GPU workload's, 64 ky each
        vmin = synth.vs_min(mesh)
        df = 0.2 * rank / world
        pairs = [(float(f + df), float(py)) for f in cfg["freqs"]
                 for py in synth.ky_list(f + df, 64, vmin)]
    ctx = Context(mesh, device=local)
    nz = ctx.nzero
    ndof_main = ctx.ndof
    nsys = len(pairs)
    freqs = [p[0] for p in pairs]
    pys = [p[1] for p in pairs]
    nslots = args.nslots
    stride = (2 * nz + 15) // 16 * 16  # 128-byte aligned ring slots
    ring = torch.empty(nslots * stride, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    setup_s = time.perf_counter() - t_setup

    def step():
        ctx.assemble_batch("B", freqs, pys, ring, stride, nslots, stream=stream)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()

    # ---------------- timed region: batched assembly
    ctx.profile(True)
    clk = Clocks(local)
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kern_ms = []
    e0.record(stream)
    for _ in range(args.steps):
        step()
        kern_ms.append(ctx.profile_ms(0))  # streaming kernel, events on the same stream
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms)
    ms_step = ms / args.steps
    value = nsys * args.steps * world / (ms / 1e3)
    # streaming kernel roofline: algorithmic bytes = 16 * NNZ per system
    kms = statistics.mean(kern_ms)
    peak, peak_kind = peaks()
    achieved = 16.0 * nz * nsys / (kms / 1e3) / 1e9
    # per step: PML delta (element + gather kernel) per distinct frequency, and
    # the streaming launches of the tuned variant (16 or, for the large-ring
    # variants 8 and 9, up to 1024 systems each, never more than the ring)
    per_launch = min(1024 if ctx.tuning()["stream_variant"] >= 8 else 16, nslots)
    launches_per_step = 2 * len(set(freqs)) + -(-nsys // per_launch)
    # DRAM bytes of one launch of the captured kernel, scaled from the small
    # case: reads by the entries, writes by entries x systems per launch
    traffic = None
    if ctx.tuning()["stream_variant"] == 8:
        traffic = (STREAM_BIG_READ_PER_ENTRY * nz +
                   STREAM_BIG_WRITE_PER_ENTRY * nz * per_launch)

    # ---------------- plain FP64 per-system path (device buffers)
    o128 = torch.empty(nz, dtype=torch.complex128, device=dev)
    o64 = torch.empty(nz, dtype=torch.complex64, device=dev)
    for k in range(2):
        ctx.assemble("B", freqs[k], pys[k], o128, o64, stream=stream)
    torch.cuda.synchronize()
    nplain = 16
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for k in range(nplain):
        ctx.assemble("B", freqs[(k * 31) % nsys], pys[(k * 31) % nsys], o128, None, stream=stream)
    p1.record(stream)
    torch.cuda.synchronize()
    plain_rate = nplain / (p0.elapsed_time(p1) / 1e3)
    del o128, o64

    # ---------------- e2e through the C ABI with host buffers
    h_cdist = torch.empty(nz, dtype=torch.complex64, pin_memory=True)
    h_e = torch.from_numpy(np.ascontiguousarray(mesh.ecoeff)).pin_memory()
    h_d = torch.from_numpy(np.ascontiguousarray(mesh.dens)).pin_memory()
    ne2e = 6
    ctx.asmble_driver("B", freqs[0], pys[0], out=h_cdist)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(ne2e):
        ctx.update_model(h_e.numpy(), h_d.numpy())
        ctx.asmble_driver("B", freqs[(k * 17) % nsys], pys[(k * 17) % nsys], out=h_cdist)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": ne2e * world / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(h_e.numel() * 8 + h_d.numel() * 8),
           "d2h_bytes_per_step": int(nz * 8),
           "path": "fem25_update_model + fem25_asmble_driver (ASMBLE_DRIVER drop-in), "
                   "COMPLEX*8 CDIST to pinned host memory"}
    del h_cdist
    # a model-update step: fem25_update_model invalidates the affine basis, so
    # the next batch rebuilds it (element basis integrals, gather, per-entry
    # primaries) before its 512 systems; wall clock around both, synchronised
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.update_model(h_e.numpy(), h_d.numpy())
    step()
    torch.cuda.synchronize()
    upd_s = max_over_ranks(time.perf_counter() - t0)
    model_update = {"s": upd_s, "assemblies_per_s": nsys * world / upd_s,
                    "basis_rebuild_s": max(0.0, upd_s - ms_step / 1e3),
                    "what": "fem25_update_model (host model upload) + one 512-system batch "
                            "that first rebuilds the affine basis"}

    # ---------------- gradient (exact lambda/mu/rho), 400x120 mesh, 32 sources x 2 pairs
    grad = None
    if not args.no_grad:
        nsrc = 32
        npool = 2
        gp = pairs[::64][:npool]
        u = synth.smooth_fields(mesh, ctx.g, gp, nsrc, seed=2027, device=dev)
        lam = synth.smooth_fields(mesh, ctx.g, gp, nsrc, seed=2028, device=dev)

        def time_grad(prec, reps=3):
            out = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=dev)
            ctx.gradient([p[0] for p in gp], [p[1] for p in gp], nsrc, u, lam, out, prec,
                         stream=stream)
            torch.cuda.synchronize()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            best = None
            for _ in range(reps):
                out.zero_()
                ev[0].record(stream)
                ctx.gradient([p[0] for p in gp], [p[1] for p in gp], nsrc, u, lam, out, prec,
                             stream=stream)
                ev[1].record(stream)
                torch.cuda.synchronize()
                ms = ev[0].elapsed_time(ev[1])
                best = ms if best is None else min(best, ms)
            return best, out

        gms, g64 = time_grad(FEM25_PREC_FP64)
        tms, g32 = time_grad(FEM25_PREC_TF32X3)
        pms, gpw = time_grad(FEM25_PREC_TF32X3_POINTWISE)
        ctx.sync_status(stream)
        rel = dict(zip(("lambda", "mu", "rho"), _per_param(torch, g32, g64)))
        prel = dict(zip(("lambda", "mu", "rho"), _per_param(torch, gpw, g64)))
        # the covariance path's two kernels on their own: accumulation (per
        # pair in an inversion loop) and contraction (once per gradient)
        fr_, py_ = [p[0] for p in gp], [p[1] for p in gp]
        acc_ms, fin_ms = [], []
        for _ in range(3):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record(stream)
            ctx.gradient_accumulate(fr_, py_, nsrc, u, lam, stream=stream)  # one k_grad_cov launch
            ev[1].record(stream)
            ctx.gradient_finalize(g32, stream=stream)  # one k_grad_cov_fin launch
            ev[2].record(stream)
            torch.cuda.synchronize()
            acc_ms.append(ev[0].elapsed_time(ev[1]))
            fin_ms.append(ev[1].elapsed_time(ev[2]))
        acc_ms, fin_ms = min(acc_ms), min(fin_ms)
        nelem_phys = int(np.sum(mesh.cdomain != ord("A")))
        units = mesh.nelem * nsrc * npool
        grad = {"metric": "gradient elem·rhs/s", "unit": "elem·rhs/s",
                "workload": "adjoint gradient: 400x120 layered mesh, 32 sources, 2 of the "
                            "8 f x 64 ky pairs; seeded smooth fields (unit RMS, lognormal "
                            "amplitude, 5 km-correlated phase)",
                "plain_fp64": units / (gms / 1e3), "ms": gms,
                "tf32x3": units / (tms / 1e3), "tf32x3_ms": tms,
                "tf32x3_rel_err_vs_fp64": rel,
                "tf32x3_form": "field covariances accumulated per element on tcgen05, "
                               "contracted once in FP64 (k_grad_cov + k_grad_cov_fin)",
                "tf32x3_accumulate_ms": acc_ms, "tf32x3_contraction_ms": fin_ms,
                "tf32x3_accumulate_elem_rhs_per_s": units / (acc_ms / 1e3),
                "tf32x3_pointwise": units / (pms / 1e3), "tf32x3_pointwise_ms": pms,
                "tf32x3_pointwise_rel_err_vs_fp64": prel,
                "units": f"{mesh.nelem} elements x {nsrc} sources x {npool} (omega,py) pairs "
                         f"({nelem_phys} non-PML elements computed)",
                "algorithmic_tflops_fp64": units * 547200 / (gms / 1e3) / 1e12}
        # covariance accumulation against HBM: the algorithmic bytes are the
        # two complex128 fields read once (2 x pairs x sources x NDOF x 16 B)
        hpk, hkind = peaks()
        fbytes = 2.0 * npool * nsrc * ctx.ndof * 16
        gbs = fbytes / (acc_ms / 1e3) / 1e9
        grad["covariance_roofline"] = {"bound": "hbm", "kernel": "k_grad_cov", "achieved": gbs,
                                       "peak": hpk, "unit": "GB/s", "frac": gbs / hpk,
                                       "peak_kind": hkind,
                                       "algorithmic_bytes": "u and lambda read once, "
                                                            f"{fbytes / 1e9:.2f} GB per launch"}
        # the launch's output too: 15 FP64 blocks of 25 x 25 per non-PML
        # element, written once (the timed launches follow a contraction, so
        # they overwrite the accumulators instead of adding to them)
        bbytes = nelem_phys * 15 * 625 * 8.0
        gbs_all = (fbytes + bbytes) / (acc_ms / 1e3) / 1e9
        grad["covariance_roofline"].update({
            "block_bytes": bbytes, "achieved_fields_and_blocks": gbs_all,
            "frac_fields_and_blocks": gbs_all / hpk})
        # the pointwise kernel against the tensor roofline: the metric's fixed
        # 547 200 flop per elem.rhs over a 3xTF32 peak (bf16 burst / 2 / 3)
        bpk, bkind = bf16_peak()
        tf = units * 547200 / (pms / 1e3) / 1e12
        grad["tf32x3_roofline"] = {"bound": "tensor", "kernel": "k_grad_tc (pointwise form)",
                                   "achieved": tf, "peak": bpk / 6.0, "unit": "TFLOP/s",
                                   "frac": tf / (bpk / 6.0),
                                   "peak_kind": f"{bkind} bf16 burst {bpk:g} / 2 (TF32) / 3 "
                                                f"(split products)"}
        # the reference-compatible drop-in (CFMAT_DIST + ADJGRAD, COMPLEX*8,
        # 'PP'): one source's virtual forces and gradient contribution
        w32 = u[0, 0].to(torch.complex64).contiguous()
        l32 = lam[0, 0].to(torch.complex64).contiguous()
        nnpinv, _, _ = ctx.ref_gradient_info()
        gl = torch.zeros(nnpinv, dtype=torch.float32, device=dev)
        p0 = pairs[0]
        ctx.cfmat_adjgrad("PP", 1.73, p0[0], p0[1], w32, l32, gl, stream=stream)
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(stream)
        nref = 3
        for _ in range(nref):
            ctx.cfmat_adjgrad("PP", 1.73, p0[0], p0[1], w32, l32, gl, stream=stream)
        ev[1].record(stream)
        torch.cuda.synchronize()
        rms = ev[0].elapsed_time(ev[1]) / nref
        grad["reference_path"] = {
            "what": "fem25_ref_gradient_dev ('PP'): CFMAT_DIST virtual forces + ADJFLAM_DIST, "
                    "one source", "ms_per_source": rms,
            "elem_rhs_per_s": mesh.nelem / (rms / 1e3), "inversion_anchors": nnpinv}
        del u, lam, w32, l32, gl
    tuning = ctx.tuning()

    del ring
    ctx.close()
    torch.cuda.empty_cache()
    ctx = None
    split = sparse = None
    if not args.no_grad and not args.small and rank == 0:
        split = split_precision_leg(local, dev)
        sparse = sparse_solve_leg(local, dev)
    pipe = None
    if not args.no_pipeline and not args.small:
        pipe = pipeline_uneven(local, dev, rank, world, max_over_ranks)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        smp = CpuSampler(1)
        smp.sample(1.0)
        cpu = smp.sample(12.0)
        smp.close()

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": max(3, args.warmup), "ms_per_step": ms_step, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded layered model; no public dataset exists for this path)",
           "config": headline_config(mesh.nelem, ndof_main, nz, nsys),
           "parallelism": f"{world} shards of distinct systems" if world > 1 else "1 GPU",
           "run": {"nslots": nslots, "slot_stride_doubles": stride, "autotuned": tuning,
                   "setup_s": round(setup_s, 2)},
           "plain_fp64": {"value": plain_rate, "unit": UNIT, "speedup_batched": value / world / plain_rate},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "traffic": traffic,
                        "traffic_unit": "bytes per launch",
                        "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum of a "
                                        "100x40 capture of the same kernel, scaled to this "
                                        "launch (reads by CSR entries, writes by entries x "
                                        "systems); null when another variant is tuned",
                        "algorithmic_bytes_per_launch": 16.0 * nz * per_launch,
                        "kernel": STREAM_KERNELS.get(tuning["stream_variant"], "k_stream"),
                        "kernel_ms": kms, "peak_kind": peak_kind,
                        "algorithmic_bytes": "16 B x NNZ per system (complex128 values written)"},
           "cpu_baseline": cpu, "e2e": e2e, "model_update_step": model_update,
           "gradient": grad, "split_precision": split, "sparse_solve": sparse, "pipeline": pipe,
           "gpu_launches": launches_per_step * args.steps, "clocks": clocks}
    if rank == 0:
        print(json.dumps(out))
    if ctx is not None:
        ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
