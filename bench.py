#!/usr/bin/env python3
"""Benchmark: batched GFN2-shaped singlepoints/s on B200, plain FP64 and mixed forms.

Workload (default): 1024 water clusters of U{8..64} rigid waters (24-192 atoms,
48-384 AOs), seeded synthetic inputs built by the cluster rules (no dataset).
One step = the full singlepoint (setup + SCF to convergence) of the whole
batch.  Both forms are timed (tb_options.precision 0 and 1) with the geometry
already resident on the device and the whole SCF loop launched as one CUDA graph
(a conditional WHILE node over one captured iteration); `value` is the faster form whose energies agree with the FP64 form
to 1e-6 Eh (config.form names it, `forms` lists both).  `e2e` times the public
tb_singlepoint_batch of that form with host buffers (the upload of the inputs
and the download of every result inside the timed region).  The working set
(about 7 GB of matrices) is far larger than L2, so no flush is needed between
steps.  `serving` is a bounded sample of the request stream (Poisson arrivals,
log-uniform 10-600 atoms) through tb_server with p50/p99 latency;
--workload serving runs the full stream report for both forms and
--workload water_box_1000 the 6000-AO structure.

Multi-GPU (torchrun): one replica per GPU, each rank its own seeded batch
(weak scaling, no data-path collective); value = all structures / max time.
`--impl reference` times the FP64 CPU restatement of the reference's singlepoint
(the reference itself does not build or run) on the host cores.
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
sys.path.insert(0, os.path.join(ROOT, "tblite-cuda_b200"))

METRIC = "GFN2 singlepoints/s at |dE|<=1e-6 Eh, mixed vs FP64 on 1 GPU; p50/p99 ms"
UNIT = "singlepoints/s"
WORKLOAD = "water_clusters_1024"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--count", type=int, default=1024, help="structures per batch")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-config2", dest="config2", action="store_false",
                    help="skip the 256-alkane summary (config 2) of the default run")
    ap.add_argument("--workload", default=WORKLOAD,
                    choices=[WORKLOAD, "alkanes_256", "water_box_1000", "serving"],
                    help="alkanes_256: 256 alkanes C20-C199, both forms with per-structure errors; "
                         "water_box_1000: one 3000-atom / 6000-AO structure, time per SCF iteration; "
                         "serving: the request stream through tb_server, both forms")
    ap.add_argument("--serving-requests", type=int, default=400,
                    help="requests of the bounded serving sample per form (0: skip)")
    ap.add_argument("--serving-rate", type=float, default=1000.0,
                    help="Poisson arrival rate per second (default above capacity: latency measures the GPU)")
    return ap.parse_args()


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def rank_seed(rank):
    """Seed of a rank's own batch (replicas: every rank its own structures)."""
    return 1001 + rank


def max_over_ranks(x, ws, device=None):
    """The largest of x over the ranks of the default process group (x on one rank)."""
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(ws, steps, per_rank_units, elapsed):
    """Whole-job throughput: the units every rank processed over the slowest rank's time."""
    return ws * steps * per_rank_units / elapsed


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.th.join(timeout=5)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def fp64_peak_tflops(torch):
    """cuBLAS DGEMM throughput measured live (the FP64 roofline denominator)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    best = 0.0
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def ncu_traffic():
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return None
    return None


def oracle_for_timing():
    """The FP64 oracle built on this host with -march=native (rebuilt here, so
    the instruction set is this CPU's), else the portable build."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    build = "portable build (-O3)"
    try:
        r = subprocess.run(["make", "-B", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle_native.so"],
                           capture_output=True, text=True, timeout=300)
        so = os.path.join(ROOT, "oracle", "liboracle_native.so")
        if r.returncode == 0 and os.path.exists(so):
            pyoracle.use_library(so)
            build = "built on this host with -O3 -march=native"
    except Exception:
        pass
    orc = pyoracle.Oracle(os.path.join(ROOT, "tblite-cuda_b200", "params", "synthetic_hco.tbp"))
    return orc, build


def lpt_sample(mols, start, count):
    """`count` consecutive structures of the workload from `start` (wrapping),
    as indices ordered largest first, so that a dynamic one-structure-per-thread
    schedule ends with small structures (balanced threads)."""
    idx = [(start + k) % len(mols) for k in range(count)]
    return sorted(idx, key=lambda i: -mols[i].nat)


def cpu_baseline(orc, build, mols, nthreads, target_s=12.0):
    """FP64 oracle (CPU restatement) on a bounded, load-balanced sample of the workload:
    at least 8 structures per thread, largest first, sized to about target_s seconds."""
    probe = lpt_sample(mols, 0, max(1, min(len(mols), nthreads)))
    t = time.perf_counter()
    orc.singlepoint_batch([mols[i] for i in probe], nthreads=nthreads)
    dt = max(time.perf_counter() - t, 1e-3)
    per = dt / len(probe) * nthreads  # seconds per structure per thread
    count = int(min(len(mols), max(8 * nthreads, target_s * nthreads / max(per, 1e-6))))
    sample = lpt_sample(mols, 0, count)
    t = time.perf_counter()
    res = orc.singlepoint_batch([mols[i] for i in sample], nthreads=nthreads)
    dt = time.perf_counter() - t
    return {"value": count / dt, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"first {count} of the {len(mols)} structures of the workload, largest first, one "
                      f"structure per thread, {dt:.1f} s; oracle {build}"}, res, sample


def time_form(capi, torch, calc, mols, args, stream, precision):
    """Device-resident batch of one form: W warm-up runs, K timed runs (CUDA events)."""
    sh = stream.cuda_stream
    batch = capi.Batch(calc, mols, profile=1, precision=precision, use_graphs=0)
    for _ in range(args.warmup):
        batch.run(sh)
    torch.cuda.synchronize()
    res = batch.results(sh)
    prof_tot, launches = {}, 0
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        t0.record(stream)
        for _ in range(args.steps):
            batch.run(sh)
            launches += batch.launches()
            for k, (la, ms, wk, un) in batch.profile().items():
                p = prof_tot.setdefault(k, [0, 0.0, 0.0, un])
                p[0] += la; p[1] += ms; p[2] += wk
        t1.record(stream)
    torch.cuda.synchronize()
    # graph-replayed runs (what a user gets with use_graphs = 1), without per-kernel events
    gb = capi.Batch(calc, mols, precision=precision, use_graphs=1)
    for _ in range(args.warmup):
        gb.run(sh)
    torch.cuda.synchronize()
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        g0.record(stream)
        for _ in range(args.steps):
            gb.run(sh)
        g1.record(stream)
    torch.cuda.synchronize()
    return dict(res=res, prof=prof_tot, launches=launches, elapsed_events=t0.elapsed_time(t1) * 1e-3,
                elapsed=g0.elapsed_time(g1) * 1e-3)


def serving_run(capi, calc, count, rate, precision, budget):
    """Poisson arrivals of log-uniform 10-600 atom water/alkane requests through tb_server."""
    from tblite_b200 import geometry
    reqs = geometry.request_stream(count=count, seed=1003, rate=rate)
    srv = capi.Server(calc, budget, max_batch=512, precision=precision, use_graphs=1)
    arrival, lat, i = {}, [], 0
    t0 = time.perf_counter()
    while len(lat) < count:
        now = time.perf_counter() - t0
        while i < count and reqs[i][0] <= now:
            arrival[srv.submit(reqs[i][1])] = reqs[i][0]
            i += 1
        resident, queued, _ = srv.step()
        now = time.perf_counter() - t0
        for t, r in srv.poll():
            lat.append(now - arrival[t])
        if resident == 0 and queued == 0 and i < count:
            time.sleep(max(0.0, min(0.002, reqs[i][0] - (time.perf_counter() - t0))))
        else:
            time.sleep(0.0002)  # the step polls; micro-batches run on their own streams
    total = time.perf_counter() - t0
    lat_ms = sorted(x * 1e3 for x in lat)
    q = lambda f: lat_ms[min(len(lat_ms) - 1, int(f * len(lat_ms)))]
    return {"requests": count, "arrival_rate_per_s": rate, "throughput": count / total, "unit": UNIT,
            "p50_ms": q(0.50), "p99_ms": q(0.99), "wall_s": total,
            "sizes": "log-uniform 10-600 atoms, 50/50 water clusters / alkanes, seed 1003"}


def main():
    args = parse()
    ws, rank, local = dist_setup(args)
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    import numpy as np
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if args.workload == "water_box_1000":
        return run_water_box(args, torch)
    if args.workload == "serving":
        return run_serving(args, torch)
    if args.workload == "alkanes_256":
        return run_alkanes(args, torch)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                               device_id=torch.device("cuda", local))
    from tblite_b200 import Calculator, capi, geometry
    calc = Calculator()
    mols = geometry.water_clusters(args.count, seed=rank_seed(rank))
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    nat = sum(m.nat for m in mols)
    nao = sum(calc.basis_size(m)[1] for m in mols)

    # ---------------- both forms, device-resident batches (value)
    sampler = ClockSampler(local)
    sampler.start()
    if ws > 1:
        dist.barrier()
    forms = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        forms[name] = time_form(capi, torch, calc, mols, args, stream, prec)
    if ws > 1:
        dist.barrier()
    clocks = sampler.stop()
    for name, f in forms.items():
        el = max_over_ranks(f["elapsed"], ws, device="cuda")
        f["value"] = job_rate(ws, args.steps, len(mols), el)
        f["ms_per_step"] = el / args.steps * 1e3
    e_fp = np.array([r["energy"] for r in forms["fp64"]["res"]])
    e_mx = np.array([r["energy"] for r in forms["mixed"]["res"]])
    forms["mixed"]["max_abs_dE_vs_fp64"] = float(np.max(np.abs(e_mx - e_fp)))
    forms["fp64"]["max_abs_dE_vs_fp64"] = 0.0
    ok = {k: f for k, f in forms.items() if f["max_abs_dE_vs_fp64"] <= 1e-6 and
          all(r["status"] == 0 for r in f["res"])}
    head_name = max(ok, key=lambda k: ok[k]["value"]) if ok else "fp64"
    head = forms[head_name]
    head_prec = 0 if head_name == "fp64" else 1
    value = head["value"]

    # ---------------- end to end through the public API (host buffers), headline form
    ids_bytes = sum(m.nat * (3 * 8 + 4) + 12 for m in mols)
    out_bytes = sum(8 * (13 + m.nat * 10) + 8 * calc.basis_size(m)[0] for m in mols)
    calc.singlepoint_batch(mols, precision=head_prec, use_graphs=1)  # warm the workspace
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    te = time.perf_counter()
    for _ in range(args.steps):
        calc.singlepoint_batch(mols, stream=sh, precision=head_prec, use_graphs=1)
    torch.cuda.synchronize()
    e2e_t = max_over_ranks(time.perf_counter() - te, ws, device="cuda")
    e2e = {"value": job_rate(ws, args.steps, len(mols), e2e_t), "unit": UNIT, "h2d_bytes_per_step": ids_bytes,
           "d2h_bytes_per_step": out_bytes}

    # ---------------- roofline of the dominant kernel class (live CUDA-event times, headline form)
    prof_tot = head["prof"]
    name, (la, ms, wk, un) = max(prof_tot.items(), key=lambda kv: kv[1][1])
    peaks, src = measured_peaks()
    if un == "flop":
        peak = fp64_peak_tflops(torch)
        achieved = wk / (ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "pipe": "fp64",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 entry)",
                "work": "canonical 4 N^3 flops per eigensolve"}
    elif un == "byte":
        peak = peaks["hbm_gbs"]
        achieved = wk / (ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{src} hbm_gbs"}
    else:
        roof = {"bound": None, "achieved": None, "peak": None, "unit": None, "frac": None}
    roof["kernel"] = name
    roof["launches"] = la
    tr = ncu_traffic()
    ent = tr.get(name) if isinstance(tr, dict) else None
    roof["traffic"] = ent.get("bytes_per_launch") if isinstance(ent, dict) else None
    if roof["traffic"] is not None:
        roof["traffic_source"] = "profiles/ncu_traffic.json: " + str(ent.get("capture", "ncu dram bytes"))
    total_ms = sum(v[1] for v in prof_tot.values())
    kernels = {k: {"launches": v[0], "ms": round(v[1], 3), "share": round(v[1] / total_ms, 4)}
               for k, v in sorted(prof_tot.items(), key=lambda kv: -kv[1][1])}

    # ---------------- serving latency (bounded sample of the request stream), both forms
    serving = None
    if rank == 0 and args.serving_requests > 0:
        free, _ = torch.cuda.mem_get_info()
        serving = {}
        for sname, sprec in (("fp64", 0), ("mixed", 1)):
            serving_run(capi, calc, min(32, args.serving_requests), args.serving_rate, sprec, int(0.5 * free))
            serving[sname] = serving_run(capi, calc, args.serving_requests, args.serving_rate, sprec,
                                         int(0.5 * free))

    # ---------------- the plain form one structure per call (no batching), for the batching gain
    one = one_per_call(calc, mols, torch, sh) if rank == 0 else None
    # the same calls with the tridiagonalisation in cluster shared memory (latency-bound calls)
    one_smem = one_per_call(calc, mols, torch, sh, smem_tridiag=True) if rank == 0 else None

    # ---------------- config 2 (256 alkanes, 122-1196 AOs): both forms, errors of the mixed form
    alk = alkanes_summary(capi, calc, torch, stream) if rank == 0 and args.config2 else None

    res = head["res"]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if head_prec == 0 else "f32+f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "form": head_name, "structures_per_gpu": len(mols),
                       "waters": "U{8..64}", "atoms": nat, "aos": nao, "seed": 1001,
                       "parallelism": f"replicas x{ws}", "l2": "inputs larger than L2 (no flush needed)",
                       "accuracy": 1.0,
                       "graphs": "whole SCF loop as one graph launch (conditional WHILE node)"},
            "e2e": e2e, "gpu_launches": launches_of(forms, head_name), "roofline": roof, "kernels": kernels,
            "clocks": clocks,
            "forms": {k: {"value": f["value"], "ms_per_step": f["ms_per_step"],
                          "ms_per_step_with_kernel_events": f["elapsed_events"] / args.steps * 1e3,
                          "max_abs_dE_vs_fp64": f["max_abs_dE_vs_fp64"],
                          "scf_iterations_mean": float(np.mean([r["iterations"] for r in f["res"]])),
                          "status_ok": int(sum(r["status"] == 0 for r in f["res"]))} for k, f in forms.items()},
            "mixed_vs_fp64": forms["mixed"]["value"] / forms["fp64"]["value"]}
    if serving is not None:
        line["serving"] = serving
    if alk is not None:
        line["alkanes_256"] = alk
    if one is not None:
        line["forms"]["fp64_one_structure_per_call"] = one
        line["forms"]["fp64_one_structure_per_call_smem_tridiag"] = one_smem
        line["batched_vs_one_per_call"] = value / one["value"]
    iters = [r["iterations"] for r in res]
    line["scf_iterations"] = {"mean": float(np.mean(iters)), "max": int(max(iters))}
    line["status_ok"] = int(sum(r["status"] == 0 for r in res))

    if rank == 0 and not args.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        orc, build = oracle_for_timing()
        cb, ores, sample = cpu_baseline(orc, build, mols, nthreads)
        line["cpu_baseline"] = cb
        de = [abs(res[i]["energy"] - o["energy"]) for i, o in zip(sample, ores)]
        line["max_abs_dE_vs_oracle"] = max(de)
        line["structures_checked_vs_oracle"] = len(sample)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def launches_of(forms, name):
    return int(forms[name]["launches"])


def one_per_call(calc, mols, torch, sh, count=48, smem_tridiag=False):
    """The plain FP64 form without batching: tb_singlepoint_batch called once per
    structure on an evenly spaced sample of the workload (host buffers);
    smem_tridiag: with the tridiagonalisation in cluster shared memory."""
    sample = [mols[int(i)] for i in range(0, len(mols), max(1, len(mols) // count))][:count]
    calc.set_smem_tridiag(64 if smem_tridiag else 0)
    try:
        # warm-up includes the largest structure, so that a first-use calibration
        # of the eigensolver choice is not timed
        for m in sample[:4] + [max(sample, key=lambda x: x.nat)]:
            calc.singlepoint_batch([m], stream=sh, precision=0)
        torch.cuda.synchronize()
        t = time.perf_counter()
        for m in sample:
            calc.singlepoint_batch([m], stream=sh, precision=0)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
    finally:
        calc.set_smem_tridiag(0)
    return {"value": len(sample) / dt, "unit": UNIT, "structures": len(sample),
            "sample": "evenly spaced structures of the batch, one tb_singlepoint_batch call each",
            "smem_tridiag": bool(smem_tridiag)}


def alkanes_summary(capi, calc, torch, stream):
    """The 256-alkane workload (config 2) inside the default run: each form one
    warm-up and one timed device-resident run (whole SCF loop as one graph),
    and the mixed form's per-structure errors against the FP64 form."""
    import numpy as np
    from tblite_b200 import geometry
    mols = geometry.alkanes(256, seed=1002)
    sh = stream.cuda_stream
    out, res = {}, {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        b = capi.Batch(calc, mols, precision=prec, use_graphs=1)
        b.run(sh)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            t0.record(stream)
            b.run(sh)
            t1.record(stream)
        torch.cuda.synchronize()
        res[name] = b.results(sh)
        el = t0.elapsed_time(t1) * 1e-3
        out[name] = {"value": len(mols) / el, "ms_per_step": el * 1e3,
                     "status_ok": int(sum(r["status"] == 0 for r in res[name])),
                     "scf_iterations_mean": float(np.mean([r["iterations"] for r in res[name]]))}
        del b
    fp, mx = res["fp64"], res["mixed"]
    de = [abs(x["energy"] - y["energy"]) for x, y in zip(mx, fp)]
    dq = [float(np.max(np.abs(np.asarray(x["qat"]) - np.asarray(y["qat"])))) for x, y in zip(mx, fp)]
    dmu = [float(np.max(np.abs(np.asarray(x["dipole"]) - np.asarray(y["dipole"])))) for x, y in zip(mx, fp)]
    out["mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["mixed_vs_fp64_errors"] = {k: {"max": float(np.max(v)), "median": float(np.median(v))}
                                   for k, v in (("dE", de), ("dq", dq), ("dmu", dmu))}
    out["config"] = {"structures": len(mols), "n": "U{20..200} (drawn 20-199)", "seed": 1002, "aos": "122-1196",
                     "accuracy": 1.0, "timing": "one warm-up and one timed run per form, CUDA events",
                     "errors": "per structure, mixed form against the plain FP64 form (both at accuracy 1: "
                               "charge spread of the convergence threshold ~1e-4 e)"}
    return out


def run_alkanes(args, torch):
    """The 256-alkane workload (C20-C199, 62-599 atoms, 122-1196 AOs): both forms
    timed as for the water clusters; per-structure |dE|, max |dq| and |dmu| of the
    mixed form against the FP64 form on every structure, and the energies of both
    forms against the FP64 oracle on the smallest structures (a bounded CPU sample)."""
    import numpy as np
    from tblite_b200 import Calculator, capi, geometry
    calc = Calculator()
    mols = geometry.alkanes(256, seed=1002)
    stream = torch.cuda.Stream()
    sampler = ClockSampler(0)
    sampler.start()
    forms = {name: time_form(capi, torch, calc, mols, args, stream, prec)
             for name, prec in (("fp64", 0), ("mixed", 1))}
    clocks = sampler.stop()
    for f in forms.values():
        f["value"] = len(mols) * args.steps / f["elapsed"]
        f["ms_per_step"] = f["elapsed"] / args.steps * 1e3

    def errs(a, b):
        return {"dE": [abs(x["energy"] - y["energy"]) for x, y in zip(a, b)],
                "dq": [float(np.max(np.abs(np.asarray(x["qat"]) - np.asarray(y["qat"])))) for x, y in zip(a, b)],
                "dmu": [float(np.max(np.abs(np.asarray(x["dipole"]) - np.asarray(y["dipole"]))))
                        for x, y in zip(a, b)]}

    fp, mx = forms["fp64"]["res"], forms["mixed"]["res"]
    e = errs(mx, fp)
    line = {"metric": METRIC, "value": max(f["value"] for f in forms.values()), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic", "clocks": clocks,
            "config": {"workload": "alkanes_256", "structures": len(mols), "n": "U{20..200} (drawn 20-199)",
                       "seed": 1002, "aos": "122-1196", "accuracy": 1.0},
            "forms": {k: {"value": f["value"], "ms_per_step": f["ms_per_step"],
                          "status_ok": int(sum(r["status"] == 0 for r in f["res"])),
                          "scf_iterations_mean": float(np.mean([r["iterations"] for r in f["res"]]))}
                      for k, f in forms.items()},
            "mixed_vs_fp64": forms["mixed"]["value"] / forms["fp64"]["value"],
            "mixed_vs_fp64_errors": {k: {"max": float(np.max(v)), "median": float(np.median(v))}
                                     for k, v in e.items()},
            "mixed_vs_fp64_errors_per_structure": e}
    if not args.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        orc, build = oracle_for_timing()
        small = sorted(range(len(mols)), key=lambda i: mols[i].nat)[:2 * nthreads]
        t = time.perf_counter()
        ores = orc.singlepoint_batch([mols[i] for i in small[::-1]], nthreads=nthreads)[::-1]
        dt = time.perf_counter() - t
        line["vs_oracle"] = {
            "structures": len(small), "oracle": build,
            "aos": f"{calc.basis_size(mols[small[0]])[1]}-{calc.basis_size(mols[small[-1]])[1]}",
            "fp64_dE_max": max(abs(fp[i]["energy"] - o["energy"]) for i, o in zip(small, ores)),
            "mixed_dE_max": max(abs(mx[i]["energy"] - o["energy"]) for i, o in zip(small, ores))}
        line["cpu_baseline"] = {"value": len(small) / dt, "unit": UNIT, "cores": nthreads, "kind": "port",
                                "sample": f"the {len(small)} smallest alkanes, one structure per thread, {dt:.1f} s"}
    print(json.dumps(line))


def run_serving(args, torch):
    """The request-stream workload: throughput and p50/p99 latency of both forms."""
    from tblite_b200 import Calculator, capi
    calc = Calculator()
    free, _ = torch.cuda.mem_get_info()
    out = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        serving_run(capi, calc, min(64, args.serving_requests), args.serving_rate, prec, int(0.5 * free))  # warm-up
        out[name] = serving_run(capi, calc, args.serving_requests, args.serving_rate, prec, int(0.5 * free))
    line = {"metric": "GFN2 singlepoints/s and p50/p99 latency, request stream, 1 GPU",
            "value": out["fp64"]["throughput"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "data": "synthetic", "config": {"workload": "request_stream", "requests": args.serving_requests,
                                            "rate_per_s": args.serving_rate},
            "forms": out}
    print(json.dumps(line))


def run_water_box(args, torch):
    """One 1000-water box (6000 AOs): time per SCF iteration and FP64 fraction."""
    from tblite_b200 import capi, geometry
    from tblite_b200 import Calculator
    calc = Calculator()
    box = geometry.water_box()
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    batch = capi.Batch(calc, [box], profile=1)
    for _ in range(max(1, args.warmup)):
        batch.run(sh)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    prof_tot = {}
    with torch.cuda.stream(stream):
        t0.record(stream)
        for _ in range(args.steps):
            batch.run(sh)
            for k, (la, ms, wk, un) in batch.profile().items():
                p = prof_tot.setdefault(k, [0, 0.0, 0.0, un])
                p[0] += la; p[1] += ms; p[2] += wk
        t1.record(stream)
    torch.cuda.synchronize()
    r = batch.results(sh)[0]
    elapsed = t0.elapsed_time(t1) * 1e-3 / args.steps
    iters = r["iterations"]
    scf_ms = sum(v[1] for k, v in prof_tot.items() if k not in ("atoms", "adjacency", "integrals", "cholesky",
                                                                   "trinv", "factor_lib", "scf_init")) / args.steps
    flops = sum(v[2] for v in prof_tot.values() if v[3] == "flop") / args.steps
    flop_ms = sum(v[1] for v in prof_tot.values() if v[3] == "flop") / args.steps
    peak = fp64_peak_tflops(torch)
    total_ms = sum(v[1] for v in prof_tot.values())
    line = {"metric": "ms per SCF iteration, one 1000-water box (6000 AOs), plain FP64", "value": scf_ms / iters,
            "unit": "ms/iteration", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed * 1e3, "higher_is_better": False, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "water_box_1000", "atoms": box.nat, "aos": calc.basis_size(box)[1],
                       "seed": 1004, "solver": "cuSOLVER Xsyevd above 1216 AOs"},
            "scf_iterations": iters, "status": r["status"], "energy": r["energy"],
            "fp64": {"achieved_tflops": flops / (flop_ms * 1e-3) / 1e12 if flop_ms else None, "peak_tflops": peak,
                     "frac": flops / (flop_ms * 1e-3) / 1e12 / peak if flop_ms else None,
                     "over": "GEMM + eigensolver kernel time"},
            "kernels": {k: {"launches": v[0], "ms": round(v[1], 3), "share": round(v[1] / total_ms, 4)}
                        for k, v in sorted(prof_tot.items(), key=lambda kv: -kv[1][1])}}
    print(json.dumps(line))


def run_reference(args, ws, rank):
    """FP64 CPU restatement of the reference singlepoint on all host cores."""
    if rank != 0:
        return
    from tblite_b200 import geometry
    orc, build = oracle_for_timing()
    mols = geometry.water_clusters(args.count, seed=1001)
    nthreads = os.cpu_count() or 1
    # each timed step: 8 structures per thread of the workload, consecutive
    # through the batch and run largest first, so that no thread idles while
    # another finishes a large cluster (the whole run stays within minutes)
    per_step = min(len(mols), 8 * nthreads)
    for w in range(args.warmup):
        orc.singlepoint_batch([mols[i] for i in lpt_sample(mols, w * nthreads, nthreads)], nthreads=nthreads)
    t = time.perf_counter()
    done = 0
    for s in range(args.steps):
        sample = lpt_sample(mols, s * per_step, per_step)
        orc.singlepoint_batch([mols[i] for i in sample], nthreads=nthreads)
        done += len(sample)
    dt = time.perf_counter() - t
    value = done / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "structures_per_step": per_step, "waters": "U{8..64}", "seed": 1001},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"{per_step} consecutive water clusters per step ({args.steps} steps), "
                                       f"largest first, one structure per thread; oracle {build}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference (tornikeo/tblite-cuda) does not compile or converge; this times its FP64 CPU "
                    "restatement (oracle/) on the same workload"}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
