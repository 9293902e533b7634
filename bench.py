#!/usr/bin/env python
"""Zip+ commit+prove throughput on B200: evals/s, per-step latency p50/p99.

One step = one plain Zip+ commit + prove of one polynomial: encode, Merkle
commitment, Fiat-Shamir transcript (root absorbed, random 256-bit prime field
sampled), alpha projection, b rows, combined row and 147 column openings.
The default workload is the Zip+ benchmark of the reference
(zip-plus/benches/zip_plus_benches.rs:37-65): num_vars 16 (65536 evaluations),
BinaryPoly<32> with Bernoulli(0.5) coefficients, IPRS rate 1/4 over F65537 with
row_len 2^14 (4 rows, depth 2), MontyField<4>, CombR Int<5>, 147 openings,
evaluation point [1; 16] (zip_common.rs:271).  Inputs are seeded synthetic.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank drives its own GPU with its own polynomials (replicas,
weak scaling); times are the max over ranks.  `--impl reference` times the
CPU restatement of the reference path (the oracle; the Rust reference cannot
be built in this image) with all host threads, on rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "zinc-plus_b200"))

import numpy as np  # noqa: E402

METRIC = "Zip+ commit+prove evals/s on 1 B200 (batched vs plain, bit-exact); p50/p99 ms"
WORKLOADS = {
    # name: (eval_kind, D, code_kind, num_vars, row_len)
    "zipplus_binpoly32_iprs_nv16": (1, 32, 0, 16, 1 << 14),
    "zipplus_binpoly32_raa_nv16": (1, 32, 1, 16, 256),
    "zip_i32_iprs_nv12": (0, 1, 0, 12, 4096),
}
DEFAULT_WORKLOAD = "zipplus_binpoly32_iprs_nv16"
L2_FLUSH_BYTES = 256 << 20


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def make_inputs(workload, count, seed):
    ek, D, _, nv, _ = WORKLOADS[workload]
    rng = np.random.default_rng(seed)
    n = 1 << nv
    if ek == 1:
        bits = rng.integers(0, 2, size=(count, n, D), dtype=np.uint8)
        w = np.left_shift(np.uint64(1), np.arange(D, dtype=np.uint64))
        return (bits.astype(np.uint64) * w).sum(axis=2, dtype=np.uint64)
    return rng.integers(-(2**15), 2**15, size=(count, n), dtype=np.int32)


def config_of(workload, num_rows, depth):
    ek, D, ck, nv, L = WORKLOADS[workload]
    code = (f"IPRS F65537 rate 1/4 row_len {L} depth {depth}" if ck == 0
            else f"RAA rate 1/4 row_len {L} (rand 0.9 StdRng seeds 1, 2)")
    return {
        "workload": workload,
        "num_vars": nv,
        "evals_per_poly": 1 << nv,
        "eval": f"BinaryPoly<{D}> u64-packed, Bernoulli(0.5)" if ek else "i32 uniform [-2^15, 2^15)",
        "code": code,
        "num_rows": num_rows,
        "field": "MontyField<4> (random 256-bit prime from the transcript)",
        "comb": "Int<5>" if ek else "Int<3>",
        "openings": 147,
        "point": f"[1; {nv}]",
        "l2": "flushed between timed steps (256 MiB device memset, untimed)",
        "parallelism": "replicas (one polynomial per step per GPU)",
    }


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clocks and clock-event reasons during the timed region: NVML read from
    a thread every 10 ms (reads only), with nvidia-smi as the fallback."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []

    def _nvml_handle(self, nv):
        try:  # the CUDA device's PCI address (CUDA and NVML may number devices differently)
            import torch
            pr = torch.cuda.get_device_properties(self.dev)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        try:
            import threading

            import pynvml as nv
            nv.nvmlInit()
            h = self._nvml_handle(nv)
            bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            self.stop_flag = threading.Event()

            def run():
                while not self.stop_flag.is_set():
                    try:
                        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.rows.append((sm, mx, [n for n, b in zip(self.NAMES, bits) if r & b]))
                    except Exception:
                        pass
                    self.stop_flag.wait(0.01)

            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            rows = list(self.rows)
            if not rows:
                return None
            sm = [r[0] for r in rows]
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(r[1] for r in rows),
                    "reasons": sorted({n for r in rows for n in r[2]}), "samples": len(rows),
                    "source": "NVML, every 10 ms over the timed region"}
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = sorted({self.NAMES[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows), "source": "nvidia-smi -lms 20"}


# ------------------------------------------------------------ CPU baseline
def cpu_commit_prove_rate(workload, seconds, max_steps, inputs):
    """Oracle (CPU restatement of the reference path) with all host threads."""
    from oracle import oracle as O

    O.build()
    ek, D, ck, nv, L = WORKLOADS[workload]
    desc = O.make_desc(ek, D, ck, nv, L)
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    O.commit_prove(desc, inputs[0], 1, [1] * nv)  # warm-up (page faults, tables)
    steps, t0 = 0, time.perf_counter()
    lat = []
    while steps < max_steps and (time.perf_counter() - t0 < seconds or steps < 1):
        t = time.perf_counter()
        O.commit_prove(desc, inputs[steps % len(inputs)], 1, [1] * nv)
        lat.append(time.perf_counter() - t)
        steps += 1
    dt = time.perf_counter() - t0
    return {"value": steps * (1 << nv) / dt, "unit": "evals/s", "cores": threads, "kind": "port",
            "sample": f"{steps} full commit+prove steps of the workload ({1 << nv} evals each), "
                      f"{dt:.1f} s, OpenMP over rows/columns/pairs like the reference's rayon",
            "latency_ms": lat}


def run_reference(args):
    """--impl reference: the oracle port on the host cores, rank 0 only."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    workload = args.workload
    ek, D, ck, nv, L = WORKLOADS[workload]
    from oracle import oracle as O

    O.build()
    desc = O.make_desc(ek, D, ck, nv, L)
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    inputs = make_inputs(workload, min(args.steps + args.warmup, 4), 1234)
    for i in range(args.warmup):
        O.commit_prove(desc, inputs[i % len(inputs)], 1, [1] * nv)
    lat = []
    t0 = time.perf_counter()
    for i in range(args.steps):
        t = time.perf_counter()
        O.commit_prove(desc, inputs[i % len(inputs)], 1, [1] * nv)
        lat.append((time.perf_counter() - t) * 1e3)
    dt = time.perf_counter() - t0
    value = args.steps * (1 << nv) / dt
    R = O.num_rows(desc)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": config_of(workload, R, 0 if ck else O.iprs_optimal_depth(L)),
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full commit+prove steps, OpenMP, the Rust "
                                   "reference is not buildable here (no cargo)"},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------ batched commit / serving
def layout_row_len(nv):
    """row_len = 2^min(nv, 14), num_rows = 2^max(0, nv - 14)."""
    return 1 << min(nv, 14)


def random_binary(rng, nv, D):
    """2^nv BinaryPoly<D> evaluations, each coefficient Bernoulli(0.5), u64-packed."""
    x = rng.bit_generator.random_raw(1 << nv).astype(np.uint64)
    return x if D == 64 else x & np.uint64((1 << D) - 1)


def run_batched_commit(Z, ctx, torch, stream, flush, reps, warm):
    """64 independent commit_single calls, num_vars uniform in 10..20, BinaryPoly<64>,
    IPRS: one zg_commit_batch (graph replay, autotuned) against 64 sequential
    zg_commit calls from the same page-locked host buffers; roots compared."""
    rng = np.random.default_rng(0x5A1F)
    nvs = [int(v) for v in rng.integers(10, 21, size=64)]
    pps = {}
    for nv in sorted(set(nvs)):
        zt = Z.ZipTypes(1, 64, 5, 4, 147)
        pps[nv] = Z.ZipPlus.setup(1 << nv, Z.IprsCode(layout_row_len(nv)), zt, ctx=ctx)
    plist = [pps[nv] for nv in nvs]
    polys = [torch.from_numpy(random_binary(rng, nv, 64)).pin_memory().numpy() for nv in nvs]
    total = sum(1 << nv for nv in nvs)

    def ev_time(fn):
        with torch.cuda.stream(stream):
            flush.zero_()
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    def batched():
        return Z.ZipPlus.commit_batch(plist, polys, ctx, Z.BatchOpts.make(lanes=4))

    def sequential():
        roots = []
        for pp, poly in zip(plist, polys):
            h, c = Z.ZipPlus.commit(pp, [poly])
            h.close()
            roots.append(c.root)
        return roots

    for _ in range(warm):
        batched()
        sequential()
    launches0 = ctx.kernel_launches
    tb, comms = [], None
    for _ in range(reps):
        ms, comms = ev_time(batched)
        tb.append(ms)
    launches = (ctx.kernel_launches - launches0) / reps
    ts, seq_roots = [], None
    for _ in range(reps):
        ms, seq_roots = ev_time(sequential)
        ts.append(ms)
    same = [c.root for c in comms] == seq_roots
    # the eight largest polynomials (num_vars 19-20) alone, one after another:
    # each fills the GPU by itself, so no batching of the 64 can beat this time
    big = [i for i, nv in enumerate(nvs) if nv >= 19]

    def sequential_big():
        for i in big:
            h, _c = Z.ZipPlus.commit(plist[i], [polys[i]])
            h.close()

    tl = []
    for _ in range(reps):
        ms, _ = ev_time(sequential_big)
        tl.append(ms)
    b, q = statistics.median(tb), statistics.median(ts)
    return {
        "workload": "64 polynomials, num_vars uniform 10..20, BinaryPoly<64> Bernoulli(0.5), "
                    "IPRS rate 1/4, row_len 2^min(nv,14); commit_single each (own Merkle tree)",
        "evals": total, "value": total / (b / 1e3), "unit": "evals/s", "ms": b,
        "sequential": {"value": total / (q / 1e3), "ms": q},
        "batched_over_sequential": q / b, "roots_equal_sequential": same,
        "largest_alone": {"polys": len(big), "evals": sum(1 << nvs[i] for i in big), "ms": statistics.median(tl),
                          "what": "only the num_vars >= 19 polynomials, committed one after another: a lower "
                                  "bound for any schedule of the 64"},
        "gpu_launches_per_call": launches, "reps": reps,
        "mode": "zg_commit_batch: same-shape groups in one launch chain, 4 lanes, autotuned "
                "kernel variants, one CUDA graph replay per call; inputs in page-locked host "
                "memory, copied to the device inside the timed region (DMA in the graph); "
                "sequential: zg_commit per polynomial from the same buffers",
    }


def run_serving(Z, ctx, torch, n_req, workers, seed=0x5A1F):
    """Poisson stream of commit+prove requests, num_vars uniform 12..22,
    BinaryPoly<32|64> 50/50, through the request server; against the plain path
    (zg_commit_prove one request at a time) on the same requests."""
    rng = np.random.default_rng(seed)
    pps, pool = {}, {}
    reqs = []
    for _ in range(n_req):
        nv = int(rng.integers(12, 23))
        D = 32 if rng.random() < 0.5 else 64
        if (D, nv) not in pps:
            zt = Z.ZipTypes(1, D, 5, 4, 147)
            pps[(D, nv)] = Z.ZipPlus.setup(1 << nv, Z.IprsCode(layout_row_len(nv)), zt, ctx=ctx)
            pool[(D, nv)] = [torch.from_numpy(random_binary(rng, nv, D)).pin_memory().numpy()
                             for _ in range(3)]
        poly = pool[(D, nv)][len(reqs) % 3]
        point = [int(v) for v in rng.integers(-(2**40), 2**40, size=nv)]
        reqs.append((pps[(D, nv)], poly, point))
    total = sum(1 << r[0].num_vars for r in reqs)
    for k, pp in pps.items():  # warm every shape
        Z.ZipPlus.commit_prove(pp, [pool[k][0]], [1] * pp.num_vars)
    t0 = time.perf_counter()
    plain_lat, plain_out = [], []
    for i, (pp, poly, pt) in enumerate(reqs):
        a = time.perf_counter()
        out = Z.ZipPlus.commit_prove(pp, [poly], pt)
        plain_lat.append((time.perf_counter() - a) * 1e3)
        if i < 32:
            plain_out.append(out)
    plain_s = time.perf_counter() - t0
    srv = Z.ZipServer(ctx, workers=workers)
    ids = [srv.submit(pp, pool[k][0], [1] * pp.num_vars) for k, pp in pps.items()]
    for i in ids:
        srv.wait(i)
    s0 = srv.stats()
    rate = 2.0 * n_req / plain_s  # arrivals at twice the plain path's request rate
    gaps = rng.exponential(1.0 / rate, size=n_req)
    t0 = time.perf_counter()
    tnext, ids = t0, []
    for (pp, poly, pt), g in zip(reqs, gaps):
        tnext += g
        d = tnext - time.perf_counter()
        if d > 0:
            time.sleep(d)
        ids.append(srv.submit(pp, poly, pt))
    res = [srv.wait(i) for i in ids]
    served_s = time.perf_counter() - t0
    st = srv.stats()
    # latency at a sustainable load: arrivals at 70% of the measured served rate
    n_light = min(n_req, 400)
    light_rate = 0.7 * n_req / served_s
    lgaps = rng.exponential(1.0 / light_rate, size=n_light)
    t1 = time.perf_counter()
    tnext, lids = t1, []
    for (pp, poly, pt), g in zip(reqs[:n_light], lgaps):
        tnext += g
        d = tnext - time.perf_counter()
        if d > 0:
            time.sleep(d)
        lids.append(srv.submit(pp, poly, pt))
    light = [srv.wait(i)[3] for i in lids]
    srv.close()
    same = all(res[i][:3] == plain_out[i] for i in range(len(plain_out)))
    lat = [r[3].latency_ms for r in res]
    q = [r[3].queue_ms for r in res]
    return {
        "workload": f"Poisson stream of {n_req} commit+prove requests, num_vars uniform 12..22, "
                    "BinaryPoly<32>/<64> 50/50 (Bernoulli(0.5)), IPRS rate 1/4, "
                    "row_len 2^min(nv,14), random i128 points; inputs in page-locked host "
                    "memory (3 distinct polynomials per shape)",
        "requests": n_req, "evals": total, "arrival_rate_per_s": rate,
        "value": total / served_s, "unit": "evals/s", "seconds": served_s,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "queue_p50": float(np.percentile(q, 50)),
                       "what": "submit -> proof written, wall clock, arrivals at 2x the "
                               "plain path's rate (the queue grows)"},
        "plain": {"value": total / plain_s, "seconds": plain_s,
                  "latency_ms": {"p50": float(np.percentile(plain_lat, 50)),
                                 "p99": float(np.percentile(plain_lat, 99))},
                  "mode": "zg_commit_prove one request at a time, no queueing"},
        "served_over_plain": plain_s / served_s,
        "latency_at_70pct_load_ms": {
            "p50": float(np.percentile([r.latency_ms for r in light], 50)),
            "p99": float(np.percentile([r.latency_ms for r in light], 99)),
            "requests": n_light, "arrival_rate_per_s": light_rate,
            "what": "same server, Poisson arrivals at 70% of the served throughput above"},
        "results_equal_plain": same, "checked": len(plain_out),
        "workers": workers, "groups": st.groups - s0.groups,
        "peak_reserved_gb": st.peak_reserved / 1e9, "budget_gb": st.budget / 1e9,
        "phase_ms": {"input": st.ms_input - s0.ms_input, "commit": st.ms_commit - s0.ms_commit,
                     "prime": st.ms_prime - s0.ms_prime, "prove": st.ms_prove - s0.ms_prove},
        "mode": "zg_server: continuous batching, HBM-budget admission, small same-shape "
                "requests share a launch chain, codewords and Merkle layers device-resident "
                "until prove",
    }


def cpr_group_arrays(rng, nv, p, L, n_mles=35):
    """MLE inners and the comb of a BigLinear CPR sumcheck group (selector,
    eq_r, 17 up and 16 down columns; degree 3) in the reference's shape: the
    folded linear constraints, times eq_r and (1 - selector).  Random field
    elements stand in for the trace, which does not change the work."""
    top = p >> (64 * (L - 1))
    mles = rng.integers(0, 2**63, size=(n_mles, 1 << nv, L), dtype=np.uint64)
    mles[..., L - 1] %= np.uint64(top)
    prods = [(int.from_bytes(rng.bytes(8 * L), "little") % p, [j]) for j in range(2, n_mles)]
    one = (1 << (64 * L)) % p
    factors = [(0, one, 1), (one, p - one, 0)]
    return mles, prods, factors


def run_sumcheck(Z, ctx, torch, stream, nv, cpu_nv, with_cpu):
    """Config 4's CPR sumcheck group (2^nv points, 35 MLEs, degree 3, a 192-bit
    MontyField<3> prime from the transcript): MultiDegreeSumcheck on the GPU with
    device-resident MLEs, against the oracle on the host cores at 2^cpu_nv points."""
    from oracle import oracle as O

    O.build()
    t = O.Transcript()
    t.absorb_slice(b"bench-sumcheck")
    L = 3
    p = t.get_prime(L)
    rng = np.random.default_rng(0x5A1F)
    mles, prods, factors = cpr_group_arrays(rng, nv, p, L)
    dev = torch.from_numpy(mles.view(np.uint8).reshape(-1)).cuda()
    torch.cuda.synchronize()
    grp = Z.SumcheckGroup(3, dev.data_ptr(), prods, n_mles=mles.shape[0], factors=factors)

    def run():
        tr = Z.PcsProverTranscript()
        out = Z.MultiDegreeSumcheck.prove_as_subprotocol(tr, p, L, nv, [grp], ctx)
        tr.close()
        return out

    for _ in range(2):
        run()
    times = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        proof = run()[0]
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    gpu_ms = statistics.median(times)
    res = {"workload": f"BigLinear CPR group: 2^{nv} points, 35 MLEs, degree 3 (33 folded linear "
                       "terms times eq_r and (1 - selector)), MontyField<3> with a transcript-sampled "
                       "192-bit prime; MLEs device-resident; MultiDegreeSumcheck",
           "value": (1 << nv) / (gpu_ms / 1e3), "unit": "hypercube points/s", "ms": gpu_ms,
           "proof_bytes": len(proof)}
    if with_cpu:
        small, sprods, sfac = cpr_group_arrays(np.random.default_rng(7), cpu_nv, p, L)
        O.set_threads(os.cpu_count() or 1)
        a = time.perf_counter()
        want = O.sumcheck_prove(O.Transcript(), p, L, cpu_nv, [(3, small, sprods, sfac)], True)
        cpu_s = time.perf_counter() - a
        dsmall = torch.from_numpy(small.view(np.uint8).reshape(-1)).cuda()
        torch.cuda.synchronize()
        tr = Z.PcsProverTranscript()
        got = Z.MultiDegreeSumcheck.prove_as_subprotocol(
            tr, p, L, cpu_nv, [Z.SumcheckGroup(3, dsmall.data_ptr(), sprods, n_mles=35,
                                               factors=sfac)], ctx)
        tr.close()
        res["cpu_baseline"] = {"value": (1 << cpu_nv) / cpu_s, "unit": "hypercube points/s",
                               "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": f"oracle MultiDegreeSumcheck at 2^{cpu_nv} points, {cpu_s:.2f} s"}
        res["proof_equal_oracle_at_cpu_size"] = got[0] == want[0]
    return res


# ------------------------------------------------------------------- ours
def algorithmic_bytes(kernel, info, nv, D):
    """Algorithmic HBM bytes of one launch of `kernel` for one polynomial."""
    R, C, L = info.num_rows, info.codeword_len, info.row_len
    N = R * L
    table = {
        "k_base_bin": N * 8 + info.base_dim * info.base_len * 4 + R * C * D * 4,
        "k_stages2_bin": R * C * D * 4 + R * C * D * 8,
        "k_tree_levels": C * 32,
        "k_stage_bin[0]": R * C * D * 4 + R * C * D * 8,
        "k_stage_bin[1+]": 2 * R * C * D * 8,
        "k_leaf_small": R * C * D * 8 + C * 32,
        "k_leaf_chunks": R * C * D * 8 + C * ((R * D * 8 + 1023) // 1024) * 32,
        "k_project_rows": N * 8 + L * 32 + N * 40,
        "k_raa_bin": N * 8 + R * C * D * 4,
    }
    return table.get(kernel)


def plain_line(Z, ctx, torch, stream, flush, spec, K, W, with_cpu, cpu_seconds, verify=False, seed=77):
    """One plain Zip/Zip+ workload, one request per step: zg_commit_prove from
    device-resident inputs (`value`) and from page-locked host inputs with the
    proof copied back (`e2e`), CUDA events on the library's stream with the L2
    flushed between steps; optionally ZipPlus::verify of the last proof (wall
    clock).  The oracle times the same workload on all host cores for a bounded
    sample (the CPU baseline)."""
    ek, D, ck, nv, L = spec
    n = 1 << nv
    zt = Z.ZipTypes(ek, D if ek else 1, 5 if ek else 3, 4, 147)
    code = Z.IprsCode(L) if ck == 0 else Z.RaaCode(L)
    pp = Z.ZipPlus.setup(n, code, zt, ctx=ctx)
    lib = Z.lib()
    rng = np.random.default_rng(seed)
    cnt = min(K + W, 8)
    if ek:
        host = np.stack([random_binary(rng, nv, D) for _ in range(cnt)])
        host_t = torch.from_numpy(host.view(np.int64)).pin_memory()
    else:
        host = rng.integers(-(2**15), 2**15, size=(cnt, n), dtype=np.int32)
        host_t = torch.from_numpy(host).pin_memory()
    dev_t = host_t.to("cuda")
    point = Z.i128_bytes([1] * nv)
    cap = pp.proof_size(1)
    proof_t = torch.empty(cap, dtype=torch.uint8).pin_memory()
    proof = C.c_void_p(proof_t.data_ptr())
    root, ev, plen = C.create_string_buffer(32), C.create_string_buffer(32), C.c_size_t(cap)

    def step(i, on_dev):
        plen.value = cap
        if on_dev:
            Z.check(lib.zg_commit_prove_d(pp.handle, C.c_void_p(dev_t[i % cnt].data_ptr()), 1,
                                          C.c_char_p(point), root, ev, proof, C.byref(plen)))
        else:
            ptrs = (C.c_void_p * 1)(host_t[i % cnt].data_ptr())
            Z.check(lib.zg_commit_prove(pp.handle, ptrs, 1, C.c_char_p(point), root, ev, proof,
                                        C.byref(plen)))

    def timed(on_dev):
        out = []
        for i in range(K):
            with torch.cuda.stream(stream):
                flush.zero_()
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step(W + i, on_dev)
            e1.record(stream)
            out.append((e0, e1))
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in out]

    for i in range(W):
        step(i, True)
        step(i, False)
    dev_ms, host_ms = timed(True), timed(False)
    res = {"num_vars": nv, "row_len": L, "num_rows": pp.num_rows,
           "eval": f"BinaryPoly<{D}> Bernoulli(0.5)" if ek else "i32 uniform [-2^15, 2^15)",
           "code": ("IPRS rate 1/4" if ck == 0 else "RAA rate 1/4"),
           "value": K * n / (sum(dev_ms) / 1e3), "unit": "evals/s", "ms": sum(dev_ms) / K,
           "e2e": {"value": K * n / (sum(host_ms) / 1e3), "unit": "evals/s", "ms": sum(host_ms) / K,
                   "h2d_bytes_per_step": int(host_t[0].numel() * host_t.element_size()),
                   "d2h_bytes_per_step": int(plen.value + 64)},
           "latency_ms": {"p50": float(np.percentile(host_ms, 50)), "p99": float(np.percentile(host_ms, 99))},
           "proof_bytes": int(plen.value)}
    vproof = bytes(proof_t[: plen.value].numpy())
    comm = Z.ZipPlusCommitment(root.raw, 1)
    if verify:
        Z.ZipPlus.verify(pp, comm, [1] * nv, ev.raw, vproof)
        vt = []
        for _ in range(5):
            a = time.perf_counter()
            Z.ZipPlus.verify(pp, comm, [1] * nv, ev.raw, vproof)
            vt.append((time.perf_counter() - a) * 1e3)
        res["verify_ms"] = statistics.median(vt)
        res["commit_prove_verify_e2e_evals_per_s"] = n / ((res["e2e"]["ms"] + res["verify_ms"]) / 1e3)
    if with_cpu:
        from oracle import oracle as O

        O.build()
        threads = os.cpu_count() or 1
        O.set_threads(threads)
        desc = O.make_desc(ek, D, ck, nv, L)
        want = O.commit_prove(desc, host[(W + K - 1) % cnt], 1, [1] * nv)
        res["equal_oracle"] = (want[0] == root.raw and want[1] == vproof and want[2] == ev.raw[:len(want[2])])
        steps, lat, t0 = 0, [], time.perf_counter()
        while steps < 50 and (time.perf_counter() - t0 < cpu_seconds or steps < 2):
            a = time.perf_counter()
            O.commit_prove(desc, host[steps % cnt], 1, [1] * nv)
            lat.append(time.perf_counter() - a)
            steps += 1
        cpu = {"value": steps * n / sum(lat), "unit": "evals/s", "cores": threads, "kind": "port",
               "sample": f"{steps} commit+prove steps of this workload, {sum(lat):.1f} s, OpenMP on {threads} "
                         "threads: base layer over rows x positions, stages over rows x chunk columns, "
                         "leaves over columns, tree pairs per level, prove over rows/columns"}
        if verify:
            a = time.perf_counter()
            rc = O.verify(desc, root.raw, 1, [1] * nv, ev.raw, vproof)
            cpu["verify_ms"] = (time.perf_counter() - a) * 1e3
            cpu["oracle_accepts_gpu_proof"] = rc == 0
        res["cpu_baseline"] = cpu
        res["e2e_over_cpu"] = res["e2e"]["value"] / cpu["value"]
    pp.close()
    return res


def run_ours(args):
    import torch

    rank, world = env_int("RANK", 0), env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    import zipgpu as Z
    from zipgpu import replicas

    workload = args.workload
    ek, D, ck, nv, L = WORKLOADS[workload]
    ctx = Z.Context(local)
    zt = Z.ZipTypes(ek, D if ek else 1, 5 if ek else 3, 4, 147)
    code = Z.IprsCode(L) if ck == 0 else Z.RaaCode(L)
    pp = Z.ZipPlus.setup(1 << nv, code, zt, ctx=ctx)
    lib = Z.lib()
    K, W = args.steps, args.warmup
    n = 1 << nv
    host = make_inputs(workload, K + W, 1000 + rank)
    dtype = torch.int64 if ek else torch.int32
    host_t = torch.from_numpy(host.view(np.int64) if ek else host).pin_memory()
    dev_t = host_t.to("cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream)
    point = Z.i128_bytes([1] * nv)
    cap = pp.proof_size(1)
    proof_t = torch.empty(cap, dtype=torch.uint8).pin_memory()  # page-locked: D2H lands in place
    proof = C.c_void_p(proof_t.data_ptr())
    root = C.create_string_buffer(32)
    ev = C.create_string_buffer(32)
    plen = C.c_size_t(cap)
    eb = host_t.element_size() * n

    def step_device(i):
        plen.value = cap
        Z.check(lib.zg_commit_prove_d(pp.handle, C.c_void_p(dev_t[i].data_ptr()), 1,
                                      C.c_char_p(point), root, ev, proof, C.byref(plen)))

    def step_host(i):
        plen.value = cap
        ptrs = (C.c_void_p * 1)(host_t[i].data_ptr())
        Z.check(lib.zg_commit_prove(pp.handle, ptrs, 1, C.c_char_p(point), root, ev, proof,
                                    C.byref(plen)))

    B = args.batch
    nl = args.lanes
    pts = (Z.i128_bytes([1] * nv)) * B
    proofs_b = [torch.empty(cap, dtype=torch.uint8).pin_memory() for _ in range(B)]
    pptrs = (C.c_void_p * B)(*[t.data_ptr() for t in proofs_b])
    plens = (C.c_size_t * B)()
    roots_b = C.create_string_buffer(32 * B)
    evs_b = C.create_string_buffer(32 * B)
    lat_b = (C.c_double * B)()
    host_b = make_inputs(workload, B, 5000 + rank)
    host_bt = torch.from_numpy(host_b.view(np.int64) if ek else host_b).pin_memory()
    dev_bt = host_bt.to("cuda")
    lat_batched = []

    def step_batched(on_device):
        for j in range(B):
            plens[j] = cap
        src = dev_bt if on_device else host_bt
        ptrs = (C.c_void_p * B)(*[src[j].data_ptr() for j in range(B)])
        Z.check(lib.zg_commit_prove_many(pp.handle, B, ptrs, 1 if on_device else 0,
                                         C.c_char_p(pts), roots_b, evs_b, pptrs, plens, nl, lat_b))
        lat_batched.extend(lat_b[j] for j in range(B))

    def timed(step):
        times = []
        for i in range(K):
            with torch.cuda.stream(stream):
                flush.zero_()
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step(W + i)
            e1.record(stream)
            times.append((e0, e1))
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in times]

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, "cuda")

    # warm-up: device path and host path
    for i in range(W):
        step_device(i)
        step_host(i)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    lat_dev = timed(step_device)
    barrier()
    total_dev = max_over_ranks(sum(lat_dev))
    barrier()
    lat_host = timed(step_host)
    barrier()
    total_host = max_over_ranks(sum(lat_host))
    proof_len = plen.value

    # batched form: B independent requests per step over `nl` lanes
    for i in range(W):
        step_batched(True)
        step_batched(False)
    lat_batched.clear()
    barrier()
    launches0 = ctx.kernel_launches
    lat_bdev = timed(lambda i: step_batched(True))
    barrier()
    launches = ctx.kernel_launches - launches0
    total_bdev = max_over_ranks(sum(lat_bdev))
    req_lat = list(lat_batched)
    barrier()
    lat_bhost = timed(lambda i: step_batched(False))
    barrier()
    total_bhost = max_over_ranks(sum(lat_bhost))
    clock_info = clocks.stop()

    # per-kernel CUDA-event timing pass (same workload, separate K steps)
    ctx.set_kernel_timing(True)
    ctx.kernel_times()
    timed(step_device)
    alltimes = ctx.kernel_times()
    ctx.set_kernel_timing(False)
    ktimes = {k: v for k, v in alltimes.items() if not k.startswith("host:")}
    host_phases = {k[5:]: round(v[1] / K, 4) for k, v in alltimes.items() if k.startswith("host:")}

    # every rank committed its own K (x B) polynomials: whole-job units over the
    # slowest rank's time (the totals above are already maxima over ranks)
    plain_value = replicas.sum_over_ranks(K * n, dist, "cuda") / (total_dev / 1e3)
    plain_e2e = replicas.sum_over_ranks(K * n, dist, "cuda") / (total_host / 1e3)
    value = replicas.sum_over_ranks(K * B * n, dist, "cuda") / (total_bdev / 1e3)
    e2e = replicas.sum_over_ranks(K * B * n, dist, "cuda") / (total_bhost / 1e3)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_kind = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    dom = max(ktimes.items(), key=lambda kv: kv[1][1]) if ktimes else None
    roofline = None
    if dom:
        name, (cnt, ms) = dom
        avg_ms = ms / cnt
        info = pp.info
        ab = algorithmic_bytes(name, info, nv, D)
        launches_per_step = cnt / K
        traffic = None
        try:
            tr = json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic.json")))
            traffic = tr.get(workload, {}).get(name)
        except Exception:
            pass
        achieved = (ab / (avg_ms / 1e3) / 1e9) if ab else None
        roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm,
                    "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                    "traffic": traffic, "algorithmic_bytes": ab, "avg_launch_ms": avg_ms,
                    "launches_per_step": launches_per_step,
                    "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)",
                    "kernel_share": {k: round(v[1] / sum(x[1] for x in ktimes.values()), 4)
                                     for k, v in sorted(ktimes.items(), key=lambda kv: -kv[1][1])}}
    # ZipPlus::verify of the last plain proof (opened positions encoded on the GPU)
    verify = None
    if rank == 0:
        vproof = bytes(proof_t[: plen.value].numpy())
        comm = Z.ZipPlusCommitment(root.raw, 1)
        pts_v = [1] * nv
        Z.ZipPlus.verify(pp, comm, pts_v, ev.raw, vproof)
        vt = []
        for _ in range(5):
            a = time.perf_counter()
            Z.ZipPlus.verify(pp, comm, pts_v, ev.raw, vproof)
            vt.append((time.perf_counter() - a) * 1e3)
        verify = {"ms": statistics.median(vt), "what": "zg_verify of one proof of the workload, wall "
                  "clock; the 147 opened codeword positions are encoded on the GPU, the rest on the host"}
        if not args.no_cpu_baseline:
            from oracle import oracle as O

            O.build()
            desc = O.make_desc(ek, D, ck, nv, L)
            a = time.perf_counter()
            rc = O.verify(desc, root.raw, 1, pts_v, ev.raw, vproof)
            verify["cpu_baseline_ms"] = (time.perf_counter() - a) * 1e3
            verify["cpu_baseline_kind"] = "port (oracle, OpenMP, full encode_wide as the reference)"
            verify["oracle_accepts"] = rc == 0
    sections = {}
    if not args.no_extra:
        with_cpu = rank == 0 and not args.no_cpu_baseline
        cs = args.cpu_seconds_per_config
        # the configurations besides the headline, each a plain line of its own
        sections["config1_zip_i32_iprs_nv12_flat"] = plain_line(
            Z, ctx, torch, stream, flush, (0, 1, 0, 12, 4096), K, W, with_cpu, cs, verify=True)
        sections["config1_zip_i32_iprs_nv12_square"] = plain_line(
            Z, ctx, torch, stream, flush, (0, 1, 0, 12, 64), K, W, with_cpu, cs, verify=True)
        sections["config2_zipplus_binpoly32_raa_nv16"] = plain_line(
            Z, ctx, torch, stream, flush, (1, 32, 1, 16, 256), K, W, with_cpu, cs, verify=True)
        sections["config2_zipplus_binpoly32_iprs_nv16_plain"] = plain_line(
            Z, ctx, torch, stream, flush, (1, 32, 0, 16, 1 << 14), K, W, with_cpu, cs, verify=True)
        nv20 = plain_line(Z, ctx, torch, stream, flush, (1, 32, 0, 20, 1 << 14), min(K, 10), W, with_cpu,
                          cs, verify=True)
        nv20["target"] = "plain GPU commit+prove >= 20x the host-CPU path at num_vars = 20 (e2e_over_cpu)"
        sections["north_star_binpoly32_iprs_nv20_plain"] = nv20
        sections["sumcheck"] = run_sumcheck(Z, ctx, torch, stream, 18, 14, with_cpu)
        sections["piop_steps"] = run_piop_steps(Z, ctx, torch, stream, 18, 14, with_cpu)
        sections["zinc_prove_mle_first"] = run_zinc_prove(Z, ctx, 18, 18, with_cpu)
        sections["batched_commit"] = run_batched_commit(Z, ctx, torch, stream, flush, reps=5, warm=2)
        sections["serving"] = run_serving(Z, ctx, torch, args.serve_requests, args.serve_workers,
                                          seed=0x5A1F + rank)
    sections["verify"] = verify
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_commit_prove_rate(workload, args.cpu_seconds, 50, host[:4])
        cpu.pop("latency_ms", None)
    if roofline:
        # the whole path against HBM: evals/s x algorithmic bytes per evaluation
        # (2 * eval bytes + 4 * codeword-entry bytes: inputs read twice, the
        # codeword written once and read back by the leaves, prove and openings)
        ebytes = 8 if ek else 4
        cw_entry = (8 * D if ck == 0 else 4 * D) if ek else 16
        bpe = 2 * ebytes + 4 * cw_entry
        roofline["path"] = {"bytes_per_eval": bpe, "achieved_gbs": value * bpe / 1e9,
                            "frac": value * bpe / 1e9 / hbm,
                            "what": "batched evals/s x bytes per evaluation over the measured HBM peak"}
        roofline["note"] = ("kernel figures are timed on the plain path (one request per step, CUDA events "
                            "per launch); value is the batched path")
        if roofline.get("kernel", "").startswith("k_leaf"):
            # the leaf hashing is bound by the integer ALU pipe: BLAKE3 compressions
            # per second against that pipe's issue rate
            info = pp.info
            per_leaf = max(1, (info.num_rows * (8 * D if ek else 16) + 63) // 64)
            comp = info.codeword_len * per_leaf
            if per_leaf <= 16 and info.codeword_len % 128 == 0:
                # the leaf kernel also reduces each block's 128 leaves to their
                # subtree root: 127 parent compressions per 128 leaves
                comp += info.codeword_len // 128 * 127
            alu_per_comp = 584  # ALU-pipe instructions per compression, ncu (profiles/)
            sm_mhz = (clock_info or {}).get("sm_mhz") or 1965.0
            sms = torch.cuda.get_device_properties(local).multi_processor_count
            peak = sms * 64 * sm_mhz * 1e6 / alu_per_comp
            achieved = comp / (roofline["avg_launch_ms"] / 1e3)
            roofline["int_alu"] = {"bound": "alu", "unit": "BLAKE3 compressions/s", "achieved": achieved,
                                   "peak": peak, "frac": achieved / peak, "compressions_per_launch": comp,
                                   "peak_basis": f"{sms} SMs x 64 ALU lanes/clk x {sm_mhz:.0f} MHz / "
                                                 f"{alu_per_comp} ALU instructions per compression (ncu)"}
    if rank == 0:
        for name, obj in sections.items():
            if obj is not None:
                print(json.dumps({"section": name, **obj}), flush=True)
        all_lat = lat_dev
        print(json.dumps({"section": "plain_headline_workload", "value": plain_value, "e2e": plain_e2e,
                          "ms_per_step": total_dev / K, "e2e_ms_per_step": total_host / K,
                          "latency_ms": {"p50": float(np.percentile(all_lat, 50)),
                                         "p99": float(np.percentile(all_lat, 99))},
                          "e2e_latency_ms": {"p50": float(np.percentile(lat_host, 50)),
                                             "p99": float(np.percentile(lat_host, 99))},
                          "host_phases_ms_per_step": host_phases,
                          "kernel_ms_per_step": {k: round(v[1] / K, 4) for k, v in
                                                 sorted(ktimes.items(), key=lambda kv: -kv[1][1])},
                          "kernel_share": roofline.pop("kernel_share", None) if roofline else None}),
              flush=True)

        def brief(name, keys):
            o = sections.get(name)
            return {k: o.get(k) for k in keys} if o else None

        summary = {
            "config1_flat": brief("config1_zip_i32_iprs_nv12_flat", ["value", "verify_ms", "e2e_over_cpu"]),
            "config1_square": brief("config1_zip_i32_iprs_nv12_square", ["value", "verify_ms", "e2e_over_cpu"]),
            "config2_raa": brief("config2_zipplus_binpoly32_raa_nv16", ["value", "e2e_over_cpu"]),
            "nv20_plain": brief("north_star_binpoly32_iprs_nv20_plain", ["value", "e2e_over_cpu"]),
            "batched_commit": brief("batched_commit", ["value", "batched_over_sequential"]),
            "serving": brief("serving", ["value", "served_over_plain", "requests"]),
            "zinc_prove": brief("zinc_prove_mle_first", ["ms", "equal_oracle_at_full_size", "oracle_verifier_accepts",
                                                         "speedup_over_cpu"]),
        }
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": total_bdev / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": config_of(workload, pp.num_rows, pp.info.depth),
            "mode": f"batched: {B} commit+prove requests per step over {nl} lanes (zg_commit_prove_many)",
            "latency_ms": {"p50": float(np.percentile(req_lat, 50)),
                           "p99": float(np.percentile(req_lat, 99))},
            "e2e": {"value": e2e, "unit": "evals/s", "h2d_bytes_per_step": eb * B,
                    "d2h_bytes_per_step": (proof_len + 64) * B, "ms_per_step": total_bhost / K},
            "plain": {"value": plain_value, "e2e": plain_e2e},
            "batched_over_plain": value / plain_value,
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clock_info,
            "summary": summary,
            "impl": "ours",
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_commit_case(nv, D):
    """Two commits of one seeded BinaryPoly<D> polynomial with 2^nv evaluations
    (IPRS, row_len 2^min(nv, 14)): a small, fixed launch sequence for ncu captures."""
    import zipgpu as Z

    ctx = Z.Context(env_int("LOCAL_RANK", 0))
    zt = Z.ZipTypes(1, D, 5, 4, 147)
    pp = Z.ZipPlus.setup(1 << nv, Z.IprsCode(layout_row_len(nv)), zt, ctx=ctx)
    poly = random_binary(np.random.default_rng(1), nv, D)
    for _ in range(2):
        hint, comm = Z.ZipPlus.commit(pp, [poly])
        hint.close()
    print(json.dumps({"commit_case": {"num_vars": nv, "D": D, "root": comm.root.hex()}}))
    return 0


def run_piop_steps(Z, ctx, torch, stream, nv, cpu_nv, with_cpu):
    """Zinc+ prover steps 3 and 6 on a BigLinear-shaped trace (16 BinaryPoly<32>
    columns and 1 integer column, 2^nv rows, a 192-bit MontyField<3> prime):
    device-resident columns through the C ABI, CUDA events on the library's
    stream; the oracle at 2^cpu_nv rows on one host core as the CPU baseline."""
    from oracle import oracle as O

    O.build()
    t = O.Transcript()
    t.absorb_slice(b"bench-piop")
    L, D, n_bin, n_int = 3, 32, 16, 1
    p = t.get_prime(L)
    rng = np.random.default_rng(0x9109)
    R = 1 << (64 * L)

    def inner(v):
        x = (v % p) * R % p
        return [(x >> (64 * i)) & ((1 << 64) - 1) for i in range(L)]

    def cols(n):
        b = rng.integers(0, 1 << 32, size=(n_bin, 1 << n), dtype=np.uint64)
        i = rng.integers(-2**40, 2**40, size=(n_int, 1 << n), dtype=np.int64)
        return b, i

    b, i = cols(nv)
    a = np.array(inner(int.from_bytes(rng.bytes(24), "little")), np.uint64)
    r = np.array([inner(int.from_bytes(rng.bytes(24), "little")) for _ in range(nv)], np.uint64)
    bd, id_ = torch.from_numpy(b.view(np.int64)).cuda(), torch.from_numpy(i).cuda()
    mles = torch.empty((n_bin + n_int) * (1 << nv) * L, dtype=torch.int64, device="cuda")
    coeffs = np.zeros((n_bin * D + n_int, L), np.uint64)
    torch.cuda.synchronize()
    mod = p.to_bytes(8 * L, "little")
    lib = Z.lib()

    def step3():
        Z.check(lib.zg_piop_eval_projection(ctx.handle, mod, L, bd.data_ptr(), n_bin, D, id_.data_ptr(), n_int,
                                            nv, a.ctypes.data, 1, mles.data_ptr()))

    def step6():
        Z.check(lib.zg_piop_lifted_evals(ctx.handle, mod, L, bd.data_ptr(), n_bin, D, id_.data_ptr(), n_int, nv,
                                         r.ctypes.data, 1, coeffs.ctypes.data))

    def timed(fn):
        for _ in range(2):
            fn()
        ts = []
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    shifts = [(k, 1) for k in range(n_bin)]  # BigLinear's down columns: the binary columns shifted by one row
    rp = np.array([inner(int.from_bytes(rng.bytes(24), "little")) for _ in range(nv)], np.uint64)

    def step5():
        tr = Z.PcsProverTranscript()
        Z.ZincPiop.multipoint_eval(ctx, tr, p, L, (mles.data_ptr(), n_bin + n_int), nv, rp, shifts)
        tr.close()

    # step 4 with BigLinear's linear constraints: the binary columns sum to the
    # integer column; down.bin[0] equals up.int; up.bin[i] equals down.bin[i]
    cons = []
    row = [1] * n_bin + [-1] + [0] * n_bin
    cons.append(row)
    row = [0] * (n_bin + 1) + [1] + [0] * (n_bin - 1)
    row[n_bin] = -1
    cons.append(row)
    for k in range(1, n_bin):
        row = [0] * (2 * n_bin + 1)
        row[k], row[n_bin + 1 + k] = 1, -1
        cons.append(row)

    def step4():
        tr = Z.PcsProverTranscript()
        Z.ZincPiop.cpr_linear_prove(ctx, tr, p, L, (mles.data_ptr(), n_bin + n_int), nv, rp, shifts, cons)
        tr.close()

    def step2():
        tr = Z.PcsProverTranscript()
        cf = Z.ZincPiop._mont_matrix(cons, p, L)
        pt2 = np.zeros((nv, L), np.uint64)
        comb2 = np.zeros((len(cons), D, L), np.uint64)
        lens = np.zeros(len(cons), np.uint32)
        src = np.array([sc for sc, _ in shifts], np.uint32)
        amt = np.array([c for _, c in shifts], np.uint32)
        Z.check(lib.zg_piop_ideal_check_linear(ctx.handle, tr.handle, mod, L, bd.data_ptr(), n_bin, D,
                                               id_.data_ptr(), n_int, nv, src.ctypes.data, amt.ctypes.data,
                                               len(shifts), len(cons), cf.ctypes.data, 1, pt2.ctypes.data,
                                               comb2.ctypes.data, lens.ctypes.data))
        tr.close()

    ms3, ms6 = timed(step3), timed(step6)
    ms5, ms4, ms2 = timed(step5), timed(step4), timed(step2)
    cells = (n_bin + n_int) << nv
    res = {"workload": f"BigLinear-shaped trace: {n_bin} BinaryPoly<{D}> + {n_int} integer columns, 2^{nv} rows, "
                       "MontyField<3> (192-bit prime from the transcript); columns resident on the device",
           "eval_projection": {"ms": ms3, "cells_per_s": cells / (ms3 / 1e3),
                               "output_bytes": cells * 8 * L},
           "lifted_evals": {"ms": ms6, "cells_per_s": cells / (ms6 / 1e3)},
           "ideal_check_linear": {"ms": ms2, "constraints": len(cons),
                                  "what": "point from the transcript, 17 up and 16 shifted columns evaluated "
                                          "coefficient-wise, constraints applied, trimmed values absorbed"},
           "cpr_linear": {"ms": ms4, "constraints": len(cons), "mles_in_sumcheck": 2 + n_bin + n_int + len(shifts),
                          "what": "folding challenge, selector, eq and down columns, degree-3 MultiDegreeSumcheck "
                                  "and the absorbed up/down evaluations over step 3's device-resident MLEs"},
           "multipoint_eval": {"ms": ms5, "shifts": len(shifts), "mles_in_sumcheck": 2 + 2 * len(shifts),
                               "what": "alphas/gammas, eq and shift selectors, precombination and the degree-2 "
                                       "MLSumcheck over step 3's device-resident MLEs"}}
    # parity at this size against the oracle on a sample of columns is in the tests;
    # here: the first MLE entries and the coefficients of the first column
    if with_cpu:
        bs, is_ = cols(cpu_nv)
        rs = r[:cpu_nv]
        a0 = time.perf_counter()
        want3 = O.piop_eval_projection(p, L, bs, D, is_, cpu_nv, a)
        c3 = time.perf_counter() - a0
        a0 = time.perf_counter()
        want6 = O.piop_lifted_evals(p, L, bs, D, is_, cpu_nv, rs)
        c6 = time.perf_counter() - a0
        got3 = Z.ZincPiop.eval_projection(ctx, p, L, bs, D, is_, cpu_nv, a)
        got6 = Z.ZincPiop.lifted_evals(ctx, p, L, bs, D, is_, cpu_nv, rs)
        cc = (n_bin + n_int) << cpu_nv
        res["cpu_baseline"] = {"eval_projection_cells_per_s": cc / c3, "lifted_evals_cells_per_s": cc / c6,
                               "cores": 1, "kind": "port",
                               "sample": f"oracle at 2^{cpu_nv} rows ({c3:.2f} s + {c6:.2f} s)"}
        # step 5 at a size the Python restatement finishes in seconds
        nv5 = 8
        m5 = O.piop_eval_projection(p, L, bs[:, : 1 << nv5], D, is_[:, : 1 << nv5], nv5, a)
        a0 = time.perf_counter()
        want5 = O.piop_multipoint_eval(O.Transcript(), p, L, m5, rp[:nv5], shifts)
        c5 = time.perf_counter() - a0
        tr = Z.PcsProverTranscript()
        got5 = Z.ZincPiop.multipoint_eval(ctx, tr, p, L, m5, nv5, rp[:nv5], shifts)
        tr.close()
        res["cpu_baseline"]["multipoint_eval_s_at_2^8_rows"] = c5
        res["equal_oracle_at_cpu_size"] = bool(np.array_equal(got3, want3) and np.array_equal(got6, want6)
                                               and got5[0] == want5[0])
    return res


def run_zinc_prove(Z, ctx, nv, cpu_nv, with_cpu):
    """The MLE-first Zinc+ prover end to end on BigLinearUair (16 BinaryPoly<32>
    columns, 1 i64 column, 16 shifts, 17 constraints; 2^nv rows; MontyField<3>;
    both tables IPRS rate 1/4 with 16 rows of 2^(nv-4), CombR Int<6>): the trace
    from host memory through zg_zinc_prove_mle_first to the Proof bytes in host
    memory, timed on the host clock (the call synchronises).  The CPU baseline is
    the oracle's C chain of the same steps at the same size on all host cores
    (its bytes must equal the GPU's), and the oracle's restated Zinc+ verifier
    must accept the GPU's proof."""
    from oracle import oracle as O
    from zipgpu import uair

    bins, ints = uair.trace(nv, 0xB16)
    shifts, coeffs = uair.signature()

    def tables(n):
        L = 1 << (n - 4)
        mk = lambda ek, D: Z.ZipPlus.setup(1 << n, Z.IprsCode(L, 0, 4), Z.ZipTypes(ek, D, 6, 3, 147), ctx=ctx)
        return mk(Z.EVAL_BINPOLY, 32), mk(Z.EVAL_I64, 1)

    pb, pi = tables(nv)
    proof = Z.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs)
    # a page-locked output buffer: the column openings arrive in place by DMA
    import torch

    pinned = torch.empty(len(proof) + (1 << 20), dtype=torch.uint8).pin_memory().numpy()
    Z.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs, out_buffer=pinned)
    ts = []
    for _ in range(3):
        a = time.perf_counter()
        again = Z.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs, out_buffer=pinned)
        ts.append((time.perf_counter() - a) * 1e3)
    ms = statistics.median(ts)
    # the reference's default path (MLE_FIRST = false) on the same trace
    cons = [[(int(c), [j]) for j, c in enumerate(row) if int(c) != 0] for row in coeffs]
    comb = Z.ZincPlusPiop.prove(pb, pi, nv, bins, 32, ints, shifts, cons, [False] * len(cons), mle_first=False)
    tc = []
    for _ in range(3):
        a = time.perf_counter()
        Z.ZincPlusPiop.prove(pb, pi, nv, bins, 32, ints, shifts, cons, [False] * len(cons), mle_first=False)
        tc.append((time.perf_counter() - a) * 1e3)
    res0 = {"combined_ms": statistics.median(tc), "combined_equals_mle_first": comb == proof}
    res = {"workload": f"BigLinearUair, 2^{nv} rows: 16 BinaryPoly<32> + 1 i64 column, 16 shifts, 17 constraints; "
                       "MontyField<3>; IPRS rate 1/4, 16 rows per table; 147 openings",
           "ms": ms, "rows_per_s": (1 << nv) / (ms / 1e3), "proof_bytes": len(proof),
           "deterministic": bytes(again) == proof, "h2d_bytes": int(bins.nbytes + ints.nbytes),
           "output": "page-locked host buffer (the column openings land in place by DMA)",
           "what": "commit both tables, prime, ideal check, evaluation projection, CPR sumcheck, multipoint "
                   "sumcheck, lifted evaluations, prove_f of both tables, Proof transcription"}
    res.update(res0)
    if with_cpu:
        O.build()
        threads = os.cpu_count() or 1
        O.set_threads(threads)
        L = 1 << (nv - 4)
        db = O.make_desc(O.EVAL_BINPOLY, 32, 0, nv, L, comb_limbs=6, field_limbs=3)
        di = O.make_desc(O.EVAL_I64, 1, 0, nv, L, comb_limbs=6, field_limbs=3)
        U = O.Uair.linear(16, 1, 32, shifts, coeffs, uair.ideal_roots())
        a = time.perf_counter()
        want = O.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=True)
        c = time.perf_counter() - a
        a = time.perf_counter()
        verdict = O.zinc_verify(db, di, nv, None, None, U, 3, proof)
        vs = time.perf_counter() - a
        res["cpu_baseline"] = {"ms": c * 1e3, "rows_per_s": (1 << nv) / c, "cores": threads, "kind": "port",
                               "sample": f"one proof by the oracle's C chain of steps 0-7 at 2^{nv} rows, OpenMP "
                                         f"on {threads} threads (commit, PIOP steps, sumchecks, prove_f)"}
        res["equal_oracle_at_full_size"] = want == proof
        res["oracle_verifier_accepts"] = verdict == 0
        res["oracle_verifier_ms"] = vs * 1e3
        res["speedup_over_cpu"] = c * 1e3 / ms
    return res


def run_zinc_prove_case(nv):
    """The MLE-first Zinc+ prover on BigLinearUair at 2^nv rows, one warm-up and
    one timed call: a fixed launch sequence for ncu launch lists."""
    import zipgpu as Z

    ctx = Z.Context(env_int("LOCAL_RANK", 0))
    out = run_zinc_prove(Z, ctx, nv, 10, False)
    print(json.dumps({"zinc_prove_case": {"num_vars": nv, "ms": out["ms"], "proof_bytes": out["proof_bytes"]}}))
    return 0


def run_sumcheck_case(nv):
    """One CPR sumcheck proof (2^nv points, device-resident MLEs), twice: a small,
    fixed launch sequence for ncu captures."""
    import torch
    import zipgpu as Z

    ctx = Z.Context(env_int("LOCAL_RANK", 0))
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = run_sumcheck(Z, ctx, torch, stream, nv, 10, False)
    print(json.dumps({"sumcheck_case": {"num_vars": nv, "ms": out["ms"]}}))
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=128, help="requests per batched step")
    ap.add_argument("--lanes", type=int, default=16, help="concurrent lanes of the batched form")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--cpu-seconds-per-config", type=float, default=4.0,
                    help="bounded CPU-baseline sample of each secondary configuration")
    ap.add_argument("--serve-requests", type=int, default=10000,
                    help="requests of the serving stream (the full stream is 10000)")
    ap.add_argument("--serve-workers", type=int, default=4)
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the secondary configurations (config 1, RAA, num_vars 20, batched "
                         "commit, serving, PIOP steps)")
    ap.add_argument("--sumcheck-case", type=int, metavar="NV",
                    help="only run the CPR sumcheck at 2^NV points (small case for ncu captures)")
    ap.add_argument("--zinc-prove-case", type=int, metavar="NV",
                    help="only run the MLE-first Zinc+ prover on BigLinear at 2^NV rows (launch lists)")
    ap.add_argument("--commit-case", type=int, nargs=2, metavar=("NV", "D"),
                    help="only commit one seeded polynomial twice (small case for ncu captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.commit_case:
        return run_commit_case(*args.commit_case)
    if args.sumcheck_case:
        return run_sumcheck_case(args.sumcheck_case)
    if args.zinc_prove_case:
        return run_zinc_prove_case(args.zinc_prove_case)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
