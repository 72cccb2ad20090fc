"""Benchmark: certificates/s (exact BZ distances) on the 1024-code uneven batch, and the
roofline of the dominant pair-sweep kernel (the tcgen05 int8 sweep of full-rank sets; the
CUDA-core POPC sweep's integer-pipe roofline is reported beside it).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--codes 1024] [--workload batch|collect|mitm|css128|...]

A step certifies every code of the batch (512 classical [n in 48..128, k in n/4..n/2] +
512 CSS [n in 40..128, ranks in n/5..n/3], seed 3; CSS codes solved with which='min').
`value` is certificates per second from device time with the inputs resident; `e2e` is
the same metric through the public C ABI from host matrices (host<->device copies inside
the timed region).  Beside them: the plain per-code drop-in over the same batch, the
reference's own plain per-code GPU path (its CUDA backend built for sm_100a) and its CPU
path on the host cores.  Under torchrun every rank certifies its own copy of the batch
(weak scaling, no collective on the data path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "certs/s batched vs plain on 1 B200 (exact d); Gcodewords/s vs int-pipe peak"
TC_OPS_PER_PAIR = 2 * 64  # int8 multiply-adds of the tensor-core filter: 64 columns per pair
POPC_PER_CLK_SM = 16     # 32-bit POPC results per clock per SM (CUDA arithmetic throughput table)
TC_ACCUMULATORS_PER_SM = 2 * 128 * 256   # tensor sweep: two 128 x 256 TMEM buffers per SM
TC_ROUND_TRIP_CYCLES = 1450              # one buffer's MMA -> read-back -> release, measured


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"sm_max_mhz": 1965.0, "hbm_gbs": 6650.0, "fallback": True}


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "25"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for nm, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def dist_setup(gpus):
    from qubitserf_b200 import dist
    return dist.init_from_env()


def max_over_ranks(pg, x):
    from qubitserf_b200 import dist
    return dist.max_over_ranks(pg, x)


def barrier(pg):
    from qubitserf_b200 import dist
    dist.barrier(pg)


def run_plain(native, codes):
    """Certify every code through the drop-in distfind_* ABI; returns (device ms, codewords,
    popc_alg, launches, distances)."""
    dev_ms = 0.0
    cw = 0
    popc = 0.0
    launches = 0
    dists = []
    for cs in codes:
        if cs.kind == "classical":
            r = native.classical_distance_raw(cs.mats[0], "bz", "gpu", 0, False)
        else:
            r = native.css_distance_raw(cs.mats[0], cs.mats[1], "bz", "M", "gpu", 0, False)
        rep = native.last_report()
        dev_ms += rep.device_ms
        cw += rep.codewords
        popc += rep.codewords * 2 * ((cs.n + 63) // 64)
        launches += rep.kernel_launches
        dists.append(r.distance)
    return dev_ms, cw, popc, launches, dists


def sample_order(codes, stride=16):
    """Every `stride`-th code, alternating the classical and CSS halves of the batch."""
    cls = [i for i in range(0, len(codes), stride) if codes[i].kind == "classical"]
    css = [i for i in range(0, len(codes), stride) if codes[i].kind != "classical"]
    out = []
    for k in range(max(len(cls), len(css))):
        out += cls[k:k + 1] + css[k:k + 1]
    return out


def cpu_baseline_sample(codes, budget_s=20.0, start=0, stride=16):
    """The reference CPU BZ path (oracle/_ref, the reference's own sources, all host
    threads) -- or the C restatement when that library is absent -- on a bounded sample of
    the batch: every `stride`-th code, alternating classical/CSS, until the budget is spent
    (stride 1 with no budget: the whole batch)."""
    from oracle.refbind import Oracle, Ref, ref_available
    kind = "reference" if ref_available() else "port"
    eng = Ref() if kind == "reference" else Oracle()
    order = sample_order(codes, stride)
    order = order[start % len(order):] + order[:start % len(order)]
    t0 = time.perf_counter()
    done = 0
    for i in order:
        cs = codes[i]
        if cs.kind == "classical":
            eng.classical(cs.mats[0])
        else:
            eng.css(cs.mats[0], cs.mats[1])
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "certs/s", "seconds": dt, "codes": done,
            "cores": os.cpu_count() if kind == "reference" else 1, "kind": kind,
            "sample": f"{done} of the {len(order)} codes at every {stride}th index of the "
                      f"{len(codes)}-code batch (classical/CSS alternating) in {dt:.1f} s"}


def plain_reference_gpu(codes, ans, budget_s=60.0):
    """The reference's own plain per-code GPU path: its distfind_* calls with backend "gpu"
    on its CUDA backend (cpp/qsf/cuda/backend_cuda.cu, built for sm_100a from its sources
    into oracle/_ref/libqubitserf_cuda.so), one code after another over the batch in index
    order until the budget is spent.  Levels of fewer than 2^18 codewords run on its CPU
    backend on all host threads, as the reference dispatches them.  Every result
    (distance, lower bound, proven, levels) is compared with the batched engine's answer on
    the same host."""
    from oracle.refbind import REF_CUDA_LIB, RefCuda
    if not REF_CUDA_LIB.exists():
        return {"unavailable": "oracle/_ref/libqubitserf_cuda.so not built"}
    eng = RefCuda()
    if not eng.available():
        return {"unavailable": "the reference's CUDA backend reports no device"}
    eng.classical(codes[0].mats[0])   # context and module load outside the timed loop
    t0 = time.perf_counter()
    done, same = 0, 0
    for cs, a in zip(codes, ans):
        if cs.kind == "classical":
            r = eng.classical(cs.mats[0])
        else:
            r = eng.css(cs.mats[0], cs.mats[1])
        same += (r.distance, r.lower_bound, r.proven, r.levels) == \
                (a.distance, a.lower_bound, a.proven, a.levels)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "certs/s", "codes": done, "seconds": dt,
            "results_equal": same, "host_threads": os.cpu_count(),
            "source": "reference distfind_* with backend gpu: its bz_enumerate kernel "
                      "(backend_cuda.cu) built for sm_100a, levels under 2^18 codewords "
                      "on its CPU backend"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--codes", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain-reference", action="store_true",
                    help="skip the reference's own per-code GPU path over the batch")
    ap.add_argument("--ref-stride", type=int, default=32,
                    help="reference arm: a step certifies every code at one residue modulo "
                         "this stride (32 codes of the 1024-code batch)")
    ap.add_argument("--ref-full", action="store_true",
                    help="reference arm: certify the whole batch once (a one-off timing; "
                         "minutes of host work)")
    ap.add_argument("--shard", action="store_true",
                    help="under torchrun: the ranks split the batch round robin (strong "
                         "scaling) instead of each certifying its own copy (weak scaling)")
    ap.add_argument("--only-resident", action="store_true",
                    help="time only the resident-input rounds (profiling runs)")
    ap.add_argument("--workload", default="batch",
                    choices=["batch", "css128", "classical128", "classical96", "collect", "mitm"],
                    help="batch = the 1024-code batch; collect = the codeaut low-weight "
                         "collector; the others certify one code")
    args = ap.parse_args()

    rank, world, local, pg = dist_setup(args.gpus)
    if args.workload == "collect":
        bench_collect(args, rank, world, local, pg)
        return
    if args.workload == "mitm":
        bench_mitm(args, rank, world, local, pg)
        return
    from qubitserf_b200 import workloads as W
    if args.workload == "batch":
        codes = W.batch_1024(args.codes)
        wname = f"batch_{args.codes}_uneven_seed3"
    else:
        one = {"css128": lambda: W.CodeSpec("css", W.single_css_128(), 128),
               "classical128": lambda: W.CodeSpec("classical", (W.single_classical_128(),), 128),
               "classical96": lambda: W.CodeSpec("classical", (W.single_classical_96(),), 96)}
        codes = [one[args.workload]()]
        args.codes = 1
        wname = {"css128": "css_n128_rank40x40_seed1_min", "classical128": "classical_n128_k40_seed2",
                 "classical96": "classical_n96_k32_seed0"}[args.workload]
    all_codes = codes
    sharded = args.shard and world > 1
    if sharded:   # strong scaling: rank r certifies codes r, r + world, ...
        from qubitserf_b200 import dist as D
        codes = D.shard(all_codes, rank, world)
    # certificates of one step over all ranks: every rank's copy, or the batch once
    units = len(all_codes) if sharded else len(all_codes) * world
    config = {"workload": wname, "codes": args.codes,
              "classical": sum(c.kind == "classical" for c in all_codes),
              "css": sum(c.kind == "css" for c in all_codes), "n_range": [40, 128],
              "parallelism": f"shard{world}" if sharded else f"replicas{world}",
              "l2": "256 MiB L2 flush before every timed step",
              "timed": "qsfb_batch_execute rounds (3 interleaved job groups), CUDA-event span "
                       "over all groups (host gaps included)"}

    if args.impl == "reference":
        if rank != 0:
            return
        if args.ref_full:
            b = cpu_baseline_sample(codes, budget_s=None, stride=1)
            print(json.dumps({"impl": "reference", "full_batch": True, "config": config, **b}),
                  flush=True)
            return
        from oracle.refbind import Oracle, Ref, ref_available
        kind = "reference" if ref_available() else "port"
        eng = Ref() if kind == "reference" else Oracle()

        def certify(i):
            cs = codes[i]
            if cs.kind == "classical":
                eng.classical(cs.mats[0])
            else:
                eng.css(cs.mats[0], cs.mats[1])

        stride = max(1, min(args.ref_stride, len(codes)))
        # warm-up steps: the library and its thread pool, on the smallest code of the batch
        small = min(range(len(codes)), key=lambda i: codes[i].n)
        for _ in range(args.warmup):
            certify(small)
        # Each step certifies one whole stratified subset of the batch: the codes at indices
        # = o (mod stride), every one of them, o rotating with the step (no time cut, so the
        # sample is not biased toward the codes that come first).
        secs, done, offsets = [], 0, []
        for k in range(args.steps):
            o = (k * 13) % stride
            idx = list(range(o, len(codes), stride))
            t0 = time.perf_counter()
            for i in idx:
                certify(i)
            secs.append(time.perf_counter() - t0)
            done += len(idx)
            offsets.append(o)
        v = done / sum(secs)
        sample = (f"{done} certificates over {args.steps} steps; step k certifies every code at "
                  f"index = (13 k mod {stride}) (mod {stride}) of the {len(codes)}-code batch "
                  f"({len(codes) // stride} codes, classical and CSS halves alike)")
        line = {"metric": METRIC, "value": v, "unit": "certs/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * sum(secs) / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                "config": config, "impl": "reference", "reference_sample": sample,
                "cpu_baseline": {"value": v, "unit": "certs/s", "seconds": sum(secs),
                                 "codes": done,
                                 "cores": os.cpu_count() if kind == "reference" else 1,
                                 "kind": kind, "sample": sample},
                "e2e": {"value": v, "unit": "certs/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    from qubitserf_b200 import _native
    if not _native.backend_available("gpu"):
        raise SystemExit("no sm_100 device visible")
    pk = peaks()
    nsm = _native.lib().qsfb_device_sms()
    batch = _native.Batch(_native.batch_items(codes))
    wpc = [2 * ((c.n + 63) // 64) for c in codes]   # POPC32 per codeword, full evaluation

    # --- device-resident throughput: prepare once, then execute the rounds K times
    # measured integer-pipe peaks (outside the timed region)
    popc_peak = _native.microbench(0)
    lop3_peak = _native.microbench(1)
    handle = batch.prepare()
    ans = None
    for _ in range(args.warmup):
        ans, st = batch.execute(handle)
    barrier(pg)
    spans, pair_ms, cw, launches, rounds = [], 0.0, 0, 0, 0
    popc_issued, zero_cw = 0, 0
    tc_ms, tc_cw = 0.0, 0
    popc_alg = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            _native.lib().qsfb_flush_l2()
            ans, st = batch.execute(handle)
            spans.append(st.device_span_ms)
            pair_ms += st.pair_ms
            cw += st.codewords
            popc_issued += st.popc_issued
            zero_cw += st.zero_codewords
            tc_ms += st.tc_ms
            tc_cw += st.tc_codewords
            launches += st.kernel_launches
            rounds = st.rounds
    # per-kernel statistics (the rooflines) from one more, untimed execution as a single job
    # group with each round's pair launches on one stream: with several groups, or pair
    # launches forked over streams, kernels overlap and their event times include others'
    os.environ["QSFB_EXEC_GROUPS"] = "1"
    os.environ["QSFB_SERIAL_PAIRS"] = "1"
    try:
        _, st1 = batch.execute(handle)
    finally:
        os.environ.pop("QSFB_EXEC_GROUPS", None)
        os.environ.pop("QSFB_SERIAL_PAIRS", None)
    k = args.steps   # every step certifies the same batch: per-step figures times the steps
    pair_ms, tc_ms, tc_cw = st1.pair_ms * k, st1.tc_ms * k, st1.tc_codewords * k
    cw, popc_issued, zero_cw = st1.codewords * k, st1.popc_issued * k, st1.zero_codewords * k
    batch.free(handle)
    span_s = max_over_ranks(pg, sum(spans) / 1000.0)
    value = units * args.steps / span_s
    dists = [a.distance for a in ans]
    assert all(a.witness_ok for a in ans), "a witness failed host verification"
    # algorithmic POPC of the full evaluation: per level work x 2W (W = 64-bit words)
    # (codewords of each code are not separated per code inside a batch: use the batch's
    #  codeword-weighted W from a plain pass below)

    if args.only_resident:
        if rank == 0:
            print(json.dumps({"workload": wname, "certs_per_s": value,
                              "ms_per_step": span_s / args.steps * 1000.0,
                              "gcodewords_per_s": cw / max(pair_ms / 1000.0, 1e-12) / 1e9,
                              "rounds": rounds, "launches": launches,
                              "device_mb": st.device_bytes / 2**20,
                              "pair_ms": st1.pair_ms, "gen_ms": st1.gen_ms,
                              "host_plan_ms": st.host_plan_seconds * 1e3,
                              "host_apply_ms": st.host_apply_seconds * 1e3,
                              "tc_share": st1.tc_codewords / max(st1.codewords, 1),
                              "tc_codewords": st1.tc_codewords, "tc_ms": st1.tc_ms,
                              "note": "pair/gen/tc times from one single-group execution"}),
                  flush=True)
        return

    # --- end to end: the one-shot public call from host matrices, K times, after untimed
    # warm-up calls of the same call (its chunk sizes and sessions differ from the resident
    # run's, and a first call would time their device allocations)
    for _ in range(max(1, args.warmup)):
        batch.run()
    e2e_t = []
    alloc0 = _native.alloc_counters()
    for _ in range(args.steps):
        t = time.perf_counter()
        ans2, st2 = batch.run()
        e2e_t.append(time.perf_counter() - t)
    alloc1 = _native.alloc_counters()
    assert [a.distance for a in ans2] == dists
    e2e_s = max_over_ranks(pg, sum(e2e_t))
    e2e = units * args.steps / e2e_s
    host_setup = st2.host_setup_seconds

    # --- the plain per-code drop-in path over the same batch (one pass, wall clock)
    t = time.perf_counter()
    pdev, pcw, ppopc, plaunch, pd = run_plain(_native, codes)
    plain_s = time.perf_counter() - t
    assert pd == dists, "plain and batched distances differ"
    plain = len(codes) / plain_s
    popc_per_cw = ppopc / max(pcw, 1)

    clocks = clk.summary()
    f_mhz = clocks.get("sm_mhz") or pk.get("sm_max_mhz", 1965.0)
    peak_popc = nsm * POPC_PER_CLK_SM * f_mhz * 1e6
    pair_s = pair_ms / 1000.0
    achieved_cw = cw / max(pair_s, 1e-12)
    # tensor-core sweep: int8 ops over its own CUDA-event time; peak = int8 dense, twice the
    # measured bf16 rate (the kernel is timed alone in short launches: burst figure)
    tc_s = max_over_ranks(pg, tc_ms / 1000.0)
    tc_ops = tc_cw * TC_OPS_PER_PAIR / max(tc_s, 1e-12)
    bf16 = pk.get("bf16_tflops")
    tc_peak = (2.0 * bf16 * 1e12) if bf16 else 2.0 * 1.59e15
    tc_traffic = tc_traffic_per_launch(tc_cw / max(args.steps, 1))
    # CUDA-core sweep: the rest of the codewords over the rest of the pair-kernel time
    cc_s = max(pair_s - tc_ms / 1000.0, 1e-12)
    cc_cw_rate = (cw - tc_cw) / cc_s
    # every code's answer in batch order on rank 0 (shards gathered; one gloo gather)
    full_dists = dists
    if sharded:
        parts = D.gather_to_root(pg, dists, world)
        full_dists = D.unshard(parts) if rank == 0 else None
    if rank != 0:
        return
    golden_ok = None
    gold = ROOT / "tests" / "golden" / "batch1024.json"
    if args.workload == "batch" and args.codes == 1024 and gold.exists():
        want = [r[0] for r in json.loads(gold.read_text())["codes"]]
        golden_ok = want == full_dists
    cpu = None if args.no_cpu_baseline else cpu_baseline_sample(all_codes)
    pref = None if args.no_plain_reference else plain_reference_gpu(codes, ans)
    line = {
        "metric": METRIC, "value": value, "unit": "certs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": span_s / args.steps * 1000.0,
        "higher_is_better": True, "scaling": "strong" if sharded else "weak",
        "vs_baseline": None, "dtype": "i8", "data": "synthetic", "config": config,
        "distances_equal_reference_golden": golden_ok,
        "plain_certs_per_s": plain, "batched_vs_plain": value / plain,
        "plain_reference_gpu": pref,
        "batched_vs_plain_reference": (value / pref["value"]) if pref and "value" in pref
                                      else None,
        "gcodewords_per_s": achieved_cw / 1e9,
        "codewords_per_step": cw / args.steps, "rounds_per_step": rounds,
        "roofline": {
            "bound": "tensor", "kernel": "pairs_tc_kernel",
            "achieved": tc_ops / 1e12, "peak": tc_peak / 1e12, "unit": "TOP/s (int8)",
            "frac": tc_ops / tc_peak, "traffic": tc_traffic,
            "algorithmic_bytes_per_launch": tc_operand_bytes_per_launch(st1.tc_operand_bytes),
            "peak_source": ("2 x measured bf16 dense (MEASURED_PEAKS.json bf16_tflops, burst)"
                            if bf16 else "2 x fallback bf16 1.59 PFLOP/s"),
            "numerator": "tensor-core codewords x 128 int8 ops (64 columns) / kernel time",
            "binding": {"resource": "TMEM capacity over the accumulator round trip: 64k "
                                    "accumulators in flight, each MMA -> commit -> read-back -> "
                                    "release before reuse (ncu: tensor pipe, TMEM, L2 and DRAM "
                                    "all below saturation)",
                        "tmem_columns_read_gbs": tc_cw * 4 / max(tc_s, 1e-12) / 1e9,
                        "tmem_bytes_per_clk_per_sm": tc_cw * 4 / max(tc_s, 1e-12) /
                                                     (nsm * f_mhz * 1e6),
                        # 65,536 accumulators per SM retire once per buffer round trip; the
                        # round trip (1,300-1,600 cycles) was measured by a clock64-stamped
                        # build of the kernel
                        "round_trip_cycles": TC_ROUND_TRIP_CYCLES,
                        "bound_pairs_per_s": TC_ACCUMULATORS_PER_SM * nsm * f_mhz * 1e6 /
                                             TC_ROUND_TRIP_CYCLES,
                        "pairs_per_s": tc_cw / max(tc_s, 1e-12),
                        "frac_of_bound": tc_cw / max(tc_s, 1e-12) /
                                         (TC_ACCUMULATORS_PER_SM * nsm * f_mhz * 1e6 /
                                          TC_ROUND_TRIP_CYCLES)},
            "codeword_share": tc_cw / max(cw, 1),
            "kernel_ms_per_step": tc_ms / max(args.steps, 1)},
        "roofline_list_generation": list_generation_roofline(st1, pk),
        "roofline_cuda_core": {
            "bound": "int-pipe (POPC on the XU pipe)", "kernel": "pairs_kernel",
            "achieved": cc_cw_rate * popc_per_cw / 1e9, "peak": popc_peak / 1e9,
            "unit": "Gpopc32/s", "frac": cc_cw_rate * popc_per_cw / popc_peak,
            "traffic": traffic_per_launch((cw - tc_cw) / max(args.steps, 1)),
            "numerator": "codewords/s of the pair kernel x 2W POPC32 of the full evaluation "
                         "(W = ceil(n/64)); the kernel issues fewer (pivot columns removed, "
                         "probe words, zero test)",
            "peak_source": "measured: qsfb_microbench POPC chains over all SMs",
            "codewords_per_step": (cw - tc_cw) / max(args.steps, 1),
            "kernel_popc_per_codeword": popc_issued / max(cw - tc_cw, 1),
            "kernel_frac": popc_issued / max(cc_s, 1e-12) / popc_peak,
            "zero_test_share": zero_cw / max(cw - tc_cw, 1),
            "lop3_peak_gops": lop3_peak / 1e9,
            "sm_mhz": f_mhz},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "certs/s", "h2d_bytes_per_step": int(batch.host_bytes),
                "d2h_bytes_per_step": int(ctypes_sizeof_answers(args.codes)),
                "call_s": st2.seconds,
                "prepare_s": st2.prepare_seconds, "host_setup_s": host_setup,
                "device_seed_s": st2.device_seed_seconds,
                "rounds_span_s": st2.device_span_ms / 1e3,
                "calls_ms": [round(x * 1e3, 2) for x in e2e_t],
                "driver_allocations": {"device": alloc1[0] - alloc0[0],
                                       "device_s": alloc1[1] - alloc0[1],
                                       "pinned": alloc1[2] - alloc0[2],
                                       "pinned_s": alloc1[3] - alloc0[3]},
                "note": "last call: prepare/host_setup/device_seed summed over the pipeline "
                        "chunks (all but the first overlap the rounds); rounds_span_s is the "
                        "merged rounds' device span"},
        "gpu_launches": launches,
        "tuning": tuning_summary(_native),
        "clocks": clocks,
        "distance_checksum": int(np.sum(np.array(full_dists, dtype=np.int64) *
                                        np.arange(1, len(full_dists) + 1))),
    }
    print(json.dumps(line), flush=True)


COLLECT = {"n": 128, "k": 64, "seed": 13, "p": 9, "keep": 20, "sample_p": 8}
COLLECT_METRIC = "codeaut low-weight collection: subset combinations/s on 1 B200"


def collect_reference_sample(G, p, keep, start=0):
    """The reference's own codeaut_bz_collect (oracle/_ref, its CPU backend, all host
    threads) on the bounded sample p = sample_p of the same generator."""
    from oracle.refbind import Ref
    ref = Ref()
    t = time.perf_counter()
    rows, combos = ref.collect(G, p, keep, threads=0)
    dt = time.perf_counter() - t
    return {"value": combos / dt, "unit": "combos/s", "cores": os.cpu_count(),
            "kind": "reference", "rows": int(rows.shape[0]),
            "sample": f"subset sizes 1..{p} of the same generator ({combos} combinations) "
                      f"in {dt:.2f} s"}


def bench_collect(args, rank, world, local, pg):
    """The codeaut collector (codeaut_bz_collect): a step collects every XOR of 1..p rows
    of a random systematic [n, k] generator with weight <= keep.  value = combinations per
    second of device time (list generation + pair sweeps, G already packed on the device by
    the call); e2e = the same combinations over the wall time of the public handle call
    (host packing, upload, sweeps, download, host sort) plus copying the rows out."""
    from qubitserf_b200 import workloads as W
    c = COLLECT
    G = W.collect_generator(c["n"], c["k"], c["seed"])
    wname = f"codeaut_collect_systematic_n{c['n']}_k{c['k']}_p{c['p']}_keep{c['keep']}_seed{c['seed']}"
    config = {"workload": wname, "n": c["n"], "k": c["k"], "p": c["p"], "keep": c["keep"],
              "parallelism": f"replicas{world}",
              "l2": "256 MiB L2 flush before every timed step (lists fit in L2)",
              "timed": "list generation + pair sweeps, CUDA events of the call"}
    if args.impl == "reference":
        if rank != 0:
            return
        for _ in range(min(args.warmup, 1)):
            collect_reference_sample(G, 3, c["keep"])
        vals, b = [], None
        for _ in range(args.steps):
            b = collect_reference_sample(G, c["sample_p"], c["keep"])
            vals.append(b["value"])
        v = float(np.mean(vals))
        print(json.dumps({"metric": COLLECT_METRIC, "value": v, "unit": "combos/s",
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                          "config": config, "impl": "reference",
                          "cpu_baseline": {**b, "value": v},
                          "e2e": {"value": v, "unit": "combos/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    from qubitserf_b200 import _native
    if not _native.backend_available("gpu"):
        raise SystemExit("no sm_100 device visible")
    popc_peak = _native.microbench(0)
    rows = None
    for _ in range(args.warmup):
        rows, combos, st = _native.collect(G, c["p"], c["keep"], stats=True)
    barrier(pg)
    dev_s, wall_s, launches, passes, hits = 0.0, 0.0, 0, 0, 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            _native.lib().qsfb_flush_l2()
            t = time.perf_counter()
            rows2, combos, st = _native.collect(G, c["p"], c["keep"], stats=True)
            wall_s += time.perf_counter() - t
            dev_s += (st.gen_ms + st.pairs_ms) / 1e3
            launches += st.launches
            passes += st.passes
            hits += st.hits
            pairs_s = st.pairs_ms / 1e3
            assert rows is None or np.array_equal(rows, rows2)
            rows = rows2
    dev_s = max_over_ranks(pg, dev_s)
    wall_s = max_over_ranks(pg, wall_s)
    value = combos * args.steps * world / dev_s
    e2e = combos * args.steps * world / wall_s
    if rank != 0:
        return
    S64 = (c["n"] + 63) // 64
    alg_popc = 2 * S64            # POPC32 per combination of the full evaluation
    achieved = combos * alg_popc / pairs_s
    # POPC32 the sweep issues per pair: the exact sum over its probe words, one for the OR
    # bounds, two for the carry-save bound
    issued = {0: st.probe_words, 2: 1, 4: 1, 6: 2}[st.filter]
    cpu = None if args.no_cpu_baseline else collect_reference_sample(G, c["sample_p"], c["keep"])
    print(json.dumps({
        "metric": COLLECT_METRIC, "value": value, "unit": "combos/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_s / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic", "config": config,
        "rows": int(rows.shape[0]), "combos_per_step": combos,
        "roofline": {"bound": "int-pipe (POPC on the XU pipe)", "kernel": "collect_pairs_kernel",
                     "achieved": achieved / 1e9, "peak": popc_peak / 1e9, "unit": "Gpopc32/s",
                     "frac": achieved / popc_peak, "traffic": None,
                     "numerator": f"combinations/s of the pair sweeps x {alg_popc} POPC32 of "
                                  "the full evaluation (2 per 64-bit word); the kernel issues "
                                  f"{issued} per pair (probe bound {st.filter} over "
                                  f"{st.probe_words} words)",
                     "kernel_frac": combos * issued / pairs_s / popc_peak,
                     "peak_source": "measured: qsfb_microbench POPC chains over all SMs",
                     "pass_rate": passes / max(combos * args.steps, 1),
                     "gen_ms": st.gen_ms, "pairs_ms": st.pairs_ms},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "combos/s", "h2d_bytes_per_step": int(G.size),
                "d2h_bytes_per_step": int(st.hits * S64 * 8),
                "seconds_per_step": wall_s / args.steps},
        "gpu_launches": launches, "clocks": clk.summary(),
        "hits_per_step": hits // max(args.steps, 1)}), flush=True)


MITM_L = 7
MITM_METRIC = "method mitm: certificates/s (exact CSS min distance) on 1 B200"


def bench_mitm(args, rank, world, local, pg):
    """Method "mitm" (meet in the middle) on the [[98, 2, 7]] toric code, which='min': a step
    is one distfind_css_distance call (host reduction, device tables and probes, one
    certificate); value and e2e are both its wall time (the inputs are two 49 x 98 matrices)."""
    from qubitserf_b200 import workloads as W
    Hx, Hz = W.toric_code(MITM_L)
    config = {"workload": f"toric_L{MITM_L}_n{2 * MITM_L * MITM_L}_mitm_min", "which": "min",
              "method": "mitm", "parallelism": f"replicas{world}",
              "timed": "wall time of distfind_css_distance (no L2 flush: tables are rebuilt "
                       "every call)"}
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle.refbind import Ref
        ref = Ref()
        Lw = W.toric_code(5)
        for _ in range(min(args.warmup, 1)):
            ref.css(*Lw, "M", method="mitm")
        ts = []
        for _ in range(args.steps):
            t = time.perf_counter()
            r = ref.css(Hx, Hz, "M", method="mitm")
            ts.append(time.perf_counter() - t)
        v = args.steps / sum(ts)
        b = {"value": v, "unit": "certs/s", "cores": os.cpu_count(), "kind": "reference",
             "sample": f"the full workload ({args.steps} certificate(s), distance {r.distance})"}
        print(json.dumps({"metric": MITM_METRIC, "value": v, "unit": "certs/s",
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                          "config": config, "impl": "reference", "cpu_baseline": b,
                          "e2e": {"value": v, "unit": "certs/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    from qubitserf_b200 import _native
    if not _native.backend_available("gpu"):
        raise SystemExit("no sm_100 device visible")
    for _ in range(args.warmup):
        r = _native.css_distance_raw(Hx, Hz, "mitm", "M", "gpu", 0, False)
    barrier(pg)
    ts, rep = [], None
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            t = time.perf_counter()
            r = _native.css_distance_raw(Hx, Hz, "mitm", "M", "gpu", 0, False)
            ts.append(time.perf_counter() - t)
            rep = _native.last_report()
    assert (r.distance, r.proven) == (MITM_L, 1)
    wall = max_over_ranks(pg, sum(ts))
    value = args.steps * world / wall
    if rank != 0:
        return
    print(json.dumps({
        "metric": MITM_METRIC, "value": value, "unit": "certs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic", "config": config, "distance": r.distance, "levels": r.levels,
        "parts_per_step": rep.codewords, "parts_per_s": rep.codewords * args.steps / wall,
        "roofline": {"bound": "integer issue (ALU pipe 71%, issue 76% under ncu): part "
                              "generation and hashing; the table lines stay in L1/L2",
                     "kernel": "mitm_probe_kernel", "achieved": None, "peak": None,
                     "frac": None, "traffic": None},
        "cpu_baseline": None,
        "e2e": {"value": value, "unit": "certs/s",
                "h2d_bytes_per_step": int(Hx.size + Hz.size), "d2h_bytes_per_step": 48},
        "gpu_launches": rep.kernel_launches, "clocks": clk.summary()}), flush=True)


def tuning_summary(native):
    """The launch shapes in effect and, when they come from the tuning table, the gain the
    tuner measured over the defaults on the same batch (its header lines)."""
    t = native.tuning()
    out = {"values": {k: v for k, v in t.items() if k != "source"}, "source": t.get("source")}
    src = str(t.get("source", ""))
    path = Path(src.split(" + ")[0])
    if path.exists():
        out["measured_gain"] = [l[2:].strip() for l in path.read_text().splitlines()
                                if l.startswith("# resident") or l.startswith("# one-shot")]
    return out


def tc_traffic_per_launch(tc_cw_per_step):
    """DRAM bytes per tensor-core launch: the committed per-codeword traffic of an ncu capture
    on a smaller batch, scaled by the codewords of an average launch of this run."""
    p = ROOT / "profiles" / "pairs_tc_kernel_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    per_cw = d.get("dram_bytes_per_codeword")
    launches = d.get("launches_per_step_full_batch")
    if per_cw is None or not launches:
        return None
    return per_cw * tc_cw_per_step / launches


def list_generation_roofline(st, pk):
    """HBM roofline of the list generation (gen_lists + expand_pm) in the statistics pass:
    the bytes it must write per step over its own CUDA-event time."""
    if not st.gen_ms:
        return None
    peak = pk.get("hbm_gbs", 6650.0)
    gbs = st.list_bytes_written / (st.gen_ms / 1e3) / 1e9
    return {"bound": "hbm", "kernel": "gen_lists_kernel + expand_pm_kernel",
            "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in pk else "fallback",
            "algorithmic_bytes_per_step": st.list_bytes_written, "ms_per_step": st.gen_ms,
            "note": "bytes written: probe words, pivot counts and +-1 rows of the lists; the "
                    "kernel is instruction-bound (ALU ~74% under ncu), not bandwidth-bound"}


def tc_operand_bytes_per_launch(operand_bytes_per_step):
    """+-1 row bytes a tensor-core launch must read at least once (the union per round of the
    row ranges each list serves), per launch of the statistics pass, for comparison with
    the DRAM traffic per launch."""
    p = ROOT / "profiles" / "pairs_tc_kernel_traffic.json"
    if not p.exists():
        return None
    launches = json.loads(p.read_text()).get("launches_per_step_full_batch")
    return operand_bytes_per_step / launches if launches else None


def traffic_per_launch(cc_cw_per_step):
    """DRAM bytes per CUDA-core pair launch: the committed per-codeword traffic of an ncu
    capture on a smaller batch, scaled by the codewords of an average launch of this run."""
    p = ROOT / "profiles" / "pairs_kernel_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    per_cw = d.get("dram_bytes_per_codeword")
    launches = d.get("launches_per_step_full_batch")
    if per_cw is None or not launches:
        return None
    return per_cw * cc_cw_per_step / launches


def ctypes_sizeof_answers(n):
    import ctypes
    from qubitserf_b200 import _native
    return ctypes.sizeof(_native.QsfbAnswer) * n


if __name__ == "__main__":
    main()
