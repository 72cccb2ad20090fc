"""Benchmark: certificates/s (exact BZ distances) on the 1024-code uneven batch, and the
integer-pipe roofline of the pair-sweep kernel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--mode batch|plain] [--codes 1024]

A step certifies every code of the batch (512 classical [n in 48..128, k in n/4..n/2] +
512 CSS [n in 40..128, ranks in n/5..n/3], seed 3; CSS codes solved with which='min').
`value` is certificates per second from device time with the inputs resident; `e2e` is
the same metric through the public C ABI from host matrices (host<->device copies inside
the timed region).  Under torchrun every rank certifies its own copy of the batch
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
POPC_PER_CLK_SM = 16     # 32-bit POPC results per clock per SM (CUDA arithmetic throughput table)


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
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
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
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ["QSFB_DEVICE"] = str(local)
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    else:
        os.environ.setdefault("QSFB_DEVICE", "0")
    return rank, world, local, pg


def max_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


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


def cpu_baseline_sample(codes, budget_s=20.0):
    """The reference CPU path (oracle/_ref when built, else the C restatement) on a bounded
    sample of the batch: every 16th code, in order, until the budget is spent."""
    from oracle.refbind import Oracle, Ref, ref_available
    kind = "reference" if ref_available() else "port"
    eng = Ref() if kind == "reference" else Oracle()
    t0 = time.perf_counter()
    done = 0
    for cs in codes[::16]:
        if cs.kind == "classical":
            eng.classical(cs.mats[0])
        else:
            eng.css(cs.mats[0], cs.mats[1])
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "certs/s", "cores": os.cpu_count() if kind == "reference" else 1,
            "kind": kind, "sample": f"{done} codes (every 16th of the 1024-code batch, in order) in {dt:.1f} s"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="plain", choices=["plain", "batch"])
    ap.add_argument("--codes", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()

    rank, world, local, pg = dist_setup(args.gpus)
    from qubitserf_b200 import workloads as W
    codes = W.batch_1024(args.codes)
    config = {"workload": f"batch_{args.codes}_uneven_seed3", "codes": args.codes,
              "classical": sum(c.kind == "classical" for c in codes),
              "css": sum(c.kind == "css" for c in codes), "n_range": [40, 128],
              "parallelism": f"replicas{world}", "l2": "inputs resident (KB per code); no flush",
              "mode": args.mode}

    if args.impl == "reference":
        if rank != 0:
            return
        steps = []
        for _ in range(args.warmup):
            pass
        for _ in range(args.steps):
            b = cpu_baseline_sample(codes, budget_s=20.0)
            steps.append(b["value"])
        v = float(np.mean(steps))
        line = {"metric": METRIC, "value": v, "unit": "certs/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v * args.codes,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic", "config": config, "impl": "reference",
                "cpu_baseline": {**b, "value": v},
                "e2e": {"value": v, "unit": "certs/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    from qubitserf_b200 import _native
    if not _native.backend_available("gpu"):
        raise SystemExit("no sm_100 device visible")
    pk = peaks()
    for _ in range(args.warmup):
        run_plain(_native, codes)
    barrier(pg)
    wall0 = time.perf_counter()
    dev_ms = cw = popc = launches = 0
    dists = None
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            a, b, c, d, dists = run_plain(_native, codes)
            dev_ms += a
            cw += b
            popc += c
            launches += d
    wall = time.perf_counter() - wall0
    wall = max_over_ranks(pg, wall)
    dev_s = max_over_ranks(pg, dev_ms / 1000.0)
    clocks = clk.summary()
    nsm = _native.lib().qsfb_device_sms()
    f_mhz = clocks.get("sm_mhz") or pk.get("sm_max_mhz", 1965.0)
    peak_popc = nsm * POPC_PER_CLK_SM * f_mhz * 1e6
    certs = args.codes * args.steps * world
    e2e = certs / wall
    if rank != 0:
        return
    cpu = None if args.no_cpu_baseline else cpu_baseline_sample(codes)
    line = {
        "metric": METRIC, "value": e2e, "unit": "certs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": wall / args.steps * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic", "config": config,
        "codewords_per_step": cw / args.steps,
        "gcodewords_per_s_kernel": cw / max(dev_s, 1e-9) / 1e9 / world,
        "roofline": {"bound": "int-pipe (POPC)", "achieved": popc / max(dev_s, 1e-9) / 1e9 / world,
                     "peak": peak_popc / 1e9, "unit": "Gpopc32/s",
                     "frac": popc / max(dev_s, 1e-9) / world / peak_popc, "traffic": None,
                     "sm_mhz_used": f_mhz},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "certs/s", "h2d_bytes_per_step": int(sum(
            sum(m.size for m in c.mats) for c in codes)), "d2h_bytes_per_step": 8 * args.codes},
        "gpu_launches": launches,
        "clocks": clocks,
        "distance_checksum": int(np.sum(np.array(dists, dtype=np.int64) * np.arange(1, len(dists) + 1))),
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
