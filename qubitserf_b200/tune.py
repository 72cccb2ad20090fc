"""Autotuner for the engine's launch shapes (no reference counterpart).

    python -m qubitserf_b200.tune [--codes 1024] [--out qubitserf_b200/tuning.txt]

Measures the 1024-code batch on the GPU it runs on and writes the table the library reads at
start (`tuning.txt` beside libqsfb200.so; keys in csrc/tuning.hpp).  The search is
coordinate descent over one knob at a time, each candidate timed in a fresh process (the
library reads its tuning once):

* device-resident rounds (`qsfb_batch_execute`, CUDA-event span, L2 flushed before each
  step): the tensor-core sweep's tile shape, its suffix tiles per job for small and large
  levels and the class boundary between them (tiles of a level's tensor plan), the
  CUDA-core loop tile (jobs per resident warp), the tensor/CUDA-core cost ratio of the
  planner, and the job groups of an execution;
* the one-shot call from host matrices (`qsfb_batch`, wall time): pipeline chunks and the
  job groups that merge them.

A candidate replaces the current value only when its median beats it by more than
`--min-gain` (default 1%) twice: once in the sweep and once more measured beside the current
value; and a group of knobs whose final values do not beat the defaults in the closing
measurement falls back to the defaults, so noise does not move the table.  Every choice gives the same
answers; the table records the candidates' times and the gain of the chosen shapes over
the defaults, measured in the same run.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent

RESIDENT_KNOBS = [
    ("tc_shape", [1, 0]),
    ("tc_job_tiles.large", [16, 8, 32]),
    ("tc_job_tiles.small", [16, 4, 8]),
    ("tc_small_tiles", [4096, 1024, 16384]),
    ("cc_jobs_per_warp", [16, 8, 32]),
    ("tc_cost_ratio", [0.6, 0.4, 0.8, 1.0]),
    ("tc_edge_div", [2, 4, 8, 16]),
    ("exec_groups", [3, 2, 4]),
]
E2E_KNOBS = [
    ("batch_chunks", [4, 1, 2, 3, 6]),
    ("overlap_groups", [3, 2, 4]),
    ("batch_first_permille", [0, 31, 62, 250]),
]
DEFAULTS = {k: v[0] for k, v in RESIDENT_KNOBS + E2E_KNOBS}


def env_for(values):
    env = dict(os.environ)
    env["QSFB_TUNING"] = "/nonexistent"   # measure from the defaults plus the overrides
    for k, v in values.items():
        env["QSFB_TUNE_" + k.replace(".", "_").upper()] = str(v)
    return env


def child(mode, codes, steps, warmup):
    """Runs in the measured process: prints the median time of `steps` executions (ms)."""
    sys.path.insert(0, str(ROOT))
    import time
    from qubitserf_b200 import _native, workloads as W
    batch = _native.Batch(_native.batch_items(W.batch_1024(codes)))
    ts = []
    if mode == "resident":
        h = batch.prepare()
        for _ in range(warmup):
            batch.execute(h)
        for _ in range(steps):
            _native.lib().qsfb_flush_l2()
            _, st = batch.execute(h)
            ts.append(st.device_span_ms)
        batch.free(h)
    else:
        for _ in range(warmup):
            batch.run()
        for _ in range(steps):
            t = time.perf_counter()
            batch.run()
            ts.append(1e3 * (time.perf_counter() - t))
    ts.sort()
    print(json.dumps({"ms": ts[len(ts) // 2], "all": ts}))


def measure(mode, values, args):
    cmd = [sys.executable, "-m", "qubitserf_b200.tune", "--child", mode, "--codes",
           str(args.codes), "--steps", str(args.steps), "--warmup", str(args.warmup)]
    p = subprocess.run(cmd, env=env_for(values), capture_output=True, text=True, cwd=str(ROOT),
                       timeout=900)
    if p.returncode != 0:
        raise RuntimeError(f"measurement failed ({values}):\n{p.stderr[-2000:]}")
    return json.loads(p.stdout.strip().splitlines()[-1])["ms"]


def search(mode, knobs, values, args, log):
    best = measure(mode, values, args)
    log.append((mode, "start", dict(values), best))
    for key, cands in knobs:
        for v in cands:
            if v == values[key]:
                continue
            trial = dict(values, **{key: v})
            ms = measure(mode, trial, args)
            log.append((mode, key, v, ms))
            print(f"  {mode:8s} {key:20s} {v!s:8s} {ms:8.3f} ms (best {best:.3f})", flush=True)
            if ms < best * (1.0 - args.min_gain):
                # a win must repeat: both measured again, side by side
                again, cur = measure(mode, trial, args), measure(mode, values, args)
                log.append((mode, key + " (again, against current)", v, again))
                if again < cur * (1.0 - args.min_gain):
                    values, best = trial, again
                else:
                    best = min(best, cur)
    return values, best


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--codes", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--min-gain", type=float, default=0.01)
    ap.add_argument("--out", default=str(PKG / "tuning.txt"))
    ap.add_argument("--child", choices=["resident", "e2e"])
    args = ap.parse_args()
    if args.child:
        child(args.child, args.codes, args.steps, args.warmup)
        return
    sys.path.insert(0, str(ROOT))
    from qubitserf_b200 import _native
    if not _native.backend_available("gpu"):
        raise SystemExit("no sm_100 device visible")
    device = _native.lib().qsfb_device_name().decode()
    log = []
    values = dict(DEFAULTS)
    base_res = measure("resident", values, args)
    base_e2e = measure("e2e", values, args)
    values, best_res = search("resident", RESIDENT_KNOBS, values, args, log)
    values, best_e2e = search("e2e", E2E_KNOBS, values, args, log)
    # the chosen table measured once more beside the defaults (same run, same box); a group
    # of knobs that does not beat its defaults there goes back to them
    final_res = measure("resident", values, args)
    final_e2e = measure("e2e", values, args)
    again_res = measure("resident", DEFAULTS, args)
    again_e2e = measure("e2e", DEFAULTS, args)
    d_res, d_e2e = (base_res + again_res) / 2, (base_e2e + again_e2e) / 2
    if final_res >= d_res:
        for key, _ in RESIDENT_KNOBS:
            values[key] = DEFAULTS[key]
        final_res = d_res
    if final_e2e >= d_e2e:
        for key, _ in E2E_KNOBS:
            values[key] = DEFAULTS[key]
        final_e2e = d_e2e
    lines = [
        "# Launch shapes of libqsfb200.so chosen by `python -m qubitserf_b200.tune` (keys: csrc/tuning.hpp).",
        f"# Measured on {device}, {datetime.date.today().isoformat()}, the {args.codes}-code uneven batch "
        "(seed 3), median of "
        f"{args.steps} steps, one fresh process per candidate.",
        f"# resident rounds: defaults {d_res:.3f} ms -> tuned {final_res:.3f} ms "
        f"({100.0 * (d_res / final_res - 1.0):+.1f}% certificates/s)",
        f"# one-shot call:   defaults {d_e2e:.3f} ms -> tuned {final_e2e:.3f} ms "
        f"({100.0 * (d_e2e / final_e2e - 1.0):+.1f}% certificates/s)",
        "# candidates (mode, knob, value, median ms):",
    ]
    for mode, key, v, ms in log:
        lines.append(f"#   {mode} {key} {v} {ms:.3f}")
    for key, _ in RESIDENT_KNOBS + E2E_KNOBS:
        lines.append(f"{key} {values[key]}")
    Path(args.out).write_text("\n".join(lines) + "\n")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
