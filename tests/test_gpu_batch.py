"""The batched engine (qsfb_batch): every answer equals the per-code drop-in path's and
the reference's golden vectors; witnesses verified; results independent of the batch mix."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_matches_per_code_path(native):
    from qubitserf_b200 import workloads as W
    codes = W.batch_1024(96)
    items = native.batch_items(codes)
    ans, st = native.Batch(items).run()
    assert st.certificates == len(codes) and st.rounds > 0
    for i, cs in enumerate(codes):
        if cs.kind == "classical":
            r = native.classical_distance_raw(cs.mats[0], "bz", "gpu", 0, False)
        else:
            r = native.css_distance_raw(*cs.mats, "bz", "M", "gpu", 0, False)
        a = ans[i]
        assert (a.distance, a.lower_bound, a.proven, a.levels) == \
            (r.distance, r.lower_bound, r.proven, r.levels), (i, cs.kind, cs.n)
        assert a.witness_ok == 1


def test_batch_golden_and_mixture(native, golden):
    names = [n for n, r in golden.results.items() if r["kind"] in ("classical", "css", "opweight")
             and n not in ("cfg_css_128",)]
    items = []
    for n in names:
        r = golden.results[n]
        m = golden.mats(n)
        if r["kind"] == "classical":
            items.append(("classical", m[0]))
        elif r["kind"] == "css":
            items.append(("css", m[0], m[1], r.get("which", "M")))
        else:
            items.append(("opweight",) + tuple(m))
    ans, _ = native.Batch(items).run()
    for n, a in zip(names, ans):
        r = golden.results[n]
        if r["kind"] == "opweight":
            assert (a.z_weight, a.x_weight) == (r["z_weight"], r["x_weight"]), n
        else:
            assert a.distance == r["distance"] and a.proven == r["proven"], n
    # the same query alone and inside a shuffled mix gives the same answer
    rng = np.random.default_rng(3)
    perm = rng.permutation(len(items))
    ans2, _ = native.Batch([items[i] for i in perm]).run()
    for k, i in enumerate(perm):
        assert (ans2[k].distance, ans2[k].levels, ans2[k].lower_bound) == \
            (ans[i].distance, ans[i].levels, ans[i].lower_bound)
    solo, _ = native.Batch([items[5]]).run()
    assert solo[0].distance == ans[5].distance and solo[0].levels == ans[5].levels


def test_batch_empty_and_trivial(native):
    ans, st = native.Batch([]).run()
    assert st.certificates == 0
    H = np.ones((1, 3), np.uint8)   # [3,2,2] even-weight code
    ans, _ = native.Batch([("classical", H)]).run()
    assert ans[0].distance == 2


def test_prepare_execute_repeatable(native):
    from qubitserf_b200 import workloads as W
    b = native.Batch(native.batch_items(W.batch_1024(40)))
    h = b.prepare()
    try:
        a1, s1 = b.execute(h)
        d1 = [(a.distance, a.levels, a.lower_bound, a.proven) for a in a1]
        a2, s2 = b.execute(h)
        d2 = [(a.distance, a.levels, a.lower_bound, a.proven) for a in a2]
    finally:
        b.free(h)
    assert d1 == d2
    assert s1.codewords == s2.codewords and s1.rounds == s2.rounds
    assert s2.device_span_ms > 0 and s2.pair_ms > 0
    a3, _ = b.run()
    assert [(a.distance, a.levels) for a in a3] == [x[:2] for x in d1]


def test_full_1024_batch_matches_reference(native):
    """All 1024 codes of the benchmark batch against the reference's own results
    (tests/golden/batch1024.json, made by make_golden.py --batch1024)."""
    import json
    import os
    from conftest import GOLDEN_DIR
    from qubitserf_b200 import workloads as W
    g = json.loads((GOLDEN_DIR / "batch1024.json").read_text())
    codes = W.batch_1024()
    ans, st = native.Batch(native.batch_items(codes)).run()
    same_host = g["meta"]["host_cores"] == os.cpu_count()
    bad = []
    for i, (a, r) in enumerate(zip(ans, g["codes"])):
        if a.distance != r[0] or a.proven != r[3] or not a.witness_ok:
            bad.append((i, a.distance, r[0]))
        if same_host and (a.levels, a.lower_bound) != (r[1], r[2]):
            bad.append((i, "levels", a.levels, r[1]))
    assert not bad, bad[:10]
    assert st.certificates == 1024


def test_one_shot_pipeline_equals_single_batch(native):
    """qsfb_batch cuts batches of 256+ queries into chunks whose jobs join the running job
    groups at round boundaries (each chunk at whatever round its preparation ends); with
    any chunk and group count, and in the caller's order or the estimated-distance order
    of the chunks, the answers, levels and codeword counts equal one prepared batch
    executed as a whole."""
    import os
    from qubitserf_b200 import workloads as W
    items = native.batch_items(W.batch_1024(300))
    b = native.Batch(items)
    h = b.prepare()
    ref, st2 = b.execute(h)                             # one batch
    b.free(h)
    want = [(r.distance, r.lower_bound, r.proven, r.levels, r.z_weight, r.x_weight)
            for r in ref]
    try:
        for chunks, groups, order in [("4", "3", "gv"), ("2", "1", "gv"), ("8", "4", "gv"),
                                      ("3", "2", "gv"), ("3", "3", "index")]:
            os.environ["QSFB_BATCH_CHUNKS"] = chunks
            os.environ["QSFB_OVERLAP_GROUPS"] = groups
            os.environ["QSFB_BATCH_ORDER"] = order
            ans, st = native.Batch(items).run()
            got = [(a.distance, a.lower_bound, a.proven, a.levels, a.z_weight, a.x_weight)
                   for a in ans]
            assert got == want, (chunks, groups)
            assert all(a.witness_ok == 1 for a in ans), (chunks, groups)
            assert st.certificates == st2.certificates == len(items)
            assert st.codewords == st2.codewords, (chunks, groups)
    finally:
        os.environ.pop("QSFB_BATCH_CHUNKS", None)
        os.environ.pop("QSFB_OVERLAP_GROUPS", None)
        os.environ.pop("QSFB_BATCH_ORDER", None)


def test_job_groups_do_not_change_answers(native):
    """Execute steps the jobs as interleaved groups (QSFB_EXEC_GROUPS, each on its own
    stream and host thread); one group and four groups give the same answers, levels and
    codeword counts, and every group's witnesses verify."""
    import os
    from qubitserf_b200 import workloads as W
    b = native.Batch(native.batch_items(W.batch_1024(400)))
    h = b.prepare()
    out = {}
    try:
        for g in ("1", "4"):
            os.environ["QSFB_EXEC_GROUPS"] = g
            a, st = b.execute(h)
            out[g] = ([(x.distance, x.lower_bound, x.proven, x.levels, x.z_weight, x.x_weight,
                        x.witness_ok) for x in a], st.codewords, st.certificates)
    finally:
        os.environ.pop("QSFB_EXEC_GROUPS", None)
        b.free(h)
    assert out["1"] == out["4"]
    assert all(t[-1] == 1 for t in out["4"][0])
