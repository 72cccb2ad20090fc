"""Random-information-set seed trials on the device against the host trials and the
reference, including rows of three and four 64-bit words (n in (128, 256]), where the
trial kernel dispatches the column's word four ways.  The seed bound decides where the BZ
levels stop, so equal `levels` and `lower_bound` mean equal seeds."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def codes():
    from qubitserf_b200 import workloads as W
    rng = np.random.default_rng(11)
    items = []
    # classical codes of small dimension (cheap for the reference) at three and four words
    for n, k in [(140, 12), (190, 14), (250, 16), (100, 20)]:
        items.append(("classical", W.classical_parity_from_rng(rng, n, k)))
    # CSS codes with n > 128 and both sides' K <= 128, distances 5-6
    rng = np.random.default_rng(12)
    for n, rx, rz in [(150, 30, 30), (170, 45, 30), (135, 25, 25)]:
        Hx, Hz = W.css_from_rng(rng, n, rx, rz)
        items.append(("css", Hx, Hz, "M"))
    return items


def answers(native, items):
    ans, _ = native.Batch(items).run()
    return [(a.distance, a.lower_bound, a.levels, a.proven, a.witness_ok) for a in ans]


def test_device_seeds_equal_host_seeds(native):
    items = codes()
    dev = answers(native, items)
    os.environ["QSFB_HOST_SEEDS"] = "1"
    try:
        host = answers(native, items)
    finally:
        os.environ.pop("QSFB_HOST_SEEDS", None)
    assert dev == host
    assert all(a[4] == 1 for a in dev), dev


def test_wide_rows_match_reference(native, ref):
    if ref is None:
        pytest.skip("reference library not present on this host")
    items = codes()
    got = answers(native, items)
    for it, g in zip(items, got):
        r = ref.classical(it[1]) if it[0] == "classical" else ref.css(it[1], it[2], "M")
        assert (g[0], g[1], g[2], g[3]) == (r.distance, r.lower_bound, r.levels, r.proven), it[0]
