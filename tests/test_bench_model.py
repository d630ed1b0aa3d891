"""CPU: the whole-build byte model used by bench.py.

The model's per-suffix terms are defined in text order (m(i) through the ISA,
C through PLCP); bench.py evaluates them from the row-order LCP alone so that
a multi-Gsym build can be reduced on the device.  These tests check that the
row-order forms equal the text-order definitions on oracle builds."""
import numpy as np

import bench
import oracle
from sufkit_b200 import synth


def _direct(text, seed=21):
    sa, isa, lcp = oracle.full_build(text)
    n = text.size
    l = lcp.astype(np.int64)
    nxt = np.append(l[1:], 0)
    row = isa.astype(np.int64)
    m = np.maximum(l[row], nxt[row])
    a_k, k = [], 1
    while True:
        a = int(np.count_nonzero(m >= seed * (1 << (k - 1))))
        if a == 0:
            break
        a_k.append(a)
        k += 1
    plcp = np.empty(n, np.int64)
    plcp[sa.astype(np.int64)] = l
    prev = np.concatenate([[0], np.maximum(plcp[:-1] - 1, 0)])
    compares = int(np.sum(plcp - prev + 1))
    return lcp, a_k, compares


def test_row_order_statistics_equal_text_order_definitions():
    rng = np.random.default_rng(11)
    texts = [synth.repeat_rich_100mbp(scale=0.001).logical_text(),
             synth.human_scale_3gbp(scale=0.0002).logical_text(),
             synth.random_text(rng, 3000, 2),
             np.concatenate([np.full(500, 2, np.uint8), np.zeros(1, np.uint8)])]
    for text in texts:
        lcp, a_k, compares = _direct(text)
        got_a, nonzero = bench.text_statistics(lcp)
        assert got_a == a_k
        assert text.size + nonzero == compares


def test_model_bytes_terms():
    n = 1000
    # seed 29n, rounds 32*(10+2), ISA emit 4n (no ISA plane), PHI 24n + 2C,
    # pack 9n (split40), byte-coded n + 8 * anchors.
    got = bench.model_bytes(n, [10, 2], 700, w_sa=5, w_isa=0, lcp_kind="byte", anchors=3)
    assert got == 29 * n + 32 * 12 + 4 * n + 24 * n + 2 * (n + 700) + 9 * n + n + 8 * 3
    raw = bench.model_bytes(n, [], 0, w_sa=4, w_isa=4, lcp_kind="raw")
    assert raw == 29 * n + 8 * n + 24 * n + 2 * n + 8 * n + 4 * n
