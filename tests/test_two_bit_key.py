"""The two-bit seed key's order properties, on every window of up to four
symbols over the logical-text alphabet (past-end, sentinel, separator, A, C,
G, T, N): the key is monotone in the windows' order, one-to-one on windows of
regular symbols and on the all-N window, and strictly ordered between such a
window and any other.  These are what let the seed sort rank every regular
window exactly and leave only rare windows to the side list.  The key here
is a restatement of two_bit_key() in sufkit_b200/csrc/doubling.cuh."""
import itertools

import pytest

LO, HI, BITS = 3, 7, 3  # codes: 0 past-end, 1 sentinel, 2 separator, 3-6 ACGT, 7 N


def exact_key(w):
    e = 0
    for c in w:
        e = (e << BITS) | c
    return e


def two_bit_key(w, hi=HI):
    s = len(w)
    k2 = 0
    irregular = 0
    for c in w:
        reg = LO <= c < LO + 4
        k2 = (k2 << 2) | (c - LO if reg else 0)
        irregular = (irregular << 1) | (0 if reg else 1)
    if irregular == 0:
        return (k2 << 2) | 1
    j = s - irregular.bit_length()
    tail = 2 * (s - j)
    head = (k2 >> tail) << tail
    if w[j] < LO:
        return head << 2
    fill = (1 << tail) - 1
    if j == 0 and hi and all(c == hi for c in w):
        return ((head | fill) << 2) | 3
    return ((head | fill) << 2) | 2


def windows(s, alphabet):
    for w in itertools.product(alphabet, repeat=s):
        if 0 in w and any(c != 0 for c in w[w.index(0):]):
            continue  # past-end only as a suffix of the window
        yield w


def rare(k):
    return (k & 1) == 0


@pytest.mark.parametrize("s", [1, 2, 3, 4])
@pytest.mark.parametrize("alphabet,hi", [(range(8), HI), (range(7), 0), (range(9), 8)])
def test_order_properties(s, alphabet, hi):
    """range(9): two symbols above T (N and one more); only windows of the
    largest one get t = 3."""
    ws = sorted(windows(s, alphabet))
    keys = [two_bit_key(w, hi) for w in ws]
    assert all(a <= b for a, b in zip(keys, keys[1:])), "not monotone"
    for a, b in zip(keys, keys[1:]):
        if not (rare(a) and rare(b)):
            assert a < b, "a regular window shares its key"
    assert max(keys).bit_length() <= 2 * s + 2


def test_rare_windows_are_the_ones_with_other_symbols():
    for w in windows(3, range(8)):
        regular = all(LO <= c < LO + 4 for c in w)
        all_n = all(c == HI for c in w)
        assert rare(two_bit_key(w)) == (not regular and not all_n)


def place(text, s):
    """The seed phase on a small text, as the kernels do it: sort by two-bit
    key (ties by position), then place the rare rows from the list sorted by
    exact key: entry idx of key k goes to row g + (idx - i0), g the first row
    of k, i0 its first entry.  Returns the positions in row order."""
    import bisect
    n = len(text)
    codes = list(text) + [0] * s  # text given as codes 1..7, 0 past the end
    windows = [tuple(codes[p:p + s]) for p in range(n)]
    keys = [two_bit_key(w) for w in windows]
    rows = sorted(range(n), key=lambda p: (keys[p], p))
    sorted_keys = [keys[p] for p in rows]
    rare_list = sorted((p for p in range(n) if rare(keys[p])), key=lambda p: exact_key(windows[p]))
    rare_keys = [keys[p] for p in rare_list]
    for idx, p in enumerate(rare_list):
        k = rare_keys[idx]
        i0 = bisect.bisect_left(rare_keys, k)
        g = bisect.bisect_left(sorted_keys, k)
        rows[g + idx - i0] = p
    return rows, windows


@pytest.mark.parametrize("seed", range(40))
def test_placement_orders_rows_by_exact_window(seed):
    import random
    rng = random.Random(seed)
    n = rng.randint(5, 200)
    body = [rng.randint(LO, LO + 3) for _ in range(n)]
    for _ in range(rng.randint(0, 5)):  # N runs
        at, length = rng.randrange(n), rng.randint(1, 10)
        body[at:at + length] = [HI] * len(body[at:at + length])
    for _ in range(rng.randint(0, 3)):  # separators
        body[rng.randrange(n)] = 2
    text = body + ([1] if rng.random() < 0.7 else [])  # the sentinel, mostly
    s = rng.randint(1, 7)
    rows, windows = place(text, s)
    assert sorted(rows) == list(range(len(text)))
    order = [exact_key(windows[p]) for p in rows]
    assert order == sorted(order)
