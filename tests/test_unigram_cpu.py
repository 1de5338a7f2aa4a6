"""The reference's unigram table from first slots (felog_unigram_starts, host
code of the CUDA library, no GPU needed).

The reference fills its 1e8 slots one by one and moves to the next word at
most once per slot (word2vec.cu:674-694); the library computes each word's
first slot from the same FP64 sums and a prefix maximum and fills the slots in
parallel.  The expanded table must equal the oracle's slot-by-slot
restatement, also where words' shares are below one slot, so that the
reference's walk lags behind the shares and some words get no slot at all.
"""
import numpy as np
import pytest

import felog_b200 as fb
import oracle_binding as ob

T = 100_000_000


def expand(start):
    """Slot a holds the last word whose first slot is <= a."""
    s = np.minimum(start.astype(np.int64), T)
    ends = np.append(s[1:], T)
    return np.repeat(np.arange(len(s), dtype=np.int32), np.maximum(ends - s, 0))


def c1_counts():
    g = fb.synth_graph(seed=0, v_target=16384, e_target=131072, holdout=0.10)
    c = ob.OracleCsr(g["edges"], g["v_num"])
    return np.asarray(ob.vocab(c.deg, 0)[1], np.int64)


def lagging_counts():
    # one dominant word (about 97% of the weight) and 3 M words of count 1
    # whose shares (~5.5e-9) are below one slot (1e-8)
    return np.concatenate([[10 ** 11, 10 ** 6, 10 ** 6], np.full(3_000_000, 1)]).astype(np.int64)


def zipf_counts():
    rng = np.random.default_rng(7)
    return np.sort(rng.zipf(1.7, size=2_000_000).clip(1, 10 ** 9))[::-1].astype(np.int64)


def single_word():
    return np.array([5], np.int64)


def with_zero_counts():
    # words of count 0 have no share; the reference's walk still passes through them one slot at a time
    return np.array([1000, 500, 0, 0, 300, 0, 7, 1, 0], np.int64)


@pytest.mark.parametrize("make", [c1_counts, lagging_counts, zipf_counts, single_word, with_zero_counts])
def test_table_from_first_slots_equals_the_reference_loop(make):
    counts = make()
    start = fb.unigram_starts(counts)
    assert np.all(np.diff(start.astype(np.int64)) > 0) and start[0] == 0
    ref = ob.unigram_table(counts)
    got = expand(start)
    assert len(got) == len(ref) == T
    np.testing.assert_array_equal(got, ref)


def test_lagging_vocabulary_leaves_words_without_slots():
    counts = lagging_counts()
    start = fb.unigram_starts(counts)
    assert start[-1] >= T  # the walk never reaches the last words


def test_unigram_starts_rejects_empty_and_oversized_input():
    L = fb.gpu_lib()
    one = np.ones(1, np.uint64)
    assert L.felog_unigram_starts(one.ctypes.data, 0, one.ctypes.data) == 1
    assert L.felog_unigram_starts(one.ctypes.data, 12_500_001, one.ctypes.data) == 1
