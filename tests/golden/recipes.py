"""Deterministic input recipes shared by the fixture generator and the tests.

A fixture stores a recipe (a few integers) instead of a large input; both
sides rebuild the input with these functions.
"""
import numpy as np

M64 = 0xFFFFFFFFFFFFFFFF


def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def pack(sents):
    off = np.zeros(len(sents) + 1, np.uint64)
    off[1:] = np.cumsum([len(s) for s in sents])
    tok = np.concatenate(sents).astype(np.uint32) if len(sents) else np.zeros(0, np.uint32)
    return tok, off


def synth_corpus(V, n_sent, seed, long_every=0, long_len=1200, max_len=8):
    """Token sequences over vertices 0..V-1 from one splitmix64 stream; every
    long_every-th sentence has long_len tokens (to reach the 1000-token cap)."""
    sents = []
    x = int(seed)
    for i in range(int(n_sent)):
        x = splitmix64(x)
        L = 1 + x % int(max_len)
        if long_every and i % long_every == long_every - 1:
            L = int(long_len)
        toks = np.empty(L, np.uint32)
        for t in range(L):
            x = splitmix64(x)
            toks[t] = (x >> 20) % V if (x & 7) else (x >> 20) % 8
        sents.append(toks)
    return sents
