"""Helpers shared by the tests (fixtures loading, key conversions)."""
import json
import os

import numpy as np

from conftest import GOLDEN

M64 = (1 << 64) - 1


def load_npz(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


def load_json(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def nlimbs(k):
    return (k + 31) // 32


def rows(a):
    """Set-comparable tuples of a (n, L) key array."""
    a = np.asarray(a, dtype=np.uint64)
    return [tuple(int(v) for v in r) for r in a]


def ecoli_packed():
    d = load_npz("ecoli_1K_packed.npz")
    return d["data"], d["offsets"], d["lengths"], d


def synth_small_packed():
    d = load_npz("synth_c2_small_packed.npz")
    return d["data"], d["offsets"], d["lengths"]


def kmer_strings(data, offsets, lengths, k):
    """All k-mer strings of packed reads (small inputs only)."""
    out = []
    for o, n in zip(offsets, lengths):
        o, n = int(o), int(n)
        by = data[o:o + (n + 3) // 4]
        codes = np.stack([(by >> 6) & 3, (by >> 4) & 3, (by >> 2) & 3, by & 3], 1).reshape(-1)[:n]
        s = "".join("ACGT"[c] for c in codes)
        out.extend(s[i:i + k] for i in range(n - k + 1))
    return out
