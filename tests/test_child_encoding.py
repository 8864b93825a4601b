"""The traversal reads a node's children as one int2: (first child, count | slot order in
3 bits each), which holds only if every node's children occupy its first slots and are
consecutive node indices.  Checked here on the oracle's trees (the reference's numbering)
for the golden cases and two seeded workloads, with the encoding decoded back to
children[].  No GPU."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden


def encode(ch):
    cnt = int((ch != -1).sum())
    if cnt == 0:
        return -1, None
    assert (ch[:cnt] != -1).all() and (ch[cnt:] == -1).all(), ch
    base = int(ch[:cnt].min())
    assert sorted(ch[:cnt] - base) == list(range(cnt)), ch  # consecutive indices
    code = cnt
    for c in range(cnt):
        code |= int(ch[c] - base) << (4 + 3 * c)
    return base, code


def decode(base, code):
    return [base + ((code >> (4 + 3 * k)) & 7) for k in range(code & 15)]


def check_tree(T):
    children = np.asarray(T.children).reshape(-1, 8)
    for ch in children:
        base, code = encode(ch)
        if code is not None:
            assert decode(base, code) == list(ch[:code & 15])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_trees(orc, name):
    g = load_golden(name)
    check_tree(orc.Tree(g["x"], g["y"], g["z"], int(g["maxmemb"])))


@pytest.mark.parametrize("maxmemb", [8, 100])
def test_seeded_trees(orc, maxmemb):
    from bit_b200 import workloads
    x, y, z, _ = workloads.clustered_blobs(20000, seed=17)
    check_tree(orc.Tree(x, y, z, maxmemb))
