"""CPU checks of the parcel initialiser shared by the device and the oracle (st_init.h):
the Hilbert decode is a bijection whose consecutive indices are unit steps (the defining
property of the curve, checked exhaustively on small curves), each cloud stays inside its
own curve segment, and the generated parcels lie inside the mesh with diameters in range."""
import numpy as np
import pytest

import oracle


@pytest.mark.parametrize("bits", [1, 2, 3, 4, 5])
def test_hilbert_decode_is_a_continuous_bijection(bits):
    n = 8 ** bits
    p = oracle.hilbert3(np.arange(n, dtype=np.uint64), bits).astype(np.int64)
    assert p.min() == 0 and p.max() == 2 ** bits - 1
    lin = (p[:, 2] << (2 * bits)) | (p[:, 1] << bits) | p[:, 0]
    assert np.unique(lin).size == n                       # every point exactly once
    step = np.abs(np.diff(p, axis=0)).sum(axis=1)
    assert (step == 1).all()                              # neighbours along the curve
    assert (p[0] == 0).all()                              # starts at the origin


def test_hilbert_decode_ten_bits_sample():
    rng = np.random.default_rng(3)
    h = rng.integers(0, 2 ** 30 - 1, 20000).astype(np.uint64)
    a = oracle.hilbert3(h, 10).astype(np.int64)
    b = oracle.hilbert3(h + 1, 10).astype(np.int64)
    assert (np.abs(a - b).sum(axis=1) == 1).all()
    assert a.max() < 1024


@pytest.mark.parametrize("pbytes", [4, 8])
def test_initialised_parcels_inside_and_clustered(pbytes):
    N, L, nc, n = (16, 12, 20), 0.1, 4, 20000
    origin, ending = (0.0, -0.05, 0.2), (0.1, 0.05, 0.4)
    boxes = []
    for c in range(nc):
        xyz, d = oracle.init_parcels(pbytes, 77, c, nc, n, N, origin, ending, 5e-6, 5e-5)
        for a in range(3):
            assert (xyz[a] >= origin[a]).all() and (xyz[a] < ending[a]).all()
        assert (d >= 5e-6).all() and (d < 5e-5).all()
        if pbytes == 4:
            assert np.array_equal(xyz, xyz.astype(np.float32).astype(np.float64))
        boxes.append(np.floor((xyz.T - np.array(origin)) / ((np.array(ending) - origin)
                                                             / np.array(N))).astype(int))
    # the four quarters of the curve occupy disjoint sets of cells
    sets = [set(map(tuple, b)) for b in boxes]
    for i in range(nc):
        for j in range(i + 1, nc):
            assert len(sets[i] & sets[j]) <= 0.02 * min(len(sets[i]), len(sets[j]))
    # same seed, same parcels; another seed, other parcels
    a1 = oracle.init_parcels(pbytes, 77, 1, nc, 100, N, origin, ending, 5e-6, 5e-5)[0]
    a2 = oracle.init_parcels(pbytes, 78, 1, nc, 100, N, origin, ending, 5e-6, 5e-5)[0]
    b1 = oracle.init_parcels(pbytes, 77, 1, nc, 100, N, origin, ending, 5e-6, 5e-5)[0]
    assert np.array_equal(a1, b1) and not np.array_equal(a1, a2)
