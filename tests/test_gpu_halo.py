"""L2GMap::update and reverse_update on the GPU: bitwise equal to the oracle's
restatement of L2GMap.cpp:126-170 (copies and ordered additions)."""
import numpy as np
import pytest
import torch

import oracle
import spmv_b200 as S
from spmv_b200 import gen

pytestmark = pytest.mark.gpu


def maps_for(local_sizes, ghosts):
    P = len(local_sizes)
    comm = S.Comm(size=P, device=0)
    return comm, S.L2GMap(comm, local_sizes, ghosts), oracle.Map(local_sizes, ghosts)


def random_map(rng, P, maxsize=50, maxg=20):
    sizes = [int(rng.integers(0, maxsize)) for _ in range(P)]
    N = sum(sizes)
    ranges = np.concatenate([[0], np.cumsum(sizes)])
    ghosts = []
    for r in range(P):
        outside = np.array([i for i in range(N) if not ranges[r] <= i < ranges[r + 1]])
        k = int(rng.integers(0, maxg)) if len(outside) else 0
        ghosts.append(np.sort(rng.choice(outside, size=k)) if k else np.zeros(0, np.int64))
    return sizes, ghosts


CASES = [("c2", 8), ("c2", 3), ("c1", 4)]


@pytest.mark.parametrize("cfg,P", CASES)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_update_bitwise(cuda_device, cfg, P, dtype):
    D = gen.distribute(gen.workload(cfg, scale=40 if cfg == "c2" else 128).A, P)
    comm, m, om = maps_for(D.local_sizes, D.ghosts)
    rng = np.random.default_rng(0)
    vecs = [rng.standard_normal(m.vec_len(q)).astype(dtype) for q in range(P)]
    ref = [v.copy() for v in vecs]
    om.update(ref)
    got = [v.copy() for v in vecs]
    m.update(got)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    dev = [torch.from_numpy(v).cuda() for v in vecs]
    m.update(dev)
    for a, b in zip(dev, ref):
        assert np.array_equal(a.cpu().numpy(), b)


@pytest.mark.parametrize("cfg,P", CASES)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_reverse_update_bitwise(cuda_device, cfg, P, dtype):
    D = gen.distribute(gen.workload(cfg, scale=40 if cfg == "c2" else 128).A, P)
    comm, m, om = maps_for(D.local_sizes, D.ghosts)
    rng = np.random.default_rng(1)
    vecs = [rng.standard_normal(m.vec_len(q)).astype(dtype) for q in range(P)]
    ref = [v.copy() for v in vecs]
    om.reverse_update(ref)
    got = [v.copy() for v in vecs]
    m.reverse_update(got)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("seed", range(8))
def test_random_maps_bitwise(cuda_device, seed):
    rng = np.random.default_rng(seed)
    P = int(rng.integers(1, 9))
    sizes, ghosts = random_map(rng, P)
    comm, m, om = maps_for(sizes, ghosts)
    vecs = [rng.standard_normal(m.vec_len(q)) for q in range(P)]
    for op in ("update", "reverse_update"):
        ref = [v.copy() for v in vecs]
        getattr(om, op)(ref)
        got = [v.copy() for v in vecs]
        getattr(m, op)(got)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), op


def test_shared_target_order(cuda_device):
    # Ranks 0 and 2 both ghost entry 4 (rank 1's first); rank 1 adds rank 0's
    # contribution first, then rank 2's (neighbour order), and the result is
    # the reference's rounding, not a reordered sum.
    sizes = [4, 1, 4]
    ghosts = [np.array([4]), np.array([0]), np.array([4])]
    comm, m, om = maps_for(sizes, ghosts)
    v = [np.array([0, 0, 0, 0, 1e16]), np.array([1.0, 5.0]),
         np.array([0, 0, 0, 0, -1e16])]
    ref = [x.copy() for x in v]
    om.reverse_update(ref)
    got = [x.copy() for x in v]
    m.reverse_update(got)
    assert np.array_equal(got[1], ref[1])
    assert got[1][0] == (1.0 + 1e16) + -1e16


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_complex_halo(cuda_device, dtype):
    rng = np.random.default_rng(5)
    sizes, ghosts = random_map(rng, 5)
    comm, m, om = maps_for(sizes, ghosts)
    real = np.float64 if dtype == np.complex128 else np.float32
    vecs = [(rng.standard_normal(m.vec_len(q)) + 1j * rng.standard_normal(m.vec_len(q)))
            .astype(dtype) for q in range(5)]
    for op in ("update", "reverse_update"):
        re = [v.real.astype(real).copy() for v in vecs]
        im = [v.imag.astype(real).copy() for v in vecs]
        getattr(om, op)(re)
        getattr(om, op)(im)
        got = [v.copy() for v in vecs]
        getattr(m, op)(got)
        for g, a, b in zip(got, re, im):
            assert np.array_equal(g.real, a) and np.array_equal(g.imag, b), op
