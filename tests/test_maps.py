"""L2GMap construction (host logic): the library's communication pattern is
bit-identical to the oracle's restatement of L2GMap.cpp:15-122 for every rank,
and the reference's errors carry its messages."""
import numpy as np
import pytest
from hypothesis import given, settings, strategies as st

import oracle
import spmv_b200 as S
from spmv_b200 import gen

FIELDS = ["neighbours", "send_count", "recv_count", "send_offset", "recv_offset",
          "indexbuf"]


def assert_same_pattern(local_sizes, ghosts):
    P = len(local_sizes)
    comm = S.Comm(size=P, device=-1)
    m = S.L2GMap(comm, local_sizes, ghosts)
    om = oracle.Map(local_sizes, ghosts)
    for r in range(P):
        for f in FIELDS:
            a, b = m.pattern(r, f), om.field(r, f)
            assert np.array_equal(a, b), (r, f, a, b)
        assert m.local_size(r) == local_sizes[r]
        assert m.num_ghosts(r) == len(ghosts[r])
        assert np.array_equal(m.ghosts(r), np.asarray(ghosts[r], np.int64))
        off = int(np.sum(local_sizes[:r]))
        assert m.global_offset(r) == off
        for i in list(range(off, off + local_sizes[r], max(1, local_sizes[r] // 7))) + \
                list(ghosts[r]):
            assert m.global_to_local(r, int(i)) == om.global_to_local(r, int(i))
    assert m.global_size() == int(np.sum(local_sizes))
    return m


@pytest.mark.parametrize("P", [1, 2, 3, 8])
def test_stencil_maps_match_oracle(P):
    W = gen.workload("c2", scale=16)
    D = gen.distribute(W.A, P)
    assert_same_pattern(D.local_sizes, D.ghosts)


def test_owner_ranges_match_oracle():
    for size in (1, 2, 3, 7, 8):
        for N in (0, 1, 5, 17, 500000):
            assert np.array_equal(gen.owner_ranges(size, N), oracle.owner_ranges(size, N))


def test_no_neighbour_quirk():
    # A rank with no neighbours keeps send_count = recv_count = {0}
    # (L2GMap.cpp:87-92) and send_offset = {L, L}.
    m = assert_same_pattern([4, 3, 5], [[4], [0], []])
    assert list(m.pattern(2, "send_count")) == [0]
    assert list(m.pattern(2, "recv_count")) == [0]
    assert list(m.pattern(2, "send_offset")) == [5, 5]


def test_empty_rank_and_duplicate_ghosts():
    assert_same_pattern([0, 4, 4], [[1, 2], [4, 4, 5], [0, 3, 3]])


def test_ghost_outside_global_range_is_error():
    comm = S.Comm(size=2, device=-1)
    with pytest.raises(S.SpmvError, match="outside the global range"):
        S.L2GMap(comm, [4, 4], [[8], []])


def test_unsorted_ghosts_message():
    comm = S.Comm(size=2, device=-1)
    with pytest.raises(S.SpmvError) as e:
        S.L2GMap(comm, [4, 4], [[6, 5], []])
    assert str(e.value) == "Ghosts must be sorted"
    with pytest.raises(RuntimeError, match="Ghosts must be sorted"):
        oracle.Map([4, 4], [[6, 5], []])


def test_ghost_in_local_range_message():
    comm = S.Comm(size=2, device=-1)
    with pytest.raises(S.SpmvError) as e:
        S.L2GMap(comm, [4, 4], [[2], []])
    assert str(e.value) == "Ghost index in local range"
    with pytest.raises(RuntimeError, match="Ghost index in local range"):
        oracle.Map([4, 4], [[2], []])


def test_global_to_local_unknown_index_is_error():
    comm = S.Comm(size=2, device=-1)
    m = S.L2GMap(comm, [4, 4], [[5], []])
    assert m.global_to_local(0, 5) == 4
    with pytest.raises(S.SpmvError, match="neither owned nor a ghost"):
        m.global_to_local(0, 6)


@settings(max_examples=60, deadline=None)
@given(st.data())
def test_random_maps_match_oracle(data):
    P = data.draw(st.integers(1, 8))
    sizes = data.draw(st.lists(st.integers(0, 12), min_size=P, max_size=P))
    N = sum(sizes)
    ranges = np.concatenate([[0], np.cumsum(sizes)])
    ghosts = []
    for r in range(P):
        outside = [i for i in range(N) if not (ranges[r] <= i < ranges[r + 1])]
        g = data.draw(st.lists(st.sampled_from(outside), max_size=8)) if outside else []
        ghosts.append(sorted(g))
    assert_same_pattern(sizes, ghosts)
