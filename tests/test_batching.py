"""Planning and packing of uneven shots into batches (host logic, no GPU)."""
import numpy as np
import pytest

from hirensi_b200 import batching as B


def _shot(rng, eqs, n, recs):
    ft = rng.standard_normal((n + 1, 3))
    return B.Shot(np.asarray(eqs), np.ones(len(eqs)), ft, np.asarray(recs, dtype=np.int32),
                  rng.standard_normal((len(recs), n + 1)))


def test_plan_sorts_by_length_and_cuts():
    lengths = [100, 400, 250, 400, 90, 300]
    batches = B.plan(lengths, max_shots=4)
    assert batches == [[1, 3, 5, 2], [0, 4]]
    with pytest.raises(ValueError):
        B.plan(lengths, max_shots=9)


def test_pack_union_masks_and_data():
    rng = np.random.default_rng(0)
    shots = [_shot(rng, [7], 30, [10, 11, 12, 20, 21, 22]),
             _shot(rng, [9, 7], 18, [20, 21, 22, 10, 11, 12, 10]),   # a duplicate receiver equation
             _shot(rng, [5], 25, [40, 41, 42])]
    b = B.pack(shots, [0, 1, 2])
    assert b.nstep == 30
    assert list(b.nstep_shot) == [30, 18, 25]
    assert list(b.src_eq) == [5, 7, 9]
    assert b.src_b.tolist() == [[0, 0, 1], [1, 1, 0], [0, 1, 0]]
    # union: first use order, equation 10 twice (shot 1 lists it twice)
    assert list(b.eqdis) == [10, 10, 11, 12, 20, 21, 22, 40, 41, 42]
    for k, s in enumerate(shots):
        assert b.rec_mask[k].sum() == len(s.eqdis)
        assert list(b.eqdis[b.slots[k]]) == list(s.eqdis)
        # data and time functions padded with zeros past the shot's length
        assert np.array_equal(b.dis[k][b.slots[k], : s.nstep + 1], s.dis)
        assert not b.dis[k][:, s.nstep + 1:].any()
        assert np.array_equal(b.ftab[k, : s.nstep + 1], s.ftab)
        assert not b.ftab[k, s.nstep + 1:].any()
    # the two copies of equation 10 in shot 1 keep its order
    assert list(b.slots[1]) == [4, 5, 6, 0, 2, 3, 1]


def test_unpack_traces_round_trip():
    rng = np.random.default_rng(1)
    shots = [_shot(rng, [1], 12, [3, 4, 5]), _shot(rng, [2], 8, [4, 5, 6, 3])]
    b = B.pack(shots, [1, 0])
    tr = np.zeros((2, len(b.eqdis), b.nstep + 1))
    for k, i in enumerate(b.shots):
        tr[k][b.slots[k], : shots[i].nstep + 1] = shots[i].dis
    out = B.unpack_traces(b, tr)
    for k, i in enumerate(b.shots):
        assert np.array_equal(out[k], shots[i].dis)
