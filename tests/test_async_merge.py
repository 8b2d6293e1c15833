"""Two-device asynchronous iteration: the merge of two iterates
(Core::read_and_solve_conflict) on the GPU against its CPU restatement."""
import numpy as np
import pytest

from libatssim_b200 import configs
from oracle import ats_oracle as O


def _three_states(n, seed):
    rng = np.random.RandomState(seed)
    begin = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    mine = begin + (1e-3 * rng.standard_normal((n, 3))).astype(np.float32)
    other = begin + (1e-3 * rng.standard_normal((n, 3))).astype(np.float32)
    # every branch: only one moved, neither moved
    mine[::5] = begin[::5]
    other[1::7] = begin[1::7]
    mine[2::11] = begin[2::11]
    other[2::11] = begin[2::11]
    return begin, mine, other


def test_merge_restatement_branches():
    b, s, o = _three_states(200, 0)
    m = O.async_merge(b, s, o, 0.5)
    only_s = np.any(s != b, 1) & np.all(o == b, 1)
    only_o = np.any(o != b, 1) & np.all(s == b, 1)
    none = np.all(s == b, 1) & np.all(o == b, 1)
    assert np.array_equal(m[only_s], s[only_s]) and np.array_equal(m[only_o], o[only_o])
    assert np.array_equal(m[none], b[none])
    both = ~(only_s | only_o | none)
    assert np.allclose(m[both], b[both] + 0.5 * ((s - b) + (o - b))[both], atol=1e-6)
    assert np.allclose(O.async_merge(b, s, o, 0.0), 0.5 * (s + o), atol=1e-7)


@pytest.mark.gpu
@pytest.mark.parametrize("weight", [0.5, 0.3, 0.0])
def test_gpu_merge_is_bit_exact(ats, weight):
    insts, prm = configs.c2(num_instances=2, seed=7, side_range=(12, 20))
    cloth = ats.Cloth(insts, **prm)
    n = cloth.nv
    begin, mine, other = _three_states(n, 3)
    cloth.set_positions(begin)
    cloth.async_fork()
    cloth.set_positions(mine)
    cloth.async_merge(other, weight)
    expect = O.async_merge(begin, mine, other, weight)
    assert np.array_equal(cloth.positions(), expect)
    # the merge is the new fork point: a second merge with an unmoved other keeps it
    cloth.async_merge(expect, weight)
    assert np.array_equal(cloth.positions(), O.async_merge(expect, expect, expect, weight))


@pytest.mark.gpu
def test_merge_without_fork_is_rejected(ats):
    insts, prm = configs.c2(num_instances=1, seed=1, side_range=(8, 8))
    cloth = ats.Cloth(insts, **prm)
    with pytest.raises(ats.AtsError):
        cloth.async_merge(cloth.positions(), 0.5)
