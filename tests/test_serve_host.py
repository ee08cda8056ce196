"""Rollout server host logic without a GPU: the HBM-budget plan."""
import pytest

from kraken_3_gpu_b200 import _native, serve, workloads
from tests import serve_ref


def _maps():
    return workloads.uneven(n=4, n_maps=3, seed=1, h_min=10, h_max=20).maps


def test_plan_fills_the_budget_with_slots():
    maps = _maps()
    cap, per = serve.plan(maps, 1 << 30)
    cap2, per2 = serve.plan(maps, 2 << 30)
    assert per == per2 and cap % 2 == 0 and cap2 % 2 == 0
    assert cap * per <= 1 << 30 < (cap + 2) * per + (16 << 20)
    assert 2 * cap - 2 <= cap2 <= 2 * cap + 2 + (16 << 20) // per
    assert serve.plan(maps, 1 << 30, max_slots=100) == (100, per)


def test_plan_counts_policy_weights_and_observation_ring():
    maps = _maps()
    _, with_policy = serve.plan(maps, 1 << 30, policy=True)
    _, without = serve.plan(maps, 1 << 30, policy=False)
    assert with_policy - without == 4 * serve.policy_params(8, 9) + 4
    _, ring = serve.plan(maps, 1 << 30, policy=False, obs_ring=128)
    assert ring - without == 128 * 56 * 4


def test_plan_rejects_a_budget_below_two_slots():
    with pytest.raises(_native.KrError) as e:
        serve.plan(_maps(), 1 << 20)
    assert e.value.code == _native.KR_ERR_CAPACITY and "budget" in str(e.value)
    with pytest.raises(_native.KrError):
        serve.plan(_maps(), 1 << 30, chunk_steps=0)


def test_eps_restatement_is_standard_normal():
    import numpy as np
    e = serve_ref.eps(7, 3, 4000)
    assert abs(e.mean()) < 0.06 and abs(e.std() - 1.0) < 0.05
    assert not np.array_equal(e, serve_ref.eps(7, 4, 4000))


def test_plan_counts_net_genomes_and_records():
    """A net server keeps a genome of the largest body (net.js layout, 16-byte
    rows) and the per-slot sense / net record in every slot; policy and net
    are exclusive."""
    maps = _maps()
    _, without = serve.plan(maps, 1 << 30, policy=False)
    _, with_net = serve.plan(maps, 1 << 30, net=True)
    stride = (serve.net_param_count(8) + 3) // 4 * 4
    assert with_net - without > 4 * stride + 4
    assert with_net - without - (4 * stride + 4) < 4096  # the record: sense state and the net's vectors
    lights = [[[100.0, 100.0, 250.0, 0.7, 0.0, 0.1]]] * len(maps)
    cap_n, _ = serve.plan(maps, 1 << 30, net=True)
    cap_l, per_l = serve.plan(maps, 1 << 30, net=True, lights=lights)
    assert per_l == with_net
    # the lights and their position table (16 B per light and step, 4,096
    # steps here) are fixed bytes, taken from the budget before the slots
    table = len(maps) * 4096 * 16
    assert cap_n - cap_l >= 2 * (table // (2 * with_net))
