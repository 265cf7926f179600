"""Batched runs (wq3d_batch_run): many uneven queues driven together must
give exactly what each queue gives when run alone, listeners included."""
import numpy as np
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import _abi
from underseamodelinglibrary_b200 import scenarios as S
from oracle_binding import OracleQueue
from test_gpu_parity import compare_eigenrays, key

pytestmark = pytest.mark.gpu


class Keep(u.eigenray_listener):
    def __init__(self):
        self.rays = []
        self.checks = []

    def add_eigenray(self, t1, t2, ray, run_id):
        self.rays.append(ray)

    def check_eigenrays(self, time, run_id):
        self.checks.append(time)


def same(ra, rb):
    assert [key(r) for r in ra] == [key(r) for r in rb]
    for x, y in zip(ra, rb):
        assert x.travel_time == y.travel_time
        assert np.array_equal(x.intensity, y.intensity) and np.array_equal(x.phase, y.phase)


def test_batch_equals_separate_runs(engine):
    """eight uneven gridded instances (1..31 AZ rays, 91..241 D/E rays,
    different end times), FP64 and FP32C mixed, each with a listener"""
    scs = S.batched_gridded(n_instances=8, seed=7, num_de=(91, 241), num_az=(1, 31), time_max=(3.0, 9.0))
    precs = [_abi.FP64 if k % 2 else _abi.FP32C for k in range(len(scs))]
    alone = []
    for sc, p in zip(scs, precs):
        q = S.build_queue(sc, u.wave_queue, precision=p)
        q.run(sc["time_max"])
        alone.append((q.take_eigenrays(), q.time()))
    qs, keeps = [], []
    for sc, p in zip(scs, precs):
        q = S.build_queue(sc, u.wave_queue, precision=p)
        kp = Keep()
        q.add_eigenray_listener(kp)
        qs.append(q)
        keeps.append(kp)
    steps, ms = u.run_batch(qs, [sc["time_max"] for sc in scs])
    assert ms > 0.0
    for q, kp, (ra, t), n, sc in zip(qs, keeps, alone, steps, scs):
        assert q.time() == t and n == len(kp.checks)
        same(kp.rays, ra)
    assert sum(len(kp.rays) for kp in keeps) > 20


def test_batch_instance_against_oracle(engine):
    """one batched instance checked against the CPU oracle"""
    scs = S.batched_gridded(n_instances=3, seed=11, num_de=(91, 151), num_az=(5, 13), time_max=(6.0, 8.0))
    qs = [S.build_queue(sc, u.wave_queue) for sc in scs]
    u.run_batch(qs, [sc["time_max"] for sc in scs])
    o = S.build_queue(scs[1], OracleQueue)
    o.run(scs[1]["time_max"])
    compare_eigenrays(qs[1].take_eigenrays(), o.take_eigenrays())


def test_batch_rejects_bad_input(engine):
    sc = S.eigenray_basic()
    q = S.build_queue(sc, u.wave_queue)
    with pytest.raises(u.EngineError):
        u.run_batch([q, q], 1.0)
