"""Eigenverbs on the GPU against the oracle and the reference's reverb
known answers: boundary and volume-layer footprints, their order, the
bounce and power thresholds, and the interleaving with reflection
notices."""
import math

import numpy as np
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import scenarios as S
from oracle_binding import OracleQueue
from test_oracle_kats import accuracy_spacing, check_bottom_eigenverbs, demo_spacing

pytestmark = pytest.mark.gpu


class Recorder(u.eigenverb_listener, u.reflection_listener):
    """keeps every eigenverb and reflection notice in arrival order"""

    def __init__(self):
        self.events = []

    def add_eigenverb(self, verb, interface_num):
        assert interface_num == verb.interface_num
        self.events.append(("verb", verb))

    def reflect(self, time, de, az, dt, grazing, speed, position, ndirection, type):
        self.events.append(("refl", (time, de, az, type)))

    def verbs(self):
        return [v for kind, v in self.events if kind == "verb"]


def key(v):
    return (v.step, v.de_index, v.az_index, v.seq, v.interface_num)


def compare_verbs(eng, orc):
    """same eigenverbs in the same order, values within FP64 rounding of
    the GPU's transcendental functions"""
    assert [key(v) for v in eng] == [key(v) for v in orc]
    for e, o in zip(eng, orc):
        for f in ("surface", "bottom", "caustic", "upper", "lower"):
            assert getattr(e, f) == getattr(o, f), (key(o), f)
        assert abs(e.travel_time - o.travel_time) < 1e-9
        for f in ("length", "width", "sound_speed"):
            assert abs(getattr(e, f) - getattr(o, f)) <= 1e-9 * abs(getattr(o, f)), (key(o), f)
        for f in ("grazing", "direction", "source_de", "source_az"):
            assert abs(getattr(e, f) - getattr(o, f)) < 1e-9, (key(o), f)
        assert abs(e.position[0] - o.position[0]) < 1e-6
        assert abs(e.position[1] - o.position[1]) < 1e-12 and abs(e.position[2] - o.position[2]) < 1e-12
        assert np.allclose(e.power, o.power, rtol=1e-9, atol=0)


def run_both(sc, setup=None):
    rec = Recorder()
    q = S.build_queue(sc, u.wave_queue)
    q.add_eigenverb_listener(rec)
    o = S.build_queue(sc, OracleQueue, eigenverbs=True)
    if setup:
        setup(q)
        setup(o)
    q.run(sc["time_max"])
    o.run(sc["time_max"])
    return rec.verbs(), o.take_eigenverbs()


def test_eigenverb_accuracy(engine):
    """reverb_test.cc:216-310 on the engine, and every eigenverb equal to
    the oracle's (bottom, surface and both sides of the 300 m layer)"""
    sc = S.eigenverb_accuracy()
    eng, orc = run_both(sc)
    bottom = [v for v in eng if v.interface_num == u.eigenverb_model.BOTTOM]
    assert check_bottom_eigenverbs(sc, bottom, accuracy_spacing, 0.1, False) >= 10
    assert {v.interface_num for v in eng} == {0, 1, 2, 3}
    compare_verbs(eng, orc)


def test_eigenverb_demo(engine):
    """reverb_test.cc:334-443 on the engine: tangent-spaced D/E, bounce
    limits of 2"""
    sc = S.eigenverb_demo()
    eng, orc = run_both(sc)
    bottom = [v for v in eng if v.interface_num == u.eigenverb_model.BOTTOM]
    assert check_bottom_eigenverbs(sc, bottom, demo_spacing, 0.5, True) >= 20
    assert all(v.surface <= 2 and v.bottom <= 2 for v in eng)
    compare_verbs(eng, orc)


def test_eigenverbs_sloped_rayleigh_with_layers(engine):
    """sloped Rayleigh workload on a reduced fan with two volume layers,
    an eigenverb power threshold and a bottom-bounce limit"""
    sc = S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=4, n_depth=4, time_max=8.0)
    sc["ocean"].add_volume(u.volume_flat(40.0, 5.0, -50.0))
    sc["ocean"].add_volume(u.volume_flat(150.0, 5.0, -45.0))

    def setup(q):
        q.eigenverb_threshold(-70.0)
        q.max_bottom(3)

    eng, orc = run_both(sc, setup)
    kinds = {v.interface_num for v in eng}
    assert {0, 1, 2, 3, 4, 5} <= kinds
    assert len(eng) > 1000
    assert all(v.bottom <= 3 for v in eng) and min(float(v.power.max()) for v in eng) >= 1e-7
    compare_verbs(eng, orc)


def test_eigenverbs_gridded_ocean(engine):
    """3-D profile_grid over 2-D boundary_grid relief with a layer: the
    gridded stepping kernels and the volume pass together"""
    sc = S.gridded_munk(seed=5, num_de=61, num_az=9, n_targets=8, time_max=12.0)
    sc["ocean"].add_volume(u.volume_flat(500.0, 10.0, -40.0))
    eng, orc = run_both(sc)
    assert len(eng) > 100
    compare_verbs(eng, orc)


def test_bounce_threshold_eigenverbs(engine):
    """reflection_test.cc:597-661 eigenverb half on the engine, equal to
    the oracle's"""
    sc = S.bounce_threshold()
    eng, orc = run_both(sc)
    assert len(eng) > 100 and all(v.bottom <= 5 and v.surface <= 3 for v in eng)
    compare_verbs(eng, orc)


def test_reflection_notice_precedes_its_eigenverb(engine):
    """a listener on both streams sees each boundary eigenverb right after
    the reflection notice of the same collision (reflection_model.cc:
    140-149, 216-225)"""
    sc = S.eigenverb_accuracy()
    rec = Recorder()
    q = S.build_queue(sc, u.wave_queue)
    q.add_eigenverb_listener(rec)
    q.add_reflection_listener(rec)
    q.run(sc["time_max"])
    boundary = 0
    for k, (kind, v) in enumerate(rec.events):
        if kind == "verb" and v.interface_num in (0, 1):
            pk, (t, de, az, typ) = rec.events[k - 1]
            assert pk == "refl" and (de, az, typ) == (v.de_index, v.az_index, v.interface_num)
            assert abs(t - v.travel_time) < 1e-12
            boundary += 1
    assert boundary > 50


def test_listener_removed_stops_eigenverbs(engine):
    """removing the last eigenverb listener stops the stream (and the
    volume pass) mid-run"""
    sc = S.eigenverb_accuracy()
    rec = Recorder()
    q = S.build_queue(sc, u.wave_queue)
    q.add_eigenverb_listener(rec)
    q.run(2.0)
    n = len(rec.events)
    assert n > 0
    q.remove_eigenverb_listener(rec)
    q.run(sc["time_max"])
    assert len(rec.events) == n
