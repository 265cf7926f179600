"""Reflection schedules (wq3d_queue_set_reflect_schedule): reflections on
their own stream, reflections inside the previous step's advance, and the
tuned choice between them must give the same listener calls, eigenrays and
fronts, bit for bit."""
import numpy as np
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import _abi
from underseamodelinglibrary_b200 import scenarios as S
from test_gpu_parity import _Log

pytestmark = pytest.mark.gpu

SCHEDULES = (_abi.REFLECT_SIDE, _abi.REFLECT_INLINE, _abi.REFLECT_AUTO)
FIELDS = ("rho", "theta", "phi", "sound_speed", "distance", "path_length", "attenuation", "phase",
          "surface", "bottom", "caustic", "upper", "lower", "on_edge")


def _run(sc, schedule, precision, time_max):
    q = S.build_queue(sc, u.wave_queue, precision=precision)
    q.set_reflect_schedule(schedule)
    lg = _Log()
    q.add_eigenray_listener(lg)
    q.add_reflection_listener(lg)
    q.run(time_max)
    return q, lg


@pytest.mark.parametrize("builder,precision,time_max", [
    (lambda: S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=12.0),
     _abi.FP32C, 12.0),
    (lambda: S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=12.0),
     _abi.FP64, 12.0),
    (lambda: S.gridded_munk(seed=5, num_de=121, num_az=13, time_max=12.0, dt=0.05), _abi.FP32C, 12.0),
    (lambda: S.std14(num_targets=40, time_max=80.0), _abi.FP32C, 80.0),
    (lambda: S.reverb_scale(num_de=91, num_az=13, n_targets=16, time_max=6.0), _abi.FP32, 6.0),
])
def test_reflect_schedules_are_bit_identical(engine, builder, precision, time_max):
    """sloped Rayleigh bottom (FP32C and FP64), gridded Munk profile over
    random bathymetry, the STD14 study area, and the reverberation-scale
    ocean in the FP32 form: every listener call (eigenrays and reflection
    notices, in order) and every field of the final fronts"""
    sc = builder()
    runs = [_run(sc, m, precision, time_max) for m in SCHEDULES]
    (qa, la), rest = runs[0], runs[1:]
    assert sum(1 for c in la.calls if c[0] == "reflect") > 50
    assert sum(1 for c in la.calls if c[0] == "ray") > 0
    for qb, lb in rest:
        assert qb.steps() == qa.steps()
        assert lb.calls == la.calls
        for which in ("prev", "curr", "next"):
            fa, fb = getattr(qa, which)(), getattr(qb, which)()
            for name in FIELDS:
                assert np.array_equal(getattr(fa, name), getattr(fb, name)), (which, name)


def test_tuned_plan_is_reused_and_changes_nothing(engine):
    """the first queue of a shape measures both schedules per bucket of
    steps; a second queue of that shape follows the plan it left: both runs
    give the same listener calls, and the schedule in use is a real one"""
    sc = S.gridded_munk(seed=9, num_de=151, num_az=13, time_max=20.0, dt=0.05)
    logs = []
    for _ in range(2):
        q = S.build_queue(sc, u.wave_queue)
        assert q.reflect_schedule() == _abi.REFLECT_AUTO
        lg = _Log()
        q.add_eigenray_listener(lg)
        q.add_reflection_listener(lg)
        q.run(sc["time_max"])
        assert q.reflect_schedule() in (_abi.REFLECT_SIDE, _abi.REFLECT_INLINE)
        logs.append(lg.calls)
    assert logs[0] == logs[1]
    assert sum(1 for c in logs[0] if c[0] == "reflect") > 50
    with pytest.raises(u.EngineError):
        q.set_reflect_schedule(7)
