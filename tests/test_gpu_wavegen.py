"""wavefront_generator tasks (wavegen/wavefront_generator.cc) run together
through wq3d_batch_run: each task's eigenray collection must equal a solo
wave_queue run of the same source with the same thresholds, bit for bit,
and an aborted task must neither run nor notify."""
import numpy as np
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import scenarios as S
from underseamodelinglibrary_b200 import types as T


def _solo(sc, pos):
    coll = u.eigenray_collection(sc["freq"], pos, sc["targets"])
    q = u.wave_queue(sc["ocean"], sc["freq"], pos, sc["de"], sc["az"], sc["dt"], sc["targets"])
    q.intensity_threshold(300.0)
    q.max_bottom(999)
    q.max_surface(999)
    q.add_eigenray_listener(coll)
    q.run(sc["time_max"])
    return coll


@pytest.mark.gpu
def test_generators_in_one_batch_match_solo_runs():
    sc = S.munk_flat(num_de=91, num_az=19, n_targets=4, time_max=20.0)
    positions = [T.wposition1(45.0, -45.0, -1000.0), T.wposition1(45.0, -45.0, -400.0)]
    got = {}

    def listener(source_id, rays, verbs):
        got[source_id] = rays

    gens = [u.wavefront_generator(sc["ocean"], p, sc["targets"], None, sc["freq"], sc["de"], sc["az"],
                                  sc["dt"], sc["time_max"], sourceID=k + 1, listener=listener)
            for k, p in enumerate(positions)]
    skipped = u.wavefront_generator(sc["ocean"], positions[0], sc["targets"], None, sc["freq"], sc["de"],
                                    sc["az"], sc["dt"], sc["time_max"], sourceID=99, listener=listener)
    skipped.abort()
    ms = u.run_wavefront_generators(gens + [skipped])
    assert ms > 0.0 and 99 not in got and not skipped.done()
    assert all(g.done() for g in gens)
    total = 0
    for k, p in enumerate(positions):
        solo = _solo(sc, p)
        batch = got[k + 1]
        for t1 in range(solo.size1()):
            for t2 in range(solo.size2()):
                a, b = solo.eigenrays(t1, t2), batch.eigenrays(t1, t2)
                assert len(a) == len(b)
                for x, y in zip(a, b):
                    assert x.travel_time == y.travel_time
                    assert np.array_equal(x.intensity, y.intensity)
                    assert (x.surface, x.bottom, x.caustic) == (y.surface, y.bottom, y.caustic)
                total += len(a)
                assert batch.total(t1, t2) is not None
    assert total > 0
