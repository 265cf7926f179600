"""eigenray_collection.dead_reckon on the reference's own test
(waveq3d/test/reverb_test.cc:74-150): a Munk deep sound channel, source
45N 45E at 1000 m, targets at 1200 m 1 deg east (46E) and 0.01 deg closer
(45.99E).  The 46E eigenrays dead reckoned to 45.99E must match the
propagated 45.99E eigenrays: travel time within 0.01 s, angles within
1 deg, identical surface / bottom / caustic / vertex counts."""
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import types as T
from underseamodelinglibrary_b200.eigenrays import eigenray_collection
from underseamodelinglibrary_b200.ocean import boundary_flat, ocean_model, profile_munk


@pytest.mark.gpu
def test_dead_reckon_reference_case():
    T.compute_earth_radius(45.0)
    profile = profile_munk()
    ocean = ocean_model(boundary_flat(), boundary_flat(4000.0), profile)
    freq = T.seq_log(10.0, 2.0, 1280.0)
    pos = T.wposition1(45.0, 45.0, -1000.0)
    de = T.seq_rayfan(-10.0, 10.0)
    az = T.seq_linear(89.0, 0.5, 91.0)
    targets = T.wposition(1, 2, 45.0, 46.0, -1200.0)
    targets.longitude(0, 1, 45.99)
    new_targets = T.wposition(1, 1, 45.0, 45.99, -1200.0)
    coll = eigenray_collection(freq, pos, targets)
    wave = u.wave_queue(ocean, freq, pos, de, az, 0.1, targets)
    wave.add_eigenray_listener(coll)
    while wave.time() < 90.0:
        wave.step()
    coll.sum_eigenrays()
    new_pos = T.wposition1()
    new_pos.rho = float(new_targets.rho[0, 0])
    new_pos.theta = float(new_targets.theta[0, 0])
    new_pos.phi = float(new_targets.phi[0, 0])
    reckoned = coll.dead_reckon(0, 0, pos, new_pos, ocean)
    theory = coll.eigenrays(0, 1)
    assert len(reckoned) > 0 and len(theory) > 0
    checked = 0
    for ray, th in zip(reckoned, theory):
        assert abs(ray.travel_time - th.travel_time) < 0.01
        for f in ("source_de", "source_az", "target_de", "target_az"):
            assert abs(getattr(ray, f) - getattr(th, f)) < 1.0, f
        for f in ("surface", "bottom", "caustic", "upper", "lower"):
            assert getattr(ray, f) == getattr(th, f), f
        checked += 1
    assert checked == min(len(reckoned), len(theory))
    # the move is about 790 m east, so travel times change by about half a second
    assert max(abs(r.travel_time - o.travel_time) for r, o in zip(reckoned, coll.eigenrays(0, 0))) > 0.1
