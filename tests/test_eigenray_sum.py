"""eigenray_collection.sum_eigenrays (the GPU's wq3d_sum_eigenrays,
sequential sums per target) against a scalar restatement of
eigenray_collection.cc:105-191, on random eigenray sets: equal within
1e-11 relative (CUDA's and the host's pow / sin / cos / log10 / atan2 may
differ in the last place)."""
import cmath
import math

import numpy as np
import pytest

from underseamodelinglibrary_b200 import types as T
from underseamodelinglibrary_b200.eigenrays import eigenray_collection
from underseamodelinglibrary_b200.waveq3d import eigenray_model

pytestmark = pytest.mark.gpu


def scalar_sum(rays, freq, coherent=True):
    nf = len(freq)
    out = {"intensity": [], "phase": []}
    time = sde = sx = sy = tde = tx = ty = wgt = max_a = 0.0
    counts = (-1,) * 5
    for f in range(nf):
        phasor = complex(0.0, 0.0)
        for r in rays:
            a = math.pow(10.0, r.intensity[f] / -20.0)
            if coherent:
                p = math.fmod(2.0 * math.pi * freq[f] * r.travel_time + r.phase[f], 2.0 * math.pi)
                phasor += complex(a * math.cos(p), a * math.sin(p))
            else:
                phasor += a
            a *= a
            wgt += a
            time += a * r.travel_time
            sde += a * r.source_de
            sx += a * math.sin(math.radians(r.source_az))
            sy += a * math.cos(math.radians(r.source_az))
            tde += a * r.target_de
            tx += a * math.sin(math.radians(r.target_az))
            ty += a * math.cos(math.radians(r.target_az))
            if a > max_a:
                max_a = a
                counts = (r.surface, r.bottom, r.caustic, r.upper, r.lower)
        out["intensity"].append(-20.0 * math.log10(max(1e-15, abs(phasor))))
        out["phase"].append(cmath.phase(phasor))
    out["travel_time"] = time / wgt
    out["source_de"] = sde / wgt
    out["source_az"] = 90.0 - math.degrees(math.atan2(sy, sx))
    out["target_de"] = tde / wgt
    out["target_az"] = 90.0 - math.degrees(math.atan2(ty, tx))
    out["counts"] = counts
    return out


def _ray(rng, nf):
    r = eigenray_model()
    r.travel_time = float(rng.uniform(1.0, 30.0))
    r.intensity = rng.uniform(40.0, 120.0, nf)
    r.phase = rng.uniform(-math.pi, math.pi, nf)
    r.source_de, r.target_de = (float(x) for x in rng.uniform(-60.0, 60.0, 2))
    r.source_az, r.target_az = (float(x) for x in rng.uniform(0.0, 360.0, 2))
    r.surface, r.bottom, r.caustic, r.upper, r.lower = (int(x) for x in rng.integers(0, 4, 5))
    return r


def test_gpu_sum_matches_scalar_restatement(engine):
    T.compute_earth_radius(45.0)
    freq = T.seq_log(100.0, 2.0, 5)
    fv = [freq[f] for f in range(freq.size())]
    targets = T.wposition(1, 3, 45.0, -45.0, -100.0)
    rng = np.random.default_rng(5)
    for coherent in (True, False):
        coll = eigenray_collection(freq, T.wposition1(45.0, -45.0, -50.0), targets, coherent=coherent)
        sets = [[_ray(rng, len(fv)) for _ in range(n)] for n in (1, 7, 40)]
        for k, rays in enumerate(sets):
            for r in rays:
                coll.add_eigenray(0, k, r)
        coll.sum_eigenrays()
        for k, rays in enumerate(sets):
            got, ref = coll.total(0, k), scalar_sum(rays, fv, coherent)
            assert np.allclose(got.intensity, ref["intensity"], rtol=1e-11, atol=0)
            assert np.allclose(got.phase, ref["phase"], rtol=1e-9, atol=1e-12)
            for f in ("travel_time", "source_de", "source_az", "target_de", "target_az"):
                assert math.isclose(getattr(got, f), ref[f], rel_tol=1e-11, abs_tol=1e-11), f
            assert (got.surface, got.bottom, got.caustic, got.upper, got.lower) == ref["counts"]


def test_empty_target_total(engine):
    T.compute_earth_radius(45.0)
    freq = T.seq_log(100.0, 2.0, 2)
    coll = eigenray_collection(freq, T.wposition1(45.0, -45.0, -50.0), T.wposition(1, 1, 45.0, -45.0, -10.0))
    coll.sum_eigenrays()
    t = coll.total(0, 0)
    assert t.intensity == [300.0, 300.0] and t.surface == -1 and math.isnan(t.travel_time)
