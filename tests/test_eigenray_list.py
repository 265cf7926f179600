"""take_eigenrays returns an eigenray_list: the engine's records copied
once into numpy arrays, each eigenray_model made when it is read.  Its
models must carry the same values, with the same Python types, as models
made field by field from the C records."""
import numpy as np

from underseamodelinglibrary_b200 import _abi
from underseamodelinglibrary_b200.waveq3d import eigenray_list, eigenray_model

FIELDS = ["travel_time", "source_de", "source_az", "target_de", "target_az", "surface", "bottom",
          "caustic", "upper", "lower", "step", "de_index", "az_index", "t1", "t2"]


def test_eigenray_list_matches_record_conversion():
    n, nf = 7, 5
    rng = np.random.default_rng(3)
    recs = (_abi.wq3d_eigenray * n)()
    for i in range(n):
        r = recs[i]
        r.time, r.source_de, r.source_az, r.target_de, r.target_az = rng.standard_normal(5)
        (r.surface, r.bottom, r.caustic, r.upper, r.lower, r.t1, r.t2, r.de, r.az) = \
            [int(x) for x in rng.integers(0, 50, 9)]
        r.step = int(rng.integers(0, 10 ** 9))
    inten, phase, sens = rng.standard_normal(n * nf), rng.standard_normal(n * nf), rng.standard_normal(n * 3)
    rec = np.ctypeslib.as_array(recs)[:n].copy()
    rays = eigenray_list(rec, inten.reshape(n, nf), phase.reshape(n, nf), sens.reshape(n, 3), "freq")
    assert len(rays) == n
    for i, a in enumerate(rays):
        b = eigenray_model.from_record(recs[i], inten[i * nf:(i + 1) * nf], phase[i * nf:(i + 1) * nf], "freq")
        for f in FIELDS:
            assert getattr(a, f) == getattr(b, f) and type(getattr(a, f)) is type(getattr(b, f)), f
        assert np.array_equal(a.intensity, b.intensity) and np.array_equal(a.phase, b.phase)
        assert np.array_equal(a.d_intensity_d_bottom, sens[3 * i:3 * i + 3])
        assert a.frequencies == "freq"
    assert rays[-1].step == recs[n - 1].step and [r.t1 for r in rays[2:5]] == [recs[k].t1 for k in range(2, 5)]
    cols = rays.arrays()
    assert np.array_equal(cols["time"], [recs[k].time for k in range(n)])
    assert cols["intensity"].shape == (n, nf) and cols["d_intensity_d_bottom"].shape == (n, 3)


def test_empty_eigenray_list():
    rec = np.ctypeslib.as_array((_abi.wq3d_eigenray * 1)())[:0].copy()
    rays = eigenray_list(rec, np.empty((0, 2)), np.empty((0, 2)), None, "f")
    assert len(rays) == 0 and list(rays) == []
