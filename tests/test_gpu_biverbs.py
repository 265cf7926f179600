"""Bistatic eigenverbs on the GPU (wq3d_biverbs) against the oracle's
restatement of biverb_generator::run and biverb_collection::add_biverb
(biverbs/biverb_generator.cc:50-72, biverbs/biverb_collection.cc:44-172):
the same (receiver, source) pairs in the same order, integer fields and
travel times equal, durations within 1e-12 relative and powers within
1e-10 relative.  The two sides differ only in the last bits of sin, cos,
asin, atan2, exp and pow; the power's exp(kappa), with |kappa| up to about
30 for faint overlaps, magnifies the last-bit differences of the bearing
between nearby footprints."""
import math

import numpy as np
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import _abi
from underseamodelinglibrary_b200 import biverbs as B
from underseamodelinglibrary_b200 import scenarios as S
from oracle_binding import load_oracle
from test_biverbs import kat_eigenverb, kat_eigenverbs

pytestmark = pytest.mark.gpu
REL = 1e-12
REL_POWER = 1e-10
INTS = ("de_index", "az_index", "source_surface", "source_bottom", "source_caustic", "source_upper",
        "source_lower", "receiver_surface", "receiver_bottom", "receiver_caustic", "receiver_upper",
        "receiver_lower", "source", "receiver")


def both(src, rcv, freq, model, **kw):
    eng = B.compute_biverbs(src, rcv, freq, model, **kw)
    orc = B.compute_biverbs(src, rcv, freq, model, lib=load_oracle(), fn="oracle_biverbs", **kw)
    return eng, orc


def compare(eng, orc):
    (er, ep), (orr, op) = eng, orc
    assert len(er) == len(orr)
    for a, b in zip(er, orr):
        for f in INTS:
            assert getattr(a, f) == getattr(b, f), f
        assert a.travel_time == b.travel_time
        for f in ("source_de", "source_az", "receiver_de", "receiver_az"):
            assert getattr(a, f) == getattr(b, f)
        assert a.duration == pytest.approx(b.duration, rel=REL, abs=0.0)
    np.testing.assert_allclose(ep, op, rtol=REL_POWER, atol=0.0)


def test_reference_case(engine):
    """biverbs_test.cc:90-158: 80 eigenverbs, monostatic, -30 dB bottom"""
    verbs, freq = kat_eigenverbs()
    eng, orc = both(verbs, verbs, freq, u.scattering_constant(-30.0))
    assert len(eng[0]) == 109
    compare(eng, orc)


def bistatic_fans(de_step=2.5, az_step=5.0):
    """analytic bottom footprints of a source at (0, 0) and a receiver
    1.1 km away, at 2 frequencies"""
    u.set_earth_radius(6371000.0)
    freq = u.seq_log(1000.0, 2.0, 2)
    out = []
    for sensor in (u.wposition1(0.0, 0.0, 0.0), u.wposition1(0.007, 0.007, 0.0)):
        verbs = []
        for az in np.arange(0.0, 360.0, az_step):
            for de in np.arange(-85.0, -4.0, de_step):
                verbs.append(kat_eigenverb(sensor, 500.0, float(de), float(az), freq))
        out.append(verbs)
    return out[0], out[1], freq


@pytest.mark.parametrize("model", [u.scattering_constant(-25.0), u.scattering_lambert(-27.0),
                                   u.scattering_chapman(7.5)], ids=["constant", "lambert", "chapman"])
def test_bistatic_fans(engine, model):
    """2,376 source x 2,376 receiver footprints at 2 frequencies: about
    58,000 overlaps; all three scattering models"""
    src, rcv, freq = bistatic_fans()
    eng, orc = both(src, rcv, freq, model)
    assert len(eng[0]) > 50000
    compare(eng, orc)


def test_power_threshold_and_search_scale(engine):
    """a power threshold drops pairs, and a larger search area finds more"""
    src, rcv, freq = bistatic_fans(de_step=5.0, az_step=10.0)
    base = both(src, rcv, freq, u.scattering_constant(-30.0))
    compare(*base)
    threshold = float(np.median(base[1][1].max(axis=1)))
    hi = both(src, rcv, freq, u.scattering_constant(-30.0), power_threshold=threshold)
    compare(*hi)
    wide = both(src, rcv, freq, u.scattering_constant(-30.0), search_scale=3.0)
    compare(*wide)
    assert 0 < len(hi[0][0]) < len(base[0][0]) < len(wide[0][0])


def test_empty_and_overflow(engine):
    """no eigenverbs on one side gives no biverbs; a buffer that is too
    small is filled and reported (WQ3D_ERR_OVERFLOW) with the full count"""
    import ctypes as C
    verbs, freq = kat_eigenverbs()
    assert len(B.compute_biverbs([], verbs, freq, u.scattering_constant(-30.0))[0]) == 0
    assert len(B.compute_biverbs(verbs, [], freq, u.scattering_constant(-30.0))[0]) == 0
    lib = _abi.load_engine()
    s, sp = B.pack_eigenverbs(verbs, 1)
    f = np.array([3000.0])
    out = (_abi.wq3d_biverb * 50)()
    power = np.zeros((50, 1))
    count = C.c_size_t()
    desc = u.scattering_constant(-30.0).desc()
    dp = C.POINTER(C.c_double)
    rc = lib.wq3d_biverbs(s, sp.ctypes.data_as(dp), 80, s, sp.ctypes.data_as(dp), 80,
                          f.ctypes.data_as(dp), 1, C.byref(desc), 6371000.0, 1.5, 1e-20, out,
                          power.ctypes.data_as(dp), 50, C.byref(count))
    assert rc == _abi.WQ3D_ERR_OVERFLOW and count.value == 109
    full, full_power = B.compute_biverbs(verbs, verbs, freq, u.scattering_constant(-30.0))
    for k in range(50):
        assert (out[k].source, out[k].receiver) == (full[k].source, full[k].receiver)
        assert power[k, 0] == full_power[k, 0]
    bad = u.scattering_constant(0.0).desc()
    bad.kind = 7
    assert lib.wq3d_biverbs(s, sp.ctypes.data_as(dp), 80, s, sp.ctypes.data_as(dp), 80, f.ctypes.data_as(dp),
                            1, C.byref(bad), 6371000.0, 1.5, 1e-20, out, power.ctypes.data_as(dp), 50,
                            C.byref(count)) == _abi.WQ3D_ERR_INVALID


def test_generator_on_propagated_eigenverbs(engine):
    """biverb_generator over the eigenverbs of a real propagation (sloped
    Rayleigh bottom, two volume layers): Lambert bottom, Chapman surface,
    constant volume scattering; each interface's collection, ordered by
    travel time, equals the oracle's pairs sorted the same way"""
    sc = S.linear_slope_rayleigh(num_de=45, num_az=7, n_range=4, n_depth=4, time_max=6.0)
    ocean = sc["ocean"]
    ocean.add_volume(u.volume_flat(40.0, 5.0, -50.0))
    ocean.bottom().scattering(u.scattering_lambert(-27.0))
    ocean.surface().scattering(u.scattering_chapman(6.0))
    q = S.build_queue(sc, u.wave_queue)
    verbs = u.eigenverb_collection(ocean.num_volume())
    q.add_eigenverb_listener(verbs)
    q.eigenverb_threshold(-80.0)
    q.run(sc["time_max"])
    done = []
    gen = B.biverb_generator(ocean, verbs, verbs, sc["freq"], listener=done.append)
    gen.run()
    assert gen.done() and done == [gen.collection()]
    coll = gen.collection()
    assert coll.num_interfaces() == 4
    total = 0
    for interface in range(4):
        vs = verbs.eigenverbs(interface)
        got = coll.biverbs(interface)
        if not vs:
            assert got == []
            continue
        recs, power = B.compute_biverbs(vs, vs, sc["freq"], ocean.scattering_model(interface),
                                        lib=load_oracle(), fn="oracle_biverbs")
        order = sorted(range(len(recs)), key=lambda k: recs[k].travel_time)
        assert len(got) == len(recs)
        for b, k in zip(got, order):
            r = recs[k]
            assert (b.source_index, b.receiver_index) == (r.source, r.receiver)
            assert b.travel_time == r.travel_time
            assert b.duration == pytest.approx(r.duration, rel=REL, abs=0.0)
            np.testing.assert_allclose(b.power, power[k], rtol=REL_POWER, atol=0.0)
        total += len(got)
    assert total > 1000


def test_high_latitude_across_the_date_line(engine):
    """footprints of a sensor at 60N, 179.99E whose fan spans longitude
    180 (the centres run from 179.92 to 180.06 deg, not wrapped): engine
    and oracle agree pair for pair (search area 3 footprint lengths and
    widths, so neighbours overlap).  Longitudes are compared as stored, so
    a receiver fan built from the same place written as -180.01 deg finds
    nothing on either side"""
    from underseamodelinglibrary_b200 import scenarios as S
    from underseamodelinglibrary_b200.eigenverbs import eigenverb_model
    u.set_earth_radius(6371000.0)
    de = np.arange(-80.0, -10.0, 2.0)
    az = np.arange(0.0, 360.0, 6.0)
    freq = np.array([2000.0])
    model = u.scattering_lambert(-27.0)

    def verbs(lat, lng):
        recs, power = S.analytic_footprints(lat, lng, 800.0, de, az, 1)
        a = np.ctypeslib.as_array(recs)
        out = []
        for k in range(len(power)):
            rec = a[k]
            v = eigenverb_model()
            v.travel_time, v.length, v.width = rec["travel_time"], rec["length"], rec["width"]
            v.position = tuple(rec["position"])
            v.direction, v.grazing, v.sound_speed = rec["direction"], rec["grazing"], rec["sound_speed"]
            v.source_de, v.source_az = rec["source_de"], rec["source_az"]
            v.de_index, v.az_index = int(rec["de"]), int(rec["az"])
            v.surface = v.bottom = v.caustic = v.upper = v.lower = 0
            v.power = power[k]
            out.append(v)
        return out

    fan = verbs(60.0, 179.99)
    lng = np.degrees(np.array([v.position[2] for v in fan]))
    assert lng.min() < 180.0 < lng.max()
    eng, orc = both(fan, fan, freq, model, search_scale=3.0)
    assert len(eng[0]) > 3 * len(fan)
    compare(eng, orc)
    other = verbs(60.0, -180.01)
    eng, orc = both(fan, other, freq, model, search_scale=3.0)
    assert len(eng[0]) == len(orc[0]) == 0
