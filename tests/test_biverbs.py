"""Bistatic eigenverbs on the CPU: the oracle pinned to the reference's
own biverb test (biverbs/test/biverbs_test.cc:90-158), and the host-side
collection order.  The GPU path is checked against the oracle in
test_gpu_biverbs.py."""
import math

import numpy as np
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import biverbs as B
from underseamodelinglibrary_b200.eigenverbs import eigenverb_model
from oracle_binding import load_oracle

DE_SPACING = 10.0
AZ_SPACING = 10.0
DEPTH = 1000.0


def kat_eigenverb(source_pos, depth, de, az, freq):
    """create_eigenverb (biverbs_test.cc:41-77): an analytic bottom
    footprint for a ray at (de, az) degrees in 1500 m/s water"""
    v = eigenverb_model()
    de_rad, az_rad = math.radians(de), math.radians(az)
    grazing = abs(de_rad)
    slant_range = depth / math.sin(grazing)
    horz_range = depth / math.tan(grazing)
    v.sound_speed = 1500.0
    v.travel_time = slant_range / v.sound_speed
    v.frequencies = freq
    v.length = 0.5 * slant_range * u.to_radians(DE_SPACING) / math.sin(grazing)
    v.width = 0.5 * slant_range * u.to_radians(AZ_SPACING) * math.cos(grazing)
    pos = u.wposition1(source_pos, horz_range, az_rad)
    pos.altitude(-depth)
    v.position = (pos.rho, pos.theta, pos.phi)
    v.direction = az_rad
    v.grazing = grazing
    v.de_index = int((90.0 + de) / DE_SPACING - 1.0)
    v.az_index = int(az / AZ_SPACING)
    v.source_de = de_rad
    v.source_az = az_rad
    v.surface = v.bottom = v.caustic = v.upper = v.lower = 0
    power = v.length * v.width / (slant_range * slant_range)
    v.power = np.full(freq.size(), power)
    return v


def kat_eigenverbs():
    """the 80 bottom eigenverbs of biverbs_test.cc:114-124 around a sensor
    at (0, 0, 0), 3 kHz"""
    u.set_earth_radius(6371000.0)
    freq = u.seq_linear(3000.0, 1.0, 1)
    sensor = u.wposition1(0.0, 0.0, 0.0)
    verbs = []
    az = 0.0
    while az <= 90.0:
        de = -90.0 + DE_SPACING
        while de < 0.0:
            verbs.append(kat_eigenverb(sensor, DEPTH, de, az, freq))
            de += DE_SPACING
        az += AZ_SPACING
    return verbs, freq


def test_oracle_biverbs_reference_case():
    """The reference's biverb case (biverbs_test.cc:90-158): 80 eigenverbs
    overlapped with themselves (a monostatic pair) under the -30 dB
    constant bottom scattering of ocean_utils::make_iso.

    The reference counts 182 biverbs there.  Its search polygon is a
    four-corner ring that is never closed, held in a closed-ring Boost
    polygon, so Boost's winding test walks only the edges A-B, B-C and C-D.
    The region that test accepts is not bounded, and which points of it
    come back then depends on the R*-tree's node boxes.  Here the search
    area is the whole quadrilateral A-B-C-D, as find_eigenverbs describes
    it: 109 biverbs, exactly the pairs that the host find_eigenverbs
    selects whose power reaches the threshold."""
    verbs, freq = kat_eigenverbs()
    assert len(verbs) == 80
    recs, power = B.compute_biverbs(verbs, verbs, freq, u.scattering_constant(-30.0),
                                    lib=load_oracle(), fn="oracle_biverbs")
    assert len(recs) == 109
    coll = u.eigenverb_collection(0)
    for v in verbs:
        coll.add_eigenverb(v, 0)
    index = {id(v): k for k, v in enumerate(verbs)}
    want = [(index[id(s)], ri) for ri, r in enumerate(verbs) for s in coll.find_eigenverbs(r, 0)]
    got = [(r.source, r.receiver) for r in recs]
    assert set(got) <= set(want) and len(want) - len(got) <= 1
    # every eigenverb finds itself: its biverb has twice its travel time
    selfs = [r for r in recs if r.source == r.receiver]
    assert len(selfs) == 80
    for r in selfs:
        assert r.travel_time == 2.0 * verbs[r.source].travel_time
    assert np.all(power >= B.biverb_collection.power_threshold)
    assert np.all(np.array([r.duration for r in recs]) > 0.0)


def test_oracle_biverb_overlap_of_identical_footprints():
    """biverb_collection.cc:115-163 for a footprint overlapped with itself
    (range 0, alpha 0): kappa = 0, so the power is 0.125 P^2 S / sqrt(det)
    with det = 0.5 (4 L^2 W^2 + (L^2 + W^2)^2 - (L^2 - W^2)^2), and the
    duration follows equation (41) with cos(2 alpha) = 1"""
    verbs, freq = kat_eigenverbs()
    v = verbs[12]
    recs, power = B.compute_biverbs([v], [v], freq, u.scattering_constant(-30.0),
                                    lib=load_oracle(), fn="oracle_biverbs")
    assert len(recs) == 1
    L2, W2 = v.length ** 2, v.width ** 2
    det = 0.5 * (2.0 * (2.0 * L2 * W2) + (L2 + W2) ** 2 - (L2 - W2) ** 2)
    want = 0.125 * v.power[0] ** 2 * 1e-3 / math.sqrt(det)
    assert power[0, 0] == pytest.approx(want, rel=1e-12)
    sigma = 0.5 * (2.0 / W2 + 2.0 / W2) / (det / (L2 * W2 * L2 * W2))
    assert recs[0].duration == pytest.approx(0.5 * math.cos(v.grazing) / 1500.0 * math.sqrt(sigma), rel=1e-12)


@pytest.mark.parametrize("model", [u.scattering_lambert(-27.0), u.scattering_chapman(8.0)])
def test_oracle_scattering_models(model):
    """scattering_lambert.h and scattering_chapman.h scale the constant
    model's biverbs by their own strength, pair by pair"""
    verbs, freq = kat_eigenverbs()
    lib = load_oracle()
    r0, p0 = B.compute_biverbs(verbs, verbs, freq, u.scattering_constant(0.0), lib=lib, fn="oracle_biverbs")
    r1, p1 = B.compute_biverbs(verbs, verbs, freq, model, lib=lib, fn="oracle_biverbs")
    assert len(r1) <= len(r0)
    keyed = {(r.source, r.receiver): p0[k, 0] for k, r in enumerate(r0)}
    for k, r in enumerate(r1):
        a, b = verbs[r.source].grazing, verbs[r.receiver].grazing
        if model.kind == u.scattering_lambert(0).kind:
            s = abs(10 ** (-2.7) * math.sin(a) * math.sin(b))
        else:
            g = 0.5 * (a + b) * 180.0 / math.pi
            beta = 158.0 * (8.0 * 1.94384449 * 3000.0 ** (1.0 / 3.0)) ** -0.58
            s = 10 ** ((2.6 - 42.4 * math.log10(beta) + 3.3 * beta * math.log10(g / 30.0 + 1e-6)) / 10.0)
        assert p1[k, 0] == pytest.approx(keyed[(r.source, r.receiver)] * s, rel=1e-12)


def test_collection_orders_by_travel_time():
    """multimap insertion (biverb_collection.cc:167-170): sorted by travel
    time, equal times in the order added, across several additions"""
    c = B.biverb_collection(1)
    assert c.num_interfaces() == 4

    class R:
        def __init__(self, t, tag):
            self.travel_time, self.tag = t, tag

    c.add_biverbs([R(2.0, "a"), R(1.0, "b"), R(2.0, "c")], 0)
    c.add_biverbs([R(2.0, "d"), R(0.5, "e")], 0)
    assert [b.tag for b in c.biverbs(0)] == ["e", "b", "a", "c", "d"]
    assert c.size(0) == 5 and c.size(1) == 0


def test_scattering_model_per_interface():
    """ocean_model::scattering picks bottom, surface, then the volume layer
    of each side (ocean_model.h:88-112); boundaries default to -300 dB"""
    bot = u.scattering_lambert(-27.0)
    ocean = u.ocean_model(u.boundary_flat(), u.boundary_flat(1000.0, None, bot), u.profile_linear())
    ocean.add_volume(u.volume_flat(300.0, 10.0, -40.0))
    ocean.add_volume(u.volume_flat(600.0, 10.0, u.scattering_chapman(5.0)))
    assert ocean.scattering_model(0) is bot
    assert ocean.scattering_model(1).p == -300.0
    assert ocean.scattering_model(2).p == -40.0 and ocean.scattering_model(3).p == -40.0
    assert ocean.scattering_model(4).kind == u.scattering_chapman(1).kind
    assert ocean.scattering_model(5).p == 5.0


def test_abi_argument_checks_without_gpu():
    """wq3d_biverbs checks its arguments before it touches the device:
    bad ones return WQ3D_ERR_INVALID with a message, and an empty side
    returns no biverbs"""
    import ctypes as C
    from underseamodelinglibrary_b200 import _abi
    lib = _abi.load_engine()
    verbs, freq = kat_eigenverbs()
    s, sp = B.pack_eigenverbs(verbs, 1)
    f = np.array([3000.0])
    dp = C.POINTER(C.c_double)
    count = C.c_size_t(99)
    desc = u.scattering_constant(-30.0).desc()

    def call(ns=80, nr=80, fp=f.ctypes.data_as(dp), nf=1, sc=C.byref(desc), R=6371000.0, scale=1.5,
             cnt=C.byref(count)):
        return lib.wq3d_biverbs(s, sp.ctypes.data_as(dp), ns, s, sp.ctypes.data_as(dp), nr, fp, nf, sc, R,
                                scale, 1e-20, None, None, 0, cnt)

    assert call(cnt=None) == _abi.WQ3D_ERR_INVALID
    assert call(sc=None) == _abi.WQ3D_ERR_INVALID
    assert call(nf=0) == _abi.WQ3D_ERR_INVALID
    assert call(R=0.0) == _abi.WQ3D_ERR_INVALID
    assert call(scale=-1.0) == _abi.WQ3D_ERR_INVALID
    bad = u.scattering_constant(0.0).desc()
    bad.kind = 3
    assert call(sc=C.byref(bad)) == _abi.WQ3D_ERR_INVALID
    assert b"scattering" in lib.wq3d_last_error_string()
    assert call(ns=0) == _abi.WQ3D_OK and count.value == 0
    count.value = 99
    assert call(nr=0) == _abi.WQ3D_OK and count.value == 0



def test_record_collection_and_lazy_list():
    """add_records keeps the multimap order across calls (stable by travel
    time, earlier calls first among equals); biverb_list reads a
    biverb_model per element and hands out the arrays"""
    from underseamodelinglibrary_b200 import _abi
    freq = u.seq_linear(3000.0, 1.0, 1)

    def recs(times, tags):
        a = np.zeros(len(times), dtype=np.ctypeslib.as_array((_abi.wq3d_biverb * 1)()).dtype).view(np.recarray)
        a.travel_time = times
        a.source = tags
        return a, np.array(times, dtype=np.float64)[:, None] * 10.0

    c = B.biverb_collection(0)
    c.add_records(*recs([2.0, 1.0, 2.0], [0, 1, 2]), freq, 0)
    c.add_records(*recs([2.0, 0.5], [3, 4]), freq, 0)
    lst = c.biverbs(0)
    assert isinstance(lst, B.biverb_list) and len(lst) == c.size(0) == 5
    assert [b.source_index for b in lst] == [4, 1, 0, 2, 3]
    assert lst[-1].power[0] == 20.0 and lst[0].frequencies is freq
    rec, power = lst.arrays()
    assert list(rec.source) == [4, 1, 0, 2, 3] and power.shape == (5, 1)
    with pytest.raises(IndexError):
        lst[5]
    assert c.biverbs(1) == [] and c.size(1) == 0


def test_generator_aborted_before_run_does_nothing():
    """thread_task::abort before execution (biverb_generator.cc:40-45): no
    device work, no collection, no notification"""
    verbs, freq = kat_eigenverbs()
    coll = u.eigenverb_collection(0)
    for v in verbs:
        coll.add_eigenverb(v, 0)
    heard = []
    ocean = u.ocean_model(u.boundary_flat(), u.boundary_flat(1000.0), u.profile_linear())
    gen = B.biverb_generator(ocean, coll, coll, freq, listener=heard.append)
    gen.abort()
    gen.run()
    assert not gen.done() and gen.collection() is None and heard == []
