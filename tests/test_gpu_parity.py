"""GPU parity: the CUDA engine (through the C ABI) against the CPU oracle.

Bar (per the engine's accuracy contract): identical eigenray topology --
the same set of (step, target, de, az) CPA brackets and the same surface /
bottom / caustic / vertex counts -- travel time within 1 us, TL within
0.1 dB, D/E and AZ within 0.01 deg.  The FP64 form runs the reference's
arithmetic in the reference's order, so in practice differences are at the
level of the last bits of CUDA's vs the host's sin/cos/exp.
"""
import math

import numpy as np
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import _abi
from underseamodelinglibrary_b200 import scenarios as S
from oracle_binding import OracleQueue

pytestmark = pytest.mark.gpu

T_TOL = 1e-6       # s
TL_TOL = 0.1       # dB
ANG_TOL = 0.01     # deg


def key(r):
    return (r.step, r.t1, r.t2, r.de_index, r.az_index)


def compare_eigenrays(eng, orc):
    E = {key(r): r for r in eng}
    O = {key(r): r for r in orc}
    assert len(E) == len(eng) and len(O) == len(orc)
    only_e = sorted(set(E) - set(O))
    only_o = sorted(set(O) - set(E))
    assert not only_e and not only_o, ("topology differs", only_e[:5], only_o[:5])
    worst = dict(t=0.0, tl=0.0, ang=0.0)
    for k, o in O.items():
        e = E[k]
        for f in ("surface", "bottom", "caustic", "upper", "lower"):
            assert getattr(e, f) == getattr(o, f), (k, f)
        worst["t"] = max(worst["t"], abs(e.travel_time - o.travel_time))
        worst["tl"] = max(worst["tl"], float(np.max(np.abs(e.intensity - o.intensity))))
        for f in ("source_de", "source_az", "target_de", "target_az"):
            worst["ang"] = max(worst["ang"], abs(getattr(e, f) - getattr(o, f)))
        assert np.allclose(e.phase, o.phase, atol=1e-9, rtol=0)
    assert worst["t"] < T_TOL, worst
    assert worst["tl"] < TL_TOL, worst
    assert worst["ang"] < ANG_TOL, worst
    return worst


def run_pair(sc, **kw):
    q = S.build_queue(sc, u.wave_queue, **kw)
    o = S.build_queue(sc, OracleQueue)
    q.run(sc["time_max"])
    o.run(sc["time_max"])
    return q, o


def test_eigenray_basic_parity(engine):
    sc = S.eigenray_basic()
    q, o = run_pair(sc)
    eng = q.take_eigenrays()
    compare_eigenrays(eng, o.take_eigenrays())
    # and the reference's own known answers, on the engine directly
    assert len(eng) == 3
    assert abs(eng[0].travel_time - 1.484018789) < 0.002 and abs(eng[0].intensity[0] - 66.9506) < 0.1
    assert abs(eng[1].travel_time - 1.995102731) < 0.002 and abs(eng[1].intensity[0] - 69.5211) < 0.1
    assert abs(eng[2].travel_time - 3.051676949) < 0.02 and abs(eng[2].intensity[0] - 73.2126) < 4.0


def test_eigenray_concave_parity(engine):
    q, o = run_pair(S.eigenray_concave())
    eng = q.take_eigenrays()
    assert len(eng) == 4
    compare_eigenrays(eng, o.take_eigenrays())


def test_eigenray_branch_pt_parity(engine):
    q, o = run_pair(S.eigenray_branch_pt())
    eng = q.take_eigenrays()
    assert len(eng) == 42
    compare_eigenrays(eng, o.take_eigenrays())


def test_proploss_gaussian_parity(engine):
    q, o = run_pair(S.proploss_gaussian())
    compare_eigenrays(q.take_eigenrays(), o.take_eigenrays())


def test_classic_ray_parity(engine):
    sc = S.eigenray_basic()
    sc["type"] = _abi.CLASSIC_RAY
    q, o = run_pair(sc)
    compare_eigenrays(q.take_eigenrays(), o.take_eigenrays())


def compare_fronts(a, b, rel=1e-11, edges=True):
    """every field of two front views; edges=False leaves out on_edge,
    which for the next front is only computed at the start of the following
    step (find_edges in detect_reflections, wave_queue.cc:197-216), so
    after a step both hold flags left from an earlier step"""
    for name in ("rho", "theta", "phi", "sound_speed", "distance", "path_length"):
        x, y = getattr(a, name), getattr(b, name)
        scale = np.maximum(np.abs(y), 1e-300)
        err = np.max(np.abs(x - y) / np.maximum(scale, 1.0 if name == "theta" else 0.0) if name != "theta"
                     else np.abs(x - y))
        assert err < rel or np.max(np.abs(x - y)) < rel * np.max(np.abs(y)) + 1e-15, (name, err)
    for k in range(3):
        x, y = a.ndirection[k], b.ndirection[k]
        assert np.max(np.abs(x - y)) <= rel * max(np.max(np.abs(y)), 1e-12), ("ndir", k)
    for name in ("surface", "bottom", "caustic", "upper", "lower") + (("on_edge",) if edges else ()):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
    assert np.allclose(a.attenuation, b.attenuation, rtol=1e-9, atol=1e-12)
    assert np.allclose(a.phase, b.phase, rtol=0, atol=1e-9)


def test_munk_refraction_fronts(engine):
    """refraction_munk_range ray fan: every front field after 950 steps"""
    sc = S.refraction_munk_range()
    q, o = run_pair(sc)
    for w in ("past", "prev", "curr", "next"):
        compare_fronts(getattr(q, w)(), getattr(o, w)(), edges=w != "next")


def test_munk_refraction_known_answers(engine):
    """refraction_test.cc:827-980 on the engine: cycle ranges within 0.01 %"""
    sc = S.refraction_munk_range()
    q = S.build_queue(sc, u.wave_queue)
    de = sc["de"]
    loop = np.zeros(de.size())
    checks = 0
    while q.time() < 95.0:
        q.step()
        P, Cc, N = q.prev(), q.curr(), q.next()
        R = u.earth_radius()
        for d in range(de.size()):
            Hp, Hc, Hn = (F.rho[d, 0] - R + 1000.0 for F in (P, Cc, N))
            if Hc * Hn < 0.0 and Cc.ndirection[0][d, 0] * de[d] > 0.0:
                loop[d] += 1.0
                Rt = loop[d] * S.MUNK_CYCLE_RANGES[d]
                Rp, Rc, Rn = (F.rho[d, 0] * u.to_radians(F.latitude()[d, 0] - 45.0) for F in (P, Cc, N))
                h = Hn - Hp
                slope = (Rn - Rp) / h
                h *= 0.5
                Rm = Rc + slope * (-Hc) + 0.5 * ((Rn - 2.0 * Rc + Rp) / (h * h)) * Hc * Hc
                assert abs(Rm - Rt) / Rt * 100.0 < 0.01
                checks += 1
    assert checks >= 29


class _Refl(u.reflection_listener):
    def __init__(self):
        self.events = []

    def reflect(self, time, de, az, dt, grazing, speed, position, ndirection, type):
        self.events.append((time, de, az, dt, grazing, speed, position.rho, position.theta,
                            position.phi, type))


def test_reflect_flat_parity(engine):
    sc = S.reflect_flat()
    q = S.build_queue(sc, u.wave_queue)
    lst = _Refl()
    q.add_reflection_listener(lst)
    q.run(sc["time_max"])
    o = S.build_queue(sc, OracleQueue, reflections=True)
    o.run(sc["time_max"])
    ref = o.take_reflections()
    assert len(lst.events) == len(ref) >= 7
    for e, r in zip(lst.events, ref):
        assert e[9] == r.type
        assert abs(e[0] - r.time) < 1e-9
        assert abs(e[4] - r.grazing) < 1e-9
        assert abs(e[6] - r.position[0]) < 1e-6
    for k, e in enumerate(lst.events):
        assert abs(e[0] - (k + 1) * 7.450560973) < 1e-4


def test_reflect_slope_known_answers(engine):
    """reflection_test.cc:283-390 on the engine, stepping one step at a
    time: bottom bounces off the 1 deg slope turn D/E by 2 deg, surface
    bounces only flip it; the final fronts match the oracle"""
    from test_oracle_kats import _de_of
    sc = S.reflect_slope()
    q = S.build_queue(sc, u.wave_queue)
    old_de = sc["de"][0]
    bounces = 0
    while q.time() < sc["time_max"]:
        q.step()
        de = _de_of(q.curr())
        if old_de * de < 0.0:
            assert abs((2.0 if old_de < 0.0 else 0.0) - (de + old_de)) < 0.001
            bounces += 1
        old_de = de
    assert bounces >= 4
    o = S.build_queue(sc, OracleQueue)
    o.run(sc["time_max"])
    assert q.time() == o.time()
    compare_fronts(q.curr(), o.curr(), rel=1e-9)


def test_bounce_threshold_parity(engine):
    """reflection_test.cc:597-661 eigenray half: bounce limits applied, and
    the eigenrays equal the oracle's"""
    q, o = run_pair(S.bounce_threshold())
    eng = q.take_eigenrays()
    assert eng and max(r.bottom for r in eng) <= 5 and max(r.surface for r in eng) <= 3
    compare_eigenrays(eng, o.take_eigenrays())


def test_munk_flat_full_parity(engine):
    """The 181 x 37 Munk workload, 100 targets, 600 steps, against the oracle."""
    q, o = run_pair(S.munk_flat())
    eng = q.take_eigenrays()
    assert len(eng) > 100
    compare_eigenrays(eng, o.take_eigenrays())


def test_linear_slope_rayleigh_reduced_parity(engine):
    """The sloped Rayleigh workload on a reduced fan and target grid."""
    sc = S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=10.0)
    q, o = run_pair(sc)
    eng = q.take_eigenrays()
    assert len(eng) > 100
    compare_eigenrays(eng, o.take_eigenrays())
    compare_fronts(q.curr(), o.curr(), rel=1e-9)


def test_linear_slope_rayleigh_full_fan_parity(engine):
    """The sloped Rayleigh workload at full D/E width against the oracle:
    all 1801 D/E rays x all 1024 targets x 5 frequencies on six AZ columns
    (every 16th column of the 91-ray fan: 0, 64, ..., 320 deg), 12 s (240
    steps).  Both the plain FP64 form and the FP32-screened form must
    reproduce the oracle's eigenrays."""
    sc = S.linear_slope_rayleigh()
    sc["az"] = u.seq_linear(0.0, 64.0, 6)
    sc["time_max"] = 12.0
    o = S.build_queue(sc, OracleQueue)
    o.run(sc["time_max"])
    orc = o.take_eigenrays()
    assert len(orc) > 2000
    for precision in (_abi.FP64, _abi.FP32C):
        q = S.build_queue(sc, u.wave_queue, precision=precision)
        q.run(sc["time_max"])
        assert q.time() == o.time()
        compare_eigenrays(q.take_eigenrays(), orc)


def test_reflect_loss_reference_values(engine):
    """The engine's loss models at the reference's known answers: the
    Rayleigh limestone preset at normal incidence and 1 kHz, 3.672875 dB
    within 4e-4 percent (ocean/test/reflect_loss_test.cc:254-278), and the
    Eckart surface loss at 10 deg against Jones et al. figures 2-5 within 1
    percent (:312-373)."""
    u.compute_earth_radius(45.0)
    oc = u.ocean_model(u.boundary_flat(), u.boundary_flat(1000.0, u.reflect_loss_rayleigh("limestone")),
                       u.profile_linear())
    a, _ = oc.reflect_loss(1, np.array([math.pi / 2]), np.array([1000.0]))
    assert abs(float(a.ravel()[0]) - 3.672875) <= 4e-4 / 100.0 * 3.672875
    for wind, freq, expect in ((4.6, 3150.0, 1.15), (4.6, 5000.0, 2.90), (14.4, 1000.0, 11.15),
                               (14.4, 5000.0, 278.76)):
        oc = u.ocean_model(u.boundary_flat(0.0, u.reflect_loss_eckart(wind)), u.boundary_flat(1000.0),
                           u.profile_linear())
        a, _ = oc.reflect_loss(0, np.array([math.radians(10.0)]), np.array([freq]))
        assert abs(float(a.ravel()[0]) - expect) <= 0.01 * expect, (wind, freq, a)


def test_nan_profile_node_reports_numeric(engine):
    """A NaN sound-speed node given to wq3d_ocean_create reaches the rays
    that cross its depth interval; the per-step finiteness check in the
    advance kernel turns that into WQ3D_ERR_NUMERIC (no fault, no trap),
    and a healthy queue runs afterwards in the same process."""
    u.compute_earth_radius(45.0)
    R = u.earth_radius()
    depth = np.linspace(0.0, 5000.0, 10)
    nodes = 1500.0 + 0.0163 * depth
    nodes[3] = np.nan
    ax = u.seq_linear(R, -5000.0 / 9.0, 10)
    freq, de, az = u.seq_log(1000.0, 1.0, 1), u.seq_rayfan(-90.0, 90.0, 31), u.seq_linear(0.0, 30.0, 7)
    pos = u.wposition1(45.0, -45.0, -1000.0)
    bad = u.ocean_model(u.boundary_flat(), u.boundary_flat(5000.0),
                        u.profile_grid(u.data_grid([ax], nodes)))
    q = u.wave_queue(bad, freq, pos, de, az, 0.1)
    with pytest.raises(u.EngineError) as ei:
        q.run(5.0)
    assert ei.value.code == _abi.WQ3D_ERR_NUMERIC
    assert "NaN or Inf" in str(ei.value)
    nodes[3] = 1500.0 + 0.0163 * depth[3]
    good = u.ocean_model(u.boundary_flat(), u.boundary_flat(5000.0),
                         u.profile_grid(u.data_grid([ax], nodes)))
    q = u.wave_queue(good, freq, pos, de, az, 0.1)
    q.run(5.0)
    assert q.time() >= 5.0


def test_cached_queue_matches_fresh(engine):
    """Queues re-initialised from the cache of destroyed queues compute
    what fresh queues compute, bit for bit: the same inputs twice, then
    another source depth and ocean on the same shapes."""
    def run(sc):
        q = S.build_queue(sc, u.wave_queue)
        q.run(sc["time_max"])
        rays = q.take_eigenrays()
        front = q.curr()
        rt = (np.array(front.rho, copy=True), np.array(front.theta, copy=True))
        del q
        return rays.arrays(), rt

    sc1 = S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=6.0)
    sc2 = S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=6.0)
    sc2["pos"] = u.wposition1(45.0, -45.0, -120.0)
    sc2["ocean"] = u.ocean_model(u.boundary_flat(), u.boundary_flat(3000.0, u.reflect_loss_rayleigh(1.5, 1.1, 0.5)),
                                 u.profile_linear(1500.0, 0.0163))
    try:
        engine.wq3d_set_queue_cache(0)
        fresh1, f1 = run(sc1)
        fresh2, f2 = run(sc2)
        engine.wq3d_set_queue_cache(2)
        outs = [run(sc1), run(sc1), run(sc2), run(sc1)]
    finally:
        engine.wq3d_set_queue_cache(2)
    for (got, front), (want, wf) in zip(outs, [(fresh1, f1), (fresh1, f1), (fresh2, f2), (fresh1, f1)]):
        assert set(got) == set(want)
        for k in want:
            assert np.array_equal(got[k], want[k]), k
        assert np.array_equal(front[0], wf[0]) and np.array_equal(front[1], wf[1])
    assert len(fresh1["time"]) > 50 and len(fresh2["time"]) > 50


def test_listener_order_and_collection(engine):
    """add_eigenray arrives in (step, t1, t2, de, az) order, check_eigenrays
    once per step; eigenray_collection sums them"""
    sc = S.eigenray_branch_pt()
    q = S.build_queue(sc, u.wave_queue)
    coll = u.eigenray_collection(sc["freq"], sc["pos"], sc["targets"])
    seen = []
    checks = []

    class L(u.eigenray_listener):
        def add_eigenray(self, t1, t2, ray, run_id):
            seen.append((ray.step, t1, t2, ray.de_index, ray.az_index))
            coll.add_eigenray(t1, t2, ray, run_id)

        def check_eigenrays(self, time, run_id):
            checks.append(time)

    q.add_eigenray_listener(L())
    n = q.run(sc["time_max"])
    assert seen == sorted(seen)
    assert len(checks) == n
    assert all(b > a for a, b in zip(checks, checks[1:]))
    coll.sum_eigenrays()
    for t in range(14):
        assert len(coll.eigenrays(t, 0)) == 3
        assert coll.total(t, 0).intensity[0] > 0.0


def test_collection_takes_whole_lists(engine):
    """An eigenray_collection alone on a queue receives each call's
    eigenrays as one list (no per-ray callback during the run); the same
    collection behind a per-ray listener must end up holding the same
    eigenrays, per target and in the same order, and the same sums."""
    sc = S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=10.0)

    class PerRay(u.eigenray_collection):
        bulk_eigenrays = False

    colls = []
    for cls in (u.eigenray_collection, PerRay):
        q = S.build_queue(sc, u.wave_queue)
        c = cls(sc["freq"], sc["pos"], sc["targets"])
        q.add_eigenray_listener(c)
        q.run(sc["time_max"] / 2)
        q.run(sc["time_max"])
        assert len(q.take_eigenrays()) == 0
        c.sum_eigenrays()
        colls.append(c)
    a, b = colls
    assert a.num_eigenrays() == b.num_eigenrays() > 10
    for t1 in range(a.size1()):
        for t2 in range(a.size2()):
            ra, rb = a.eigenrays(t1, t2), b.eigenrays(t1, t2)
            assert [key(r) for r in ra] == [key(r) for r in rb]
            for x, y in zip(ra, rb):
                assert x.travel_time == y.travel_time
                assert np.array_equal(x.intensity, y.intensity) and np.array_equal(x.phase, y.phase)
            if ra:
                assert a.initial_time(t1, t2) == b.initial_time(t1, t2)
                assert np.array_equal(a.total(t1, t2).intensity, b.total(t1, t2).intensity)


def test_chunking_and_timing_mode_are_bit_identical(engine):
    """one step at a time, graph-replayed chunks and event-timed direct
    launches give identical eigenrays and fronts"""
    sc = S.munk_flat(num_de=91, num_az=19, n_targets=5, time_max=20.0)
    a = S.build_queue(sc, u.wave_queue)
    b = S.build_queue(sc, u.wave_queue)
    c = S.build_queue(sc, u.wave_queue)
    c.set_timing(True)
    a.run(sc["time_max"])
    while b.time() < sc["time_max"]:
        b.step()
    c.run(sc["time_max"])
    ra, rb, rc = a.take_eigenrays(), b.take_eigenrays(), c.take_eigenrays()
    assert [key(r) for r in ra] == [key(r) for r in rb] == [key(r) for r in rc]
    for x, y, z in zip(ra, rb, rc):
        assert x.travel_time == y.travel_time == z.travel_time
        assert np.array_equal(x.intensity, y.intensity) and np.array_equal(x.intensity, z.intensity)
    fa, fb = a.curr(), b.curr()
    assert np.array_equal(fa.rho, fb.rho) and np.array_equal(fa.theta, fb.theta)


def test_ocean_point_evaluations(engine):
    """profile, boundary and reflection-loss models against the oracle"""
    from oracle_binding import load_oracle
    import ctypes as C
    lib = load_oracle()
    u.compute_earth_radius(45.0)
    src = u.wposition1(45.0, -45.0, -50.0)
    for prof in (u.profile_munk(), u.profile_linear(1500.0, 0.0163), u.profile_linear(1480.0, 0.02, 500.0, 0.01),
                 u.profile_catenary(1500.0, 1500.0, 1000.0), u.profile_n2(1550.0, 1.2)):
        for flat in (False, True):
            prof.flat_earth(flat)
            bottom = u.boundary_slope(src, 200.0, -0.09, 0.01, u.reflect_loss_rayleigh(1.5, 1.1, 0.5))
            oc = u.ocean_model(u.boundary_flat(0.0, u.reflect_loss_eckart(10.0)), bottom, prof)
            R = u.earth_radius()
            rho = R - np.linspace(0.0, 5000.0, 101)
            th = np.full(101, src.theta)
            ph = np.full(101, src.phi)
            c, g = oc.sound_speed(rho, th, ph)
            od = oc.descriptor()
            co = np.empty(101)
            go = np.empty(303)
            lib.oracle_sound_speed(C.byref(od), R, 101, _abi.as_dp(rho), _abi.as_dp(th), _abi.as_dp(ph),
                                   _abi.as_dp(co), _abi.as_dp(go))
            assert np.allclose(c, co, rtol=1e-13, atol=0)
            assert np.allclose(g.ravel(), go, rtol=1e-11, atol=1e-15)
    th = src.theta + np.linspace(-0.01, 0.01, 51)
    ph = src.phi + np.linspace(-0.01, 0.01, 51)
    h, n = oc.height(1, th, ph)
    ho = np.empty(51)
    no = np.empty(153)
    z = np.zeros(51)
    lib.oracle_height(C.byref(od), 1, 51, _abi.as_dp(z), _abi.as_dp(th), _abi.as_dp(ph), _abi.as_dp(ho),
                      _abi.as_dp(no))
    assert np.array_equal(h, ho)
    for prof in (u.profile_linear(1500.0), u.profile_linear(1500.0, u.attenuation_constant(0.003))):
        oc2 = u.ocean_model(u.boundary_flat(), u.boundary_flat(3000.0), prof)
        rho = u.earth_radius() - np.linspace(0.0, 3000.0, 31)
        dist = np.linspace(0.0, 500.0, 31)
        freq = np.array([10.0, 900.0, 3000.0, 20000.0])
        a = oc2.attenuation(rho, dist, freq)
        ao = np.empty(31 * 4)
        od2 = oc2.descriptor()
        lib.oracle_attenuation(C.byref(od2), u.earth_radius(), 31, _abi.as_dp(rho), _abi.as_dp(dist), 4,
                               _abi.as_dp(freq), _abi.as_dp(ao))
        assert np.allclose(a.ravel(), ao, rtol=1e-14, atol=0)
    graz = np.linspace(0.0, math.pi / 2, 91)
    freq = np.array([100.0, 1000.0, 3000.0])
    for which in (0, 1):
        a, p = oc.reflect_loss(which, graz, freq)
        ao = np.empty(91 * 3)
        po = np.empty(91 * 3)
        lib.oracle_reflect_loss(C.byref(od), which, 91, _abi.as_dp(graz), 3, _abi.as_dp(freq),
                                _abi.as_dp(ao), _abi.as_dp(po))
        assert np.allclose(a.ravel(), ao, rtol=1e-12, atol=1e-12)
        if which == 1:
            assert np.allclose(p.ravel(), po, rtol=0, atol=1e-12)


def test_source_clamp(engine):
    """proploss_test.cc:250-280 on the engine"""
    u.compute_earth_radius(45.0)
    ocean = u.ocean_model(u.boundary_flat(), u.boundary_flat(1000.0), u.profile_linear())
    freq, de, az = u.seq_linear(1000.0, 1.0, 1), u.seq_rayfan(), u.seq_linear(-20.0, 5.0, 20.0)
    q = u.wave_queue(ocean, freq, u.wposition1(45.0, -45.0, 10.0), de, az, 0.1)
    assert abs(q.source_pos().altitude() + 0.1) < 1e-7
    q = u.wave_queue(ocean, freq, u.wposition1(45.0, -45.0, -1010.0), de, az, 0.1)
    assert abs(q.source_pos().altitude() - (-1000.0 + 0.1)) < 1e-6


def test_overflow_is_reported(engine):
    """a candidate buffer too small for one step's eigenrays reports
    WQ3D_ERR_OVERFLOW instead of dropping paths silently"""
    sc = S.eigenray_branch_pt()
    q = S.build_queue(sc, u.wave_queue, eigenray_capacity=1)
    with pytest.raises(u.EngineError) as ei:
        q.run(sc["time_max"])
    assert ei.value.code == _abi.WQ3D_ERR_OVERFLOW


def test_abort_between_chunks(engine):
    sc = S.eigenray_basic()
    q = S.build_queue(sc, u.wave_queue)
    q.abort()
    with pytest.raises(u.EngineError) as ei:
        q.step(5)
    assert ei.value.code == _abi.WQ3D_ERR_ABORTED
    q.step(5)  # the flag is consumed; propagation continues
    assert q.steps() == 5


def _identical(ra, rb):
    assert [key(r) for r in ra] == [key(r) for r in rb]
    for x, y in zip(ra, rb):
        assert x.travel_time == y.travel_time
        assert np.array_equal(x.intensity, y.intensity)
        assert (x.source_de, x.source_az, x.target_de, x.target_az) == \
            (y.source_de, y.source_az, y.target_de, y.target_az)
        assert (x.surface, x.bottom, x.caustic, x.upper, x.lower) == \
            (y.surface, y.bottom, y.caustic, y.upper, y.lower)


@pytest.mark.parametrize("builder", [
    lambda: S.munk_flat(),
    lambda: S.linear_slope_rayleigh(num_de=451, num_az=31, n_range=16, n_depth=16, time_max=20.0),
    lambda: S.eigenray_branch_pt(),
])
def test_fp32c_screen_matches_fp64(engine, builder):
    """The FP32C form screens CPA comparisons in FP32 and falls back to the
    FP64 expression inside its error bound, so every eigenray must equal
    the FP64 form's, bit for bit."""
    sc = builder()
    a = S.build_queue(sc, u.wave_queue, precision=_abi.FP64)
    b = S.build_queue(sc, u.wave_queue, precision=_abi.FP32C)
    a.run(sc["time_max"])
    b.run(sc["time_max"])
    ra, rb = a.take_eigenrays(), b.take_eigenrays()
    assert len(ra) > 0
    _identical(ra, rb)


def test_fp32c_matches_oracle_on_sloped_workload(engine):
    sc = S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=10.0)
    q = S.build_queue(sc, u.wave_queue, precision=_abi.FP32C)
    o = S.build_queue(sc, OracleQueue)
    q.run(sc["time_max"])
    o.run(sc["time_max"])
    compare_eigenrays(q.take_eigenrays(), o.take_eigenrays())


class _Log(u.eigenray_listener, u.reflection_listener):
    """records every listener call in order"""

    def __init__(self):
        self.calls = []

    def add_eigenray(self, t1, t2, ray, run_id):
        self.calls.append(("ray", t1, t2, ray.travel_time, tuple(ray.intensity), ray.source_de, ray.source_az))

    def check_eigenrays(self, time, run_id):
        self.calls.append(("check", time))

    def reflect(self, time, de, az, dt, grazing, speed, position, ndirection, type):
        self.calls.append(("reflect", time, de, az, dt, grazing, speed,
                           (position.rho, position.theta, position.phi), tuple(ndirection), type))


@pytest.mark.parametrize("precision", [_abi.FP64, _abi.FP32C])
def test_queued_chunks_match_single_chunks(engine, precision):
    """A run of many chunks queues chunk c+1 before it delivers chunk c and
    reflects each chunk's first step beside the previous chunk's last CPA
    search.  Stepping one partial chunk at a time does neither, and every
    listener call must come out the same, in the same order."""
    sc = S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=10.0)
    a = S.build_queue(sc, u.wave_queue, precision=precision)
    b = S.build_queue(sc, u.wave_queue, precision=precision)
    la, lb = _Log(), _Log()
    for q, lg in ((a, la), (b, lb)):
        q.add_eigenray_listener(lg)
        q.add_reflection_listener(lg)
    a.run(sc["time_max"])
    n = a.steps()
    assert n > 3 * 16
    while b.steps() < n:
        b.step(5)
        b.step(2)
    # the stepped queue may run a few steps past the run: compare the calls
    # of the run's steps
    checks = [i for i, c in enumerate(lb.calls) if c[0] == "check"]
    cut = checks[n - 1] + 1
    assert sum(1 for c in la.calls if c[0] == "reflect") > 100
    assert sum(1 for c in la.calls if c[0] == "ray") > 10
    assert la.calls == lb.calls[:cut]


def test_reverb_scale_reduced_parity(engine):
    """The reverberation-scale environment (gridded random ocean, Eckart
    surface loss at 10 m/s, 32 frequencies 100 Hz - 10 kHz) on a reduced
    fan and target set, FP32C engine against the oracle."""
    sc = S.reverb_scale(num_de=181, num_az=19, n_targets=32, time_max=5.0)
    q = S.build_queue(sc, u.wave_queue, precision=_abi.FP32C)
    o = S.build_queue(sc, OracleQueue)
    q.run(sc["time_max"])
    o.run(sc["time_max"])
    eng = q.take_eigenrays()
    assert len(eng) > 10 and len(eng[0].intensity) == 32
    compare_eigenrays(eng, o.take_eigenrays())


@pytest.mark.parametrize("builder,t_max", [
    (lambda: S.munk_flat(), 5e-6),
    (lambda: S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=10.0), 1e-6),
    (lambda: S.eigenray_basic(), 1e-7),
])
def test_fp32_form_error_envelope(engine, builder, t_max):
    """The FP32 propagation form (sound speed, gradient and ray derivatives
    in single precision) against the FP64 form: the same eigenrays and
    counts, TL within 0.1 dB, angles within 1e-3 deg, travel time within
    the form's measured drift (the rounding of c in FP32, about 8e-8
    relative, accumulates along the path: 3 us after the Munk workload's
    60 s, 0.7 us after the sloped workload's 10 s)."""
    from underseamodelinglibrary_b200.eigenrays import form_errors
    sc = builder()
    a = S.build_queue(sc, u.wave_queue, precision=_abi.FP64)
    b = S.build_queue(sc, u.wave_queue, precision=_abi.FP32)
    a.run(sc["time_max"])
    b.run(sc["time_max"])
    ra, rb = a.take_eigenrays(), b.take_eigenrays()
    assert len(ra) > 0
    e = form_errors(rb, ra)
    assert e["only_test"] == 0 and e["only_ref"] == 0 and e["counts_differ"] == 0, e
    assert e["travel_time_s"]["max"] <= t_max, e
    assert e["intensity_db"]["max"] <= 0.1, e
    for k in ("source_de_deg", "source_az_deg", "target_de_deg", "target_az_deg"):
        assert e[k]["max"] <= 1e-3, (k, e)


def test_fp32_form_refuses_the_adjoint(engine):
    from underseamodelinglibrary_b200 import adjoint as A
    sc = A.AdjointScenario(num_de=31, num_az=7, n_steps=20, n_targets=4, max_range=5e3)
    q = sc.queue(A.munk_nodes(), precision=_abi.FP32)
    with pytest.raises(u.EngineError) as ei:
        q.enable_adjoint(10, 40)
    assert ei.value.code == _abi.WQ3D_ERR_UNSUPPORTED
