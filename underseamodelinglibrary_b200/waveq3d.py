"""Drop-in mirror of USML's WaveQ3D wave_queue API over the CUDA engine.

``wave_queue(ocean, freq, pos, de, az, time_step, target_pos, type)`` keeps
the reference constructor (waveq3d/wave_queue.h:122-126), ``step()``,
``time()``, ``source_pos()``, the front accessors ``curr()/next()/prev()/
past()``, the wave_thresholds setters and the listener registration of
eigenray_notifier / reflection_notifier.  All propagation runs in
libwq3d.so on the GPU; this module only marshals arguments and dispatches
listener callbacks in the reference's order.
"""
import ctypes as C
from collections.abc import Sequence

import numpy as np

from . import _abi
from .eigenverbs import eigenverb_model
from .types import earth_radius, wposition1


class eigenray_model:
    """eigenrays/eigenray_model.h:24-102 plus the CPA bracket (step, de, az)."""

    __slots__ = ("travel_time", "intensity", "phase", "source_de", "source_az",
                 "target_de", "target_az", "surface", "bottom", "caustic", "upper",
                 "lower", "frequencies", "step", "de_index", "az_index", "t1", "t2",
                 "d_intensity_d_bottom")

    @classmethod
    def from_record(cls, rec, intensity, phase, freq):
        r = cls()
        r.travel_time = rec.time
        r.intensity = np.array(intensity, dtype=np.float64)
        r.phase = np.array(phase, dtype=np.float64)
        r.source_de = rec.source_de
        r.source_az = rec.source_az
        r.target_de = rec.target_de
        r.target_az = rec.target_az
        r.surface = rec.surface
        r.bottom = rec.bottom
        r.caustic = rec.caustic
        r.upper = rec.upper
        r.lower = rec.lower
        r.frequencies = freq
        r.step = rec.step
        r.de_index = rec.de
        r.az_index = rec.az
        r.t1 = rec.t1
        r.t2 = rec.t2
        r.d_intensity_d_bottom = None
        return r


class eigenray_list(Sequence):
    """The eigenrays of one ``take_eigenrays`` call.  The records are held
    as numpy arrays (one copy out of the engine); an ``eigenray_model`` is
    made when an element is read, so a caller that only wants the arrays
    (``arrays()``) or the count pays no per-ray Python cost."""

    __slots__ = ("_rec", "_inten", "_phase", "_sens", "_freq")

    def __init__(self, rec, inten, phase, sens, freq):
        self._rec = rec
        self._inten = inten
        self._phase = phase
        self._sens = sens
        self._freq = freq

    def __len__(self):
        return len(self._rec)

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[j] for j in range(*i.indices(len(self)))]
        n = len(self._rec)
        i = int(i)
        if i < 0:
            i += n
        if not 0 <= i < n:
            raise IndexError("eigenray index out of range")
        (t, sde, saz, tde, taz, sf, bt, cs, up, lo, t1, t2, de, az, _pad, step) = self._rec[i].item()
        r = eigenray_model()
        r.travel_time = t
        r.intensity = self._inten[i].copy()
        r.phase = self._phase[i].copy()
        r.source_de, r.source_az, r.target_de, r.target_az = sde, saz, tde, taz
        r.surface, r.bottom, r.caustic, r.upper, r.lower = sf, bt, cs, up, lo
        r.frequencies = self._freq
        r.step, r.de_index, r.az_index, r.t1, r.t2 = step, de, az, t1, t2
        r.d_intensity_d_bottom = None if self._sens is None else self._sens[i].copy()
        return r

    def __iter__(self):
        for i in range(len(self._rec)):
            yield self[i]

    @property
    def records(self):
        """the engine's wq3d_eigenray records (numpy structured array)"""
        return self._rec

    def arrays(self):
        """All eigenrays as columns: the record fields (travel time as
        "time", CPA bracket as "step", "de", "az"), intensity and phase
        [n, frequencies] and, with sensitivities on, d_intensity_d_bottom
        [n, 3]."""
        out = {name: self._rec[name] for name in self._rec.dtype.names if name != "pad"}
        out["intensity"] = self._inten
        out["phase"] = self._phase
        if self._sens is not None:
            out["d_intensity_d_bottom"] = self._sens
        return out


class eigenray_listener:
    """eigenrays/eigenray_listener.h:41-53."""

    def add_eigenray(self, t1, t2, ray, run_id):
        raise NotImplementedError

    def check_eigenrays(self, time, run_id):
        pass


class reflection_listener:
    """waveq3d/reflection_listener.h:46-49."""

    def reflect(self, time, de, az, dt, grazing, speed, position, ndirection, type):
        raise NotImplementedError


class wave_front_view:
    """Host copy of one wavefront (wave_front.h:152-258)."""

    def __init__(self, getter, q, which, num_de, num_az, nf, check=None):
        n = num_de * num_az
        shape = (num_de, num_az)
        self.num_de, self.num_az = num_de, num_az
        f = {k: np.empty(n) for k in ("rho", "theta", "phi", "c", "dist", "plen")}
        vec = {k: [np.empty(n) for _ in range(3)] for k in ("pg", "nd", "ng", "sg")}
        att = np.empty(n * nf)
        ph = np.empty(n * nf)
        ints = {k: np.empty(n, dtype=np.int32) for k in ("surface", "bottom", "caustic", "upper", "lower")}
        edge = np.empty(n, dtype=np.uint8)
        v = _abi.wq3d_front_view()
        v.rho, v.theta, v.phi = (_abi.as_dp(f["rho"]), _abi.as_dp(f["theta"]), _abi.as_dp(f["phi"]))
        for k in range(3):
            v.pos_grad[k] = _abi.as_dp(vec["pg"][k])
            v.ndir[k] = _abi.as_dp(vec["nd"][k])
            v.ndir_grad[k] = _abi.as_dp(vec["ng"][k])
            v.sound_grad[k] = _abi.as_dp(vec["sg"][k])
        v.sound_speed = _abi.as_dp(f["c"])
        v.distance = _abi.as_dp(f["dist"])
        v.path_length = _abi.as_dp(f["plen"])
        v.attenuation = _abi.as_dp(att)
        v.phase = _abi.as_dp(ph)
        for k, a in ints.items():
            setattr(v, k, a.ctypes.data_as(C.POINTER(C.c_int32)))
        v.on_edge = edge.ctypes.data_as(C.POINTER(C.c_uint8))
        rc = getter(q, which, C.byref(v))
        if check is not None:
            check(rc)
        self.rho = f["rho"].reshape(shape)
        self.theta = f["theta"].reshape(shape)
        self.phi = f["phi"].reshape(shape)
        self.pos_gradient = [a.reshape(shape) for a in vec["pg"]]
        self.ndirection = [a.reshape(shape) for a in vec["nd"]]
        self.ndir_gradient = [a.reshape(shape) for a in vec["ng"]]
        self.sound_gradient = [a.reshape(shape) for a in vec["sg"]]
        self.sound_speed = f["c"].reshape(shape)
        self.distance = f["dist"].reshape(shape)
        self.path_length = f["plen"].reshape(shape)
        self.attenuation = att.reshape(num_de, num_az, nf)
        self.phase = ph.reshape(num_de, num_az, nf)
        for k, a in ints.items():
            setattr(self, k, a.reshape(shape))
        self.on_edge = edge.reshape(shape).astype(bool)

    def altitude(self):
        return self.rho - earth_radius()

    def latitude(self):
        return 90.0 - self.theta * (180.0 / np.pi)


def make_queue_desc(freq, pos, de, az, time_step, target_pos=None, type=_abi.HYBRID_GAUSSIAN,
                    precision=_abi.FP64, device=0, eigenray_capacity=0, run_id=0):
    """Fills a wq3d_queue_desc from reference-style arguments.  Returns the
    descriptor and the numpy arrays it points into (keep them alive)."""
    d = _abi.wq3d_queue_desc()
    fr = np.ascontiguousarray(freq.data, dtype=np.float64)
    dv = np.ascontiguousarray(de.data, dtype=np.float64)
    di = np.ascontiguousarray(de.increments, dtype=np.float64)
    av = np.ascontiguousarray(az.data, dtype=np.float64)
    ai = np.ascontiguousarray(az.increments, dtype=np.float64)
    keep = [fr, dv, di, av, ai]
    d.freq, d.num_freq = _abi.as_dp(fr), fr.size
    d.source[0], d.source[1], d.source[2] = pos.rho, pos.theta, pos.phi
    d.de, d.de_inc, d.num_de = _abi.as_dp(dv), _abi.as_dp(di), dv.size
    d.az, d.az_inc, d.num_az = _abi.as_dp(av), _abi.as_dp(ai), av.size
    d.time_step = float(time_step)
    if target_pos is not None:
        tg = target_pos.packed()
        keep.append(tg)
        d.targets = _abi.as_dp(tg)
        d.num_targets1, d.num_targets2 = target_pos.size1(), target_pos.size2()
    d.spreading = int(type)
    d.precision = int(precision)
    d.earth_radius = earth_radius()
    d.eigenray_capacity = int(eigenray_capacity)
    d.device = int(device)
    d.run_id = int(run_id)
    return d, keep


class wave_queue:
    CLASSIC_RAY = _abi.CLASSIC_RAY
    HYBRID_GAUSSIAN = _abi.HYBRID_GAUSSIAN

    def __init__(self, ocean, freq, pos, de, az, time_step, target_pos=None,
                 type=_abi.HYBRID_GAUSSIAN, precision=_abi.FP64, device=0,
                 eigenray_capacity=0, run_id=0):
        self._lib = _abi.load_engine()
        self._ocean = ocean
        self._freq = freq
        self._de = de
        self._az = az
        self._targets = target_pos
        d, self._keep = make_queue_desc(freq, pos, de, az, time_step, target_pos, type,
                                        precision, device, eigenray_capacity, run_id)
        h = C.c_void_p()
        _abi.check(self._lib, self._lib.wq3d_queue_create(ocean.handle(), C.byref(d), C.byref(h)))
        self._q = h
        self._time_step = float(time_step)
        self._eig_listeners = []
        self._refl_listeners = []
        self._verb_listeners = []
        self._run_id = int(run_id)
        self._thresh = _abi.wq3d_thresholds(300.0, 300.0, 999, 999, 999, 999, 999)
        self._cb = None

    def __del__(self):
        if getattr(self, "_q", None) is not None:
            try:
                self._lib.wq3d_queue_destroy(self._q)
            except Exception:
                pass
            self._q = None

    # ---------------- reference accessors ----------------
    def time(self):
        t = C.c_double()
        _abi.check(self._lib, self._lib.wq3d_queue_time(self._q, C.byref(t)))
        return t.value

    def time_step(self):
        return self._time_step

    def num_de(self):
        return self._de.size()

    def num_az(self):
        return self._az.size()

    def source_de(self, i):
        return self._de[i]

    def source_az(self, i):
        return self._az[i]

    def frequencies(self):
        return self._freq

    def targets(self):
        return self._targets

    def runID(self, id=None):
        if id is None:
            return self._run_id
        self._run_id = int(id)

    def source_pos(self):
        s = (C.c_double * 3)()
        _abi.check(self._lib, self._lib.wq3d_queue_source(self._q, s))
        p = wposition1()
        p.rho, p.theta, p.phi = s[0], s[1], s[2]
        return p

    def steps(self):
        v = C.c_int64()
        _abi.check(self._lib, self._lib.wq3d_queue_steps(self._q, C.byref(v)))
        return v.value

    def _front(self, which):
        return wave_front_view(self._lib.wq3d_queue_get_front, self._q, which, self.num_de(),
                               self.num_az(), self._freq.size(),
                               check=lambda rc: _abi.check(self._lib, rc))

    def past(self):
        return self._front(_abi.FRONT_PAST)

    def prev(self):
        return self._front(_abi.FRONT_PREV)

    def curr(self):
        return self._front(_abi.FRONT_CURR)

    def next(self):
        return self._front(_abi.FRONT_NEXT)

    # ---------------- wave_thresholds (wave_thresholds.h:54-182) ----------------
    def _push_thresholds(self):
        _abi.check(self._lib, self._lib.wq3d_queue_set_thresholds(self._q, C.byref(self._thresh)))

    def intensity_threshold(self, value):
        self._thresh.intensity = abs(float(value))
        self._push_thresholds()

    def eigenverb_threshold(self, value):
        """power threshold in dB (wave_thresholds.h:87-89)"""
        self._thresh.eigenverb = abs(float(value))
        self._push_thresholds()

    def max_bottom(self, v):
        self._thresh.max_bottom = int(v)
        self._push_thresholds()

    def max_surface(self, v):
        self._thresh.max_surface = int(v)
        self._push_thresholds()

    def max_caustic(self, v):
        self._thresh.max_caustic = int(v)
        self._push_thresholds()

    def max_upper(self, v):
        self._thresh.max_upper = int(v)
        self._push_thresholds()

    def max_lower(self, v):
        self._thresh.max_lower = int(v)
        self._push_thresholds()

    # ---------------- listeners ----------------
    def _install_callbacks(self):
        if not self._eig_listeners and not self._refl_listeners and not self._verb_listeners:
            _abi.check(self._lib, self._lib.wq3d_queue_set_callbacks(self._q, None, None))
            self._cb = None
            self._bulk_listeners = []
            return
        freq = self._freq
        # listeners that take a whole list at once (eigenray_collection) get
        # it after each step() / run() call instead of one callback per ray,
        # unless a per-ray listener is registered too
        per_ray = [l for l in self._eig_listeners if not getattr(l, "bulk_eigenrays", False)]
        self._bulk_listeners = [] if per_ray else list(self._eig_listeners)
        want_rays = bool(per_ray)

        def add(ctx, t1, t2, rec, inten, phase, nf, run_id):
            r = eigenray_model.from_record(rec.contents, inten[:nf], phase[:nf], freq)
            for l in self._eig_listeners:
                l.add_eigenray(t1, t2, r, run_id)

        def check(ctx, time, run_id):
            for l in self._eig_listeners:
                l.check_eigenrays(time, run_id)

        def reflect(ctx, rp):
            r = rp.contents
            pos = wposition1()
            pos.rho, pos.theta, pos.phi = r.position[0], r.position[1], r.position[2]
            nd = (r.ndirection[0], r.ndirection[1], r.ndirection[2])
            for l in self._refl_listeners:
                l.reflect(r.time, r.de, r.az, r.dt, r.grazing, r.speed, pos, nd, r.type)

        def verb(ctx, vp, power, nf, interface_num):
            v = eigenverb_model.from_record(vp.contents, power[:nf], freq)
            for l in self._verb_listeners:
                l.add_eigenverb(v, interface_num)

        if not want_rays and not self._refl_listeners and not self._verb_listeners:
            _abi.check(self._lib, self._lib.wq3d_queue_set_callbacks(self._q, None, None))
            self._cb = None
            return
        cb = _abi.wq3d_callbacks()
        cb.add_eigenray = _abi.ADD_EIGENRAY(add) if want_rays else _abi.ADD_EIGENRAY()
        cb.check_eigenrays = _abi.CHECK_EIGENRAYS(check) if want_rays else _abi.CHECK_EIGENRAYS()
        cb.reflect = _abi.REFLECT(reflect) if self._refl_listeners else _abi.REFLECT()
        cb.add_eigenverb = _abi.ADD_EIGENVERB(verb) if self._verb_listeners else _abi.ADD_EIGENVERB()
        self._cb = cb
        _abi.check(self._lib, self._lib.wq3d_queue_set_callbacks(self._q, C.byref(cb), None))

    def add_eigenray_listener(self, listener):
        if listener not in self._eig_listeners:
            self._eig_listeners.append(listener)
        self._install_callbacks()

    def remove_eigenray_listener(self, listener):
        if listener in self._eig_listeners:
            self._eig_listeners.remove(listener)
        self._install_callbacks()

    def add_reflection_listener(self, listener):
        if listener not in self._refl_listeners:
            self._refl_listeners.append(listener)
        self._install_callbacks()

    def remove_reflection_listener(self, listener):
        if listener in self._refl_listeners:
            self._refl_listeners.remove(listener)
        self._install_callbacks()

    def add_eigenverb_listener(self, listener):
        """eigenverb_notifier::add_eigenverb_listener (eigenverb_notifier.h)"""
        if listener not in self._verb_listeners:
            self._verb_listeners.append(listener)
        self._install_callbacks()

    def remove_eigenverb_listener(self, listener):
        if listener in self._verb_listeners:
            self._verb_listeners.remove(listener)
        self._install_callbacks()

    # ---------------- propagation ----------------
    def _deliver_bulk(self):
        """hands the eigenrays of the last call to the list-taking listeners"""
        if getattr(self, "_bulk_listeners", None):
            rays = self.take_eigenrays()
            if len(rays):
                for l in self._bulk_listeners:
                    l.add_eigenray_list(rays)

    def step(self, nsteps=1):
        """wave_queue::step() (wave_queue.cc:155-192); nsteps > 1 runs several."""
        try:
            _abi.check(self._lib, self._lib.wq3d_queue_step(self._q, int(nsteps)))
        finally:
            self._deliver_bulk()

    def run(self, time_max):
        """``while (time() < time_max) step();`` in one call."""
        n = C.c_size_t()
        try:
            _abi.check(self._lib, self._lib.wq3d_queue_run(self._q, float(time_max), C.byref(n)))
        finally:
            self._deliver_bulk()
        return n.value

    def abort(self):
        _abi.check(self._lib, self._lib.wq3d_queue_abort(self._q))

    def take_eigenrays(self):
        """Eigenrays found since the last call (when no eigenray listener is
        registered), in the reference's delivery order, as an eigenray_list
        (a sequence of eigenray_model)."""
        n = C.c_size_t()
        _abi.check(self._lib, self._lib.wq3d_queue_take_eigenrays(self._q, None, None, None, 0, C.byref(n)))
        cnt = n.value
        nf = self._freq.size()
        sens = None
        if getattr(self, "_sens", False):
            sens = np.empty(max(cnt, 1) * 3)
            _abi.check(self._lib, self._lib.wq3d_queue_sensitivities(self._q, _abi.as_dp(sens), cnt, C.byref(n)))
        recs = (_abi.wq3d_eigenray * max(cnt, 1))()
        inten = np.empty(max(cnt, 1) * nf)
        phase = np.empty(max(cnt, 1) * nf)
        _abi.check(self._lib, self._lib.wq3d_queue_take_eigenrays(self._q, recs, _abi.as_dp(inten),
                                                                  _abi.as_dp(phase), cnt, C.byref(n)))
        rec = np.ctypeslib.as_array(recs)[:cnt].copy()
        return eigenray_list(rec, inten[:cnt * nf].reshape(cnt, nf), phase[:cnt * nf].reshape(cnt, nf),
                             None if sens is None else sens[:cnt * 3].reshape(cnt, 3), self._freq)

    def enable_sensitivity(self):
        """exact d(intensity)/d(bottom density ratio, speed ratio,
        attenuation) on every eigenray (wq3d_queue_enable_sensitivity);
        call before the first step"""
        _abi.check(self._lib, self._lib.wq3d_queue_enable_sensitivity(self._q))
        self._sens = True

    def enable_adjoint(self, checkpoint_interval=50, max_steps=100000, max_eigenrays=0):
        """Records what the reverse sweep needs (wq3d_queue_enable_adjoint):
        ray states every ``checkpoint_interval`` steps and each eigenray's
        partial derivatives; call before the first step."""
        _abi.check(self._lib, self._lib.wq3d_queue_enable_adjoint(self._q, int(checkpoint_interval),
                                                                  int(max_steps), int(max_eigenrays)))

    def adjoint(self, rays, w_tl, w_time, num_nodes):
        """The reverse sweep (wq3d_queue_adjoint): sum_k w_tl[k] dTL_k/dc +
        w_time[k] dT_k/dc over the profile grid's nodes c, for the
        eigenrays ``rays`` (an eigenray_list this queue returned).  Returns
        (gradient, device milliseconds)."""
        rec = np.ascontiguousarray(rays.records if hasattr(rays, "records") else rays)
        n = rec.shape[0]
        wt = np.ascontiguousarray(w_tl, dtype=np.float64).reshape(-1)
        wtt = np.ascontiguousarray(w_time, dtype=np.float64).reshape(-1)
        if wt.size != n or wtt.size != n:
            raise ValueError("one TL weight and one travel-time weight per eigenray")
        grad = np.zeros(int(num_nodes))
        ms = C.c_double()
        _abi.check(self._lib, self._lib.wq3d_queue_adjoint(
            self._q, rec.ctypes.data_as(C.c_void_p), _abi.as_dp(wt), _abi.as_dp(wtt), n,
            _abi.as_dp(grad), grad.size, C.byref(ms)))
        return grad, ms.value

    def adjoint_state(self, ray, step, component, num_nodes):
        """d (component of ray's state after step) / d profile nodes
        (wq3d_queue_adjoint_state): the reverse sweep seeded on one state
        value; components 0-17 are rho, theta, phi and the normalised
        direction of the prev, curr and next fronts"""
        grad = np.zeros(int(num_nodes))
        _abi.check(self._lib, self._lib.wq3d_queue_adjoint_state(self._q, int(ray), int(step), int(component),
                                                                 _abi.as_dp(grad), grad.size))
        return grad

    def count_eigenverbs(self, on=True):
        """builds eigenverbs and counts them per interface instead of
        delivering them (wq3d_queue_count_eigenverbs)"""
        _abi.check(self._lib, self._lib.wq3d_queue_count_eigenverbs(self._q, 1 if on else 0))

    def eigenverb_counts(self):
        """eigenverbs counted per interface number since counting began"""
        out = (C.c_uint64 * (2 + 2 * _abi.MAX_VOLUME))()
        _abi.check(self._lib, self._lib.wq3d_queue_eigenverb_counts(self._q, out))
        return [int(x) for x in out]

    def set_timing(self, on):
        _abi.check(self._lib, self._lib.wq3d_queue_set_timing(self._q, 1 if on else 0))

    def set_reflect_schedule(self, schedule):
        """where a step's reflections run (wq3d_queue_set_reflect_schedule):
        _abi.REFLECT_AUTO (tuned), REFLECT_SIDE or REFLECT_INLINE; the
        results do not depend on it"""
        _abi.check(self._lib, self._lib.wq3d_queue_set_reflect_schedule(self._q, int(schedule)))

    def reflect_schedule(self):
        """the schedule in use: REFLECT_SIDE, REFLECT_INLINE, or
        REFLECT_AUTO while still tuning"""
        v = C.c_int()
        _abi.check(self._lib, self._lib.wq3d_queue_reflect_schedule(self._q, C.byref(v)))
        return v.value

    def timing(self, reset=False):
        """device milliseconds since the last reset (wq3d_queue_timing): the
        whole step/run calls, and per kernel while timing mode is on"""
        t = _abi.wq3d_timing()
        _abi.check(self._lib, self._lib.wq3d_queue_timing(self._q, C.byref(t), 1 if reset else 0))
        return {"total_ms": t.ms_total, "advance_ms": t.ms_advance, "reflect_ms": t.ms_reflect,
                "cpa_ms": t.ms_cpa, "eigenray_ms": t.ms_eigenray, "launches": t.launches}


def run_batch(queues, time_max):
    """Runs several wave_queues concurrently on one GPU, each until its
    time() reaches its time_max (wq3d_batch_run; the reference runs one
    wavefront_generator task per queue on a thread pool).  ``time_max`` is
    one value or one per queue.  Listeners are called per queue in
    reference order.  Returns (steps per queue, device milliseconds)."""
    queues = list(queues)
    n = len(queues)
    tm = np.broadcast_to(np.asarray(time_max, dtype=np.float64), (n,)).copy()
    handles = (C.c_void_p * n)(*[q._q for q in queues])
    steps = (C.c_size_t * n)()
    ms = C.c_double()
    lib = _abi.load_engine()
    try:
        _abi.check(lib, lib.wq3d_batch_run(handles, n, _abi.as_dp(tm), steps, C.byref(ms)))
    finally:
        for q in queues:
            q._deliver_bulk()
    return [int(x) for x in steps], ms.value
