"""eigenray_collection: per-target eigenray store and coherent sum.

Mirrors eigenrays/eigenray_collection.{h,cc}: ``add_eigenray`` keeps a list
per target (eigenray_collection.cc:90-100) and ``sum_eigenrays`` forms the
coherent (or incoherent) phasor sum per frequency with power-weighted
averages of time and angles (eigenray_collection.cc:105-191).
"""
import math

import numpy as np

from .types import to_degrees, to_radians, wposition1
from .waveq3d import eigenray_listener, eigenray_model


class eigenray_total:
    __slots__ = ("travel_time", "intensity", "phase", "source_de", "source_az",
                 "target_de", "target_az", "surface", "bottom", "caustic", "upper", "lower")


class eigenray_collection(eigenray_listener):
    def __init__(self, frequencies, source_pos, target_pos, sourceID=0, targetIDs=None,
                 coherent=True):
        self._freq = frequencies
        self._source = source_pos
        self._targets = target_pos
        self._sourceID = sourceID
        self._coherent = coherent
        n1, n2 = target_pos.size1(), target_pos.size2()
        self._rays = [[[] for _ in range(n2)] for _ in range(n1)]
        self._initial = [[0.0] * n2 for _ in range(n1)]
        self._total = [[None] * n2 for _ in range(n1)]
        self._targetIDs = targetIDs
        self._num = 0

    def size1(self):
        return self._targets.size1()

    def size2(self):
        return self._targets.size2()

    def num_eigenrays(self):
        return self._num

    # a wave_queue hands this listener each call's eigenrays as one list
    # (add_eigenray_list) instead of calling add_eigenray once per ray
    bulk_eigenrays = True

    def add_eigenray(self, t1, t2, ray, run_id=0):
        self._rays[t1][t2].append(ray)
        old = self._initial[t1][t2]
        if old <= 0.0 or old > ray.travel_time:
            self._initial[t1][t2] = ray.travel_time
        self._num += 1

    def add_eigenray_list(self, rays):
        """add_eigenray for every ray of an eigenray_list, in its order (the
        reference's delivery order), each to its own target.  The rays stay
        rows of the list's record arrays until they are read; a subclass
        that overrides add_eigenray gets one call per ray."""
        if type(self).add_eigenray is not eigenray_collection.add_eigenray:
            for ray in rays:
                self.add_eigenray(ray.t1, ray.t2, ray)
            return
        rec = rays.records
        t1s, t2s, times = rec["t1"].tolist(), rec["t2"].tolist(), rec["time"].tolist()
        for k in range(len(t1s)):
            t1, t2, t = t1s[k], t2s[k], times[k]
            self._rays[t1][t2].append((rays, k))
            old = self._initial[t1][t2]
            if old <= 0.0 or old > t:
                self._initial[t1][t2] = t
        self._num += len(t1s)

    def _entries(self, t1, t2):
        """the target's eigenrays, rows of added lists made into
        eigenray_model objects on first read"""
        lst = self._rays[t1][t2]
        for k, e in enumerate(lst):
            if isinstance(e, tuple):
                lst[k] = e[0][e[1]]
        return lst

    def eigenrays(self, t1, t2):
        return list(self._entries(t1, t2))

    def dead_reckon(self, t1, t2, source_new, target_new, profile):
        """eigenray_collection::dead_reckon (eigenray_collection.cc:361-368):
        the eigenrays of target (t1, t2) moved to a new source position, then
        to a new target position, by dead_reckon_one.  ``profile`` is the
        ocean_model (or profile_model) whose sound speed and attenuation are
        used."""
        rays = dead_reckon_one(self._entries(t1, t2), self._source, source_new, profile)
        old_target = wposition1()
        old_target.rho = float(self._targets.rho[t1, t2])
        old_target.theta = float(self._targets.theta[t1, t2])
        old_target.phi = float(self._targets.phi[t1, t2])
        return dead_reckon_one(rays, old_target, target_new, profile)

    def initial_time(self, t1, t2):
        return self._initial[t1][t2]

    def total(self, t1, t2):
        return self._total[t1][t2]

    def sum_eigenrays(self):
        """eigenray_collection::sum_eigenrays (eigenray_collection.cc:
        105-191) on the GPU (wq3d_sum_eigenrays): per target, the coherent
        (or incoherent) phasor sum of its eigenrays at each frequency, in
        the order they were added, and the power-weighted travel time, D/E
        and AZ; the strongest path gives the counts."""
        import ctypes as C

        from . import _abi
        lib = _abi.load_engine()
        nf = self._freq.size()
        n1, n2 = self.size1(), self.size2()
        fv = np.ascontiguousarray([self._freq[f] for f in range(nf)], dtype=np.float64)
        rays = [(t1, t2, r) for t1 in range(n1) for t2 in range(n2) for r in self._rays[t1][t2]]
        n = len(rays)
        rec = (_abi.wq3d_eigenray * max(n, 1))()
        inten = np.zeros((max(n, 1), nf))
        phase = np.zeros((max(n, 1), nf))
        # rows still held by their eigenray_list are copied list by list
        recs = np.ctypeslib.as_array(rec)
        groups = {}
        for k, (t1, t2, r) in enumerate(rays):
            if isinstance(r, tuple):
                g = groups.setdefault(id(r[0]), (r[0], [], []))
                g[1].append(k)
                g[2].append(r[1])
                continue
            e = rec[k]
            e.time, e.source_de, e.source_az = r.travel_time, r.source_de, r.source_az
            e.target_de, e.target_az = r.target_de, r.target_az
            e.surface, e.bottom, e.caustic, e.upper, e.lower = r.surface, r.bottom, r.caustic, r.upper, r.lower
            e.t1, e.t2 = t1, t2
            inten[k] = r.intensity
            phase[k] = r.phase
        for lst, dst, rows in groups.values():
            dst, rows = np.asarray(dst), np.asarray(rows)
            recs[dst] = lst.records[rows]
            inten[dst] = lst._inten[rows]
            phase[dst] = lst._phase[rows]
        tot = (_abi.wq3d_eigenray * (n1 * n2))()
        ti = np.empty((n1 * n2, nf))
        tp = np.empty((n1 * n2, nf))
        _abi.check(lib, lib.wq3d_sum_eigenrays(C.cast(rec, C.c_void_p), _abi.as_dp(inten), _abi.as_dp(phase), n,
                                               _abi.as_dp(fv), nf, n1, n2, 1 if self._coherent else 0,
                                               C.cast(tot, C.c_void_p), _abi.as_dp(ti), _abi.as_dp(tp)))
        for t in range(n1 * n2):
            o = tot[t]
            out = eigenray_total()
            out.travel_time, out.source_de, out.source_az = o.time, o.source_de, o.source_az
            out.target_de, out.target_az = o.target_de, o.target_az
            out.surface, out.bottom, out.caustic, out.upper, out.lower = o.surface, o.bottom, o.caustic, o.upper, o.lower
            out.intensity = [float(x) for x in ti[t]]
            out.phase = [float(x) for x in tp[t]]
            self._total[t // n2][t % n2] = out


def _evaluator(profile):
    """an object with sound_speed / attenuation point evaluations"""
    if hasattr(profile, "sound_speed") and hasattr(profile, "attenuation") and hasattr(profile, "handle"):
        return profile
    from .ocean import boundary_flat, ocean_model
    return ocean_model(boundary_flat(), boundary_flat(1.0e4), profile)


def dead_reckon_one(eigenrays, oldpos, newpos, profile):
    """eigenray_collection::dead_reckon_one (eigenray_collection.cc:373-446):
    adjusts eigenrays for a small move of one sensor.  The move, in the local
    tangent plane at the old position, is projected on each ray's launch
    direction (source D/E and AZ, also for a moving target, as the reference
    does); travel time changes by that range over the sound speed at the old
    position, and intensity by the change of 20 log10(r) plus attenuation
    over r (r = travel time x sound speed).  A move of less than 1 mm returns
    the eigenrays unchanged."""
    dr_rho = newpos.rho - oldpos.rho
    dr_th = (newpos.theta - oldpos.theta) * oldpos.rho
    dr_ph = (newpos.phi - oldpos.phi) * (oldpos.rho * math.sin(oldpos.theta))
    if dr_rho * dr_rho + dr_th * dr_th + dr_ph * dr_ph < 1e-6:
        return list(eigenrays)
    rays = list(eigenrays)
    if not rays:
        return []
    ev = _evaluator(profile)
    c, _ = ev.sound_speed([oldpos.rho], [oldpos.theta], [oldpos.phi])
    sound_speed = float(c[0])
    freq = rays[0].frequencies
    fv = np.array([freq(k) for k in range(freq.size())], dtype=np.float64)
    r1 = np.empty(len(rays))
    r2 = np.empty(len(rays))
    out = []
    for n, ray in enumerate(rays):
        de = to_radians(ray.source_de)
        az = to_radians(ray.source_az)
        cos_de, sin_de = math.cos(de), math.sin(de)
        cos_az, sin_az = math.cos(az), math.sin(az)
        dr = dr_rho * sin_de + dr_th * (-cos_de * cos_az) + dr_ph * (cos_de * sin_az)
        new = eigenray_model()
        for name in eigenray_model.__slots__:
            setattr(new, name, getattr(ray, name, None))
        new.travel_time = ray.travel_time + dr / sound_speed
        r1[n] = ray.travel_time * sound_speed
        r2[n] = r1[n] + dr
        out.append(new)
    rho = np.full(len(rays), oldpos.rho)
    a1 = ev.attenuation(rho, r1, fv)
    a2 = ev.attenuation(rho, r2, fv)
    for n, (ray, new) in enumerate(zip(rays, out)):
        inten = np.array(ray.intensity, dtype=np.float64)
        offset = inten - 20.0 * np.log10(r1[n]) - a1[n]
        new.intensity = 20.0 * np.log10(r2[n]) + a2[n] + offset
        new.phase = np.array(ray.phase, dtype=np.float64)
    return out


def form_errors(test, ref):
    """Differences between two eigenray sets of the same propagation (two
    arithmetic forms, or the engine and the oracle), matched on the CPA
    bracket (step, t1, t2, D/E index, AZ index): the counts found in one set
    only, and for the matched eigenrays the largest and 99th-percentile
    absolute differences of travel time (s), intensity (dB, every
    frequency), source D/E and AZ and target D/E and AZ (deg).  ``test`` and
    ``ref`` are eigenray_lists (take_eigenrays)."""
    def table(rays):
        a = rays.arrays()
        keys = list(zip(a["step"].tolist(), a["t1"].tolist(), a["t2"].tolist(), a["de"].tolist(),
                        a["az"].tolist()))
        return a, {k: i for i, k in enumerate(keys)}
    at, it = table(test)
    ar, ir = table(ref)
    common = sorted(set(it) & set(ir))
    out = {"matched": len(common), "only_test": len(it) - len(common), "only_ref": len(ir) - len(common)}
    if not common:
        return out
    jt = np.array([it[k] for k in common])
    jr = np.array([ir[k] for k in common])
    cols = {"travel_time_s": ("time", 1.0), "intensity_db": ("intensity", 1.0),
            "source_de_deg": ("source_de", 1.0), "source_az_deg": ("source_az", 1.0),
            "target_de_deg": ("target_de", 1.0), "target_az_deg": ("target_az", 1.0)}
    for name, (col, _) in cols.items():
        d = np.abs(np.asarray(at[col])[jt] - np.asarray(ar[col])[jr])
        if name.endswith("az_deg"):
            d = np.minimum(d, 360.0 - d)
        d = d.ravel()
        out[name] = {"max": float(d.max()), "p99": float(np.percentile(d, 99))}
    counts = ("surface", "bottom", "caustic", "upper", "lower")
    out["counts_differ"] = int(sum(np.count_nonzero(np.asarray(at[c])[jt] != np.asarray(ar[c])[jr]) for c in counts))
    return out
