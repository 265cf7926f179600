"""eigenray_collection: per-target eigenray store and coherent sum.

Mirrors eigenrays/eigenray_collection.{h,cc}: ``add_eigenray`` keeps a list
per target (eigenray_collection.cc:90-100) and ``sum_eigenrays`` forms the
coherent (or incoherent) phasor sum per frequency with power-weighted
averages of time and angles (eigenray_collection.cc:105-191).
"""
import cmath
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

    def add_eigenray(self, t1, t2, ray, run_id=0):
        self._rays[t1][t2].append(ray)
        old = self._initial[t1][t2]
        if old <= 0.0 or old > ray.travel_time:
            self._initial[t1][t2] = ray.travel_time
        self._num += 1

    def eigenrays(self, t1, t2):
        return list(self._rays[t1][t2])

    def dead_reckon(self, t1, t2, source_new, target_new, profile):
        """eigenray_collection::dead_reckon (eigenray_collection.cc:361-368):
        the eigenrays of target (t1, t2) moved to a new source position, then
        to a new target position, by dead_reckon_one.  ``profile`` is the
        ocean_model (or profile_model) whose sound speed and attenuation are
        used."""
        rays = dead_reckon_one(self._rays[t1][t2], self._source, source_new, profile)
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
        105-191), one target at a time with numpy.  Every sum runs in the
        reference's order (frequency, then eigenray) as a sequential
        cumulative sum: the phasor of each frequency, and the weights
        a^2 = 10^(-I/10) with the weighted travel time, D/E and the unit
        vectors of AZ.  The strongest path (first largest weight) gives the
        counts."""
        nf = self._freq.size()
        fv = np.array([self._freq[f] for f in range(nf)], dtype=np.float64)
        two_pi = 2.0 * math.pi
        for t1 in range(self.size1()):
            for t2 in range(self.size2()):
                rays = self._rays[t1][t2]
                tot = eigenray_total()
                n = len(rays)
                if n == 0:
                    tot.intensity = [-20.0 * math.log10(1e-15)] * nf
                    tot.phase = [0.0] * nf
                    tot.travel_time = tot.source_de = tot.target_de = float("nan")
                    tot.source_az = tot.target_az = 90.0 - to_degrees(math.atan2(0.0, 0.0))
                    tot.surface = tot.bottom = tot.caustic = tot.upper = tot.lower = -1
                    self._total[t1][t2] = tot
                    continue
                amp = np.power(10.0, np.array([r.intensity for r in rays], dtype=np.float64).T / -20.0)
                if self._coherent:
                    tt = np.array([r.travel_time for r in rays], dtype=np.float64)
                    ph = np.array([r.phase for r in rays], dtype=np.float64).T
                    p = np.fmod(two_pi * fv[:, None] * tt[None, :] + ph, two_pi)
                    re = np.cumsum(amp * np.cos(p), axis=1)[:, -1]
                    im = np.cumsum(amp * np.sin(p), axis=1)[:, -1]
                else:
                    re = np.cumsum(amp, axis=1)[:, -1]
                    im = np.zeros(nf)
                tot.intensity = [float(x) for x in -20.0 * np.log10(np.maximum(1e-15, np.hypot(re, im)))]
                tot.phase = [float(x) for x in np.arctan2(im, re)]
                w = (amp * amp).ravel()  # (frequency, eigenray) order
                wgt = float(np.cumsum(w)[-1])

                def wsum(v):
                    return float(np.cumsum(w * np.tile(np.asarray(v, dtype=np.float64), nf))[-1])

                saz = np.radians([r.source_az for r in rays])
                taz = np.radians([r.target_az for r in rays])
                nan = float("nan")
                tot.travel_time = wsum([r.travel_time for r in rays]) / wgt if wgt else nan
                tot.source_de = wsum([r.source_de for r in rays]) / wgt if wgt else nan
                tot.source_az = 90.0 - to_degrees(math.atan2(wsum(np.cos(saz)), wsum(np.sin(saz))))
                tot.target_de = wsum([r.target_de for r in rays]) / wgt if wgt else nan
                tot.target_az = 90.0 - to_degrees(math.atan2(wsum(np.cos(taz)), wsum(np.sin(taz))))
                j = int(np.argmax(w))
                if w[j] > 0.0:
                    best = rays[j % n]
                    tot.surface, tot.bottom, tot.caustic = best.surface, best.bottom, best.caustic
                    tot.upper, tot.lower = best.upper, best.lower
                else:
                    tot.surface = tot.bottom = tot.caustic = tot.upper = tot.lower = -1
                self._total[t1][t2] = tot


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
