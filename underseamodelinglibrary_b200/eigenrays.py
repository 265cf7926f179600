"""eigenray_collection: per-target eigenray store and coherent sum.

Mirrors eigenrays/eigenray_collection.{h,cc}: ``add_eigenray`` keeps a list
per target (eigenray_collection.cc:90-100) and ``sum_eigenrays`` forms the
coherent (or incoherent) phasor sum per frequency with power-weighted
averages of time and angles (eigenray_collection.cc:105-191).
"""
import cmath
import math

from .types import to_degrees, to_radians
from .waveq3d import eigenray_listener


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

    def initial_time(self, t1, t2):
        return self._initial[t1][t2]

    def total(self, t1, t2):
        return self._total[t1][t2]

    def sum_eigenrays(self):
        nf = self._freq.size()
        for t1 in range(self.size1()):
            for t2 in range(self.size2()):
                rays = self._rays[t1][t2]
                tot = eigenray_total()
                tot.intensity = [0.0] * nf
                tot.phase = [0.0] * nf
                time = source_de = saz_x = saz_y = target_de = taz_x = taz_y = 0.0
                surface = bottom = caustic = upper = lower = -1
                wgt = 0.0
                max_a = 0.0
                for f in range(nf):
                    phasor = complex(0.0, 0.0)
                    for ray in rays:
                        a = math.pow(10.0, ray.intensity[f] / -20.0)
                        if self._coherent:
                            p = 2.0 * math.pi * self._freq[f] * ray.travel_time + ray.phase[f]
                            p = math.fmod(p, 2.0 * math.pi)
                            phasor += complex(a * math.cos(p), a * math.sin(p))
                        else:
                            phasor += a
                        a *= a
                        wgt += a
                        time += a * ray.travel_time
                        source_de += a * ray.source_de
                        saz_x += a * math.sin(to_radians(ray.source_az))
                        saz_y += a * math.cos(to_radians(ray.source_az))
                        target_de += a * ray.target_de
                        taz_x += a * math.sin(to_radians(ray.target_az))
                        taz_y += a * math.cos(to_radians(ray.target_az))
                        if a > max_a:
                            max_a = a
                            surface, bottom, caustic = ray.surface, ray.bottom, ray.caustic
                            upper, lower = ray.upper, ray.lower
                    tot.intensity[f] = -20.0 * math.log10(max(1e-15, abs(phasor)))
                    tot.phase[f] = cmath.phase(phasor)
                tot.travel_time = time / wgt if wgt else float("nan")
                tot.source_de = source_de / wgt if wgt else float("nan")
                tot.source_az = 90.0 - to_degrees(math.atan2(saz_y, saz_x))
                tot.target_de = target_de / wgt if wgt else float("nan")
                tot.target_az = 90.0 - to_degrees(math.atan2(taz_y, taz_x))
                tot.surface, tot.bottom, tot.caustic = surface, bottom, caustic
                tot.upper, tot.lower = upper, lower
                self._total[t1][t2] = tot
