"""Eigenverbs: Gaussian-beam footprints where rays meet a boundary or a
volume scattering layer, and the listener and collection that receive them
(eigenverbs/eigenverb_model.h, eigenverb_listener.h,
eigenverb_collection.h).  The propagator builds them on the GPU; this
module holds the host-side objects a caller works with."""
import numpy as np

from . import _abi

BOTTOM = _abi.VERB_BOTTOM
SURFACE = _abi.VERB_SURFACE
VOLUME_UPPER = _abi.VERB_VOLUME_UPPER
VOLUME_LOWER = _abi.VERB_VOLUME_LOWER


class eigenverb_model:
    """eigenverbs/eigenverb_model.h:34-150 plus the step and the order of
    the ray's events in it.  ``position`` holds (rho, theta, phi)."""

    BOTTOM, SURFACE, VOLUME_UPPER, VOLUME_LOWER = BOTTOM, SURFACE, VOLUME_UPPER, VOLUME_LOWER

    __slots__ = ("travel_time", "frequencies", "power", "length", "width", "position",
                 "direction", "grazing", "sound_speed", "de_index", "az_index", "source_de",
                 "source_az", "surface", "bottom", "caustic", "upper", "lower", "step", "seq",
                 "interface_num")

    @classmethod
    def from_record(cls, rec, power, freq):
        v = cls()
        v.travel_time = rec.travel_time
        v.frequencies = freq
        v.power = np.array(power, dtype=np.float64)
        v.length = rec.length
        v.width = rec.width
        v.position = (rec.position[0], rec.position[1], rec.position[2])
        v.direction = rec.direction
        v.grazing = rec.grazing
        v.sound_speed = rec.sound_speed
        v.de_index = rec.de
        v.az_index = rec.az
        v.source_de = rec.source_de
        v.source_az = rec.source_az
        v.surface = rec.surface
        v.bottom = rec.bottom
        v.caustic = rec.caustic
        v.upper = rec.upper
        v.lower = rec.lower
        v.step = rec.step
        v.seq = rec.seq
        v.interface_num = rec.interface_num
        return v


class eigenverb_listener:
    """eigenverbs/eigenverb_listener.h:23-41."""

    def add_eigenverb(self, verb, interface_num):
        raise NotImplementedError


class eigenverb_collection(eigenverb_listener):
    """eigenverb_collection(num_volumes) (eigenverb_collection.h): one list
    per interface -- bottom, surface, then the upper and lower side of each
    volume layer."""

    def __init__(self, num_volumes=0):
        self._collection = [[] for _ in range((1 + int(num_volumes)) * 2)]

    def num_interfaces(self):
        return len(self._collection)

    def size(self, interface_num):
        return len(self._collection[interface_num])

    def eigenverbs(self, interface_num):
        return list(self._collection[interface_num])

    def add_eigenverb(self, verb, interface_num):
        self._collection[interface_num].append(verb)

    #: size of the search area of find_eigenverbs, in footprint lengths and
    #: widths (eigenverb_collection.cc:32)
    search_scale = 1.5

    def find_eigenverbs(self, bounding_verb, interface_num):
        """eigenverb_collection::find_eigenverbs (eigenverb_collection.cc:
        60-93): the eigenverbs of one interface whose centres lie strictly
        inside the quadrilateral, in (latitude, longitude), whose corners are
        search_scale x length ahead of and behind the bounding eigenverb
        along its direction and search_scale x width to either side.  The
        reference queries an R-tree; the corners are convex, so this tests
        each centre against the four edges at once (in insertion order)."""
        from .types import wposition1
        verbs = self._collection[interface_num]
        if not verbs:
            return []
        pos = wposition1()
        pos.rho, pos.theta, pos.phi = bounding_verb.position
        d, s = bounding_verb.direction, self.search_scale
        corners = [wposition1(pos, s * bounding_verb.length, d),
                   wposition1(pos, s * bounding_verb.width, d + np.pi / 2),
                   wposition1(pos, s * bounding_verb.length, d + np.pi),
                   wposition1(pos, s * bounding_verb.width, d + np.pi + np.pi / 2)]
        cx = np.array([c.latitude() for c in corners])
        cy = np.array([c.longitude() for c in corners])
        th = np.array([v.position[1] for v in verbs])
        ph = np.array([v.position[2] for v in verbs])
        x = 90.0 - np.degrees(th)
        y = np.degrees(ph)
        cross = np.empty((4, len(verbs)))
        for k in range(4):
            x1, y1, x2, y2 = cx[k], cy[k], cx[(k + 1) % 4], cy[(k + 1) % 4]
            cross[k] = (x2 - x1) * (y - y1) - (y2 - y1) * (x - x1)
        inside = np.all(cross > 0.0, axis=0) | np.all(cross < 0.0, axis=0)
        return [verbs[i] for i in np.nonzero(inside)[0]]
