"""Bistatic eigenverbs (biverbs/): the overlap of the eigenverbs a source
lays on each interface with those a receiver lays there, the input of the
reference's reverberation time series.

``biverb_generator`` follows biverb_generator::run
(biverbs/biverb_generator.cc:39-82): for every interface, each receiver
eigenverb is overlapped with the source eigenverbs that
eigenverb_collection::find_eigenverbs finds under it, scaled by the
interface's scattering strength, and kept when its power reaches
``biverb_collection.power_threshold``.  All of that runs on the GPU in
one ``wq3d_biverbs`` call per interface; the collection keeps each
interface's biverbs ordered by travel time, as the reference's multimap
does."""
import ctypes as C
from collections.abc import Sequence

import numpy as np

from . import _abi


def _freq_array(frequencies):
    f = frequencies.data if hasattr(frequencies, "data") else frequencies
    return np.ascontiguousarray(np.asarray(f, dtype=np.float64).ravel())


_VERB_FIELDS = ("travel_time", "length", "width", "direction", "grazing", "sound_speed", "source_de",
                "source_az")
_VERB_INTS = (("de", "de_index"), ("az", "az_index"), ("surface", "surface"), ("bottom", "bottom"),
              ("caustic", "caustic"), ("upper", "upper"), ("lower", "lower"))


def pack_eigenverbs(verbs, num_freq):
    """eigenverb_model list -> (wq3d_eigenverb array, power (n, num_freq)),
    filled a column at a time"""
    n = len(verbs)
    recs = (_abi.wq3d_eigenverb * max(n, 1))()
    power = np.zeros((n, num_freq))
    if n == 0:
        return recs, power
    a = np.ctypeslib.as_array(recs)[:n]
    for f in _VERB_FIELDS:
        a[f] = [getattr(v, f) for v in verbs]
    for f, attr in _VERB_INTS:
        a[f] = [int(getattr(v, attr)) for v in verbs]
    a["position"] = [v.position for v in verbs]
    p = [np.asarray(v.power, dtype=np.float64) for v in verbs]
    power[:] = np.stack([np.broadcast_to(x, (num_freq,)) for x in p])
    return recs, power


def compute_biverbs(src_verbs, rcv_verbs, frequencies, scattering, search_scale=1.5,
                    power_threshold=1e-20, lib=None, fn="wq3d_biverbs"):
    """The biverbs of one interface, in (receiver, source) order: returns
    (records, power (n, num_freq)).  The records are a numpy record array
    over the library's wq3d_biverb layout (fields read as attributes:
    ``recs[k].travel_time``).  ``scattering`` is an ocean scattering model
    (scattering_constant, _lambert, _chapman)."""
    lib = lib or _abi.load_engine()
    freq = _freq_array(frequencies)
    nf = freq.size
    s, sp = pack_eigenverbs(src_verbs, nf)
    r, rp = pack_eigenverbs(rcv_verbs, nf)
    desc = scattering.desc()
    dp = C.POINTER(C.c_double)
    count = C.c_size_t()
    call = getattr(lib, fn)

    def run(capacity):
        out = (_abi.wq3d_biverb * max(capacity, 1))()
        power = np.zeros((max(capacity, 1), nf))
        rc = call(s, sp.ctypes.data_as(dp), len(src_verbs), r, rp.ctypes.data_as(dp), len(rcv_verbs),
                  freq.ctypes.data_as(dp), nf, C.byref(desc), _earth(), float(search_scale),
                  float(power_threshold), out, power.ctypes.data_as(dp), capacity, C.byref(count))
        return rc, out, power

    capacity = max(1024, 4 * (len(src_verbs) + len(rcv_verbs)))
    rc, out, power = run(capacity)
    if rc == _abi.WQ3D_ERR_OVERFLOW:
        rc, out, power = run(count.value)
    if rc != 0:
        msg = lib.wq3d_last_error_string() if hasattr(lib, "wq3d_last_error_string") else b""
        raise _abi.EngineError(rc, msg.decode() if msg else "")
    n = count.value
    recs = np.ctypeslib.as_array(out)[:n].copy().view(np.recarray)
    return recs, power[:n].copy()


def _earth():
    from .types import earth_radius
    return earth_radius()


class biverb_model:
    """biverbs/biverb_model.h:24-104, plus the indices of the source and
    receiver eigenverbs it overlaps."""

    __slots__ = ("travel_time", "frequencies", "power", "duration", "de_index", "az_index",
                 "source_de", "source_az", "receiver_de", "receiver_az", "source_surface",
                 "source_bottom", "source_caustic", "source_upper", "source_lower",
                 "receiver_surface", "receiver_bottom", "receiver_caustic", "receiver_upper",
                 "receiver_lower", "source_index", "receiver_index")

    @classmethod
    def from_record(cls, rec, power, frequencies):
        """from a wq3d_biverb record (ctypes or numpy record)"""
        b = cls()
        b.travel_time = rec.travel_time
        b.frequencies = frequencies
        b.power = np.array(power, dtype=np.float64)
        b.duration = rec.duration
        b.de_index = rec.de_index
        b.az_index = rec.az_index
        b.source_de, b.source_az = rec.source_de, rec.source_az
        b.receiver_de, b.receiver_az = rec.receiver_de, rec.receiver_az
        b.source_surface, b.source_bottom = rec.source_surface, rec.source_bottom
        b.source_caustic, b.source_upper, b.source_lower = rec.source_caustic, rec.source_upper, rec.source_lower
        b.receiver_surface, b.receiver_bottom = rec.receiver_surface, rec.receiver_bottom
        b.receiver_caustic, b.receiver_upper = rec.receiver_caustic, rec.receiver_upper
        b.receiver_lower = rec.receiver_lower
        b.source_index, b.receiver_index = rec.source, rec.receiver
        return b


class biverb_list(Sequence):
    """The biverbs of one interface over record arrays: a biverb_model is
    made when an element is read, so a caller that wants the arrays
    (``arrays()``) or the count pays no per-biverb Python cost."""

    __slots__ = ("_rec", "_power", "_freq")

    def __init__(self, rec, power, frequencies):
        self._rec = rec
        self._power = power
        self._freq = frequencies

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
            raise IndexError("biverb index out of range")
        return biverb_model.from_record(self._rec[i], self._power[i], self._freq)

    def __iter__(self):
        for i in range(len(self._rec)):
            yield self[i]

    def __eq__(self, other):
        return list(self) == list(other) if isinstance(other, (list, biverb_list)) else NotImplemented

    def arrays(self):
        """(records as a numpy record array, power (n, num_freq))"""
        return self._rec, self._power


class biverb_collection:
    """biverb_collection(num_volumes) (biverbs/biverb_collection.h:36-119):
    one list per interface, ordered by travel time; biverbs of equal
    travel time keep the order in which they were added."""

    #: smallest power (largest over frequency) a biverb must reach
    #: (biverb_collection.cc:28)
    power_threshold = 1e-20

    def __init__(self, num_volumes=0):
        n = (1 + int(num_volumes)) * 2
        self._collection = [[] for _ in range(n)]
        self._records = [None] * n      # (records, power, frequencies) per interface

    def num_interfaces(self):
        return len(self._collection)

    def size(self, interface_num):
        r = self._records[interface_num]
        return len(self._collection[interface_num]) + (0 if r is None else len(r[0]))

    def biverbs(self, interface_num):
        r = self._records[interface_num]
        if r is None:
            return list(self._collection[interface_num])
        if not self._collection[interface_num]:
            return biverb_list(*r)
        merged = list(biverb_list(*r)) + self._collection[interface_num]
        merged.sort(key=lambda b: b.travel_time)
        return merged

    def add_biverbs(self, biverbs, interface_num):
        """inserts, as the reference's multimap insert does: after every
        biverb of equal or smaller travel time already held"""
        merged = self._collection[interface_num] + list(biverbs)
        merged.sort(key=lambda b: b.travel_time)
        self._collection[interface_num] = merged

    def add_records(self, records, power, frequencies, interface_num):
        """the records of one wq3d_biverbs call, kept as arrays; inserted as
        add_biverbs does (a stable sort by travel time)"""
        old = self._records[interface_num]
        if old is not None:
            records = np.concatenate([old[0], records]).view(np.recarray)
            power = np.concatenate([old[1], power])
        order = np.argsort(records.travel_time, kind="stable")
        self._records[interface_num] = (records[order], power[order], frequencies)


class biverb_generator:
    """biverb_generator(src_eigenverbs, rcv_eigenverbs) for one sensor pair
    (biverbs/biverb_generator.cc:26-82).  The reference takes the ocean and
    frequencies from process-wide singletons; here they are arguments.
    ``listener`` is called with the collection when the task completes
    (notify_update)."""

    def __init__(self, ocean, src_eigenverbs, rcv_eigenverbs, frequencies, listener=None):
        self.ocean = ocean
        self.src_eigenverbs = src_eigenverbs
        self.rcv_eigenverbs = rcv_eigenverbs
        self.frequencies = frequencies
        self.listener = listener
        self._collection = None
        self._abort = False
        self._done = False

    def abort(self):
        self._abort = True

    def done(self):
        return self._done

    def collection(self):
        return self._collection

    def run(self):
        if self._abort:
            return
        coll = biverb_collection(self.ocean.num_volume())
        src, rcv = self.src_eigenverbs, self.rcv_eigenverbs
        for interface in range(rcv.num_interfaces()):
            rv = rcv.eigenverbs(interface)
            sv = src.eigenverbs(interface) if interface < src.num_interfaces() else []
            if rv and sv:
                recs, power = compute_biverbs(sv, rv, self.frequencies,
                                              self.ocean.scattering_model(interface),
                                              search_scale=src.search_scale,
                                              power_threshold=biverb_collection.power_threshold)
                coll.add_records(recs, power, self.frequencies, interface)
            if self._abort:
                return
        self._collection = coll
        self._done = True
        if self.listener is not None:
            self.listener(coll)
