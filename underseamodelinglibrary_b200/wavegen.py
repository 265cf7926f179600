"""wavefront_generator: one propagation task per source (wavegen/
wavefront_generator.{h,cc}).

The reference runs each task on a thread of its pool: build a wave_queue
for the source, attach an eigenray_collection (when there are targets)
and an eigenverb_collection (when the source computes reverberation),
step until the time limit, sum the eigenrays and hand both collections to
the source's wavefront listeners.  Here a task does the same with the GPU
engine, and ``run_wavefront_generators`` advances many tasks together in
one ``wq3d_batch_run`` (each keeps its own queue, streams and graphs)
instead of one host thread each.  Sensors, platforms and the wavefront
netCDF file are not part of this library; the source is given by its
position and an ID, and the listener is a callable."""
from ._abi import WQ3D_ERR_ABORTED, EngineError
from .eigenrays import eigenray_collection
from .eigenverbs import eigenverb_collection
from .waveq3d import run_batch, wave_queue


class wavefront_generator:
    """wavefront_generator(source, targets, targetIDs, frequencies, de_fan,
    az_fan, time_step, time_maximum, intensity_threshold, max_bottom,
    max_surface) (wavefront_generator.cc:20-39).  ``listener`` is called as
    listener(sourceID, eigenray_collection, eigenverb_collection) when the
    task completes (sensor_model::notify_wavefront_listeners)."""

    def __init__(self, ocean, source_position, target_positions, targetIDs, frequencies, de_fan,
                 az_fan, time_step, time_maximum, intensity_threshold=300.0, max_bottom=999,
                 max_surface=999, compute_reverb=False, sourceID=0, listener=None,
                 precision=None):
        self.ocean = ocean
        self.source_position = source_position
        self.target_positions = target_positions
        self.targetIDs = targetIDs
        self.frequencies = frequencies
        self.de_fan = de_fan
        self.az_fan = az_fan
        self.time_step = float(time_step)
        self.time_maximum = float(time_maximum)
        self.intensity_threshold = float(intensity_threshold)
        self.max_bottom = int(max_bottom)
        self.max_surface = int(max_surface)
        self.compute_reverb = bool(compute_reverb)
        self.sourceID = sourceID
        self.listener = listener
        self.precision = precision
        self.eigenrays = None
        self.eigenverbs = None
        self._abort = False
        self._done = False
        self._queue = None

    def abort(self):
        """thread_task::abort: a task aborted before it runs does nothing; a
        running one stops after the chunk in flight and notifies nobody."""
        self._abort = True
        if self._queue is not None:
            self._queue.abort()

    def done(self):
        return self._done

    def _has_targets(self):
        t = self.target_positions
        return t is not None and t.size1() > 0 and t.size2() > 0

    def _prepare(self):
        """the queue with thresholds and collections (wavefront_generator.cc:
        52-80)"""
        kw = {} if self.precision is None else {"precision": self.precision}
        targets = self.target_positions if self._has_targets() else None
        q = wave_queue(self.ocean, self.frequencies, self.source_position, self.de_fan, self.az_fan,
                       self.time_step, targets, **kw)
        q.intensity_threshold(self.intensity_threshold)
        q.max_bottom(self.max_bottom)
        q.max_surface(self.max_surface)
        self.eigenrays = eigenray_collection(self.frequencies, self.source_position,
                                             self.target_positions, self.sourceID, self.targetIDs) \
            if self._has_targets() else None
        if self.eigenrays is not None:
            q.add_eigenray_listener(self.eigenrays)
        self.eigenverbs = eigenverb_collection(self.ocean.num_volume())
        if self.compute_reverb:
            q.add_eigenverb_listener(self.eigenverbs)
        self._queue = q
        return q

    def _finish(self):
        """sum the eigenrays and notify (wavefront_generator.cc:113-126)"""
        if self.eigenrays is not None:
            self.eigenrays.sum_eigenrays()
        self._done = True
        self._queue = None
        if self.listener is not None:
            self.listener(self.sourceID, self.eigenrays, self.eigenverbs)

    def run(self):
        """wavefront_generator::run for this task alone."""
        if self._abort:
            return
        q = self._prepare()
        try:
            q.run(self.time_maximum)
        except EngineError as e:
            if e.code != WQ3D_ERR_ABORTED:
                raise
            self._queue = None
            return
        self._finish()


def run_wavefront_generators(generators):
    """Runs the tasks that are not aborted together on one GPU
    (wq3d_batch_run); each is then summed and notified as run() does.
    Returns the device milliseconds of the batch.  Aborting a task while
    the batch runs ends the whole batch with an EngineError
    (WQ3D_ERR_ABORTED) and notifies nobody."""
    todo = [g for g in generators if not g._abort]
    if not todo:
        return 0.0
    queues = [g._prepare() for g in todo]
    _, ms = run_batch(queues, [g.time_maximum for g in todo])
    for g in todo:
        if g._abort:
            g._queue = None
            continue
        g._finish()
    return ms
