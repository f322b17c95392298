"""ctypes binding of the C ABI (include/itsu.h) in lib/libitsu_b200.so.

There is no fallback: if the library is missing or no B200 is visible, the calls raise.
Results come back in the same canonical dict form as the oracle, so tests compare them field
by field.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .gen import CLUSTER_DTYPE

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "lib", "libitsu_b200.so")

# itsu_cluster_in: the 24-byte input record of the compact host calls
CLUSTER_IN_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("id", "<i4"), ("alpha", "<f4"), ("mc", "<i4")])


# itsu_cluster_track: the 16-byte input record of the track host calls (roads and labels only)
CLUSTER_TRACK_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("mc", "<i4")])


def track_clusters(clusters) -> np.ndarray:
    """The 16-byte input records of clusters (coordinates and MC id)."""
    out = np.zeros(len(clusters), CLUSTER_TRACK_DTYPE)
    for k in CLUSTER_TRACK_DTYPE.names:
        out[k] = clusters[k]
    return out


def compact_clusters(clusters) -> np.ndarray:
    """The 24-byte input records of 36-byte clusters (the fields clustering computes dropped)."""
    out = np.zeros(len(clusters), CLUSTER_IN_DTYPE)
    for k in CLUSTER_IN_DTYPE.names:
        out[k] = clusters[k]
    return out


TRACKLET_DTYPE = np.dtype([("c1", "<i4"), ("c2", "<i4"), ("tan_lambda", "<f4"), ("phi", "<f4")])
CELL_DTYPE = np.dtype(
    [("c1", "<i4"), ("c2", "<i4"), ("c3", "<i4"), ("t1", "<i4"), ("t2", "<i4"), ("nx", "<f4"), ("ny", "<f4"),
     ("nz", "<f4"), ("curvature", "<f4"), ("level", "<i4")]
)
ROAD_DTYPE = np.dtype([("cells", "<i4", (5,)), ("size", "<i4"), ("label", "<i4"), ("fake", "u1"), ("pad", "u1", (3,))])
REPORT_COUNTS_DTYPE = np.dtype([("labels", "<i4"), ("correct", "<i4"), ("duplicate", "<i4"), ("fake", "<i4")])

OK, ERR_INVALID, ERR_CAPACITY, ERR_TIMEOUT, ERR_CUDA, ERR_NOMEM, ERR_STATE = range(7)
FLAG_NO_GROW = 1
FLAG_STREAM_HOST = 2


class ItsuError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


STATUS_NAMES = {OK: "ITSU_OK", ERR_INVALID: "ITSU_ERR_INVALID", ERR_CAPACITY: "ITSU_ERR_CAPACITY",
                ERR_TIMEOUT: "ITSU_ERR_TIMEOUT", ERR_CUDA: "ITSU_ERR_CUDA", ERR_NOMEM: "ITSU_ERR_NOMEM",
                ERR_STATE: "ITSU_ERR_STATE"}


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("flags", ctypes.c_uint32), ("max_clusters", ctypes.c_int64),
                ("max_tracklets", ctypes.c_int64), ("max_cells", ctypes.c_int64), ("max_neighbours", ctypes.c_int64),
                ("max_roads", ctypes.c_int64), ("max_events", ctypes.c_int32), ("stream_chunk_clusters", ctypes.c_int32)]


class Counts(ctypes.Structure):
    _fields_ = [("clusters", ctypes.c_int32 * 7), ("tracklets", ctypes.c_int32 * 6), ("cells", ctypes.c_int32 * 5),
                ("neighbours", ctypes.c_int32 * 4), ("roads", ctypes.c_int32)]


class Results(ctypes.Structure):
    _fields_ = [("clusters", ctypes.c_void_p * 7), ("index_tables", ctypes.c_void_p * 6), ("tracklets", ctypes.c_void_p * 6),
                ("tracklets_lookup", ctypes.c_void_p * 5), ("cells", ctypes.c_void_p * 5), ("cells_lookup", ctypes.c_void_p * 4),
                ("neighbour_offsets", ctypes.c_void_p * 4), ("neighbours", ctypes.c_void_p * 4), ("roads", ctypes.c_void_p)]


class KernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 40), ("ms", ctypes.c_float), ("launches", ctypes.c_int32)]


class Frames(ctypes.Structure):
    _fields_ = [("clusters", ctypes.c_void_p), ("frame_offsets", ctypes.c_void_p), ("vertices", ctypes.c_void_p),
                ("vertex_frame", ctypes.c_void_p), ("n_frames", ctypes.c_int32), ("n_vertices", ctypes.c_int32)]


class Tune(ctypes.Structure):
    _fields_ = [("band", ctypes.c_int32), ("threads_per_block", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("prune", ctypes.c_int32), ("ms", ctypes.c_float), ("events_per_group", ctypes.c_int32)]


class MemoryUsage(ctypes.Structure):
    _fields_ = [("device_bytes", ctypes.c_int64), ("clusters_capacity", ctypes.c_int64), ("events_capacity", ctypes.c_int64),
                ("capacity", ctypes.c_int64 * 4), ("used", ctypes.c_int64 * 4), ("cell_entries_capacity", ctypes.c_int64)]


class Batch(ctypes.Structure):
    _fields_ = [("clusters", ctypes.c_void_p), ("layer_offsets", ctypes.c_void_p), ("vertices", ctypes.c_void_p),
                ("n_events", ctypes.c_int32), ("reserved_", ctypes.c_int32), ("n_clusters", ctypes.c_int64)]


MLP_INPUTS, MLP_HIDDEN = 8, 64
MLP_PARAMS = MLP_HIDDEN * MLP_INPUTS + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_HIDDEN + 1


TRACKLET_LAYERS = 6
GATE_HIDDEN = 16
GATE_PARAMS = GATE_HIDDEN * MLP_INPUTS + GATE_HIDDEN + GATE_HIDDEN * GATE_HIDDEN + GATE_HIDDEN + GATE_HIDDEN + 1


def _model_fields(hidden):
    return [("w1", (ctypes.c_float * MLP_INPUTS) * hidden), ("b1", ctypes.c_float * hidden),
            ("w2", (ctypes.c_float * hidden) * hidden), ("b2", ctypes.c_float * hidden),
            ("w3", ctypes.c_float * hidden), ("b3", ctypes.c_float), ("mean", ctypes.c_float * MLP_INPUTS),
            ("inv_std", ctypes.c_float * MLP_INPUTS), ("logit_threshold", ctypes.c_float)]


class PrefilterModel(ctypes.Structure):
    """itsu_prefilter_model: the pair prefilter (8 -> 64 -> 64 -> 1, GELU)."""
    _fields_ = _model_fields(MLP_HIDDEN)
    N_PARAMS = MLP_PARAMS

    def params(self) -> np.ndarray:
        """The trainable parameters as one float32 array (w1, b1, w2, b2, w3, b3)."""
        return np.frombuffer(bytes(self), np.float32, self.N_PARAMS).copy()

    def arrays(self) -> dict:
        return dict(w1=np.ctypeslib.as_array(self.w1).copy(), b1=np.ctypeslib.as_array(self.b1).copy(),
                    w2=np.ctypeslib.as_array(self.w2).copy(), b2=np.ctypeslib.as_array(self.b2).copy(),
                    w3=np.ctypeslib.as_array(self.w3).copy(), b3=float(self.b3),
                    mean=np.ctypeslib.as_array(self.mean).copy(), inv_std=np.ctypeslib.as_array(self.inv_std).copy(),
                    logit_threshold=float(self.logit_threshold))


class GateModel(ctypes.Structure):
    """itsu_gate_model: the tracklet gate (per-layer |dphi| and |dz| windows, then 8 -> 16 -> 16 -> 1,
    ReLU); same field order."""
    _fields_ = _model_fields(GATE_HIDDEN) + [("dphi_window", ctypes.c_float * TRACKLET_LAYERS),
                                              ("dz_window", ctypes.c_float * TRACKLET_LAYERS),
                                              ("mlp_layers", ctypes.c_int32)]
    N_PARAMS = GATE_PARAMS
    params = PrefilterModel.params
    arrays = PrefilterModel.arrays


class GateSamples(ctypes.Structure):
    _fields_ = [("features", ctypes.c_void_p), ("labels", ctypes.c_void_p), ("capacity", ctypes.c_int64),
                ("road_tracklets", ctypes.c_void_p), ("road_capacity", ctypes.c_int64), ("n_tracklets", ctypes.c_int64),
                ("n_roads", ctypes.c_int64)]


class PrefilterSamples(ctypes.Structure):
    _fields_ = [("features", ctypes.c_void_p), ("labels", ctypes.c_void_p), ("capacity", ctypes.c_int64),
                ("road_cells", ctypes.c_void_p), ("road_keys", ctypes.c_void_p), ("road_fake", ctypes.c_void_p),
                ("road_capacity", ctypes.c_int64), ("n_cells", ctypes.c_int64), ("n_roads", ctypes.c_int64)]


class TrainConfig(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int64), ("batch", ctypes.c_int32), ("reserved_", ctypes.c_int32), ("lr", ctypes.c_float),
                ("lr_final", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
                ("weight_decay", ctypes.c_float), ("pos_weight", ctypes.c_float), ("seed", ctypes.c_uint64)]


_lib = None

# (name, restype, argtypes) of every entry point declared in include/itsu.h
SIGNATURES = [
    ("itsu_version", ctypes.c_char_p, []),
    ("itsu_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("itsu_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("itsu_config_default", None, [ctypes.POINTER(Config)]),
    ("itsu_context_create", ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]),
    ("itsu_context_destroy", None, [ctypes.c_void_p]),
    ("itsu_context_set_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("itsu_context_stream", ctypes.c_void_p, [ctypes.c_void_p]),
    ("itsu_pvc_initialize", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("itsu_compute_layer_tracklets", ctypes.c_int, [ctypes.c_void_p]),
    ("itsu_compute_layer_cells", ctypes.c_int, [ctypes.c_void_p]),
    ("itsu_find_cells_neighbours", ctypes.c_int, [ctypes.c_void_p]),
    ("itsu_find_tracks", ctypes.c_int, [ctypes.c_void_p]),
    ("itsu_compute_montecarlo_labels", ctypes.c_int, [ctypes.c_void_p]),
    ("itsu_get_counts", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(Counts)]),
    ("itsu_copy_results", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(Results)]),
    ("itsu_clusters_to_tracks", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
      ctypes.POINTER(ctypes.c_int32)]),
    ("itsu_batch_run", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Batch)]),
    ("itsu_batch_run_host", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64,
      ctypes.c_void_p]),
    ("itsu_batch_run_host_compact", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64,
      ctypes.c_void_p]),
    ("itsu_atan2f_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]),
    ("itsu_batch_run_host_tracks", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64,
      ctypes.c_void_p]),
    ("itsu_batch_launch", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Batch)]),
    ("itsu_batch_status", ctypes.c_int, [ctypes.c_void_p]),
    ("itsu_batch_roads_device", ctypes.c_int,
     [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]),
    ("itsu_frames_run_host", ctypes.c_int,
     [ctypes.c_void_p, ctypes.POINTER(Frames), ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    ("itsu_relaunch", ctypes.c_int, [ctypes.c_void_p]),
    ("itsu_memory_usage_get", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(MemoryUsage)]),
    ("itsu_batch_road_count", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    ("itsu_roads_report", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    ("itsu_kernels_per_run", ctypes.c_int32, []),
    ("itsu_multiplicity_band", ctypes.c_int32, [ctypes.c_int64, ctypes.c_int32]),
    ("itsu_autotune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(Tune)]),
    ("itsu_get_tune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(Tune)]),
    ("itsu_set_tune", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Tune)]),
    ("itsu_pvc_initialize_noalloc", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("itsu_batch_profile", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    ("itsu_prefilter_init", None, [ctypes.POINTER(PrefilterModel), ctypes.c_uint64]),
    ("itsu_train_config_default", None, [ctypes.POINTER(TrainConfig)]),
    ("itsu_prefilter_save", ctypes.c_int, [ctypes.POINTER(PrefilterModel), ctypes.c_char_p]),
    ("itsu_prefilter_load", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(PrefilterModel)]),
    ("itsu_prefilter_set_model", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PrefilterModel)]),
    ("itsu_prefilter_get_model", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PrefilterModel)]),
    ("itsu_prefilter_enable", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ("itsu_prefilter_export", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PrefilterSamples)]),
    ("itsu_prefilter_score", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    ("itsu_prefilter_train", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(TrainConfig), ctypes.c_void_p]),
    ("itsu_prefilter_gradient", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_float, ctypes.c_void_p,
      ctypes.POINTER(ctypes.c_float)]),
    ("itsu_gate_init", None, [ctypes.POINTER(GateModel), ctypes.c_uint64]),
    ("itsu_gate_save", ctypes.c_int, [ctypes.POINTER(GateModel), ctypes.c_char_p]),
    ("itsu_gate_load", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(GateModel)]),
    ("itsu_gate_set_model", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GateModel)]),
    ("itsu_gate_get_model", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GateModel)]),
    ("itsu_gate_enable", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ("itsu_gate_export", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GateSamples)]),
    ("itsu_gate_score", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    ("itsu_gate_train", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(TrainConfig), ctypes.c_void_p]),
    ("itsu_gate_gradient", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_float, ctypes.c_void_p,
      ctypes.POINTER(ctypes.c_float)]),
]


def prefilter_init(seed: int) -> PrefilterModel:
    """A fresh seeded model (host only)."""
    m = PrefilterModel()
    load().itsu_prefilter_init(ctypes.byref(m), seed)
    return m


def train_config(**kw) -> TrainConfig:
    cfg = TrainConfig()
    load().itsu_train_config_default(ctypes.byref(cfg))
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def prefilter_save(model: PrefilterModel, path: str):
    L = load()
    st = L.itsu_prefilter_save(ctypes.byref(model), path.encode())
    if st != OK:
        raise ItsuError(st, L.itsu_last_error(None).decode())


def prefilter_load(path: str) -> PrefilterModel:
    L = load()
    m = PrefilterModel()
    st = L.itsu_prefilter_load(path.encode(), ctypes.byref(m))
    if st != OK:
        raise ItsuError(st, L.itsu_last_error(None).decode())
    return m


def gate_init(seed: int) -> GateModel:
    """A fresh seeded tracklet gate (host only)."""
    m = GateModel()
    load().itsu_gate_init(ctypes.byref(m), seed)
    return m


def gate_save(model: GateModel, path: str):
    L = load()
    st = L.itsu_gate_save(ctypes.byref(model), path.encode())
    if st != OK:
        raise ItsuError(st, L.itsu_last_error(None).decode())


def gate_load(path: str) -> GateModel:
    L = load()
    m = GateModel()
    st = L.itsu_gate_load(path.encode(), ctypes.byref(m))
    if st != OK:
        raise ItsuError(st, L.itsu_last_error(None).decode())
    return m


def load(path: str = LIB_PATH):
    """Load the library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError("libitsu_b200.so not found at %s: run `make -C tracking-itsu_b200`" % path)
        L = ctypes.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else ctypes.c_void_p(0)


class Context:
    """One itsu_context: a device arena and stream."""

    def __init__(self, device: int = 0, flags: int = 0, **caps):
        self.lib = load()
        cfg = Config()
        self.lib.itsu_config_default(ctypes.byref(cfg))
        cfg.device = device
        cfg.flags = flags
        for k, v in caps.items():
            setattr(cfg, k, v)
        h = ctypes.c_void_p()
        st = self.lib.itsu_context_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != OK:
            raise ItsuError(st, self.lib.itsu_last_error(None).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.itsu_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != OK:
            raise ItsuError(st, self.lib.itsu_last_error(self.h).decode())

    def set_stream(self, stream_handle: int):
        self._check(self.lib.itsu_context_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    @property
    def stream(self) -> int:
        return self.lib.itsu_context_stream(self.h) or 0

    # ---- per vertex ----
    @staticmethod
    def _layer_args(layers, vertex):
        layers = [np.ascontiguousarray(l, dtype=CLUSTER_DTYPE) for l in layers]
        ptrs = (ctypes.c_void_p * 7)(*[l.ctypes.data if len(l) else None for l in layers])
        counts = (ctypes.c_int32 * 7)(*[len(l) for l in layers])
        v = (ctypes.c_float * 3)(*[float(x) for x in vertex])
        return layers, ptrs, counts, v

    def initialize(self, layers, vertex):
        keep, ptrs, counts, v = self._layer_args(layers, vertex)
        self._check(self.lib.itsu_pvc_initialize(self.h, ptrs, counts, v))

    def run_stages(self, layers, vertex):
        """PrimaryVertexContext::initialize then every Tracker stage, one call per stage."""
        self.initialize(layers, vertex)
        for fn in (self.lib.itsu_compute_layer_tracklets, self.lib.itsu_compute_layer_cells,
                   self.lib.itsu_find_cells_neighbours, self.lib.itsu_find_tracks, self.lib.itsu_compute_montecarlo_labels):
            self._check(fn(self.h))

    def counts(self, event: int = 0) -> Counts:
        c = Counts()
        self._check(self.lib.itsu_get_counts(self.h, event, ctypes.byref(c)))
        return c

    def results(self, event: int = 0) -> dict:
        """Host copies of every output of one event, in the oracle's canonical form."""
        c = self.counts(event)
        res = dict(
            clusters=[np.zeros(c.clusters[l], CLUSTER_DTYPE) for l in range(7)],
            index_tables=np.zeros((6, 401), np.int32),
            tracklets=[np.zeros(c.tracklets[l], TRACKLET_DTYPE) for l in range(6)],
            trk_lookup=[np.zeros(c.clusters[l + 1], np.int32) for l in range(5)],
            cells=[np.zeros(c.cells[l], CELL_DTYPE) for l in range(5)],
            cell_lookup=[np.zeros(c.tracklets[l + 1], np.int32) for l in range(4)],
            nb_offsets=[np.zeros(c.cells[l + 1] + 1, np.int32) for l in range(4)],
            nb=[np.zeros(c.neighbours[l], np.int32) for l in range(4)],
            roads=np.zeros(c.roads, ROAD_DTYPE),
        )
        r = Results()
        for l in range(7):
            r.clusters[l] = res["clusters"][l].ctypes.data if c.clusters[l] else None
        for l in range(6):
            r.index_tables[l] = res["index_tables"][l].ctypes.data
            r.tracklets[l] = res["tracklets"][l].ctypes.data if c.tracklets[l] else None
        for l in range(5):
            r.tracklets_lookup[l] = res["trk_lookup"][l].ctypes.data if len(res["trk_lookup"][l]) else None
            r.cells[l] = res["cells"][l].ctypes.data if c.cells[l] else None
        for l in range(4):
            r.cells_lookup[l] = res["cell_lookup"][l].ctypes.data if len(res["cell_lookup"][l]) else None
            r.neighbour_offsets[l] = res["nb_offsets"][l].ctypes.data
            r.neighbours[l] = res["nb"][l].ctypes.data if c.neighbours[l] else None
        r.roads = res["roads"].ctypes.data if c.roads else None
        self._check(self.lib.itsu_copy_results(self.h, event, ctypes.byref(r)))
        res["roads"]["pad"] = 0
        return res

    def run_vertex(self, layers, vertex) -> dict:
        self.run_stages(layers, vertex)
        return self.results(0)

    def clusters_to_tracks(self, layers, vertex) -> np.ndarray:
        """Whole path for one vertex in one call; returns its roads."""
        keep, ptrs, counts, v = self._layer_args(layers, vertex)
        n = ctypes.c_int32()
        self._check(self.lib.itsu_clusters_to_tracks(self.h, ptrs, counts, v, None, 0, ctypes.byref(n)))
        roads = np.zeros(n.value, ROAD_DTYPE)
        self._check(self.lib.itsu_clusters_to_tracks(self.h, ptrs, counts, v, _ptr(roads), n.value, ctypes.byref(n)))
        roads["pad"] = 0
        return roads

    # ---- batches ----
    def memory_usage(self) -> dict:
        """itsu_memory_usage_get: arena bytes, capacities and the last run's totals."""
        m = MemoryUsage()
        self._check(self.lib.itsu_memory_usage_get(self.h, ctypes.byref(m)))
        names = ("tracklets", "cells", "neighbours", "roads")
        return dict(device_bytes=m.device_bytes, clusters_capacity=m.clusters_capacity, events_capacity=m.events_capacity,
                    capacity=dict(zip(names, list(m.capacity))), used=dict(zip(names, list(m.used))),
                    cell_entries_capacity=m.cell_entries_capacity)

    def roads_report(self, label_maps, roads=None, run_offsets=None, run_event=None, n_runs=None):
        """itsu_roads_report: the road classes (ITSU_ROAD_*: 0 unreported, 1 correct, 2 duplicate,
        3 fake) and per-event counts (labels, correct, duplicate, fake) of IOUtils::writeRoadsReport.
        label_maps: one LABEL_DTYPE array per event (itsu.io.read_reference_labels). roads and
        run_offsets on the host, or neither for the device-resident roads of the last batch or frames
        run (n_runs: its run count). run_event maps runs (vertices) to events (default: run r is
        event r)."""
        from .io import labels_for_report

        labels, label_offsets = labels_for_report(label_maps)
        n_events = len(label_maps)
        if roads is not None:
            roads = np.ascontiguousarray(roads, ROAD_DTYPE)
            if len(roads) == 0:
                roads = np.zeros(1, ROAD_DTYPE)  # a valid pointer: the offsets say there are none
            run_offsets = np.ascontiguousarray(run_offsets, np.int32)
            n_runs = len(run_offsets) - 1
            n_roads = int(run_offsets[-1])
        else:
            if n_runs is None:
                raise ValueError("n_runs is required for the device-resident roads")
            n = ctypes.c_int64()
            self._check(self.lib.itsu_batch_road_count(self.h, ctypes.byref(n)))
            n_roads = n.value
        rev = None if run_event is None else np.ascontiguousarray(run_event, np.int32)
        cls = np.zeros(max(n_roads, 1), np.uint8)
        counts = np.zeros(max(n_events, 1), REPORT_COUNTS_DTYPE)
        self._check(self.lib.itsu_roads_report(
            self.h, _ptr(roads) if roads is not None else None, _ptr(run_offsets) if roads is not None else None,
            _ptr(rev) if rev is not None else None, n_runs, _ptr(labels) if len(labels) else None, _ptr(label_offsets),
            n_events, cls.ctypes.data, counts.ctypes.data))
        return cls[:n_roads], counts[:n_events]

    def batch_run_host(self, clusters, layer_offsets, vertices, roads_capacity=None):
        """Host in / host out over a batch; returns (roads, road_offsets)."""
        clusters = np.ascontiguousarray(clusters, CLUSTER_DTYPE)
        layer_offsets = np.ascontiguousarray(layer_offsets, np.int32)
        vertices = np.ascontiguousarray(vertices, np.float32)
        n_events = (len(layer_offsets) - 1) // 7
        offs = np.zeros(n_events + 1, np.int32)
        if roads_capacity is None:
            self._check(self.lib.itsu_batch_run_host(self.h, _ptr(clusters), _ptr(layer_offsets), _ptr(vertices), n_events,
                                                     None, 0, _ptr(offs)))
            roads_capacity = int(offs[-1])
        roads = np.zeros(roads_capacity, ROAD_DTYPE)
        self._check(self.lib.itsu_batch_run_host(self.h, _ptr(clusters), _ptr(layer_offsets), _ptr(vertices), n_events,
                                                 _ptr(roads), roads_capacity, _ptr(offs)))
        roads = roads[: offs[-1]].copy()
        roads["pad"] = 0
        return roads, offs

    def _batch_run_host_records(self, fn_name, dtype, records, layer_offsets, vertices, roads_capacity):
        records = np.ascontiguousarray(records, dtype)
        fn = getattr(self.lib, fn_name)
        layer_offsets = np.ascontiguousarray(layer_offsets, np.int32)
        vertices = np.ascontiguousarray(vertices, np.float32)
        n_events = (len(layer_offsets) - 1) // 7
        offs = np.zeros(n_events + 1, np.int32)
        if roads_capacity is None:
            self._check(fn(self.h, _ptr(records), _ptr(layer_offsets), _ptr(vertices), n_events, None, 0, _ptr(offs)))
            roads_capacity = int(offs[-1])
        roads = np.zeros(roads_capacity, ROAD_DTYPE)
        self._check(fn(self.h, _ptr(records), _ptr(layer_offsets), _ptr(vertices), n_events, _ptr(roads), roads_capacity,
                       _ptr(offs)))
        roads = roads[: offs[-1]].copy()
        roads["pad"] = 0
        return roads, offs

    def atan2f_device(self, y_ptr, x_ptr, out_ptr, n):
        """The device's correctly rounded atan2 on n device-resident argument pairs."""
        self._check(self.lib.itsu_atan2f_device(self.h, ctypes.c_void_p(y_ptr), ctypes.c_void_p(x_ptr),
                                                ctypes.c_void_p(out_ptr), n))

    def batch_run_host_compact(self, clusters_in, layer_offsets, vertices, roads_capacity=None):
        """batch_run_host with 24-byte input records (CLUSTER_IN_DTYPE); returns (roads, road_offsets)."""
        return self._batch_run_host_records("itsu_batch_run_host_compact", CLUSTER_IN_DTYPE, clusters_in, layer_offsets,
                                            vertices, roads_capacity)

    def batch_run_host_tracks(self, clusters_track, layer_offsets, vertices, roads_capacity=None):
        """batch_run_host with 16-byte input records (CLUSTER_TRACK_DTYPE); returns (roads, road_offsets)."""
        return self._batch_run_host_records("itsu_batch_run_host_tracks", CLUSTER_TRACK_DTYPE, clusters_track, layer_offsets,
                                            vertices, roads_capacity)

    def batch_device(self, clusters_ptr, layer_offsets_ptr, vertices_ptr, n_events, n_clusters) -> Batch:
        b = Batch()
        b.clusters, b.layer_offsets, b.vertices = clusters_ptr, layer_offsets_ptr, vertices_ptr
        b.n_events, b.n_clusters = n_events, n_clusters
        return b

    def batch_run(self, batch: Batch):
        self._check(self.lib.itsu_batch_run(self.h, ctypes.byref(batch)))

    def batch_launch(self, batch: Batch):
        self._check(self.lib.itsu_batch_launch(self.h, ctypes.byref(batch)))

    def batch_status(self):
        self._check(self.lib.itsu_batch_status(self.h))

    def profile(self, repeats: int = 5) -> list:
        """(kernel name, mean ms) for every kernel of the last batch, timed one by one."""
        n = self.lib.itsu_kernels_per_run() + 8  # the learned form launches more
        arr = (KernelTime * n)()
        cnt = ctypes.c_int32()
        self._check(self.lib.itsu_batch_profile(self.h, repeats, arr, n, ctypes.byref(cnt)))
        return [(arr[k].name.decode(), float(arr[k].ms)) for k in range(min(cnt.value, n))]

    def frames_run_host(self, clusters, frame_offsets, vertices, vertex_frame, roads_capacity=None):
        """Pile-up frames: each frame's clusters once, one run per vertex; returns (roads, road_offsets)."""
        clusters = np.ascontiguousarray(clusters, CLUSTER_DTYPE)
        frame_offsets = np.ascontiguousarray(frame_offsets, np.int32)
        vertices = np.ascontiguousarray(vertices, np.float32)
        vertex_frame = np.ascontiguousarray(vertex_frame, np.int32)
        f = Frames()
        f.clusters, f.frame_offsets, f.vertices, f.vertex_frame = (_ptr(clusters).value, _ptr(frame_offsets).value,
                                                                   _ptr(vertices).value, _ptr(vertex_frame).value)
        f.n_frames, f.n_vertices = (len(frame_offsets) - 1) // 7, len(vertex_frame)
        offs = np.zeros(f.n_vertices + 1, np.int32)
        if roads_capacity is None:
            self._check(self.lib.itsu_frames_run_host(self.h, ctypes.byref(f), None, 0, _ptr(offs)))
            roads_capacity = int(offs[-1])
        roads = np.zeros(roads_capacity, ROAD_DTYPE)
        self._check(self.lib.itsu_frames_run_host(self.h, ctypes.byref(f), _ptr(roads), roads_capacity, _ptr(offs)))
        roads = roads[: offs[-1]].copy()
        roads["pad"] = 0
        return roads, offs

    def relaunch(self):
        self._check(self.lib.itsu_relaunch(self.h))

    def autotune(self, repeats: int = 3) -> dict:
        """Tune the launch shape for the band of the last run; returns the chosen entry."""
        t = Tune()
        self._check(self.lib.itsu_autotune(self.h, repeats, ctypes.byref(t)))
        return dict(band=t.band, threads_per_block=t.threads_per_block, blocks_per_sm=t.blocks_per_sm, prune=t.prune, ms=t.ms,
                    events_per_group=t.events_per_group)

    def set_tune(self, band: int, threads_per_block: int, blocks_per_sm: int, prune: int = 1, events_per_group: int = 0):
        t = Tune(band, threads_per_block, blocks_per_sm, prune, 0.0, events_per_group)
        self._check(self.lib.itsu_set_tune(self.h, ctypes.byref(t)))

    def get_tune(self, band: int) -> dict:
        t = Tune()
        self._check(self.lib.itsu_get_tune(self.h, band, ctypes.byref(t)))
        return dict(band=t.band, threads_per_block=t.threads_per_block, blocks_per_sm=t.blocks_per_sm, prune=t.prune, ms=t.ms,
                    events_per_group=t.events_per_group)

    # ---- learned prefilter ----

    def prefilter_set_model(self, model: PrefilterModel):
        self._check(self.lib.itsu_prefilter_set_model(self.h, ctypes.byref(model)))

    def prefilter_get_model(self) -> PrefilterModel:
        m = PrefilterModel()
        self._check(self.lib.itsu_prefilter_get_model(self.h, ctypes.byref(m)))
        return m

    def prefilter_enable(self, enable: bool = True):
        self._check(self.lib.itsu_prefilter_enable(self.h, 1 if enable else 0))

    def prefilter_export(self, features=0, labels=0, capacity=0, road_cells=0, road_keys=0, road_fake=0, road_capacity=0):
        """Device pointers (ints) of the buffers to fill; returns (n_cells, n_roads)."""
        s = PrefilterSamples()
        s.features, s.labels, s.capacity = features or None, labels or None, capacity
        s.road_cells, s.road_keys, s.road_fake, s.road_capacity = road_cells or None, road_keys or None, road_fake or None, road_capacity
        self._check(self.lib.itsu_prefilter_export(self.h, ctypes.byref(s)))
        return s.n_cells, s.n_roads

    def prefilter_score(self, features_ptr: int, n: int, logits_ptr: int):
        self._check(self.lib.itsu_prefilter_score(self.h, ctypes.c_void_p(features_ptr), n, ctypes.c_void_p(logits_ptr)))

    def prefilter_train(self, features_ptr: int, labels_ptr: int, n: int, cfg: TrainConfig) -> np.ndarray:
        losses = np.zeros(max(int(cfg.steps), 1), np.float32)
        self._check(self.lib.itsu_prefilter_train(self.h, ctypes.c_void_p(features_ptr), ctypes.c_void_p(labels_ptr), n,
                                                  ctypes.byref(cfg), _ptr(losses)))
        return losses[:int(cfg.steps)]

    def prefilter_gradient(self, features_ptr: int, labels_ptr: int, n: int, pos_weight: float = 1.0):
        grad = np.zeros(MLP_PARAMS, np.float32)
        loss = ctypes.c_float()
        self._check(self.lib.itsu_prefilter_gradient(self.h, ctypes.c_void_p(features_ptr), ctypes.c_void_p(labels_ptr), n,
                                                     pos_weight, _ptr(grad), ctypes.byref(loss)))
        return grad, loss.value

    # ---- learned tracklet gate ----

    def gate_set_model(self, model: GateModel):
        self._check(self.lib.itsu_gate_set_model(self.h, ctypes.byref(model)))

    def gate_get_model(self) -> GateModel:
        m = GateModel()
        self._check(self.lib.itsu_gate_get_model(self.h, ctypes.byref(m)))
        return m

    def gate_enable(self, enable: bool = True):
        self._check(self.lib.itsu_gate_enable(self.h, 1 if enable else 0))

    def gate_export(self, features=0, labels=0, capacity=0, road_tracklets=0, road_capacity=0):
        """Device pointers (ints) of the buffers to fill; returns (n_tracklets, n_roads)."""
        s = GateSamples()
        s.features, s.labels, s.capacity = features or None, labels or None, capacity
        s.road_tracklets, s.road_capacity = road_tracklets or None, road_capacity
        self._check(self.lib.itsu_gate_export(self.h, ctypes.byref(s)))
        return s.n_tracklets, s.n_roads

    def gate_score(self, features_ptr: int, n: int, logits_ptr: int):
        self._check(self.lib.itsu_gate_score(self.h, ctypes.c_void_p(features_ptr), n, ctypes.c_void_p(logits_ptr)))

    def gate_train(self, features_ptr: int, labels_ptr: int, n: int, cfg: TrainConfig) -> np.ndarray:
        losses = np.zeros(max(int(cfg.steps), 1), np.float32)
        self._check(self.lib.itsu_gate_train(self.h, ctypes.c_void_p(features_ptr), ctypes.c_void_p(labels_ptr), n,
                                             ctypes.byref(cfg), _ptr(losses)))
        return losses[:int(cfg.steps)]

    def gate_gradient(self, features_ptr: int, labels_ptr: int, n: int, pos_weight: float = 1.0):
        grad = np.zeros(GATE_PARAMS, np.float32)
        loss = ctypes.c_float()
        self._check(self.lib.itsu_gate_gradient(self.h, ctypes.c_void_p(features_ptr), ctypes.c_void_p(labels_ptr), n,
                                                pos_weight, _ptr(grad), ctypes.byref(loss)))
        return grad, loss.value
