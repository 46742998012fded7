"""B200-native GustANN all-in-GPU search path.

Python mirror of the reference's host interface (``gustann::GustANN``,
src/ssd_search.hpp:18-83) over the C ABI of ``libgann.so`` (include/gann.h):

    g = GustANN(DataType.UINT8)
    g.init_pure_mem(GustANNConfig(index_file, pq_file_prefix, nav_graph_prefix), use_gpu_mem=True)
    g.search(qdata, num_queries, topk, ef_search, nns, distances, found_cnt, stats)

Errors are raised as :class:`GustANNError` carrying the ABI status code (the
reference aborts, exits or throws instead). The search runs only through the
CUDA library; there is no CPU fallback, and importing fails loudly when the
library has not been built.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "libgann.so"
_lib = None

GANN_OK, GANN_EINVAL, GANN_EIO, GANN_EFORMAT, GANN_ECUDA, GANN_ENOMEM, GANN_EKERNEL, GANN_ERANGE, GANN_EBUSY = range(9)
GANN_OPEN_NO_VALIDATE, GANN_OPEN_HOST_PAGES = 1, 2
PREC_FP32, PREC_BF16, PREC_BF16X3, PREC_BF16_CC = 0, 1, 2, 3
ENTRY_NAV_WALK, ENTRY_NEAREST_PIVOT = 0, 1


class DataType(enum.IntEnum):
    """gustann::DataType, src/common.hpp:22-25."""

    UINT8 = 0
    FLOAT = 1


@dataclass
class GustANNConfig:
    """gustann::GustANNConfig, src/ssd_search.hpp:18-23."""

    index_file: str = ""
    pq_file_prefix: str = ""
    nav_graph_prefix: str = ""


@dataclass
class GustANNStats:
    """gustann::GustANNStats, src/ssd_search.hpp:25-27 (seconds)."""

    run_time: float = 0.0


class GustANNError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[gann status {code}] {msg}")
        self.code = code


class BatchOpts(ctypes.Structure):
    """gann_batch_opts_t (include/gann.h)."""

    _fields_ = [("precision", ctypes.c_int32), ("beam_width", ctypes.c_int32), ("hash_bits", ctypes.c_int32),
                ("entry", ctypes.c_int32), ("reserved", ctypes.c_int32 * 4)]


class ServerOpts(ctypes.Structure):
    """gann_server_opts_t (include/gann.h)."""

    _fields_ = [("max_batch", ctypes.c_int32), ("streams", ctypes.c_int32), ("topk_max", ctypes.c_int32),
                ("ef_max", ctypes.c_int32), ("precision", ctypes.c_int32), ("beam_width", ctypes.c_int32),
                ("hash_bits", ctypes.c_int32), ("max_wait_us", ctypes.c_int32), ("min_batch", ctypes.c_int32),
                ("mem_budget_kib", ctypes.c_int32), ("entry", ctypes.c_int32), ("reserved", ctypes.c_int32 * 5)]


class LoadStats(ctypes.Structure):
    """gann_load_stats_t (include/gann.h)."""

    _fields_ = [("offered_qps", ctypes.c_double), ("achieved_qps", ctypes.c_double), ("submitted", ctypes.c_int64),
                ("rejected", ctypes.c_int64), ("completed", ctypes.c_int64), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("p999_ms", ctypes.c_double), ("mean_ms", ctypes.c_double)]


class GannInfo(ctypes.Structure):
    _fields_ = [
        ("num_points", ctypes.c_int64), ("dim", ctypes.c_int64), ("max_degree", ctypes.c_int64),
        ("medoid", ctypes.c_int64), ("node_len", ctypes.c_int64), ("nodes_per_page", ctypes.c_int64),
        ("num_pages", ctypes.c_int64), ("pq_chunks", ctypes.c_int32), ("dtype", ctypes.c_int32),
        ("has_nav", ctypes.c_int32), ("nav_points", ctypes.c_int32), ("nav_max_degree", ctypes.c_int32),
        ("device", ctypes.c_int32), ("device_bytes", ctypes.c_int64),
        ("host_pages", ctypes.c_int32), ("reserved0", ctypes.c_int32), ("host_bytes", ctypes.c_int64),
    ]


_P = ctypes.c_void_p
_I = ctypes.c_int
_SIGNATURES = {
    "gann_open": (_I, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _I, _I, ctypes.POINTER(_P)]),
    "gann_close": (_I, [_P]),
    "gann_get_info": (_I, [_P, ctypes.POINTER(GannInfo)]),
    "gann_search": (_I, [_P, _P, _I, _I, _I, _P, _P, _P, ctypes.POINTER(ctypes.c_double)]),
    "gann_search_device": (_I, [_P, _P, _I, _I, _I, _P, _P, _P, _P]),
    "gann_search_device_ex": (_I, [_P, _P, _I, _I, _I, _P, _P, _P, _P, _P, _P]),
    "gann_search_batch": (_I, [_P, _P, _I, _P, _P, _I, _I, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_double)]),
    "gann_search_batch_device": (_I, [_P, _P, _I, _P, _P, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "gann_search_batch_noalloc": (_I, [_P, _P, _I, _I, _I, _P, _P, _P, _P, _P]),
    "gann_batch_graph_create": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, ctypes.POINTER(_P)]),
    "gann_batch_graph_launch": (_I, [_P, _P]),
    "gann_batch_graph_destroy": (_I, [_P]),
    "gann_cache_hot_records": (_I, [_P, _P, _I, _I, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "gann_pq_tables": (_I, [_P, _P, _I, _I, _P]),
    "gann_autotune": (_I, [_P, _P, _I, _I, _I, _I, _P, ctypes.POINTER(ctypes.c_double)]),
    "gann_server_start": (_I, [_P, ctypes.POINTER(ServerOpts), ctypes.POINTER(_P)]),
    "gann_server_submit": (_I, [_P, _P, _I, _I, ctypes.c_uint64]),
    "gann_server_request_bytes": (ctypes.c_int64, [_P, _I, _I]),
    "gann_nearest_pivots": (_I, [_P, _P, _I, _P, _P, _P]),
    "gann_server_poll": (_I, [_P, _I, _P, _P, _P, _P, _P, ctypes.POINTER(_I)]),
    "gann_server_stop": (_I, [_P]),
    "gann_server_open_loop": (_I, [_P, _P, _I, _P, _P, ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                                   ctypes.POINTER(LoadStats)]),
    "gann_check": (_I, [_P, _P]),
    "gann_set_fma": (_I, [_P, _I, _I]),
    "gann_last_error": (ctypes.c_char_p, []),
    "gann_sample_pivots": (_I, [ctypes.c_int64, ctypes.c_int64, ctypes.c_uint32, _P]),
    "gann_build_prune": (_I, [_P, _I, ctypes.c_int64, _I, _P, _P, ctypes.c_int64, _I, _I, ctypes.c_float, _P, _P]),
}


def lib() -> ctypes.CDLL:
    """Load libgann.so (built in-tree by gustann_b200/build.py)."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise ImportError(f"{_LIB_PATH} is missing: run `python gustann_b200/build.py` "
                              "(the search path has no CPU fallback)")
        L = ctypes.CDLL(str(_LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def _check(rc: int) -> None:
    if rc != GANN_OK:
        msg = lib().gann_last_error()
        raise GustANNError(rc, msg.decode() if msg else "")


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


_CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy


def _stream(stream):
    """None -> NULL (the handle's stream); 0 (torch's legacy default stream) ->
    cudaStreamLegacy; anything else is passed through."""
    if stream is None:
        return None
    return _CUDA_STREAM_LEGACY if stream == 0 else stream


def sample_pivots(num_data: int, num_samp: int, seed: int = 114514) -> np.ndarray:
    """The pivot-graph sample of bin/gen_small_file.cpp:12-25 (sorted global ids)."""
    out = np.empty(num_samp, dtype=np.int32)
    _check(lib().gann_sample_pivots(num_data, num_samp, seed, _ptr(out)))
    return out


class GustANN:
    """gustann::GustANN (src/ssd_search.hpp:29-83), all-in-GPU mode."""

    def __init__(self, data_type: DataType = DataType.FLOAT):
        self.data_type = DataType(data_type)
        self._h = None

    def init_pure_mem(self, config: GustANNConfig, use_gpu_mem: bool = True, validate: bool = True) -> None:
        """GustANN::init_pure_mem (src/ssd_search.cu:108-112). ``use_gpu_mem=True``
        (``-G``) makes the records resident in HBM; ``False`` keeps them in pinned
        host memory that the kernels read over PCIe/C2C (src/pure_mem.cu:51-66),
        with codes, pivots and the pivot graph in HBM. Results are the same."""
        if self._h is not None:
            self.close()
        h = _P()
        nav = config.nav_graph_prefix.encode() if config.nav_graph_prefix else None
        _check(lib().gann_open(config.index_file.encode(), config.pq_file_prefix.encode(), nav,
                               int(self.data_type),
                               (0 if validate else GANN_OPEN_NO_VALIDATE) |
                               (0 if use_gpu_mem else GANN_OPEN_HOST_PAGES), ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        if self._h is None:
            raise GustANNError(GANN_EINVAL, "not initialised: call init_pure_mem first")
        return self._h

    def info(self) -> dict:
        inf = GannInfo()
        _check(lib().gann_get_info(self.handle, ctypes.byref(inf)))
        return {f: getattr(inf, f) for f, _ in GannInfo._fields_}

    def set_fma(self, table: bool, exact: bool) -> None:
        _check(lib().gann_set_fma(self.handle, int(table), int(exact)))

    def search(self, qdata: np.ndarray, num_queries: int, topk: int, ef_search: int, nns: np.ndarray,
               distances: np.ndarray, found_cnt: np.ndarray, stats: GustANNStats | None = None) -> None:
        """GustANN::search (src/ssd_search.hpp:78-80): fills nns (nq x topk int32),
        distances (nq x topk float32, squared L2) and found_cnt (nq int32)."""
        q = np.ascontiguousarray(qdata, dtype=np.float32)
        for a, dt in ((nns, np.int32), (distances, np.float32), (found_cnt, np.int32)):
            if a.dtype != dt or not a.flags.c_contiguous:
                raise GustANNError(GANN_EINVAL, "output buffers must be C-contiguous int32/float32/int32")
        if q.size < num_queries * self.info()["dim"] or nns.size < num_queries * topk or \
                distances.size < num_queries * topk or found_cnt.size < num_queries:
            raise GustANNError(GANN_EINVAL, "buffer smaller than num_queries requires")
        t = ctypes.c_double(0.0)
        _check(lib().gann_search(self.handle, _ptr(q), int(num_queries), int(topk), int(ef_search),
                                 _ptr(nns), _ptr(distances), _ptr(found_cnt), ctypes.byref(t)))
        if stats is not None:
            stats.run_time = t.value

    def query(self, q: np.ndarray, topk: int, ef_search: int):
        """Convenience form of :meth:`search` returning (ids, distances, found, seconds)."""
        q = np.ascontiguousarray(q, dtype=np.float32)
        nq = q.shape[0]
        nns = np.zeros((nq, topk), np.int32)
        dis = np.zeros((nq, topk), np.float32)
        fnd = np.zeros(nq, np.int32)
        st = GustANNStats()
        self.search(q, nq, topk, ef_search, nns, dis, fnd, st)
        return nns, dis, fnd, st.run_time

    def search_device(self, d_q: int, nq: int, topk: int, ef_search: int, d_nns: int, d_dists: int,
                      d_found: int, stream: int | None = None) -> None:
        """Device-pointer form (gann_search_device); enqueued without a host sync.
        ``stream``: a cudaStream_t value (0 = the legacy default stream, as torch
        reports it), or None for the handle's own stream."""
        _check(lib().gann_search_device(self.handle, d_q, nq, topk, ef_search, d_nns, d_dists, d_found,
                                        _stream(stream)))

    def search_device_ex(self, d_q: int, nq: int, topk: int, ef_search: int, d_nns: int, d_dists: int,
                         d_found: int, d_hops: int = 0, d_bytes: int = 0, stream: int | None = None) -> None:
        """gann_search_device_ex: also writes per-query hop and gathered-byte counters."""
        _check(lib().gann_search_device_ex(self.handle, d_q, nq, topk, ef_search, d_nns, d_dists, d_found,
                                           d_hops or None, d_bytes or None, _stream(stream)))

    @staticmethod
    def _opts(precision, beam_width, hash_bits, entry=ENTRY_NAV_WALK):
        o = BatchOpts()
        o.precision, o.beam_width, o.hash_bits, o.entry = int(precision), int(beam_width), int(hash_bits), int(entry)
        return o

    def search_batch(self, q: np.ndarray, topk, ef_search, precision: int = PREC_BF16, beam_width: int = 0,
                     hash_bits: int = 0, entry: int = ENTRY_NAV_WALK):
        """Batched search (gann_search_batch). ``topk`` / ``ef_search`` are ints or
        per-query int arrays. Returns (ids nq x kmax, distances, found, seconds)."""
        q = np.ascontiguousarray(q, dtype=np.float32)
        nq = q.shape[0]
        karr = None if np.isscalar(topk) else np.ascontiguousarray(topk, dtype=np.int32)
        larr = None if np.isscalar(ef_search) else np.ascontiguousarray(ef_search, dtype=np.int32)
        kmax = int(topk) if karr is None else int(karr.max(initial=1))
        lmax = int(ef_search) if larr is None else int(larr.max(initial=1))
        nns = np.zeros((nq, kmax), np.int32)
        dis = np.zeros((nq, kmax), np.float32)
        fnd = np.zeros(nq, np.int32)
        t = ctypes.c_double(0.0)
        o = self._opts(precision, beam_width, hash_bits, entry)
        _check(lib().gann_search_batch(self.handle, _ptr(q), nq, None if karr is None else _ptr(karr),
                                       None if larr is None else _ptr(larr), kmax, lmax, ctypes.byref(o),
                                       _ptr(nns), _ptr(dis), _ptr(fnd), ctypes.byref(t)))
        return nns, dis, fnd, t.value

    def search_batch_device(self, d_q: int, nq: int, d_topk: int, d_ef: int, topk_max: int, ef_max: int,
                            d_nns: int, d_dists: int, d_found: int, d_hops: int = 0, d_bytes: int = 0,
                            precision: int = PREC_BF16, beam_width: int = 0, hash_bits: int = 0,
                            stream: int | None = None, entry: int = ENTRY_NAV_WALK) -> None:
        o = self._opts(precision, beam_width, hash_bits, entry)
        _check(lib().gann_search_batch_device(self.handle, d_q, nq, d_topk or None, d_ef or None, topk_max, ef_max,
                                              ctypes.byref(o), d_nns, d_dists, d_found, d_hops or None,
                                              d_bytes or None, _stream(stream)))

    def nearest_pivots(self, d_q: int, nq: int, d_pivot: int, d_node: int, stream: int | None = None) -> None:
        """gann_nearest_pivots: per query, the nearest pivot's row and node id (device buffers)."""
        _check(lib().gann_nearest_pivots(self.handle, d_q, nq, d_pivot or None, d_node or None, _stream(stream)))

    def autotune(self, d_q: int, nq: int, topk: int, ef_search: int, precision: int = PREC_BF16):
        """gann_autotune: returns (beam_width, hash_bits, seconds) of the fastest
        configuration, which becomes this handle's default."""
        o = BatchOpts()
        t = ctypes.c_double(0.0)
        _check(lib().gann_autotune(self.handle, d_q, nq, topk, ef_search, int(precision), ctypes.byref(o),
                                   ctypes.byref(t)))
        return o.beam_width, o.hash_bits, t.value

    def pq_tables(self, q: np.ndarray, precision: int) -> np.ndarray:
        """PQ tables (nq x M x 256, FP32 view) as the given precision builds them."""
        q = np.ascontiguousarray(q, dtype=np.float32)
        M = self.info()["pq_chunks"]
        out = np.zeros((q.shape[0], M, 256), np.float32)
        _check(lib().gann_pq_tables(self.handle, _ptr(q), q.shape[0], int(precision), _ptr(out)))
        return out

    def cache_hot_records(self, d_q: int, nq: int, ef_search: int, max_bytes: int) -> int:
        """gann_cache_hot_records (host-memory records only): copy the records a
        sample batch of nq device queries expands most into HBM, up to max_bytes.
        Returns the number of records cached."""
        n = ctypes.c_int64(0)
        _check(lib().gann_cache_hot_records(self.handle, d_q, nq, ef_search, int(max_bytes), ctypes.byref(n)))
        return n.value

    def check(self, stream: int | None = None) -> None:
        _check(lib().gann_check(self.handle, _stream(stream)))

    def close(self) -> None:
        if self._h is not None:
            lib().gann_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchGraph:
    """A batched search captured once as a CUDA graph (gann_batch_graph_*).
    The device buffers (ints are device addresses) are fixed at capture; each
    launch processes the number of queries held in the device int at ``d_nq``."""

    def __init__(self, index: GustANN, max_nq: int, topk_max: int, ef_max: int, d_q: int, d_nq: int, d_nns: int,
                 d_dists: int, d_found: int, d_topk: int = 0, d_ef: int = 0, precision: int = PREC_BF16,
                 beam_width: int = 0, hash_bits: int = 0):
        self.index = index
        o = index._opts(precision, beam_width, hash_bits)
        self._g = _P()
        _check(lib().gann_batch_graph_create(index.handle, max_nq, topk_max, ef_max, ctypes.byref(o), d_q,
                                             d_topk or None, d_ef or None, d_nq, d_nns, d_dists, d_found,
                                             ctypes.byref(self._g)))

    def launch(self, stream: int | None = None) -> None:
        _check(lib().gann_batch_graph_launch(self._g, _stream(stream)))

    def destroy(self) -> None:
        if self._g:
            lib().gann_batch_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Server:
    """Continuous-batching server over one open index (gann_server_*)."""

    def __init__(self, index: GustANN, max_batch: int = 1024, streams: int = 4, topk_max: int = 100,
                 ef_max: int = 512, precision: int = PREC_BF16X3, beam_width: int = 0, hash_bits: int = 0,
                 max_wait_us: int = 100, min_batch: int = 0, mem_budget_kib: int = 0, entry: int = ENTRY_NAV_WALK):
        self.index = index
        self.dim = index.info()["dim"]
        o = ServerOpts()
        (o.max_batch, o.streams, o.topk_max, o.ef_max, o.precision, o.beam_width, o.hash_bits, o.max_wait_us,
         o.min_batch, o.mem_budget_kib, o.entry) = (max_batch, streams, topk_max, ef_max, precision, beam_width,
                                                    hash_bits, max_wait_us, min_batch, mem_budget_kib, entry)
        self.topk_max = topk_max
        self._s = _P()
        _check(lib().gann_server_start(index.handle, ctypes.byref(o), ctypes.byref(self._s)))

    def request_bytes(self, topk: int, ef_search: int) -> int:
        """The admission charge of one request (gann_server_request_bytes)."""
        return int(lib().gann_server_request_bytes(self._s, topk, ef_search))

    def submit(self, query: np.ndarray, topk: int, ef_search: int, tag: int) -> bool:
        """False when the server's request budget is full (GANN_EBUSY)."""
        q = np.ascontiguousarray(query, dtype=np.float32).reshape(-1)
        rc = lib().gann_server_submit(self._s, _ptr(q), int(topk), int(ef_search), int(tag))
        if rc == GANN_EBUSY:
            return False
        _check(rc)
        return True

    def poll(self, max_results: int = 4096):
        tags = np.zeros(max_results, np.uint64)
        ids = np.zeros((max_results, self.topk_max), np.int32)
        dis = np.zeros((max_results, self.topk_max), np.float32)
        fnd = np.zeros(max_results, np.int32)
        lat = np.zeros(max_results, np.float64)
        n = ctypes.c_int(0)
        _check(lib().gann_server_poll(self._s, max_results, _ptr(tags), _ptr(ids), _ptr(dis), _ptr(fnd), _ptr(lat),
                                      ctypes.byref(n)))
        k = n.value
        return tags[:k], ids[:k], dis[:k], fnd[:k], lat[:k]

    def open_loop(self, queries: np.ndarray, rate_qps: float, seconds: float, topk=None, ef_search=None,
                  seed: int = 1) -> dict:
        q = np.ascontiguousarray(queries, dtype=np.float32)
        ka = None if topk is None else np.ascontiguousarray(topk, dtype=np.int32)
        la = None if ef_search is None else np.ascontiguousarray(ef_search, dtype=np.int32)
        st = LoadStats()
        _check(lib().gann_server_open_loop(self._s, _ptr(q), q.shape[0], None if ka is None else _ptr(ka),
                                           None if la is None else _ptr(la), float(rate_qps), float(seconds),
                                           int(seed), ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in LoadStats._fields_}

    def stop(self) -> None:
        if self._s:
            lib().gann_server_stop(self._s)
            self._s = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass
