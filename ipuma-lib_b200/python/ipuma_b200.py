"""ctypes binding of the C ABI in include/ipuma_b200.h.

Loads the in-tree ``libipuma_b200.so`` (built by ``make -C ipuma-lib_b200``);
there is no fallback: a missing library or device raises.  Used by the
tests, ``bench.py`` and ``__graft_entry__``; C and C++ callers link the
library directly.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "libipuma_b200.so")

OK = 0
ERR_INVALID_ARG = -1
ERR_CUDA = -2
ERR_NO_DEVICE = -3
ERR_TOO_LONG = -4
ERR_OUT_OF_BUCKETS = -5
ERR_BAD_SEQUENCE = -6
ERR_TIMEOUT = -7
ERR_NO_MEMORY = -8
ERR_UNKNOWN_JOB = -9
ERR_DEVICE = -10
ERR_CLOSED = -11

SIM = {"na": 0, "blosum50": 1, "blosum62": 2, "simple": 3}
DT = {"na": 0, "aa": 1, "str": 2}

# Every symbol include/ipuma_b200.h declares.
EXPORTS = [
    "ipuma_last_error", "ipuma_version", "ipuma_device_count", "ipuma_encode",
    "ipuma_select_matrix", "ipuma_input_buffer_words", "ipuma_gpu_create", "ipuma_gpu_destroy",
    "ipuma_gpu_set_option", "ipuma_gpu_run_buffer", "ipuma_gpu_submit_buffer", "ipuma_gpu_poll",
    "ipuma_gpu_join", "ipuma_gpu_compare", "ipuma_gpu_compare_device", "ipuma_gpu_last_stats",
    "ipuma_gpu_run_buffer_device", "ipuma_measure_int_peak", "ipuma_gpu_compare_noalloc",
    "ipuma_gpu_autotune", "ipuma_gpu_tuning", "ipuma_server_create", "ipuma_server_submit",
    "ipuma_server_poll", "ipuma_server_wait", "ipuma_server_get_stats", "ipuma_server_close",
    "ipuma_server_destroy", "ipuma_server_add_sequences", "ipuma_server_submit_resident",
    "ipuma_gpu_reserve", "ipuma_gpu_join_stats", "ipuma_host_alloc", "ipuma_host_free",
    "ipuma_gpu_compare_packed", "ipuma_pack_codes", "ipuma_gpu_compare_device_packed",
]

KERNEL_NAMES = {0: "k_batched<s32,L32,K16>", 1: "k_batched<s16x2,L16,K4>",
                2: "k_batched<s16x2,L16,K8>", 3: "k_batched<s16x2,L16,K12>",
                4: "k_batched<s16x2,L16,K16>", 5: "k_batched<s16x2,L32,K12>",
                6: "k_batched<s16x2,L32,K16>", 7: "k_batched<s32,L32,K16> rerun",
                8: "k_plain<K>", 9: "k_exact", 10: "k_thread<s16x2,K16>",
                11: "k_batched<s16x2,L16,K6>", 12: "k_batched<s16x2,L16,K10>",
                13: "k_batched<s16x2,L16,K14>", 14: "k_batched<s16x2,L16,K5>",
                15: "k_batched<s16x2,L16,K7>", 16: "k_batched<s16x2,L16,K9>",
                17: "k_batched<s16x2,L16,K11>", 18: "k_batched<s16x2,L16,K13>",
                19: "k_batched<s16x2,L16,K15>", 20: "k_hybrid<b16x2->s32,L32,K16>",
                21: "k_plain16<K>", 22: "k_batched<s16x2,L8,K8>",
                23: "k_batched<s16x2,L8,K10>", 24: "k_batched<s16x2,L8,K12>",
                25: "k_batched<s16x2,L8,K14>", 26: "k_batched<s16x2,L8,K16>",
                27: "k_strips<s16x2,L32,K16> team"}
MAX_TIMED = 24  # IPUMA_MAX_TIMED


class SwConfig(ctypes.Structure):
    _fields_ = [("gap_init", ctypes.c_int32), ("gap_extend", ctypes.c_int32),
                ("match_value", ctypes.c_int32), ("mismatch_value", ctypes.c_int32),
                ("ambiguity_value", ctypes.c_int32), ("similarity", ctypes.c_int32),
                ("datatype", ctypes.c_int32)]


class AlgoConfig(ctypes.Structure):
    _fields_ = [("tiles_used", ctypes.c_int32), ("max_ab", ctypes.c_int32),
                ("max_batches", ctypes.c_int32), ("bufsize", ctypes.c_int32),
                ("vtype", ctypes.c_int32), ("fill_algo", ctypes.c_int32),
                ("forward_only", ctypes.c_int32), ("use_remote_buffer", ctypes.c_int32),
                ("transmission_programs", ctypes.c_int32), ("io_tiles", ctypes.c_int32)]


class Pair(ctypes.Structure):
    _fields_ = [("a_off", ctypes.c_int64), ("b_off", ctypes.c_int64), ("a_len", ctypes.c_int32),
                ("b_len", ctypes.c_int32)]


PAIR_DTYPE = np.dtype([("a_off", "<i8"), ("b_off", "<i8"), ("a_len", "<i4"), ("b_len", "<i4")])
assert PAIR_DTYPE.itemsize == ctypes.sizeof(Pair) == 24


class Stats(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("cells", ctypes.c_int64), ("pairs", ctypes.c_int64),
                ("s32_pairs", ctypes.c_int64), ("overflow_reruns", ctypes.c_int64),
                ("launches", ctypes.c_int32), ("used_graph", ctypes.c_int32),
                ("n_timed", ctypes.c_int32), ("timed_kind", ctypes.c_int32 * MAX_TIMED),
                ("timed_ms", ctypes.c_double * MAX_TIMED), ("timed_cells", ctypes.c_int64 * MAX_TIMED),
                ("chunks", ctypes.c_int32), ("n_trace", ctypes.c_int32),
                ("trace_kind", ctypes.c_int32 * MAX_TIMED),
                ("trace_start_ms", ctypes.c_double * MAX_TIMED),
                ("trace_end_ms", ctypes.c_double * MAX_TIMED),
                ("trace_cells", ctypes.c_int64 * MAX_TIMED),
                ("host_check_ms", ctypes.c_double), ("host_wall_ms", ctypes.c_double)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("n_scorings", ctypes.c_int32), ("scorings", ctypes.POINTER(SwConfig)),
                ("forward_only", ctypes.c_int32), ("slots", ctypes.c_int32),
                ("pool_bytes", ctypes.c_int64), ("max_batch_pairs", ctypes.c_int32),
                ("device", ctypes.c_int32), ("one_request_per_batch", ctypes.c_int32),
                ("max_batch_cells", ctypes.c_int64), ("reserve_b_len", ctypes.c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("submitted", "completed", "queued", "batches",
                                               "pairs", "cells", "max_batch_pairs",
                                               "pool_bytes", "pool_used", "max_pool_used")] + \
               [("busy_ms", ctypes.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libipuma_b200.so is not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_size_t
        L.ipuma_last_error.restype = ctypes.c_char_p
        L.ipuma_version.restype = ctypes.c_char_p
        L.ipuma_device_count.restype = i32
        L.ipuma_encode.argtypes = [i32, ctypes.c_char_p, sz, vp]
        L.ipuma_select_matrix.argtypes = [i32, i32, i32, i32, vp, sz, vp, vp]
        L.ipuma_input_buffer_words.argtypes = [ctypes.POINTER(AlgoConfig)]
        L.ipuma_input_buffer_words.restype = i64
        L.ipuma_gpu_create.argtypes = [ctypes.POINTER(SwConfig), ctypes.POINTER(AlgoConfig), i32,
                                       ctypes.POINTER(vp)]
        L.ipuma_gpu_destroy.argtypes = [vp]
        L.ipuma_gpu_destroy.restype = None
        L.ipuma_gpu_set_option.argtypes = [vp, ctypes.c_char_p, i64]
        L.ipuma_gpu_run_buffer.argtypes = [vp, vp, sz, vp, sz]
        L.ipuma_gpu_submit_buffer.argtypes = [vp, vp, sz, vp, sz, ctypes.POINTER(ctypes.c_uint64)]
        L.ipuma_gpu_poll.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(i32)]
        L.ipuma_gpu_join.argtypes = [vp, ctypes.c_uint64, i64]
        L.ipuma_gpu_join_stats.argtypes = [vp, ctypes.c_uint64, i64, ctypes.POINTER(Stats)]
        L.ipuma_gpu_compare.argtypes = [vp, vp, sz, vp, i32, vp, vp, vp]
        L.ipuma_gpu_compare_packed.argtypes = [vp, vp, sz, i32, vp, i32, vp, vp, vp]
        L.ipuma_pack_codes.argtypes = [vp, sz, i32, vp]
        L.ipuma_gpu_compare_device.argtypes = [vp, vp, sz, vp, i32, i32, i32, vp, vp, vp, vp]
        L.ipuma_gpu_compare_device_packed.argtypes = [vp, vp, sz, i32, vp, i32, i32, i32, vp, vp, vp, vp]
        L.ipuma_gpu_last_stats.argtypes = [vp, ctypes.POINTER(Stats)]
        L.ipuma_gpu_run_buffer_device.argtypes = [vp, vp, sz, vp, sz, vp]
        L.ipuma_measure_int_peak.argtypes = [i32, ctypes.POINTER(ctypes.c_double)]
        L.ipuma_gpu_autotune.argtypes = [vp, ctypes.c_char_p]
        L.ipuma_gpu_reserve.argtypes = [vp, i32, i32, i32]
        L.ipuma_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
        L.ipuma_server_submit.argtypes = [vp, i32, vp, sz, vp, i32, ctypes.POINTER(ctypes.c_uint64)]
        L.ipuma_server_add_sequences.argtypes = [vp, vp, sz, ctypes.POINTER(i32)]
        L.ipuma_server_submit_resident.argtypes = [vp, i32, i32, vp, i32,
                                                   ctypes.POINTER(ctypes.c_uint64)]
        L.ipuma_server_poll.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(i32)]
        L.ipuma_server_wait.argtypes = [vp, ctypes.c_uint64, i64, vp, vp, vp,
                                        ctypes.POINTER(ctypes.c_double)]
        L.ipuma_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
        L.ipuma_server_close.argtypes = [vp]
        L.ipuma_server_destroy.argtypes = [vp]
        L.ipuma_server_destroy.restype = None
        L.ipuma_gpu_tuning.argtypes = [vp, ctypes.c_char_p, sz]
        L.ipuma_gpu_compare_noalloc.argtypes = [ctypes.POINTER(SwConfig), i32, vp, sz, vp, i32, i32,
                                                vp, vp, vp, vp]
        _lib = L
    return _lib


class IpumaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("ipuma error %d: %s" % (code, msg))
        self.code = code


def _check(rc):
    if rc != OK:
        raise IpumaError(rc, lib().ipuma_last_error().decode())


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else ctypes.c_void_p(0)


def last_error() -> str:
    return lib().ipuma_last_error().decode()


def device_count() -> int:
    return int(lib().ipuma_device_count())


def measure_int_peak(device: int = 0) -> float:
    """Lane-ops/s of the s16x2 cell-update instruction mix on `device`."""
    v = ctypes.c_double()
    _check(lib().ipuma_measure_int_peak(device, ctypes.byref(v)))
    return v.value


def encode(datatype: str, s: str) -> np.ndarray:
    b = s.encode("latin-1")
    out = np.zeros(len(b), dtype=np.uint8)
    _check(lib().ipuma_encode(DT[datatype], b, len(b), _ptr(out)))
    return out


def packed_bytes(n_codes: int, bits: int) -> int:
    """Bytes of n_codes residues packed at `bits` per residue."""
    return (n_codes * bits + 7) // 8


def device_packed_bytes(n_codes: int, bits: int) -> int:
    """Bytes a device copy of packed codes must hold for
    compare_device_packed: rounded up to a word, plus one word."""
    return ((packed_bytes(n_codes, bits) + 3) // 4) * 4 + 4


def pack_codes(codes: np.ndarray, bits: int = 4, out: np.ndarray | None = None) -> np.ndarray:
    """Packs codes for the packed compare calls (ipuma_pack_codes): a
    little-endian bit stream, residue r in bits [bits*r, bits*r + bits);
    bits = 5 (codes < 32), 4 (codes < 16) or 2 (A, T, C, G = codes 1..4 as
    code - 1).  `out` may be a preallocated (e.g. pinned) uint8 array of at
    least ceil(n * bits / 8) bytes."""
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    nb = packed_bytes(codes.size, bits)
    if out is None:
        out = np.zeros(nb, dtype=np.uint8)
    assert out.dtype == np.uint8 and out.size >= nb and out.flags.c_contiguous
    _check(lib().ipuma_pack_codes(_ptr(codes), codes.size, bits, _ptr(out)))
    return out


def pack_codes4(codes: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
    return pack_codes(codes, 4, out)


def select_matrix(similarity: str, match=1, mismatch=-1, ambiguity=-1) -> np.ndarray:
    out = np.zeros(32 * 32, dtype=np.int8)
    m = ctypes.c_int32()
    n = ctypes.c_int32()
    _check(lib().ipuma_select_matrix(SIM[similarity], match, mismatch, ambiguity, _ptr(out),
                                     out.size, ctypes.byref(m), ctypes.byref(n)))
    return out[: m.value * n.value].reshape(m.value, n.value).copy()


def sw_config(gap_init=0, gap_extend=-1, match=1, mismatch=-1, ambiguity=-1, similarity="na",
              datatype="na") -> SwConfig:
    return SwConfig(gap_init, gap_extend, match, mismatch, ambiguity, SIM[similarity], DT[datatype])


def algo_config(tiles_used=1, max_ab=300, max_batches=20, bufsize=3000, vtype=0, fill_algo=0,
                forward_only=False, use_remote_buffer=False, transmission_programs=1,
                io_tiles=0) -> AlgoConfig:
    return AlgoConfig(tiles_used, max_ab, max_batches, bufsize, vtype, fill_algo,
                      int(bool(forward_only)), int(bool(use_remote_buffer)),
                      transmission_programs, io_tiles)


def input_buffer_words(algo: AlgoConfig) -> int:
    return int(lib().ipuma_input_buffer_words(ctypes.byref(algo)))


class Engine:
    """One engine on one GPU (ipuma_gpu_create / ipuma_gpu_destroy)."""

    def __init__(self, sw: SwConfig, algo: AlgoConfig | None = None, device: int = 0):
        self.sw = sw
        self.algo = algo if algo is not None else algo_config()
        h = ctypes.c_void_p()
        _check(lib().ipuma_gpu_create(ctypes.byref(self.sw), ctypes.byref(self.algo), device,
                                      ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().ipuma_gpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, name: str, value: int):
        _check(lib().ipuma_gpu_set_option(self.h, name.encode(), int(value)))

    def autotune(self, cache_path: str | None = None):
        _check(lib().ipuma_gpu_autotune(self.h, cache_path.encode() if cache_path else None))

    def reserve(self, n: int, max_a_len: int, max_b_len: int):
        """Grows the device buffers for compare_device calls up to this size."""
        _check(lib().ipuma_gpu_reserve(self.h, n, max_a_len, max_b_len))

    def tuning(self) -> dict:
        import json
        buf = ctypes.create_string_buffer(4096)
        _check(lib().ipuma_gpu_tuning(self.h, buf, 4096))
        return json.loads(buf.value.decode())

    def stats(self) -> Stats:
        st = Stats()
        _check(lib().ipuma_gpu_last_stats(self.h, ctypes.byref(st)))
        return st

    def compare(self, codes: np.ndarray, pairs: np.ndarray):
        """Host buffers in, (score, arange, brange) out, in pair order."""
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        pairs = np.ascontiguousarray(pairs, dtype=PAIR_DTYPE)
        n = pairs.shape[0]
        score = np.zeros(n, dtype=np.int32)
        ar = np.zeros(n, dtype=np.int32)
        br = np.zeros(n, dtype=np.int32)
        _check(lib().ipuma_gpu_compare(self.h, _ptr(codes), codes.size, _ptr(pairs), n,
                                       _ptr(score), _ptr(ar), _ptr(br)))
        return score, ar, br

    def compare_into(self, codes: np.ndarray, pairs: np.ndarray, score, ar, br):
        """Like compare() but into caller buffers (e.g. pinned host arrays)."""
        _check(lib().ipuma_gpu_compare(self.h, _ptr(codes), codes.size, _ptr(pairs),
                                       pairs.shape[0], _ptr(score), _ptr(ar), _ptr(br)))

    def compare_packed(self, packed: np.ndarray, n_codes: int, pairs: np.ndarray, bits: int = 4):
        """compare() on packed codes (pack_codes); n_codes residues."""
        packed = np.ascontiguousarray(packed, dtype=np.uint8)
        assert packed.size >= (n_codes * bits + 7) // 8
        pairs = np.ascontiguousarray(pairs, dtype=PAIR_DTYPE)
        n = pairs.shape[0]
        out = [np.zeros(n, dtype=np.int32) for _ in range(3)]
        self.compare_packed_into(packed, n_codes, pairs, *out, bits=bits)
        return tuple(out)

    def compare_packed_into(self, packed: np.ndarray, n_codes: int, pairs: np.ndarray, score, ar, br,
                            bits: int = 4):
        """compare_packed() into caller buffers (e.g. pinned host arrays)."""
        _check(lib().ipuma_gpu_compare_packed(self.h, _ptr(packed), n_codes, bits, _ptr(pairs),
                                              pairs.shape[0], _ptr(score), _ptr(ar), _ptr(br)))

    def compare_device(self, d_codes: int, n_codes: int, d_pairs: int, n: int, max_a: int,
                       max_b: int, d_score: int, d_ar: int, d_br: int, stream: int = 0):
        """Device pointers (ints) in and out; enqueued on `stream`."""
        _check(lib().ipuma_gpu_compare_device(self.h, ctypes.c_void_p(d_codes), n_codes,
                                              ctypes.c_void_p(d_pairs), n, max_a, max_b,
                                              ctypes.c_void_p(d_score), ctypes.c_void_p(d_ar),
                                              ctypes.c_void_p(d_br), ctypes.c_void_p(stream)))

    def compare_device_packed(self, d_packed: int, n_codes: int, bits: int, d_pairs: int, n: int,
                              max_a: int, max_b: int, d_score: int, d_ar: int, d_br: int,
                              stream: int = 0):
        """compare_device on packed codes the kernels read directly
        (device_packed_bytes(n_codes, bits) bytes at d_packed)."""
        _check(lib().ipuma_gpu_compare_device_packed(self.h, ctypes.c_void_p(d_packed), n_codes, bits,
                                                     ctypes.c_void_p(d_pairs), n, max_a, max_b,
                                                     ctypes.c_void_p(d_score), ctypes.c_void_p(d_ar),
                                                     ctypes.c_void_p(d_br), ctypes.c_void_p(stream)))

    def run_buffer(self, inputs: np.ndarray) -> np.ndarray:
        inputs = np.ascontiguousarray(inputs, dtype=np.int32)
        total = self.algo.tiles_used * self.algo.max_batches
        results = np.zeros(3 * total, dtype=np.int32)
        _check(lib().ipuma_gpu_run_buffer(self.h, _ptr(inputs), inputs.size, _ptr(results),
                                          results.size))
        return results

    def run_buffer_device(self, d_inputs: int, n_inputs: int, d_results: int, n_results: int,
                          stream: int = 0):
        _check(lib().ipuma_gpu_run_buffer_device(self.h, ctypes.c_void_p(d_inputs), n_inputs,
                                                 ctypes.c_void_p(d_results), n_results,
                                                 ctypes.c_void_p(stream)))

    def submit_buffer(self, inputs: np.ndarray, results: np.ndarray) -> int:
        job = ctypes.c_uint64()
        _check(lib().ipuma_gpu_submit_buffer(self.h, _ptr(inputs), inputs.size, _ptr(results),
                                             results.size, ctypes.byref(job)))
        return job.value

    def poll(self, job: int) -> bool:
        done = ctypes.c_int32()
        _check(lib().ipuma_gpu_poll(self.h, job, ctypes.byref(done)))
        return bool(done.value)

    def join(self, job: int, timeout_ms: int = -1):
        _check(lib().ipuma_gpu_join(self.h, job, timeout_ms))

    def join_stats(self, job: int, timeout_ms: int = -1) -> "Stats":
        """join() returning the job's own statistics."""
        st = Stats()
        _check(lib().ipuma_gpu_join_stats(self.h, job, timeout_ms, ctypes.byref(st)))
        return st


def compare_noalloc(sw: SwConfig, forward_only: bool, d_codes: int, n_codes: int, d_pairs: int,
                    n: int, max_b: int, d_score: int, d_ar: int, d_br: int, stream: int = 0) -> int:
    """ipuma_gpu_compare_noalloc on device pointers (ints); returns the status."""
    return lib().ipuma_gpu_compare_noalloc(ctypes.byref(sw), int(bool(forward_only)),
                                           ctypes.c_void_p(d_codes), n_codes,
                                           ctypes.c_void_p(d_pairs), n, max_b,
                                           ctypes.c_void_p(d_score), ctypes.c_void_p(d_ar),
                                           ctypes.c_void_p(d_br), ctypes.c_void_p(stream))


class Server:
    """Serving loop (ipuma_server_*): continuous batching of requests."""

    def __init__(self, scorings, forward_only=True, slots=4, pool_bytes=0, max_batch_pairs=0,
                 device=0, one_request_per_batch=False, max_batch_cells=0, reserve_b_len=0):
        self._scorings = (SwConfig * len(scorings))(*scorings)
        cfg = ServerConfig(len(scorings), self._scorings, int(bool(forward_only)), slots,
                           pool_bytes, max_batch_pairs, device, int(bool(one_request_per_batch)),
                           max_batch_cells, reserve_b_len)
        h = ctypes.c_void_p()
        _check(lib().ipuma_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h

    def submit(self, kind: int, codes: np.ndarray, pairs: np.ndarray) -> int:
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        pairs = np.ascontiguousarray(pairs, dtype=PAIR_DTYPE)
        rid = ctypes.c_uint64()
        _check(lib().ipuma_server_submit(self.h, kind, _ptr(codes), codes.size, _ptr(pairs),
                                         pairs.shape[0], ctypes.byref(rid)))
        return rid.value

    def add_sequences(self, codes: np.ndarray) -> int:
        """Uploads a code array once; returns its resident set id."""
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        sid = ctypes.c_int32()
        _check(lib().ipuma_server_add_sequences(self.h, _ptr(codes), codes.size, ctypes.byref(sid)))
        return sid.value

    def submit_resident(self, kind: int, set_id: int, pairs: np.ndarray) -> int:
        """Queues pairs whose offsets index resident set `set_id`."""
        pairs = np.ascontiguousarray(pairs, dtype=PAIR_DTYPE)
        rid = ctypes.c_uint64()
        _check(lib().ipuma_server_submit_resident(self.h, kind, set_id, _ptr(pairs), pairs.shape[0],
                                                  ctypes.byref(rid)))
        return rid.value

    def poll(self, rid: int) -> bool:
        d = ctypes.c_int32()
        _check(lib().ipuma_server_poll(self.h, rid, ctypes.byref(d)))
        return bool(d.value)

    def wait(self, rid: int, n: int, timeout_ms: int = -1):
        score = np.zeros(n, np.int32)
        ar = np.zeros(n, np.int32)
        br = np.zeros(n, np.int32)
        lat = ctypes.c_double()
        _check(lib().ipuma_server_wait(self.h, rid, timeout_ms, _ptr(score), _ptr(ar), _ptr(br),
                                       ctypes.byref(lat)))
        return score, ar, br, lat.value

    def stats(self) -> ServerStats:
        st = ServerStats()
        _check(lib().ipuma_server_get_stats(self.h, ctypes.byref(st)))
        return st

    def close(self):
        _check(lib().ipuma_server_close(self.h))

    def destroy(self):
        if self.h:
            lib().ipuma_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.destroy()


def make_pairs(a_off, a_len, b_off, b_len) -> np.ndarray:
    p = np.zeros(len(a_len), dtype=PAIR_DTYPE)
    p["a_off"] = a_off
    p["a_len"] = a_len
    p["b_off"] = b_off
    p["b_len"] = b_len
    return p
