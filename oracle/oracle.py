"""CPU oracle for the batched affine-gap Smith-Waterman path (ctypes wrapper).

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker or the timed CPU reference.  The product
library never imports it.

Three CPU implementations are reachable from here:

* ``sw_batch``           -- the C restatement in ``sw_oracle.c`` of the codelet
                            recurrence ``SWAffine::compute``
                            (src/codelets/codelet_batch_affine.cpp:37-127);
* ``ref_codelet_pairs`` / ``ref_codelet_run_buffer``
                         -- the reference's own codelets compiled for the host
                            (``oracle/_ref/libref_codelet.so``);
* ``ref_ssw_pairs``      -- the reference's vendored SSW library driven like its
                            cpusw benchmark (``oracle/_ref/libref_ssw.so``).

The swatlib tables (encoders, NA/BLOSUM matrices) come from
``tests/golden/tables.json``, which ``tests/golden/make_golden.py`` extracts
from the reference's src/swatlib/encoding.h:26-72 and
src/swatlib/similarity.h:17-94.  ``select_matrix`` restates
``swatlib::selectMatrix`` / ``scaleMatrix`` (src/swatlib/similarity.cpp:18-33,89-105)
and ``encode`` restates ``Encoding`` (src/swatlib/encoding.cpp:38-49).
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
TABLES_JSON = os.path.join(REPO, "tests", "golden", "tables.json")

_lib = None
_ref_codelet = None
_ref_ssw = None
_tables = None

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i8p = ctypes.POINTER(ctypes.c_int8)


def _ptr(arr, typ):
    return arr.ctypes.data_as(typ)


def build(with_ref: bool = False) -> None:
    """Builds liboracle.so (and the reference libraries when the tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if with_ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = ctypes.CDLL(path)
        _lib.oracle_sw_batch.argtypes = [
            _u8p, _i64p, _i32p, _i64p, _i32p, ctypes.c_int64, _i8p, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p, _i32p, _i32p]
        _lib.oracle_sw_batch.restype = None
        _lib.oracle_max_threads.restype = ctypes.c_int
    return _lib


def have_ref() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_codelet.so"))


def have_ssw() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_ssw.so"))


def ref_codelet():
    global _ref_codelet
    if _ref_codelet is None:
        _ref_codelet = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_codelet.so"))
        for pre in ("ref_codelet_batch", "ref_codelet_multi"):
            f = getattr(_ref_codelet, pre + "_pairs")
            f.argtypes = [_u8p, _i64p, _i32p, _i64p, _i32p, ctypes.c_int64, ctypes.c_int,
                          ctypes.c_int, ctypes.c_int, _i8p, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, _i32p, _i32p, _i32p]
            f.restype = ctypes.c_int
            g = getattr(_ref_codelet, pre + "_run_buffer")
            g.argtypes = [_i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, ctypes.c_int, ctypes.c_int, _i8p, ctypes.c_int,
                          ctypes.c_int, ctypes.c_int, _i32p]
            g.restype = ctypes.c_int
    return _ref_codelet


def ref_ssw():
    global _ref_ssw
    if _ref_ssw is None:
        _ref_ssw = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_ssw.so"))
        _ref_ssw.ref_ssw_pairs.argtypes = [
            _u8p, _i64p, _i32p, _i64p, _i32p, ctypes.c_int64, _i8p, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p, _i32p, _i32p, _i32p, _i32p]
        _ref_ssw.ref_ssw_pairs.restype = ctypes.c_int
    return _ref_ssw


# --------------------------------------------------------------------------
# swatlib tables
# --------------------------------------------------------------------------

def tables() -> dict:
    global _tables
    if _tables is None:
        with open(TABLES_JSON) as f:
            _tables = json.load(f)
    return _tables


def code_table(datatype: str) -> np.ndarray:
    """127-entry char->code table like Encoding::Encoding (encoding.cpp:38-49).

    Entries default to the code of '\\0'; upper and lower case both map.
    """
    t = tables()
    mapping = t["NA_CODE"] if datatype == "na" else t["AA_CODE"]
    term = mapping["\\0"]
    table = np.full(127, term, dtype=np.uint8)
    for key, val in mapping.items():
        if key == "\\0":
            continue
        table[ord(key)] = val
        table[ord(key.lower())] = val
    return table


def encode(datatype: str, s: str) -> np.ndarray:
    tab = code_table(datatype)
    b = np.frombuffer(s.encode("latin-1"), dtype=np.uint8)
    return tab[b]


def select_matrix(similarity: str, match: int = 1, mismatch: int = -1,
                  ambiguity: int = -1) -> np.ndarray:
    """swatlib::selectMatrix (similarity.cpp:89-105) with scaleMatrix (:18-33)."""
    t = tables()
    if similarity == "na":
        base = np.array(t["NA_SUBSTITUTION"], dtype=np.int8).reshape(16, 16)
        out = np.where(base != 0, np.int8(match), np.int8(mismatch)).astype(np.int8)
        flat = out.reshape(-1)
        m, n = base.shape
        for i in range(m):
            flat[i] = ambiguity
            flat[i * n] = ambiguity
        return flat.reshape(m, n)
    if similarity == "blosum50":
        return np.array(t["BLOSUM50"], dtype=np.int8).reshape(25, 25)
    if similarity == "blosum62":
        return np.array(t["BLOSUM62"], dtype=np.int8).reshape(25, 25)
    raise ValueError("No matrix for similarity " + similarity)


# --------------------------------------------------------------------------
# batch helpers
# --------------------------------------------------------------------------

def pack_pairs(a_codes, b_codes):
    """Concatenates per-pair code arrays into (codes, a_off, a_len, b_off, b_len)."""
    n = len(a_codes)
    a_len = np.array([len(x) for x in a_codes], dtype=np.int32)
    b_len = np.array([len(x) for x in b_codes], dtype=np.int32)
    a_off = np.zeros(n, dtype=np.int64)
    b_off = np.zeros(n, dtype=np.int64)
    parts = []
    pos = 0
    for p in range(n):
        a_off[p] = pos
        parts.append(np.asarray(a_codes[p], dtype=np.uint8))
        pos += a_len[p]
        b_off[p] = pos
        parts.append(np.asarray(b_codes[p], dtype=np.uint8))
        pos += b_len[p]
    codes = np.concatenate(parts) if parts else np.zeros(0, dtype=np.uint8)
    if codes.size == 0:
        codes = np.zeros(1, dtype=np.uint8)
    return codes, a_off, a_len, b_off, b_len


def _arrs(codes, a_off, a_len, b_off, b_len):
    return (np.ascontiguousarray(codes, dtype=np.uint8), np.ascontiguousarray(a_off, dtype=np.int64),
            np.ascontiguousarray(a_len, dtype=np.int32), np.ascontiguousarray(b_off, dtype=np.int64),
            np.ascontiguousarray(b_len, dtype=np.int32))


def sw_batch(codes, a_off, a_len, b_off, b_len, sim, gap_init, gap_extend,
             forward_only=False, nthreads=0):
    """C restatement of the codelet over many pairs -> (score, arange, brange)."""
    codes, a_off, a_len, b_off, b_len = _arrs(codes, a_off, a_len, b_off, b_len)
    sim = np.ascontiguousarray(sim, dtype=np.int8)
    n = a_len.size
    score = np.zeros(n, dtype=np.int32)
    ar = np.zeros(n, dtype=np.int32)
    br = np.zeros(n, dtype=np.int32)
    lib().oracle_sw_batch(_ptr(codes, _u8p), _ptr(a_off, _i64p), _ptr(a_len, _i32p),
                          _ptr(b_off, _i64p), _ptr(b_len, _i32p), n, _ptr(sim, _i8p),
                          sim.shape[1], int(gap_init), int(gap_extend), int(bool(forward_only)),
                          int(nthreads), _ptr(score, _i32p), _ptr(ar, _i32p), _ptr(br, _i32p))
    return score, ar, br


def ref_codelet_pairs(codes, a_off, a_len, b_off, b_len, sim, gap_init, gap_extend,
                      forward_only=False, nthreads=0, variant="batch"):
    """The reference codelet itself (host build) over many pairs."""
    codes, a_off, a_len, b_off, b_len = _arrs(codes, a_off, a_len, b_off, b_len)
    sim = np.ascontiguousarray(sim, dtype=np.int8)
    n = a_len.size
    score = np.zeros(n, dtype=np.int32)
    ar = np.zeros(n, dtype=np.int32)
    br = np.zeros(n, dtype=np.int32)
    f = getattr(ref_codelet(), "ref_codelet_%s_pairs" % variant)
    rc = f(_ptr(codes, _u8p), _ptr(a_off, _i64p), _ptr(a_len, _i32p), _ptr(b_off, _i64p),
           _ptr(b_len, _i32p), n, int(gap_init), int(gap_extend), int(bool(forward_only)),
           _ptr(sim, _i8p), sim.shape[0], sim.shape[1], int(nthreads), _ptr(score, _i32p),
           _ptr(ar, _i32p), _ptr(br, _i32p))
    if rc != 0:
        raise RuntimeError("reference codelet harness rejected the input (offsets > 2^31)")
    return score, ar, br


def ref_codelet_run_buffer(inputs, tiles_used, max_batches, bufsize, max_ab, sim, gap_init,
                           gap_extend, forward_only=False, nthreads=0, variant="batch"):
    """Runs the reference codelet over a full ipuma input buffer -> results buffer."""
    inputs = np.ascontiguousarray(inputs, dtype=np.int32)
    sim = np.ascontiguousarray(sim, dtype=np.int8)
    results = np.zeros(3 * tiles_used * max_batches, dtype=np.int32)
    f = getattr(ref_codelet(), "ref_codelet_%s_run_buffer" % variant)
    f(_ptr(inputs, _i32p), tiles_used, max_batches, bufsize, max_ab, int(gap_init),
      int(gap_extend), int(bool(forward_only)), _ptr(sim, _i8p), sim.shape[0], sim.shape[1],
      int(nthreads), _ptr(results, _i32p))
    return results


def ref_ssw_pairs(codes, a_off, a_len, b_off, b_len, sim, gap_open, gap_ext,
                  report_begin=False, nthreads=0):
    """Reference SSW (cpusw-style) -> (score, a_end, b_end, a_begin, b_begin)."""
    codes, a_off, a_len, b_off, b_len = _arrs(codes, a_off, a_len, b_off, b_len)
    sim = np.ascontiguousarray(sim, dtype=np.int8)
    n = a_len.size
    outs = [np.zeros(n, dtype=np.int32) for _ in range(5)]
    ref_ssw().ref_ssw_pairs(_ptr(codes, _u8p), _ptr(a_off, _i64p), _ptr(a_len, _i32p),
                            _ptr(b_off, _i64p), _ptr(b_len, _i32p), n, _ptr(sim, _i8p),
                            sim.shape[0], int(gap_open), int(gap_ext), int(bool(report_begin)),
                            int(nthreads), *[_ptr(o, _i32p) for o in outs])
    return tuple(outs)


def unpack_range(v):
    """Splits packed ranges into (begin, end) like simple-test.cpp:64-70."""
    v = np.asarray(v, dtype=np.int64) & 0xFFFFFFFF
    return (v & 0xFFFF).astype(np.int32), (v >> 16).astype(np.int32)
