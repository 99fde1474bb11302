"""Open-loop serving benchmark on top of the serving loop (ipuma_server_*).

Builds a Poisson request stream -- request sizes log-uniform in
[min_pairs, max_pairs], each request a contiguous slice of pairs of one
workload (scoring kind) -- and replays it through libipuma_loadgen.so
(C++ submitter and waiter threads), so that the submission rate is not
limited by Python.  Reports throughput and latency percentiles.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

import ipuma_b200 as ib

LOADGEN = os.path.join(os.path.dirname(ib.LIB_PATH), "libipuma_loadgen.so")
_lg = None


def loadgen():
    global _lg
    if _lg is None:
        ib.lib()
        L = ctypes.CDLL(LOADGEN)
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        L.ipuma_loadgen_run.argtypes = [vp, i32, vp, vp, vp, i64, vp, vp, vp, vp, vp, i32, i32, vp,
                                        vp, ctypes.POINTER(ctypes.c_double)]
        L.ipuma_loadgen_run.restype = ctypes.c_int
        _lg = L
    return _lg


def schedule(workloads, offered_gcups, duration_s, min_pairs=1, max_pairs=4096, probs=None,
             seed=0):
    """Arrival times, kinds, first pair and pair count of each request."""
    rng = np.random.default_rng(seed)
    k = len(workloads)
    probs = np.full(k, 1.0 / k) if probs is None else np.asarray(probs, float)
    # mean cells per request: mean pairs per request x mean cells per pair
    lo, hi = np.log(min_pairs), np.log(max_pairs + 1)
    mean_pairs = (max_pairs + 1 - min_pairs) / (hi - lo) if max_pairs > min_pairs else min_pairs
    cells_pp = np.array([wl.cells / wl.n for wl in workloads])
    mean_cells = mean_pairs * float(np.dot(probs, cells_pp))
    rate = offered_gcups * 1e9 / mean_cells
    n = max(1, int(rate * duration_s))
    arrival = np.cumsum(rng.exponential(1.0 / rate, n))
    kind = rng.choice(k, size=n, p=probs).astype(np.int32)
    count = np.floor(np.exp(rng.uniform(lo, hi, n))).astype(np.int32).clip(min_pairs, max_pairs)
    first = np.zeros(n, np.int64)
    for j, wl in enumerate(workloads):
        m = kind == j
        first[m] = rng.integers(0, np.maximum(1, wl.n - count[m] + 1))
        count[m] = np.minimum(count[m], wl.n)
    return arrival, kind, first, count, rate


def run(server, workloads, arrival, kind, first, count, submitters=4, waiters=8, set_ids=None,
        pairs=None):
    """Replays the schedule.  With `set_ids` (one resident set per workload,
    holding that workload's codes) requests carry only pair descriptors."""
    if pairs is None:
        pairs = [ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len) for wl in workloads]
    codes = [np.ascontiguousarray(wl.codes) for wl in workloads]
    k = len(workloads)
    codes_p = (ctypes.c_void_p * k)(*[c.ctypes.data for c in codes])
    pairs_p = (ctypes.c_void_p * k)(*[p.ctypes.data for p in pairs])
    ncodes = np.array([c.size for c in codes], np.int64)
    n = arrival.size
    lat = np.zeros(n, np.float64)
    st = np.zeros(n, np.int32)
    wall = ctypes.c_double()
    arrival = np.ascontiguousarray(arrival, np.float64)
    kind = np.ascontiguousarray(kind, np.int32)
    first = np.ascontiguousarray(first, np.int64)
    count = np.ascontiguousarray(count, np.int32)
    sets = None if set_ids is None else np.ascontiguousarray(set_ids, np.int32)
    rc = loadgen().ipuma_loadgen_run(server.h, k, codes_p, ncodes.ctypes.data, pairs_p, n,
                                     arrival.ctypes.data, kind.ctypes.data, first.ctypes.data,
                                     count.ctypes.data, None if sets is None else sets.ctypes.data,
                                     submitters, waiters, lat.ctypes.data, st.ctypes.data,
                                     ctypes.byref(wall))
    if rc != 0:
        raise RuntimeError("loadgen failed: %d" % rc)
    cells = 0
    for j, wl in enumerate(workloads):
        m = np.nonzero(kind == j)[0]
        cum = np.concatenate([[0], np.cumsum(wl.a_len.astype(np.int64) * wl.b_len.astype(np.int64))])
        cells += int((cum[first[m] + count[m]] - cum[first[m]]).sum())
    ok = st == 0
    return {
        "requests": int(n), "failed": int((~ok).sum()), "wall_s": wall.value,
        "gcups": cells / max(wall.value, 1e-9) / 1e9, "cells": cells,
        "p50_ms": float(np.percentile(lat[ok], 50)) if ok.any() else None,
        "p95_ms": float(np.percentile(lat[ok], 95)) if ok.any() else None,
        "p99_ms": float(np.percentile(lat[ok], 99)) if ok.any() else None,
        "mean_pairs_per_request": float(count.mean()),
    }


def mix_peak(device_gcups, workloads, probs=None):
    """Batched-engine throughput of a request mix: each workload's device
    GCUPS weighted by its expected share of the mix's cells."""
    k = len(workloads)
    probs = np.full(k, 1.0 / k) if probs is None else np.asarray(probs, float)
    cpp = np.array([wl.cells / wl.n for wl in workloads])
    share = probs * cpp / float(np.dot(probs, cpp))
    return 1.0 / float(np.sum(share / np.asarray(device_gcups, float)))


def sweep(server, workloads, peak_gcups, loads, duration_s, min_pairs, max_pairs, set_ids=None,
          seed=0, max_requests=None, warmup_s=0.3):
    """One open-loop run per offered load (fraction of `peak_gcups`) on
    `server`, after a short warm-up run at half load; `set_ids` (resident
    sets holding each workload's codes) sends pair descriptors only.
    Returns a list of result dicts."""
    pairs = [ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len) for wl in workloads]
    if warmup_s > 0:
        arrival, kind, first, count, _ = schedule(workloads, 0.5 * peak_gcups, warmup_s, min_pairs,
                                                  max_pairs, seed=seed + 999)
        run(server, workloads, arrival, kind, first, count, set_ids=set_ids, pairs=pairs)
    out = []
    for j, load in enumerate(loads):
        arrival, kind, first, count, rate = schedule(workloads, load * peak_gcups, duration_s,
                                                     min_pairs, max_pairs, seed=seed + j)
        if max_requests and arrival.size > max_requests:
            keep = max_requests
            arrival, kind, first, count = arrival[:keep], kind[:keep], first[:keep], count[:keep]
        b0 = server.stats()
        r = run(server, workloads, arrival, kind, first, count, set_ids=set_ids, pairs=pairs)
        b1 = server.stats()
        nb = int(b1.batches - b0.batches)
        r.update({"offered_load": load, "offered_gcups": load * peak_gcups,
                  "requests_per_s": rate, "batches": nb,
                  "mean_pairs_per_batch": float(b1.pairs - b0.pairs) / max(1, nb),
                  "fraction_of_peak": r["gcups"] / peak_gcups})
        out.append(r)
    return out
