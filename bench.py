"""Benchmark: bit-exact GCUPS of the batched affine-gap Smith-Waterman engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
    python bench.py --impl reference ...

One step = one pass of the engine over the whole synthetic batch (default:
1,000,000 DNA pairs, |A| ~ U[50,250], |B| lognormal median 300 clipped to
[100, 1000], +1/-1, gap open/extend 1/1, forward pass, score + end
coordinates).  `value` times the persistent cost-binned engine on
device-resident inputs (2-bit DNA / 5-bit protein codes read packed by the
kernels, ipuma_gpu_compare_device_packed, captured pipeline replayed);
`e2e` times the host-buffer C ABI call (ipuma_gpu_compare_packed) with
pinned inputs and outputs, copies included.  `targets` holds the single-GPU targets of the
engine: the batched engine against the plain one-launch-per-batch kernel (in
s32 and in s16x2 lanes, on the same pairs in the reference wire format) on
the 200,000-pair protein batch and the 500,000-pair heavy-tailed protein
batch, the serving loop at 64-pair requests, and strip teams (the warps of a
block sharing one long pair couple's strips) on a small batch of long pairs.

`--gpus N` runs N ranks, one per GPU (it re-launches itself through
torch.distributed.run when WORLD_SIZE is unset): every rank aligns its own
batch (weak scaling), no collective on the data path, timing is the maximum
over ranks.

`--impl reference` times the reference's CPU implementation of the path
(its vendored StripedSmithWaterman library driven like its cpusw benchmark,
oracle/_ref/libref_ssw.so, all host threads) on bounded samples.
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "ipuma-lib_b200", "python"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

LANE_OPS_PER_CELL = 7  # E: 2, F: 2, H: 2, running max: 1 (int lane-ops)
METRIC = "bit-exact GCUPS (forward pass, score + end coordinates)"

# DRAM bytes (read + write) per forward-pass cell of the dominant launch,
# from one ncu capture of that kernel on the same workload
# (profiles/k_batched_s16x2_L16_K15_dna_1m.md: a launch reads the codes of
# its own pairs, so its traffic scales with its cells).
TRAFFIC_PER_CELL = {"dna_batched": 0.00622}


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dna_batched",
                    choices=["dna_plain", "dna_batched", "protein", "protein_mixed"])
    ap.add_argument("--pairs", type=int, default=0, help="override the pair count")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-targets", action="store_true",
                    help="skip the protein and serving targets (run at N=1 only)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the serving-loop sweep (run at N=1 only)")
    ap.add_argument("--serving-seconds", type=float, default=1.5,
                    help="arrival window of each offered-load point")
    ap.add_argument("--target-reps", type=int, default=3,
                    help="timed replays per arm of each protein target")
    ap.add_argument("--long-pairs-only", action="store_true",
                    help="print only the strip-team comparison on the small batch of long "
                         "pairs (one JSON object; the case of its ncu summary)")
    ap.add_argument("--option", action="append", default=[], metavar="NAME=VALUE",
                    help="engine option (ipuma_gpu_set_option) for the batched engines")
    return ap.parse_args(argv)


OPTIONS = {}  # engine options from --option, applied to every batched engine


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch_ranks(args, argv=None, timeout_s=3600):
    """Re-runs this script as `args.gpus` ranks under torch.distributed.run
    (rendezvous on 127.0.0.1), when it was started as a single process.
    Rank 0 prints the JSON line; returns the launcher's exit status."""
    argv = sys.argv[1:] if argv is None else argv
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", str(args.gpus), "--master-addr", "127.0.0.1",
           "--master-port", str(_free_port()), os.path.abspath(__file__)] + list(argv)
    return subprocess.run(cmd, timeout=timeout_s).returncode


def max_over_ranks(dist, x, device):
    """Largest value of `x` over all ranks (identity without a process group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


SEEDS = {"dna_plain": 1000, "dna_batched": 1001, "protein": 1002, "protein_mixed": 1003}


def make_workload(name, pairs=0, seed_offset=0):
    import workloads
    fn = workloads.CONFIGS[name]
    kw = {}
    if pairs:
        kw["n"] = pairs
    return fn(seed=SEEDS[name] + seed_offset, **kw)


def _gen_workload(name):
    """Worker of the spawned generator pool (module-level: picklable)."""
    return make_workload(name)


def config_of(wl, extra=None):
    """The `config` object of a bench line (both arms use the same keys)."""
    c = {"workload": wl.name, "pairs_per_gpu": wl.n, "cells_per_gpu": wl.cells, "seed": wl.seed,
         "scoring": "%s match %d mismatch %d gapInit %d gapExtend %d"
                    % (wl.similarity, wl.match, wl.mismatch, wl.gap_init, wl.gap_extend)}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout_s=5.0):
        """Blocks until nvidia-smi printed its first sample (its start-up
        takes longer than a short timed region)."""
        t0 = time.perf_counter()
        while self.proc is not None and not self.lines and time.perf_counter() - t0 < timeout_s:
            time.sleep(0.01)

    def mark(self):
        """Index of the next sample: samples from here on are taken during
        the timed region."""
        return len(self.lines)

    def stop(self, first=0, last=None):
        """Stops sampling; summarises samples [first, last) (the timed
        region), plus the one sample that straddles its end."""
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        if last is None:
            last = len(self.lines)
        time.sleep(0.12)  # the sample covering the end of the region
        self.lines = self.lines[first:last + 1]
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def algorithmic_bytes(wl):
    """Bytes a launch must move: packed sequences (2-bit DNA, 5-bit protein),
    16 B of pair descriptor in and 12 B of results out per pair."""
    bits = 2 if wl.datatype == "na" else 5
    seq = (wl.a_len.astype(np.int64) + wl.b_len.astype(np.int64)) * bits / 8.0
    return float(seq.sum() + wl.n * (16 + 12))


def build_wire(wl, max_batches=128):
    """Reference wire buffer (Seqs || Meta) with `max_batches` consecutive
    pairs per tile and bufsize = the largest tile's bytes."""
    n = wl.n
    tiles = (n + max_batches - 1) // max_batches
    need = (wl.a_len.astype(np.int64) + wl.b_len.astype(np.int64))
    tile_of = np.arange(n) // max_batches
    slot = np.arange(n) % max_batches
    tile_bytes = np.bincount(tile_of, weights=need, minlength=tiles).astype(np.int64)
    bufsize = int(((tile_bytes.max() + 15) // 16) * 16)
    words_per_tile = (bufsize + 3) // 4
    inputs = np.zeros(tiles * words_per_tile + tiles * max_batches * 4, dtype=np.int32)
    seq = inputs[: tiles * words_per_tile].view(np.uint8)
    start_in_tile = np.cumsum(need) - need - np.repeat(
        np.concatenate([[0], np.cumsum(tile_bytes)[:-1]]), np.bincount(tile_of, minlength=tiles))
    a_pos = tile_of * (words_per_tile * 4) + start_in_tile
    b_pos = a_pos + wl.a_len
    import workloads as w
    a_codes = w._gather(wl.codes, wl.a_off, wl.a_len)
    b_codes = w._gather(wl.codes, wl.b_off, wl.b_len)

    def scatter(pos, ln, src):
        ln = ln.astype(np.int64)
        idx = np.repeat(pos - np.concatenate([[0], np.cumsum(ln)[:-1]]), ln) + np.arange(int(ln.sum()))
        seq[idx] = src
    scatter(a_pos, wl.a_len, a_codes)
    scatter(b_pos, wl.b_len, b_codes)
    meta = inputs[tiles * words_per_tile:].reshape(tiles * max_batches, 4)
    g = tile_of * max_batches + slot
    meta[g, 0] = wl.a_len
    meta[g, 1] = start_in_tile
    meta[g, 2] = wl.b_len
    meta[g, 3] = start_in_tile + wl.a_len
    return tiles, max_batches, bufsize, inputs, g


def cpu_baseline(wl, seconds):
    """The reference codelet compiled for the host (oracle/_ref), all cores,
    on a bounded sample of the same workload (or the oracle port if the
    reference library is absent)."""
    import oracle
    sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
    use_ref = oracle.have_ref()
    cores = os.cpu_count() or 1
    run = (lambda sub: oracle.ref_codelet_pairs(sub.codes, sub.a_off, sub.a_len, sub.b_off,
                                                sub.b_len, sim, wl.gap_init, wl.gap_extend,
                                                forward_only=True, nthreads=cores)) if use_ref else \
          (lambda sub: oracle.sw_batch(sub.codes, sub.a_off, sub.a_len, sub.b_off, sub.b_len, sim,
                                       wl.gap_init, wl.gap_extend, forward_only=True,
                                       nthreads=cores))
    rng = np.random.default_rng(99)
    idx = rng.choice(wl.n, size=min(wl.n, 2000), replace=False)
    cal = wl.subset(np.sort(idx))
    t0 = time.perf_counter()
    run(cal)
    dt = time.perf_counter() - t0
    rate = cal.cells / max(dt, 1e-6)
    target = max(int(rate * seconds), cal.cells)
    frac = min(1.0, target / wl.cells)
    m = max(1, int(wl.n * frac))
    idx = np.sort(rng.choice(wl.n, size=m, replace=False))
    sub = wl.subset(idx)
    t0 = time.perf_counter()
    run(sub)
    dt = time.perf_counter() - t0
    return {"value": sub.cells / dt / 1e9, "unit": "GCUPS", "cores": cores,
            "kind": "reference" if use_ref else "port",
            "sample": "%d of %d pairs drawn uniformly (%.3g cells, %.1f s), forward pass; %s" % (
                m, wl.n, sub.cells, dt,
                "reference SWAffine codelet compiled for the host, OpenMP over pair chunks"
                if use_ref else "oracle restatement (C), OpenMP over pairs")}


def oracle_sample(wl, got, n=3000, seed=3):
    """Mismatching fields of `got` (3 x n results) on a uniform sample of
    pairs against the oracle."""
    import oracle
    rng = np.random.default_rng(seed)
    chk = np.sort(rng.choice(wl.n, size=min(wl.n, n), replace=False))
    sub = wl.subset(chk)
    sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
    want = oracle.sw_batch(sub.codes, sub.a_off, sub.a_len, sub.b_off, sub.b_len, sim,
                           wl.gap_init, wl.gap_extend, forward_only=True)
    return int(chk.size), int(sum((got[k][chk] != want[k]).sum() for k in range(3)))


def code_bits(wl):
    """Packed width of a workload's codes: 2 bits when every residue is A, C,
    G or T, 4 for other nucleic-acid codes, 5 for amino acids."""
    if wl.datatype == "aa":
        return 5
    return 2 if bool(((wl.codes >= 1) & (wl.codes <= 4)).all()) else 4


class DeviceBatch:
    """A workload resident on the device with one engine (forward pass).
    Its codes stay packed on the device (code_bits) and the kernels read
    them packed (ipuma_gpu_compare_device_packed)."""

    def __init__(self, ib, torch, wl, dev, local, stream):
        self.ib, self.torch, self.wl, self.dev, self.stream = ib, torch, wl, dev, stream
        sw = ib.sw_config(wl.gap_init, wl.gap_extend, wl.match, wl.mismatch, wl.ambiguity,
                          wl.similarity, wl.datatype)
        self.sw = sw
        self.eng = ib.Engine(sw, ib.algo_config(forward_only=True), device=local)
        for k, v in OPTIONS.items():
            self.eng.set_option(k, v)
        t0 = time.perf_counter()
        self.eng.autotune(os.environ.get("IPUMA_TUNE_CACHE"))
        self.tune_s = time.perf_counter() - t0
        self.pairs_np = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
        self.bits = code_bits(wl)
        buf = np.zeros(ib.device_packed_bytes(wl.codes.size, self.bits), np.uint8)
        ib.pack_codes(wl.codes, self.bits, buf)
        self.d_codes = torch.from_numpy(buf).to(dev)
        self.d_pairs = torch.from_numpy(self.pairs_np.view(np.uint8)).to(dev)
        self.d_out = torch.zeros(3, wl.n, dtype=torch.int32, device=dev)
        self.max_a, self.max_b = int(wl.a_len.max()), int(wl.b_len.max())

    def step(self):
        o = self.d_out
        self.eng.compare_device_packed(self.d_codes.data_ptr(), self.wl.codes.size, self.bits,
                                       self.d_pairs.data_ptr(), self.wl.n, self.max_a, self.max_b,
                                       o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr(),
                                       self.stream.cuda_stream)

    def timed(self, reps, warmup):
        """Device ms per replay of the captured pipeline, and the results the
        timed replays wrote (the output is cleared before them)."""
        torch = self.torch
        self.eng.set_option("graphs", 1)
        for _ in range(warmup):
            self.step()
        self.d_out.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        for _ in range(reps):
            self.step()
        e1.record(self.stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, self.d_out.cpu().numpy()

    def launch_breakdown(self):
        """One untimed step with every launch timed alone (sequential), and
        one with the concurrent launches traced on the device."""
        ib = self.ib
        self.eng.set_option("graphs", 0)
        self.eng.set_option("time_launches", 1)
        self.step()
        st = self.eng.stats()
        self.eng.set_option("time_launches", 0)
        timed = [(ib.KERNEL_NAMES.get(st.timed_kind[k], str(st.timed_kind[k])), st.timed_ms[k],
                  st.timed_cells[k]) for k in range(st.n_timed)]
        self.eng.set_option("trace", 1)
        self.step()
        st = self.eng.stats()
        self.eng.set_option("trace", 0)
        trace = [{"kernel": ib.KERNEL_NAMES.get(st.trace_kind[k], str(st.trace_kind[k])),
                  "start_ms": round(st.trace_start_ms[k], 3), "end_ms": round(st.trace_end_ms[k], 3),
                  "gcells": round(st.trace_cells[k] / 1e9, 3)} for k in range(st.n_trace)]
        return timed, trace

    def plain(self, reps, warmup, got, local):
        """The plain one-launch-per-batch kernel on the same pairs in the
        wire format, s32 and s16x2 lanes, checked bit for bit against the
        batched engine's results `got` on every pair."""
        ib, torch, wl = self.ib, self.torch, self.wl
        tiles, mb, bufsize, inputs, slot_of = build_wire(wl)
        algo = ib.algo_config(tiles_used=tiles, max_batches=mb, bufsize=bufsize, max_ab=self.max_a,
                              forward_only=True)
        peng = ib.Engine(self.sw, algo, device=local)
        d_in = torch.from_numpy(inputs).to(self.dev)
        d_res = torch.zeros(3 * tiles * mb, dtype=torch.int32, device=self.dev)
        total = tiles * mb
        out = {"wire_layout": {"tiles": tiles, "max_batches": mb, "bufsize": bufsize}}
        peng.set_option("scheduler", 1)
        for lanes in (32, 16):
            peng.set_option("plain_lanes", lanes)
            for _ in range(max(1, warmup)):
                peng.run_buffer_device(d_in.data_ptr(), d_in.numel(), d_res.data_ptr(),
                                       d_res.numel(), self.stream.cuda_stream)
            d_res.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            for _ in range(reps):
                peng.run_buffer_device(d_in.data_ptr(), d_in.numel(), d_res.data_ptr(),
                                       d_res.numel(), self.stream.cuda_stream)
            e1.record(self.stream)
            torch.cuda.synchronize()
            pms = e0.elapsed_time(e1) / reps
            r = d_res.cpu().numpy()
            same = all(np.array_equal(r[k * total + slot_of], got[k]) for k in range(3))
            out["s32" if lanes == 32 else "s16x2"] = {
                "gcups": wl.cells / (pms * 1e-3) / 1e9, "ms_per_batch": pms,
                "bit_identical_to_batched": bool(same)}
        del d_in, d_res
        peng.close()
        return out

    def close(self):
        self.eng.close()


def protein_target(ib, torch, wl, dev, local, stream, reps):
    """Batched engine vs both plain arms on one protein workload."""
    db = DeviceBatch(ib, torch, wl, dev, local, stream)
    ms, got = db.timed(reps, 2)
    gcups = wl.cells / (ms * 1e-3) / 1e9
    checked, mism = oracle_sample(wl, got, n=1000)
    timed, trace = db.launch_breakdown()
    plain = db.plain(reps, 1, got, local)
    db.close()
    return {
        "pairs": wl.n, "cells": wl.cells, "codes": "%d-bit packed, read by the kernels" % db.bits,
        "batched_gcups": gcups, "batched_ms": ms,
        "plain_s32_gcups": plain["s32"]["gcups"], "plain_s16x2_gcups": plain["s16x2"]["gcups"],
        "ratio_vs_plain_s32": gcups / plain["s32"]["gcups"],
        "ratio_vs_plain_s16x2": gcups / plain["s16x2"]["gcups"],
        "plain_bit_identical": plain["s32"]["bit_identical_to_batched"] and
                               plain["s16x2"]["bit_identical_to_batched"],
        "oracle_sample": {"pairs": checked, "mismatching_fields": mism},
        # Device trace of one step, summarised: the span of its class launches
        # and its longest launch.
        "trace_span_ms": max((t["end_ms"] for t in trace), default=None),
        "trace_longest": max(trace, key=lambda t: t["end_ms"] - t["start_ms"], default=None),
    }


def long_pair_target(ib, reps=3):
    """A small batch of long pairs through the host-buffer call: 296 unrelated
    6000 x 6000 protein pairs (148 two-pair items, one per SM), with strip
    teams (the default of a forward-only engine) and with one warp per item
    (team_warps 0).  The results of both must be identical and match the
    oracle on a sample."""
    import oracle
    n, length = 296, 6000
    rng = np.random.default_rng(20)
    codes = rng.integers(0, 20, 2 * n * length).astype(np.uint8)
    off = np.arange(2 * n, dtype=np.int64) * length
    lens = np.full(n, length, dtype=np.int32)
    pairs = ib.make_pairs(off[0::2], lens, off[1::2], lens)
    sw = ib.sw_config(-11, -1, 1, -1, -1, "blosum62", "aa")
    ms, res = {}, {}
    for warps in (8, 0):
        with ib.Engine(sw, ib.algo_config(forward_only=True)) as e:
            e.set_option("team_warps", warps)
            e.compare(codes, pairs)  # warm-up: autotuning and buffers
            best = float("inf")
            for _ in range(reps):
                t0 = time.perf_counter()
                res[warps] = e.compare(codes, pairs)
                best = min(best, time.perf_counter() - t0)
            ms[warps] = best * 1e3
    chk = np.array([0, n // 2, n - 1])
    want = oracle.sw_batch(codes, pairs["a_off"][chk], pairs["a_len"][chk], pairs["b_off"][chk],
                           pairs["b_len"][chk], oracle.select_matrix("blosum62"), -11, -1,
                           forward_only=True)
    mism = int(sum((res[8][k][chk] != want[k]).sum() for k in range(3)))
    return {"pairs": n, "lengths": "%d x %d" % (length, length), "call": "ipuma_gpu_compare, host buffers",
            "teams_of_8_ms": ms[8], "one_warp_per_item_ms": ms[0], "speedup": ms[0] / ms[8],
            "teams_gcups": n * length * length / (ms[8] * 1e-3) / 1e9,
            "bit_identical": all(np.array_equal(a, b) for a, b in zip(res[8], res[0])),
            "oracle_sample": {"pairs": int(chk.size), "mismatching_fields": mism}}


def serving_section(args, ib, dev, local, wls, peak):
    """Open-loop Poisson sweep of the serving loop on resident sequence sets:
    50% DNA / 50% protein requests (subsets of the DNA and protein
    workloads), 64-pair requests and 1-4096-pair requests, against one
    request per device batch (no coalescing)."""
    import serving
    scorings = [ib.sw_config(wl.gap_init, wl.gap_extend, wl.match, wl.mismatch, wl.ambiguity,
                             wl.similarity, wl.datatype) for wl in wls]

    def server(one=False):
        return ib.Server(scorings, slots=4, pool_bytes=4 << 30, device=local,
                         one_request_per_batch=one)

    dur = args.serving_seconds

    def slim(rs):
        return [{"offered_load": r["offered_load"], "gcups": round(r["gcups"], 1),
                 "fraction_of_peak": round(r["fraction_of_peak"], 4),
                 "p50_ms": round(r["p50_ms"], 2) if r["p50_ms"] is not None else None,
                 "p99_ms": round(r["p99_ms"], 2) if r["p99_ms"] is not None else None,
                 "requests": r["requests"], "failed": r["failed"]} for r in rs]

    t0 = time.perf_counter()
    res = {"workload": "poisson requests, 50%% DNA / 50%% protein, %d + %d pair pools, "
                       "%.1f s arrival window per point, 4 slots" % (wls[0].n, wls[1].n, dur),
           "peak_gcups": peak}
    with server() as srv:
        sets = [srv.add_sequences(wl.codes) for wl in wls]
        res["pairs_64_resident"] = slim(serving.sweep(srv, wls, peak, [0.5, 0.8, 0.85, 0.9], dur, 64, 64,
                                                      set_ids=sets, seed=30))
        res["sizes_1_4096_resident"] = slim(serving.sweep(srv, wls, peak, [0.5, 0.8], dur, 1, 4096,
                                                          set_ids=sets, seed=10))
        res["pairs_64_staged"] = slim(serving.sweep(srv, wls, peak, [0.8], dur, 64, 64, seed=40))
    with server(True) as srv:
        sets = [srv.add_sequences(wl.codes) for wl in wls]
        res["per_request_baseline_64"] = slim(serving.sweep(srv, wls, peak, [0.8], dur, 64, 64,
                                                            set_ids=sets, seed=60,
                                                            max_requests=4000))
    res["seconds"] = time.perf_counter() - t0
    return res


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    import oracle
    if not oracle.have_ssw():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libref_ssw.so not built (needs the reference tree at build time)"}))
        return 0
    wl = make_workload(args.workload, args.pairs)
    sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
    gap_open = -(wl.gap_init + wl.gap_extend)
    gap_ext = -wl.gap_extend
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(7)
    # calibrate a per-step sample of ~4 s
    cal = wl.subset(np.sort(rng.choice(wl.n, size=min(wl.n, 4000), replace=False)))
    t0 = time.perf_counter()
    oracle.ref_ssw_pairs(cal.codes, cal.a_off, cal.a_len, cal.b_off, cal.b_len, sim, gap_open,
                         gap_ext, report_begin=False, nthreads=cores)
    rate = cal.cells / max(time.perf_counter() - t0, 1e-6)
    m = max(1000, min(wl.n, int(wl.n * min(1.0, rate * 4.0 / wl.cells))))
    subs = [wl.subset(np.sort(rng.choice(wl.n, size=m, replace=False)))
            for _ in range(min(3, args.steps + args.warmup))]
    times, cells = [], []
    for k in range(args.warmup + args.steps):
        sub = subs[k % len(subs)]
        t0 = time.perf_counter()
        oracle.ref_ssw_pairs(sub.codes, sub.a_off, sub.a_len, sub.b_off, sub.b_len, sim,
                             gap_open, gap_ext, report_begin=False, nthreads=cores)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
            cells.append(sub.cells)
    value = sum(cells) / sum(times) / 1e9
    line = {
        "impl": "reference", "metric": METRIC,
        "value": value, "unit": "GCUPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16/int32",
        "data": "synthetic",
        "config": config_of(wl, {"sample_pairs_per_step": m}),
        "cpu_baseline": {"value": value, "unit": "GCUPS", "cores": cores, "kind": "reference",
                         "sample": "%d of %d pairs per step; reference StripedSmithWaterman "
                                   "(extern/include/ssw) driven like cpusw/aligners.hpp, "
                                   "ssw_init per pair, %d threads" % (m, wl.n, cores)},
        "e2e": {"value": value, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main(argv=None):
    args = parse(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args, argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.long_pairs_only:
        import ipuma_b200 as ib
        print(json.dumps(long_pair_target(ib)), flush=True)
        return 0

    ws, rank, local = dist_env()
    for kv in args.option:
        k, v = kv.split("=", 1)
        OPTIONS[k] = int(v)
    single = ws == 1
    want_targets = single and not args.no_targets
    # The protein target workloads take tens of seconds to generate: spawned
    # workers (no CUDA in them) make them while the DNA batch runs.
    pool = futs = None
    if want_targets:
        import concurrent.futures as cf
        import multiprocessing as mp
        pool = cf.ProcessPoolExecutor(max_workers=2, mp_context=mp.get_context("spawn"))
        futs = {name: pool.submit(_gen_workload, name) for name in ("protein_mixed", "protein")}

    import torch
    import ipuma_b200 as ib
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    wl = make_workload(args.workload, args.pairs, seed_offset=rank)
    db = DeviceBatch(ib, torch, wl, dev, local, stream)
    tuning = db.eng.tuning()
    tuning["seconds"] = db.tune_s

    # Timed replays of the captured pipeline (CUDA graph) of this shape.
    db.eng.set_option("graphs", 1)
    for _ in range(args.warmup):
        db.step()
    launches_per_step = db.eng.stats().launches
    used_graph = bool(db.eng.stats().used_graph)
    db.d_out.zero_()  # the parity check below reads what the timed replays wrote
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    clocks.wait_first()
    torch.cuda.synchronize()
    clk_first = clocks.mark()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        db.step()
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop(clk_first, clocks.mark())
    ms = max_over_ranks(dist, ev0.elapsed_time(ev1), dev)
    ms_step = ms / args.steps
    total_cells = wl.cells * ws
    value = total_cells / (ms_step * 1e-3) / 1e9
    got = db.d_out.cpu().numpy()
    checked, mism = oracle_sample(wl, got)
    zero_rows = int((got[0] == 0).sum())

    # Per-launch timing (each launch alone) and the device trace of the
    # concurrent launches: two untimed steps after the timed region.
    timed, trace = db.launch_breakdown()
    dom = max(timed, key=lambda x: x[1]) if timed else None

    plain = None
    if single and not args.no_plain:
        plain = db.plain(max(1, min(args.steps, 5)), args.warmup, got, local)
        plain["speedup_batched_vs_plain_s32"] = value / plain["s32"]["gcups"]
        plain["speedup_batched_vs_plain_s16x2"] = value / plain["s16x2"]["gcups"]

    # End to end through the host-buffer C ABI call, pinned host memory,
    # timed over `steps` calls: ipuma_gpu_compare_packed with the codes
    # packed as on the device (code_bits); the one-byte path
    # (ipuma_gpu_compare) is timed beside it.
    e2e = None
    if not args.no_e2e:
        h_codes = torch.from_numpy(wl.codes).pin_memory()
        h_pairs = torch.from_numpy(db.pairs_np.view(np.uint8)).pin_memory()
        h_out = torch.zeros(3, wl.n, dtype=torch.int32).pin_memory()
        codes_np = h_codes.numpy()
        pairs_view = h_pairs.numpy().view(ib.PAIR_DTYPE)
        out_np = h_out.numpy()
        bits = code_bits(wl)
        h_packed = torch.empty(ib.packed_bytes(wl.codes.size, bits), dtype=torch.uint8).pin_memory()
        packed_np = ib.pack_codes(wl.codes, bits, h_packed.numpy())

        def run_bytes():
            db.eng.compare_into(codes_np, pairs_view, out_np[0], out_np[1], out_np[2])

        def run_packed():
            db.eng.compare_packed_into(packed_np, wl.codes.size, pairs_view, out_np[0], out_np[1],
                                       out_np[2], bits=bits)

        def time_call(call):
            for _ in range(max(1, args.warmup)):
                call()
            out_np[:] = 0
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                call()
            wall = max_over_ranks(dist, (time.perf_counter() - t0) / args.steps, dev)
            st = db.eng.stats()
            return wall, int(st.chunks), bool(np.array_equal(out_np, got)), st

        wall_b, chunks_b, same_b, _ = time_call(run_bytes)
        bytes_path = {"value": total_cells / wall_b / 1e9, "ms_per_step": wall_b * 1e3,
                      "h2d_bytes_per_step": int(wl.codes.nbytes + db.pairs_np.nbytes),
                      "bit_identical_to_device_run": same_b, "chunks": chunks_b,
                      "call": "ipuma_gpu_compare (one byte per residue)"}
        wall, chunks, same, st = time_call(run_packed)
        e2e = {"value": total_cells / wall / 1e9, "unit": "GCUPS",
               "h2d_bytes_per_step": int(packed_np.nbytes + db.pairs_np.nbytes),
               "d2h_bytes_per_step": int(3 * 4 * wl.n), "ms_per_step": wall * 1e3,
               "last_call_ms": {"device_span": st.total_ms,  # first copy to last result, CUDA events
                                "host_check": st.host_check_ms, "host_wall": st.host_wall_ms},
               "bit_identical_to_device_run": same, "chunks": chunks,
               "call": "ipuma_gpu_compare_packed (%d-bit codes, read packed by the kernels)" % bits,
               "bytes_path": bytes_path}
        e2e["timing"] = ("host wall clock around each of %d calls (validation, H2D, kernels, D2H; "
                         "uploads of later chunks overlap the kernels of earlier ones); the codes "
                         "are encoded and packed once before timing, as a caller holding 2-bit "
                         "sequences would" % args.steps)

    peaks, peak_src = measured_peaks()
    int_peak = ib.measure_int_peak(local)
    rl = None
    if dom:
        name, dms, dcells = dom
        achieved = dcells * LANE_OPS_PER_CELL / (dms * 1e-3) / 1e9
        tpc = TRAFFIC_PER_CELL.get(args.workload)
        rl = {"bound": "int_issue", "kernel": name, "achieved": achieved,
              "peak": int_peak / 1e9, "unit": "G int lane-ops/s", "frac": achieved * 1e9 / int_peak,
              "per_unit": "%d lane-ops per cell; %d cells in this launch" % (LANE_OPS_PER_CELL, dcells),
              "launch_ms": dms, "peak_source": "ipuma_measure_int_peak (s16x2 DPX mix, this GPU)",
              "traffic": (dcells * tpc) if tpc else None,
              "traffic_unit": "bytes per launch (ncu dram__bytes_read+write per cell x launch cells)"}
    algo_bytes = algorithmic_bytes(wl)
    roof_hbm = {"bound": "hbm", "achieved": algo_bytes / (ms_step * 1e-3) / 1e9,
                "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                "frac": algo_bytes / (ms_step * 1e-3) / 1e9 / peaks.get("hbm_gbs", 1.0),
                "traffic": None, "peak_source": peak_src,
                "per_unit": "packed sequence bytes + 28 B per pair"}

    targets = None
    srv = None
    if want_targets:
        wls = {name: f.result() for name, f in futs.items()}
        pool.shutdown()
        tg = {"what": "1 GPU: the batched engine against the plain one-launch-per-batch kernel "
                      "(s32 and s16x2 lanes, same pairs in the wire format) on the mixed-length "
                      "protein batches, target >= 3x; the serving loop at 64-pair requests, "
                      "target >= 80% of the device rate with p99 < 50 ms; strip teams on a small "
                      "batch of long pairs against one warp per item"}
        tg["protein_mixed_500k"] = protein_target(ib, torch, wls["protein_mixed"], dev, local,
                                                  stream, args.target_reps)
        tg["protein_200k"] = protein_target(ib, torch, wls["protein"], dev, local, stream,
                                            args.target_reps)
        tg["long_pairs_small_batch"] = long_pair_target(ib)
        if plain:
            tg["dna_batched_1m"] = {"batched_gcups": value,
                                    "plain_s32_gcups": plain["s32"]["gcups"],
                                    "plain_s16x2_gcups": plain["s16x2"]["gcups"],
                                    "ratio_vs_plain_s32": plain["speedup_batched_vs_plain_s32"],
                                    "ratio_vs_plain_s16x2": plain["speedup_batched_vs_plain_s16x2"]}
        if not args.no_serving and wl.datatype == "na":
            import serving
            swl = [wl.subset(np.arange(min(wl.n, 400_000))),
                   wls["protein"].subset(np.arange(min(wls["protein"].n, 100_000)))]
            peak = serving.mix_peak([value, tg["protein_200k"]["batched_gcups"]], swl)
            srv = serving_section(args, ib, dev, local, swl, peak)
            tg["serving_64_pairs"] = [p for p in srv["pairs_64_resident"]
                                      if p["offered_load"] in (0.8, 0.85, 0.9)]
        pm = tg["protein_mixed_500k"]
        met = {"protein_mixed_3x_plain_s32": pm["ratio_vs_plain_s32"] >= 3.0,
               "protein_mixed_3x_plain_s16x2": pm["ratio_vs_plain_s16x2"] >= 3.0}
        if "serving_64_pairs" in tg:
            met["serving_64_pairs_80pct_p99_under_50ms"] = any(
                p["fraction_of_peak"] >= 0.8 and p["p99_ms"] is not None and p["p99_ms"] < 50
                for p in tg["serving_64_pairs"])
        tg["met"] = met
        targets = tg

    cpu = None
    if rank == 0 and single and not args.no_cpu_baseline:
        cpu = cpu_baseline(wl, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value, "unit": "GCUPS", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "s16x2 (int32 rerun)",
            "data": "synthetic",
            "config": config_of(wl, {
                "l2": "inputs larger than L2 (%.0f MB of %d-bit codes, %.0f MB of pair "
                      "descriptors per GPU)" % (db.d_codes.numel() / 1e6, db.bits, db.pairs_np.nbytes / 1e6),
                "codes": "%d-bit packed on the device, read by the kernels" % db.bits,
                "engine": "persistent cost-binned (compare_device)", "cuda_graph": used_graph}),
            "targets": targets,
            "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps,
            "roofline": rl,
            "roofline_hbm": roof_hbm,
            "cpu_baseline": cpu,
            "clocks": clk,
            "parity": {"checked_pairs": checked, "mismatching_fields": mism,
                       "zero_score_pairs": zero_rows,
                       "against": "oracle (C restatement of SWAffine::compute), on the output "
                                  "of the timed replays (cleared before them)"},
            "plain": plain,
            "launch_breakdown_ms": [{"kernel": n, "ms": round(m, 4), "cells": c} for n, m, c in timed],
            "trace": trace,
            "autotune": tuning,
            "serving": srv,
        }
        print(json.dumps(line))
    db.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
