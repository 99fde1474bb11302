"""GPU tests of asynchronous wire-buffer jobs (ipuma_gpu_submit_buffer /
ipuma_gpu_join_stats), the path of SWAlgorithm::async_submit_prepared_remote_compare
and blocking_join_prepared_remote_compare (src/ipu_batch_affine.cpp of the
reference).

Jobs alternate between two device buffer sets and streams, upload only the
tiles up to the last one with a non-zero Meta word, and report their own
statistics.  Every case checks the results against the oracle, whatever
ran before on either buffer set and in whichever order the jobs are joined.
"""
import numpy as np
import pytest

import ipuma_b200 as ib
import oracle
import workloads

pytestmark = pytest.mark.gpu


def _wire(wl, idx, tiles, max_batches, bufsize):
    """Fills tiles in order (the reference's fillFirst) with the pairs
    `idx` of `wl`; returns (algo, inputs, slot of each pair)."""
    algo = ib.algo_config(tiles_used=tiles, max_batches=max_batches, bufsize=bufsize)
    inputs = np.zeros(ib.input_buffer_words(algo), dtype=np.int32)
    seq = inputs.view(np.uint8)
    tile_bytes = ((bufsize + 3) // 4) * 4
    meta = inputs[tiles * ((bufsize + 3) // 4):].reshape(tiles, max_batches, 4)
    slot_of = np.full(len(idx), -1)
    t = s = used = 0
    for k, p in enumerate(idx):
        a, b = wl.seqs(p)
        need = a.size + b.size
        if s == max_batches or used + need > bufsize:
            t, s, used = t + 1, 0, 0
        assert t < tiles, "workload does not fit the wire buffer"
        base = t * tile_bytes + used
        seq[base:base + a.size] = a
        seq[base + a.size:base + need] = b
        meta[t, s] = (a.size, used, b.size, used + a.size)
        slot_of[k] = t * max_batches + s
        used += need
        s += 1
    return algo, inputs, slot_of


def _engine(wl, algo, forward_only=False):
    algo.forward_only = int(forward_only)
    sw = ib.sw_config(wl.gap_init, wl.gap_extend, wl.match, wl.mismatch, wl.ambiguity,
                      wl.similarity, wl.datatype)
    return ib.Engine(sw, algo)


def _want(wl, idx, forward_only=False, gap_init=None, gap_extend=None):
    sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
    return oracle.sw_batch(wl.codes, wl.a_off[idx], wl.a_len[idx], wl.b_off[idx], wl.b_len[idx],
                           sim, wl.gap_init if gap_init is None else gap_init,
                           wl.gap_extend if gap_extend is None else gap_extend,
                           forward_only=forward_only)


def _check(res, slot_of, total, want, label):
    got = (res[slot_of], res[total + slot_of], res[2 * total + slot_of])
    for g, w, name in zip(got, want, ("score", "arange", "brange")):
        bad = np.nonzero(g != w)[0]
        assert bad.size == 0, "%s %s: %d pairs differ, first %d" % (label, name, bad.size, bad[0])


def _cells(wl, idx):
    return int((wl.a_len[idx].astype(np.int64) * wl.b_len[idx]).sum())


def test_jobs_in_flight_joined_in_reverse_order_with_their_own_stats():
    wl = workloads.dna_batched(n=9_000, seed=61)
    tiles, mb, buf = 100, 64, 80_000
    parts = [np.arange(0, 2_000), np.arange(2_000, 6_500), np.arange(6_500, 7_000)]
    bufs = [_wire(wl, idx, tiles, mb, buf) for idx in parts]
    algo = bufs[0][0]
    total = tiles * mb
    order = [0, 1, 2, 0, 1, 2, 1]
    with _engine(wl, algo) as e:
        outs = [np.full(3 * total, -7, np.int32) for _ in order]
        jobs = [e.submit_buffer(bufs[k][1], o) for k, o in zip(order, outs)]
        stats = {}
        for j in reversed(jobs):
            stats[j] = e.join_stats(j, timeout_ms=120_000)
        for j, k, o in zip(jobs, order, outs):
            _check(o, bufs[k][2], total, _want(wl, parts[k]), "job %d (input %d)" % (j, k))
            st = stats[j]
            assert st.cells == _cells(wl, parts[k])
            assert st.pairs == total
            assert 0 < st.kernel_ms <= st.total_ms
        # the engine's last statistics are those of the job joined last
        assert e.stats().cells == stats[jobs[0]].cells


def test_trimmed_uploads_after_full_buffers_on_both_sets():
    """A job that uses only the first tiles follows jobs that filled every
    tile on the same device buffers: the tail of Meta is cleared on the
    device, so stale slots of earlier jobs never reappear."""
    wl = workloads.dna_batched(n=6_000, seed=62)
    tiles, mb, buf = 24, 200, 120_000
    full_idx = np.arange(0, 4_800)
    part_idx = np.arange(4_800, 5_100)
    algo, full, full_slots = _wire(wl, full_idx, tiles, mb, buf)
    _, part, part_slots = _wire(wl, part_idx, tiles, mb, buf)
    meta = part[tiles * ((buf + 3) // 4):].reshape(tiles, mb, 4)
    used_tiles = np.nonzero(meta.reshape(tiles, -1).any(axis=1))[0]
    assert used_tiles.max() < tiles // 4
    full_meta = full[tiles * ((buf + 3) // 4):].reshape(tiles, mb, 4)
    assert full_meta[tiles - 1].any()
    total = tiles * mb
    want_full, want_part = _want(wl, full_idx), _want(wl, part_idx)
    with _engine(wl, algo) as e:
        fresh = e.run_buffer(part)
        _check(fresh, part_slots, total, want_part, "fresh partial")
        seq = [full, full, part, part, full, part, full, part]
        outs = [np.full(3 * total, -7, np.int32) for _ in seq]
        jobs = [e.submit_buffer(x, o) for x, o in zip(seq, outs)]
        for j in jobs:
            e.join(j, timeout_ms=120_000)
    for x, o in zip(seq, outs):
        if x is full:
            _check(o, full_slots, total, want_full, "full")
        else:
            _check(o, part_slots, total, want_part, "partial")
            # every slot, used or empty, as on the first run of the engine
            np.testing.assert_array_equal(o, fresh)


def test_pinned_and_pageable_results():
    torch = pytest.importorskip("torch")
    wl = workloads.protein(n=1_500, seed=63)
    idx = np.arange(wl.n)
    algo, inputs, slots = _wire(wl, idx, tiles=30, max_batches=64, bufsize=60_000)
    total = 30 * 64
    want = _want(wl, idx)
    pinned_in = torch.from_numpy(inputs).pin_memory()
    with _engine(wl, algo) as e:
        pinned_out = [torch.full((3 * total,), -7, dtype=torch.int32).pin_memory() for _ in range(3)]
        pageable_out = [np.full(3 * total, -7, np.int32) for _ in range(3)]
        jobs = []
        for p, q in zip(pinned_out, pageable_out):
            jobs.append(e.submit_buffer(pinned_in.numpy(), p.numpy()))
            jobs.append(e.submit_buffer(inputs, q))
        for j in jobs:
            e.join(j, timeout_ms=120_000)
    for p, q in zip(pinned_out, pageable_out):
        _check(p.numpy(), slots, total, want, "pinned")
        _check(q, slots, total, want, "pageable")


def test_overflow_counts_belong_to_their_job():
    """A job with pairs scoring above int16 and a job without run
    interleaved; each reports the rerun count it has when run alone."""
    wl = workloads.protein_mixed(n=1_200, seed=64, long_identical_frac=0.01)
    want_all = _want(wl, np.arange(wl.n), forward_only=True)
    high = np.nonzero(want_all[0] > 32767)[0]
    low = np.nonzero(want_all[0] < 2000)[0][:600]
    assert high.size >= 3
    idx_h = np.concatenate([high, low[:100]])
    tiles, mb = 40, 40
    buf = int(2 * (wl.a_len[idx_h] + wl.b_len[idx_h]).max() + 64)
    algo, in_h, slots_h = _wire(wl, idx_h, tiles, mb, buf)
    _, in_l, slots_l = _wire(wl, low, tiles, mb, buf)
    total = tiles * mb
    with _engine(wl, algo, forward_only=True) as e:
        ref = {}
        for name, x in (("h", in_h), ("l", in_l)):
            res = np.zeros(3 * total, np.int32)  # must outlive the join
            j = e.submit_buffer(x, res)
            ref[name] = e.join_stats(j, timeout_ms=120_000).overflow_reruns
        seq = [("h", in_h), ("l", in_l), ("l", in_l), ("h", in_h), ("l", in_l)]
        outs = [np.zeros(3 * total, np.int32) for _ in seq]
        jobs = [e.submit_buffer(x, o) for (_, x), o in zip(seq, outs)]
        got = {j: e.join_stats(j, timeout_ms=120_000) for j in reversed(jobs)}
    assert ref["l"] == 0
    for (name, _), j, o in zip(seq, jobs, outs):
        assert got[j].overflow_reruns == ref[name], name
        if name == "h":
            _check(o, slots_h, total, _want(wl, idx_h, forward_only=True), "high")
        else:
            _check(o, slots_l, total, _want(wl, low, forward_only=True), "low")


@pytest.mark.parametrize("gap_init,gap_extend", [(0, 0), (2, -1)])
def test_exact_path_jobs_and_chunks(gap_init, gap_extend):
    """Scorings outside the wavefront kernels' range run the exact kernel,
    whose row scratch is one engine buffer: wire jobs stay on one buffer
    set and host-buffer compares stay in one chunk."""
    wl = workloads.dna_batched(n=1_000, seed=65)
    wl.gap_init, wl.gap_extend = gap_init, gap_extend
    idx = np.arange(wl.n)
    algo, inputs, slots = _wire(wl, idx, tiles=20, max_batches=64, bufsize=60_000)
    total = 20 * 64
    want = _want(wl, idx)
    with _engine(wl, algo) as e:
        outs = [np.zeros(3 * total, np.int32) for _ in range(3)]
        jobs = [e.submit_buffer(inputs, o) for o in outs]
        for j in jobs:
            e.join(j, timeout_ms=120_000)
        e.set_option("chunks", 4)
        pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
        got = e.compare(wl.codes, pairs)
        assert e.stats().chunks == 1
    for o in outs:
        _check(o, slots, total, want, "exact wire")
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)
