"""Serving loop (ipuma_server_*): continuous batching on one GPU.

* every request's result is the same alone and in the mix (bit-exact; the
  alone run is the engine's host-buffer call on that request only);
* admission by free device memory: a small pool makes batches wait for
  memory and splits big requests, results unchanged;
* host-side failures: a pair that cannot fit the pool is refused, a closed
  server refuses submissions but finishes queued work, waits time out.
"""
import threading

import numpy as np
import pytest

import ipuma_b200 as ib
import oracle
import serving
import workloads

pytestmark = pytest.mark.gpu


def _scorings(wls):
    return [ib.sw_config(wl.gap_init, wl.gap_extend, wl.match, wl.mismatch, wl.ambiguity,
                         wl.similarity, wl.datatype) for wl in wls]


def _requests(wls, n_req, seed, max_pairs=300):
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n_req):
        k = int(rng.integers(0, len(wls)))
        cnt = int(np.exp(rng.uniform(0, np.log(max_pairs))))
        cnt = max(1, min(cnt, wls[k].n))
        first = int(rng.integers(0, wls[k].n - cnt + 1))
        reqs.append((k, first, cnt))
    return reqs


def _request_data(wl, first, cnt):
    p = ib.make_pairs(wl.a_off[first:first + cnt], wl.a_len[first:first + cnt],
                      wl.b_off[first:first + cnt], wl.b_len[first:first + cnt])
    return wl.codes, p


def _alone(wls, reqs, forward_only):
    out = []
    engines = [ib.Engine(sc, ib.algo_config(forward_only=forward_only)) for sc in _scorings(wls)]
    try:
        for k, first, cnt in reqs:
            codes, p = _request_data(wls[k], first, cnt)
            out.append(engines[k].compare(codes, p))
    finally:
        for e in engines:
            e.close()
    return out


def _serve(server, wls, reqs, threads=4):
    results = [None] * len(reqs)

    def worker(t):
        mine = []
        for i in range(t, len(reqs), threads):
            k, first, cnt = reqs[i]
            codes, p = _request_data(wls[k], first, cnt)
            mine.append((i, server.submit(k, codes, p), cnt))
        for i, rid, cnt in mine:
            results[i] = server.wait(rid, cnt, timeout_ms=120_000)

    ts = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return results


@pytest.mark.parametrize("forward_only", [True, False])
def test_same_result_alone_and_in_the_mix(forward_only):
    wls = [workloads.dna_batched(n=6000, seed=81), workloads.protein(n=3000, seed=82)]
    reqs = _requests(wls, 60, seed=83)
    alone = _alone(wls, reqs, forward_only)
    with ib.Server(_scorings(wls), forward_only=forward_only, slots=3,
                   max_batch_pairs=2048) as srv:
        mixed = _serve(srv, wls, reqs)
        st = srv.stats()
    assert st.completed == len(reqs) and st.batches < len(reqs)  # requests were coalesced
    for i, ((sa, aa, ba), (sm, am, bm, lat)) in enumerate(zip(alone, mixed)):
        np.testing.assert_array_equal(sa, sm, err_msg="request %d score" % i)
        np.testing.assert_array_equal(aa, am, err_msg="request %d arange" % i)
        np.testing.assert_array_equal(ba, bm, err_msg="request %d brange" % i)
        assert lat > 0
    # and against the oracle on a few requests
    for i in range(0, len(reqs), 15):
        k, first, cnt = reqs[i]
        wl = wls[k]
        sub = wl.subset(np.arange(first, first + cnt))
        sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
        want = oracle.sw_batch(sub.codes, sub.a_off, sub.a_len, sub.b_off, sub.b_len, sim,
                               wl.gap_init, wl.gap_extend, forward_only=forward_only)
        np.testing.assert_array_equal(mixed[i][0], want[0])
        np.testing.assert_array_equal(mixed[i][1], want[1])
        np.testing.assert_array_equal(mixed[i][2], want[2])


def test_small_pool_admission_and_split_requests():
    wl = workloads.protein(n=4000, seed=84)
    reqs = [(0, 0, 1500), (0, 1500, 1000), (0, 2500, 1500)]
    alone = _alone([wl], reqs, True)
    # 1 MiB pool: a batch may use half (about 700 of these pairs), so every
    # request is split and the three slots wait for each other's memory.
    with ib.Server(_scorings([wl]), slots=3, pool_bytes=1 << 20) as srv:
        mixed = _serve(srv, [wl], reqs, threads=3)
        st = srv.stats()
    assert st.batches > len(reqs)
    assert st.max_pool_used <= st.pool_bytes
    for (sa, aa, ba), (sm, am, bm, _) in zip(alone, mixed):
        np.testing.assert_array_equal(sa, sm)
        np.testing.assert_array_equal(aa, am)
        np.testing.assert_array_equal(ba, bm)


@pytest.mark.parametrize("forward_only", [True, False])
def test_resident_sets_match_staged_requests(forward_only):
    """Requests into resident sequence sets, mixed with requests that carry
    their codes, give the same results as each request alone."""
    wls = [workloads.dna_batched(n=5000, seed=91), workloads.protein(n=2500, seed=92)]
    reqs = _requests(wls, 48, seed=93)
    alone = _alone(wls, reqs, forward_only)
    pairs = [ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len) for wl in wls]
    with ib.Server(_scorings(wls), forward_only=forward_only, slots=3,
                   max_batch_pairs=1500) as srv:
        sets = [srv.add_sequences(wl.codes) for wl in wls]
        ids = []
        for i, (k, first, cnt) in enumerate(reqs):
            if i % 3 == 2:
                codes, p = _request_data(wls[k], first, cnt)
                ids.append(srv.submit(k, codes, p))
            else:
                ids.append(srv.submit_resident(k, sets[k], pairs[k][first:first + cnt]))
        got = [srv.wait(rid, cnt) for rid, (_, _, cnt) in zip(ids, reqs)]
        with pytest.raises(ib.IpumaError):
            srv.submit_resident(0, 7, pairs[0][:1])  # unknown set
        bad = pairs[0][:1].copy()
        bad["a_off"] = wls[0].codes.size
        with pytest.raises(ib.IpumaError):
            srv.submit_resident(0, sets[0], bad)  # outside the set
    for i, ((sa, aa, ba), (sm, am, bm, _)) in enumerate(zip(alone, got)):
        np.testing.assert_array_equal(sa, sm, err_msg="request %d score" % i)
        np.testing.assert_array_equal(aa, am, err_msg="request %d arange" % i)
        np.testing.assert_array_equal(ba, bm, err_msg="request %d brange" % i)


def test_oversize_pair_is_refused():
    with ib.Server(_scorings([workloads.dna_batched(n=8, seed=1)]), pool_bytes=1 << 20) as srv:
        codes = np.ones(700_000, np.uint8)
        with pytest.raises(ib.IpumaError) as ei:
            srv.submit(0, codes, ib.make_pairs([0], [1], [1], [699_999]))
        assert ei.value.code in (ib.ERR_NO_MEMORY, ib.ERR_INVALID_ARG)
        s, _, _, _ = srv.wait(srv.submit(0, codes[:8], ib.make_pairs([0], [4], [4], [4])), 1)
        assert s[0] == 4


def test_closed_server_refuses_but_finishes_queued_work():
    wl = workloads.dna_batched(n=2000, seed=85)
    with ib.Server(_scorings([wl]), slots=2) as srv:
        codes, p = _request_data(wl, 0, 2000)
        rid = srv.submit(0, codes, p)
        srv.close()
        with pytest.raises(ib.IpumaError) as ei:
            srv.submit(0, codes, p)
        assert ei.value.code == ib.ERR_CLOSED
        s, _, _, _ = srv.wait(rid, 2000)
    sim = oracle.select_matrix("na", 1, -1, -1)
    want = oracle.sw_batch(wl.codes, wl.a_off, wl.a_len, wl.b_off, wl.b_len, sim, 0, -1,
                           forward_only=True)
    np.testing.assert_array_equal(s, want[0])


def test_wait_timeout_then_success():
    wl = workloads.protein(n=20000, seed=86)
    with ib.Server(_scorings([wl]), slots=1) as srv:
        codes, p = _request_data(wl, 0, wl.n)
        rid = srv.submit(0, codes, p)
        with pytest.raises(ib.IpumaError) as ei:
            srv.wait(rid, wl.n, timeout_ms=0)
        assert ei.value.code == ib.ERR_TIMEOUT
        s, _, _, lat = srv.wait(rid, wl.n)
        assert lat > 0 and s.max() > 0
        with pytest.raises(ib.IpumaError) as ei:
            srv.wait(rid, wl.n)
        assert ei.value.code == ib.ERR_UNKNOWN_JOB


@pytest.mark.parametrize("resident", [False, True])
def test_open_loop_load_generator(resident):
    """The C++ load generator replays a Poisson stream; every request
    completes and latencies are recorded."""
    wls = [workloads.dna_batched(n=20000, seed=87), workloads.protein(n=10000, seed=88)]
    arrival, kind, first, count, rate = serving.schedule(wls, offered_gcups=200, duration_s=1.0,
                                                         max_pairs=512, seed=89)
    with ib.Server(_scorings(wls), slots=4) as srv:
        sets = [srv.add_sequences(wl.codes) for wl in wls] if resident else None
        res = serving.run(srv, wls, arrival, kind, first, count, set_ids=sets)
    assert res["failed"] == 0 and res["requests"] == arrival.size
    assert res["p99_ms"] >= res["p50_ms"] > 0
