// loadgen.cpp -- open-loop load generator for the serving loop (benchmark
// support, built as libipuma_loadgen.so next to the engine library).
//
// The caller precomputes a request schedule (arrival time, scoring kind,
// first pair and pair count within that kind's pair array).  `submitters`
// threads submit request i at its arrival time (Poisson stream from the
// caller), `waiters` threads wait for the requests and record each one's
// latency as the server measured it (submission to completion).  With
// `set_ids` the requests go to ipuma_server_submit_resident (kind k's pairs
// index resident set set_ids[k]); without, each request carries its codes.
#include <atomic>
#include <chrono>
#include <cstdint>
#include <thread>
#include <vector>

#include "ipuma_b200.h"

extern "C" int ipuma_loadgen_run(ipuma_server* srv, int32_t n_kinds, const uint8_t* const* codes,
                                 const int64_t* n_codes, const ipuma_pair* const* pairs, int64_t n_req,
                                 const double* arrival_s, const int32_t* kind, const int64_t* first,
                                 const int32_t* count, const int32_t* set_ids, int32_t submitters,
                                 int32_t waiters, double* latency_ms,
                                 int32_t* status, double* wall_s) {
  using Clock = std::chrono::steady_clock;
  if (!srv || n_req < 0 || submitters < 1 || waiters < 1) return IPUMA_ERR_INVALID_ARG;
  std::vector<std::atomic<uint64_t>> ids(n_req);
  for (auto& x : ids) x.store(0);
  std::vector<int32_t> sub_status(n_req, IPUMA_OK);
  const auto t0 = Clock::now();
  std::atomic<int64_t> last_done_ns{0};
  std::vector<std::thread> threads;
  for (int t = 0; t < submitters; ++t) {
    threads.emplace_back([&, t] {
      for (int64_t i = t; i < n_req; i += submitters) {
        const auto when = t0 + std::chrono::nanoseconds((int64_t)(arrival_s[i] * 1e9));
        std::this_thread::sleep_until(when);
        const int k = kind[i];
        uint64_t id = 0;
        const int rc =
            set_ids ? ipuma_server_submit_resident(srv, k, set_ids[k], pairs[k] + first[i], count[i], &id)
                    : ipuma_server_submit(srv, k, codes[k], (size_t)n_codes[k], pairs[k] + first[i], count[i], &id);
        sub_status[i] = rc;
        ids[i].store(rc == IPUMA_OK ? id : ~uint64_t(0));
      }
    });
  }
  for (int w = 0; w < waiters; ++w) {
    threads.emplace_back([&, w] {
      for (int64_t i = w; i < n_req; i += waiters) {
        uint64_t id;
        while ((id = ids[i].load()) == 0) std::this_thread::sleep_for(std::chrono::microseconds(20));
        if (id == ~uint64_t(0)) {
          status[i] = sub_status[i];
          latency_ms[i] = -1;
          continue;
        }
        double lat = 0;
        status[i] = ipuma_server_wait(srv, id, -1, nullptr, nullptr, nullptr, &lat);
        latency_ms[i] = lat;
        const int64_t ns = std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - t0).count();
        int64_t prev = last_done_ns.load();
        while (ns > prev && !last_done_ns.compare_exchange_weak(prev, ns)) {
        }
      }
    });
  }
  for (auto& th : threads) th.join();
  *wall_s = last_done_ns.load() * 1e-9;
  return IPUMA_OK;
}
