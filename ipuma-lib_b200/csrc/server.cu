// server.cu -- the serving loop: continuous batching of alignment requests.
//
// Requests (host code arrays + pairs, one scoring configuration each) are
// queued by ipuma_server_submit and returned through ipuma_server_wait.
// `slots` worker threads, each with its own engine and CUDA stream, take
// whatever is queued -- the oldest request's scoring, as many of its pairs
// and of the following requests' as fit a device batch -- stage it through
// pinned memory into a region of the server's device pool, run the
// cost-binned engine on it and scatter the results back per request.  A
// request that arrives while batches run on other slots joins the next
// batch a slot forms, so work of different requests overlaps on the
// device; a large request is split across batches.  A batch holds at most
// max_batch_pairs pairs and (beyond its first pair) max_batch_cells cells,
// which bounds how long a request waits behind one batch.
//
// Resident sequence sets: a caller that aligns against the same sequences
// again and again uploads them once (ipuma_server_add_sequences); requests
// then carry only pair descriptors into that set and batches stage nothing
// but pairs.  A batch holds requests of one scoring and one set.  A set of
// A/C/G/T codes only also gets a 2-bit copy, which the nucleic-acid batches
// on it read.
//
// Engines for every slot and scoring are created, autotuned (one scoring
// after the other) and given device buffers for reserve_b_len rows when
// the server starts, so no request waits for an engine, a tuning run or an
// allocation that synchronises the device.
//
// Admission by free HBM: the device pool (one allocation made when the
// server starts, sized from the free device memory) is carved per batch by
// a first-fit allocator; a slot that cannot get the bytes for its batch
// waits until running batches return theirs.  A request that cannot fit
// even an empty pool is refused at submission.
//
// Locking: one mutex guards the queues and the pool; requests in flight
// live in 64 shards (id % 64), each with its own mutex and condition
// variable, and count their unfinished pairs in an atomic, so completing
// one request wakes only the waiters of its shard.
//
// Failure handling is on the host: a closed server refuses submissions,
// waits have timeouts, and a failing batch marks its requests failed
// (their waiters get the error) without stopping the other slots.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "errors.h"
#include "ipuma_b200.h"

using ipuma_internal::fail;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id = 0;
  int kind = 0;
  int set = -1;          // resident sequence set, -1: codes travel with the request
  std::vector<uint8_t> codes;
  std::vector<ipuma_pair> pairs;
  std::vector<int32_t> score, arange, brange;
  int64_t cells = 0;
  int next = 0;                   // first pair not yet given to a batch (queue mutex)
  std::atomic<int> remaining{0};  // pairs not yet finished
  std::atomic<int> error{IPUMA_OK};
  std::string message;            // shard mutex
  bool done = false;              // shard mutex
  Clock::time_point t_submit, t_done;
};

// Part of a request carried by one batch.
struct Chunk {
  std::shared_ptr<Request> req;
  int first, count;
};

// First-fit allocator over the device pool (offsets in bytes).
class Pool {
 public:
  explicit Pool(size_t size) : size_(size) { free_[0] = size; }
  bool alloc(size_t bytes, size_t* off) {
    bytes = (bytes + 255) & ~size_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes, at = it->first + bytes;
        free_.erase(it);
        if (rest) free_[at] = rest;
        used_ += bytes;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t size() const { return size_; }
  size_t used() const { return used_; }

 private:
  size_t size_, used_ = 0;
  std::map<size_t, size_t> free_;
};

size_t batch_bytes(size_t codes, size_t pairs) {
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  return up(codes) + up(pairs * sizeof(ipuma_pair)) + up(pairs * 3 * sizeof(int32_t));
}

struct ResidentSet {
  uint8_t* d_codes = nullptr;
  size_t n_codes = 0;
  // 2-bit copy (ipuma_pack_codes) when every code is A, C, G or T (1..4):
  // nucleic-acid batches on the set read it through
  // ipuma_gpu_compare_device_packed, whose profiles hold four letters.
  uint8_t* d_packed2 = nullptr;
};

constexpr int kShards = 64;

struct Shard {
  std::mutex mu;
  std::condition_variable cv;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
};

}  // namespace

struct ipuma_server {
  ipuma_server_config cfg{};
  std::vector<ipuma_sw_config> scorings;
  int device = 0;
  uint8_t* d_pool = nullptr;
  size_t pool_size = 0;
  std::vector<std::vector<ipuma_engine*>> engines;  // [slot][scoring]
  // Queue state, under `mu`.
  std::mutex mu;
  std::condition_variable cv_work;  // work queued / pool freed / closing
  std::unique_ptr<Pool> pool;
  std::vector<ResidentSet> sets;    // append-only; freed at destroy
  // Requests with pairs not yet batched, one FIFO per (scoring, set).
  std::map<std::pair<int, int>, std::deque<std::shared_ptr<Request>>> queues;
  int64_t n_queued = 0;
  bool closing = false;
  std::vector<std::thread> workers;
  // Requests in flight, by id.
  Shard shards[kShards];
  std::atomic<uint64_t> next_id{1};
  // Statistics (under `mu` unless atomic).
  std::atomic<int64_t> submitted{0}, completed{0};
  int64_t batches = 0, pairs_done = 0, cells_done = 0;
  int64_t max_batch_pairs_seen = 0, max_pool_used = 0;
  double busy_ms = 0;

  Shard& shard(uint64_t id) { return shards[id % kShards]; }
};

namespace {

struct SlotState {
  std::vector<ipuma_engine*> engines;  // one per scoring, owned by the server
  cudaStream_t stream = nullptr;
  uint8_t* h_codes = nullptr;
  ipuma_pair* h_pairs = nullptr;
  int32_t* h_out = nullptr;
  size_t cap_codes = 0, cap_pairs = 0;
};

// Marks `count` pairs of a request finished; the last ones complete it.
void finish_pairs(ipuma_server* s, const std::shared_ptr<Request>& r, int count) {
  if (r->remaining.fetch_sub(count, std::memory_order_acq_rel) != count) return;
  Shard& sh = s->shard(r->id);
  {
    std::lock_guard<std::mutex> lk(sh.mu);
    r->done = true;
    r->t_done = Clock::now();
  }
  s->completed.fetch_add(1, std::memory_order_relaxed);
  sh.cv.notify_all();
}

void fail_chunks(ipuma_server* s, std::vector<Chunk>& chunks, int code, const std::string& msg) {
  for (auto& c : chunks) {
    {
      std::lock_guard<std::mutex> lk(s->shard(c.req->id).mu);
      if (c.req->error.load() == IPUMA_OK) {
        c.req->error.store(code);
        c.req->message = msg;
      }
    }
    finish_pairs(s, c.req, c.count);
  }
}

void worker_loop(ipuma_server* s, int slot_index) {
  SlotState st;
  st.engines = s->engines[slot_index];
  cudaSetDevice(s->device);
  cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking);
  st.cap_pairs = (size_t)s->cfg.max_batch_pairs;
  st.cap_codes = st.cap_pairs * 2048;  // grows on demand
  cudaHostAlloc((void**)&st.h_codes, st.cap_codes, cudaHostAllocDefault);
  cudaHostAlloc((void**)&st.h_pairs, st.cap_pairs * sizeof(ipuma_pair), cudaHostAllocDefault);
  cudaHostAlloc((void**)&st.h_out, st.cap_pairs * 3 * sizeof(int32_t), cudaHostAllocDefault);
  const int64_t cell_cap = s->cfg.max_batch_cells;

  while (true) {
    std::vector<Chunk> chunks;
    size_t codes_bytes = 0, npairs = 0, pool_off = 0, pool_len = 0;
    int kind = 0, set = -1;
    ResidentSet rs;
    int maxA = 1, maxB = 1;
    int64_t cells = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->closing || s->n_queued > 0; });
      if (s->n_queued == 0) break;  // closing and drained
      // Continuous batching: the queue (scoring, sequence set) whose head
      // request is the oldest, then every request of that queue that still
      // fits this batch.
      auto qi = s->queues.end();
      for (auto it = s->queues.begin(); it != s->queues.end(); ++it)
        if (!it->second.empty() &&
            (qi == s->queues.end() || it->second.front()->t_submit < qi->second.front()->t_submit))
          qi = it;
      kind = qi->first.first;
      set = qi->first.second;
      if (set >= 0) rs = s->sets[set];
      auto& q = qi->second;
      while (!q.empty()) {
        std::shared_ptr<Request> r = q.front();
        int take = 0;
        size_t bytes = 0;
        while (r->next + take < (int)r->pairs.size() && npairs + take < st.cap_pairs) {
          const ipuma_pair& p = r->pairs[r->next + take];
          const size_t add = set >= 0 ? 0 : (size_t)p.a_len + (size_t)p.b_len;
          const int64_t c = (int64_t)p.a_len * p.b_len;
          if (npairs + take > 0 &&
              (batch_bytes(codes_bytes + bytes + add, npairs + take + 1) > s->pool_size / 2 ||
               cells + c > cell_cap))
            break;
          bytes += add;
          cells += c;
          ++take;
        }
        if (take > 0) {
          chunks.push_back({r, r->next, take});
          r->next += take;
          npairs += take;
          codes_bytes += bytes;
        }
        if (r->next < (int)r->pairs.size()) break;  // batch full
        q.pop_front();
        s->n_queued--;
        if (s->cfg.one_request_per_batch) break;
      }
      // Admission by free device memory: wait for the pool.
      pool_len = batch_bytes(std::max<size_t>(codes_bytes, 1), npairs);
      // (A batch never exceeds half the pool and slots holding pool bytes
      // are running, so this wait ends.)
      while (!s->pool->alloc(pool_len, &pool_off)) s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
      s->max_pool_used = std::max<int64_t>(s->max_pool_used, (int64_t)s->pool->used());
    }
    // Stage the batch in pinned memory (pair offsets rebased; pairs into a
    // resident set keep theirs and stage no codes).
    if (codes_bytes > st.cap_codes) {
      cudaFreeHost(st.h_codes);
      st.cap_codes = codes_bytes * 2;
      cudaHostAlloc((void**)&st.h_codes, st.cap_codes, cudaHostAllocDefault);
    }
    size_t pos = 0, k = 0;
    for (auto& c : chunks) {
      const Request& r = *c.req;
      if (set >= 0) {
        std::memcpy(st.h_pairs + k, r.pairs.data() + c.first, sizeof(ipuma_pair) * c.count);
        for (int i = 0; i < c.count; ++i) {
          const ipuma_pair& p = st.h_pairs[k + i];
          maxA = std::max(maxA, p.a_len);
          maxB = std::max(maxB, p.b_len);
        }
        k += c.count;
        continue;
      }
      for (int i = 0; i < c.count; ++i, ++k) {
        const ipuma_pair& p = r.pairs[c.first + i];
        ipuma_pair q{(int64_t)pos, (int64_t)(pos + p.a_len), p.a_len, p.b_len};
        std::memcpy(st.h_codes + pos, r.codes.data() + p.a_off, p.a_len);
        std::memcpy(st.h_codes + pos + p.a_len, r.codes.data() + p.b_off, p.b_len);
        pos += (size_t)p.a_len + p.b_len;
        st.h_pairs[k] = q;
        maxA = std::max(maxA, p.a_len);
        maxB = std::max(maxB, p.b_len);
      }
    }
    uint8_t* d_codes = set >= 0 ? rs.d_codes : s->d_pool + pool_off;
    const size_t n_codes_batch = set >= 0 ? rs.n_codes : codes_bytes;
    size_t o = (std::max<size_t>(codes_bytes, 1) + 255) & ~size_t(255);
    ipuma_pair* d_pairs = reinterpret_cast<ipuma_pair*>(s->d_pool + pool_off + o);
    o += (npairs * sizeof(ipuma_pair) + 255) & ~size_t(255);
    int32_t* d_out = reinterpret_cast<int32_t*>(s->d_pool + pool_off + o);
    const auto t0 = Clock::now();
    int rc = IPUMA_OK;
    std::string msg;
    if (npairs > 0) {
      if ((set < 0 && cudaMemcpyAsync(d_codes, st.h_codes, codes_bytes, cudaMemcpyHostToDevice, st.stream) !=
                          cudaSuccess) ||
          cudaMemcpyAsync(d_pairs, st.h_pairs, npairs * sizeof(ipuma_pair), cudaMemcpyHostToDevice, st.stream) !=
              cudaSuccess) {
        rc = IPUMA_ERR_CUDA;
        msg = "copy to the device failed";
      }
    }
    if (rc == IPUMA_OK && npairs > 0) {
      if (set >= 0 && rs.d_packed2 && s->scorings[kind].datatype == IPUMA_DT_NUCLEIC_ACID)
        rc = ipuma_gpu_compare_device_packed(st.engines[kind], rs.d_packed2, rs.n_codes, 2, d_pairs, (int32_t)npairs,
                                             maxA, maxB, d_out, d_out + npairs, d_out + 2 * npairs, st.stream);
      else
        rc = ipuma_gpu_compare_device(st.engines[kind], d_codes, n_codes_batch, d_pairs, (int32_t)npairs, maxA, maxB,
                                      d_out, d_out + npairs, d_out + 2 * npairs, st.stream);
      if (rc) msg = ipuma_last_error();
    }
    if (rc == IPUMA_OK && npairs > 0) {
      if (cudaMemcpyAsync(st.h_out, d_out, npairs * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost, st.stream) !=
              cudaSuccess ||
          cudaStreamSynchronize(st.stream) != cudaSuccess) {
        rc = IPUMA_ERR_CUDA;
        msg = "copy from the device failed";
      }
    }
    const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->pool->release(pool_off, pool_len);
      s->busy_ms += ms;
      if (rc == IPUMA_OK) {
        s->batches++;
        s->pairs_done += (int64_t)npairs;
        s->cells_done += cells;
        s->max_batch_pairs_seen = std::max<int64_t>(s->max_batch_pairs_seen, (int64_t)npairs);
      }
    }
    s->cv_work.notify_all();
    if (rc != IPUMA_OK) {
      fail_chunks(s, chunks, rc, msg);
      continue;
    }
    // Scatter results back per request (each chunk's range belongs to this
    // batch alone; finish_pairs publishes them under the shard mutex).
    size_t idx = 0;
    for (auto& c : chunks) {
      Request& r = *c.req;
      std::memcpy(r.score.data() + c.first, st.h_out + idx, sizeof(int32_t) * c.count);
      std::memcpy(r.arange.data() + c.first, st.h_out + npairs + idx, sizeof(int32_t) * c.count);
      std::memcpy(r.brange.data() + c.first, st.h_out + 2 * npairs + idx, sizeof(int32_t) * c.count);
      idx += c.count;
      finish_pairs(s, c.req, c.count);
    }
  }
  cudaFreeHost(st.h_codes);
  cudaFreeHost(st.h_pairs);
  cudaFreeHost(st.h_out);
  cudaStreamDestroy(st.stream);
}

// Queues a prepared request (results sized here) and hands out its id.
int enqueue(ipuma_server* s, const std::shared_ptr<Request>& r, uint64_t* req) {
  const size_t n = r->pairs.size();
  r->score.assign(n, 0);
  r->arange.assign(n, 0);
  r->brange.assign(n, 0);
  r->remaining.store((int)n);
  r->t_submit = Clock::now();
  r->id = s->next_id.fetch_add(1);
  // Registered before it is queued, so a worker may finish it at once.
  Shard& sh = s->shard(r->id);
  {
    std::lock_guard<std::mutex> lk(sh.mu);
    if (n == 0) {
      r->done = true;
      r->t_done = r->t_submit;
    }
    sh.live[r->id] = r;
  }
  bool closed = false;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->closing) {
      closed = true;
    } else if (n > 0) {
      s->queues[{r->kind, r->set}].push_back(r);
      s->n_queued++;
    }
  }
  if (closed) {
    std::lock_guard<std::mutex> lk(sh.mu);
    sh.live.erase(r->id);
    return fail(IPUMA_ERR_CLOSED, "server is closed");
  }
  s->submitted.fetch_add(1, std::memory_order_relaxed);
  if (n == 0)
    s->completed.fetch_add(1, std::memory_order_relaxed);
  else
    s->cv_work.notify_one();
  *req = r->id;
  return IPUMA_OK;
}

bool pair_ok(const ipuma_pair& p, size_t n_codes) {
  return p.a_len >= 0 && p.b_len >= 0 && p.a_len <= 65535 && p.b_len <= 65535 && p.a_off >= 0 && p.b_off >= 0 &&
         (size_t)p.a_off + p.a_len <= n_codes && (size_t)p.b_off + p.b_len <= n_codes;
}

}  // namespace

extern "C" {

int ipuma_server_create(const ipuma_server_config* cfg, ipuma_server** out) {
  if (!cfg || !out || cfg->n_scorings < 1 || !cfg->scorings) return fail(IPUMA_ERR_INVALID_ARG, "bad server configuration");
  std::unique_ptr<ipuma_server> s(new ipuma_server());
  s->cfg = *cfg;
  s->scorings.assign(cfg->scorings, cfg->scorings + cfg->n_scorings);
  s->cfg.scorings = nullptr;
  if (s->cfg.slots <= 0) s->cfg.slots = 4;
  if (s->cfg.max_batch_pairs <= 0) s->cfg.max_batch_pairs = 262144;
  // 4e9 cells: ~2 ms of device time; measured on B200 with 64-pair
  // requests, 2e9 saturated at 80 % of the device rate, 4e9 sustains 90 %
  // with p99 15 ms, 8e9 adds little.
  if (s->cfg.max_batch_cells <= 0) s->cfg.max_batch_cells = 20000000000LL;
  if (s->cfg.reserve_b_len <= 0) s->cfg.reserve_b_len = 2048;
  s->cfg.reserve_b_len = std::min(s->cfg.reserve_b_len, 65535);
  s->device = cfg->device;
  if (cudaSetDevice(s->device) != cudaSuccess) return fail(IPUMA_ERR_NO_DEVICE, "cannot use device %d", s->device);
  size_t freeB = 0, totalB = 0;
  if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) return fail(IPUMA_ERR_CUDA, "cudaMemGetInfo failed");
  size_t pool = cfg->pool_bytes > 0 ? (size_t)cfg->pool_bytes : freeB / 4;
  if (pool > freeB / 2) pool = freeB / 2;
  if (pool < (1u << 20)) return fail(IPUMA_ERR_NO_MEMORY, "not enough free device memory for the pool");
  if (cudaMalloc(&s->d_pool, pool) != cudaSuccess) return fail(IPUMA_ERR_NO_MEMORY, "pool allocation failed");
  s->pool.reset(new Pool(pool));
  s->pool_size = pool;
  // Engines for every slot and scoring: tuned and given their buffers here,
  // one after the other.
  ipuma_algo_config algo{1, 300, 20, 3000, 0, 0, s->cfg.forward_only, 0, 1, 0};
  s->engines.assign(s->cfg.slots, std::vector<ipuma_engine*>(s->scorings.size(), nullptr));
  int rc = IPUMA_OK;
  for (int i = 0; i < s->cfg.slots && rc == IPUMA_OK; ++i)
    for (size_t k = 0; k < s->scorings.size() && rc == IPUMA_OK; ++k) {
      rc = ipuma_gpu_create(&s->scorings[k], &algo, s->device, &s->engines[i][k]);
      if (rc == IPUMA_OK) rc = ipuma_gpu_autotune(s->engines[i][k], nullptr);
      if (rc == IPUMA_OK)
        rc = ipuma_gpu_reserve(s->engines[i][k], s->cfg.max_batch_pairs, s->cfg.reserve_b_len, s->cfg.reserve_b_len);
    }
  if (rc != IPUMA_OK) {
    const std::string msg = ipuma_last_error();
    for (auto& row : s->engines)
      for (auto* e : row)
        if (e) ipuma_gpu_destroy(e);
    cudaFree(s->d_pool);
    return fail(rc, "%s", msg.c_str());
  }
  for (int i = 0; i < s->cfg.slots; ++i) s->workers.emplace_back(worker_loop, s.get(), i);
  *out = s.release();
  return IPUMA_OK;
}

int ipuma_server_add_sequences(ipuma_server* s, const uint8_t* codes, size_t n_codes, int32_t* set_id) {
  if (!s || !set_id || (!codes && n_codes)) return fail(IPUMA_ERR_INVALID_ARG, "bad sequence set");
  if (cudaSetDevice(s->device) != cudaSuccess) return fail(IPUMA_ERR_NO_DEVICE, "cannot use device %d", s->device);
  ResidentSet rs;
  rs.n_codes = n_codes;
  if (cudaMalloc(&rs.d_codes, std::max<size_t>(n_codes, 1)) != cudaSuccess) {
    cudaGetLastError();
    return fail(IPUMA_ERR_NO_MEMORY, "no device memory for a set of %zu bytes", n_codes);
  }
  if (n_codes && cudaMemcpy(rs.d_codes, codes, n_codes, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(rs.d_codes);
    return fail(IPUMA_ERR_CUDA, "copying the sequence set failed");
  }
  if (n_codes && std::all_of(codes, codes + n_codes, [](uint8_t c) { return c >= 1 && c <= 4; })) {
    // Packed arrays are read a word at a time: whole words plus one.
    const size_t bytes = ((n_codes * 2 + 7) / 8 + 3) / 4 * 4 + 8;
    std::vector<uint8_t> packed(bytes, 0);
    if (ipuma_pack_codes(codes, n_codes, 2, packed.data()) == IPUMA_OK &&
        cudaMalloc(&rs.d_packed2, bytes) == cudaSuccess &&
        cudaMemcpy(rs.d_packed2, packed.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaFree(rs.d_packed2);
      rs.d_packed2 = nullptr;
    }
    cudaGetLastError();  // a failed copy only leaves the set without its 2-bit form
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->closing) {
    cudaFree(rs.d_codes);
    cudaFree(rs.d_packed2);
    return fail(IPUMA_ERR_CLOSED, "server is closed");
  }
  *set_id = (int32_t)s->sets.size();
  s->sets.push_back(rs);
  return IPUMA_OK;
}

int ipuma_server_submit(ipuma_server* s, int32_t kind, const uint8_t* codes, size_t n_codes,
                        const ipuma_pair* pairs, int32_t n, uint64_t* req) {
  if (!s || !req || n < 0 || (n > 0 && (!pairs || (!codes && n_codes))))
    return fail(IPUMA_ERR_INVALID_ARG, "bad submission");
  if (kind < 0 || kind >= (int)s->scorings.size()) return fail(IPUMA_ERR_INVALID_ARG, "unknown scoring kind %d", kind);
  auto r = std::make_shared<Request>();
  r->kind = kind;
  // Copy only the sequences the pairs use, offsets rebased to the copy.
  size_t need = 0;
  for (int i = 0; i < n; ++i) {
    const ipuma_pair& p = pairs[i];
    if (!pair_ok(p, n_codes)) return fail(IPUMA_ERR_INVALID_ARG, "pair %d lies outside the code array", i);
    if (batch_bytes((size_t)p.a_len + p.b_len, 1) > s->pool_size / 2)
      return fail(IPUMA_ERR_NO_MEMORY, "pair %d does not fit the device pool", i);
    need += (size_t)p.a_len + p.b_len;
    r->cells += (int64_t)p.a_len * p.b_len;
  }
  r->codes.resize(need);
  r->pairs.resize(n);
  size_t pos = 0;
  for (int i = 0; i < n; ++i) {
    const ipuma_pair& p = pairs[i];
    std::memcpy(r->codes.data() + pos, codes + p.a_off, p.a_len);
    std::memcpy(r->codes.data() + pos + p.a_len, codes + p.b_off, p.b_len);
    r->pairs[i] = ipuma_pair{(int64_t)pos, (int64_t)(pos + p.a_len), p.a_len, p.b_len};
    pos += (size_t)p.a_len + p.b_len;
  }
  return enqueue(s, r, req);
}

int ipuma_server_submit_resident(ipuma_server* s, int32_t kind, int32_t set_id, const ipuma_pair* pairs,
                                 int32_t n, uint64_t* req) {
  if (!s || !req || n < 0 || (n > 0 && !pairs)) return fail(IPUMA_ERR_INVALID_ARG, "bad submission");
  if (kind < 0 || kind >= (int)s->scorings.size()) return fail(IPUMA_ERR_INVALID_ARG, "unknown scoring kind %d", kind);
  size_t n_codes;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (set_id < 0 || set_id >= (int)s->sets.size()) return fail(IPUMA_ERR_INVALID_ARG, "unknown sequence set %d", set_id);
    n_codes = s->sets[set_id].n_codes;
  }
  auto r = std::make_shared<Request>();
  r->kind = kind;
  r->set = set_id;
  for (int i = 0; i < n; ++i) {
    const ipuma_pair& p = pairs[i];
    if (!pair_ok(p, n_codes)) return fail(IPUMA_ERR_INVALID_ARG, "pair %d lies outside the sequence set", i);
    r->cells += (int64_t)p.a_len * p.b_len;
  }
  r->pairs.assign(pairs, pairs + n);
  return enqueue(s, r, req);
}

int ipuma_server_poll(ipuma_server* s, uint64_t req, int32_t* done) {
  if (!s || !done) return fail(IPUMA_ERR_INVALID_ARG, "null argument");
  Shard& sh = s->shard(req);
  std::lock_guard<std::mutex> lk(sh.mu);
  auto it = sh.live.find(req);
  if (it == sh.live.end()) return fail(IPUMA_ERR_UNKNOWN_JOB, "unknown request %llu", (unsigned long long)req);
  *done = it->second->done ? 1 : 0;
  return IPUMA_OK;
}

int ipuma_server_wait(ipuma_server* s, uint64_t req, int64_t timeout_ms, int32_t* score, int32_t* arange,
                      int32_t* brange, double* latency_ms) {
  if (!s) return fail(IPUMA_ERR_INVALID_ARG, "null server");
  Shard& sh = s->shard(req);
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(sh.mu);
    auto it = sh.live.find(req);
    if (it == sh.live.end()) return fail(IPUMA_ERR_UNKNOWN_JOB, "unknown request %llu", (unsigned long long)req);
    r = it->second;
    auto pred = [&] { return r->done; };
    if (timeout_ms < 0) {
      sh.cv.wait(lk, pred);
    } else if (!sh.cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
      return fail(IPUMA_ERR_TIMEOUT, "request %llu not finished after %lld ms", (unsigned long long)req,
                  (long long)timeout_ms);
    }
    sh.live.erase(r->id);
    if (r->error.load() != IPUMA_OK) return fail(r->error.load(), "request failed: %s", r->message.c_str());
  }
  const size_t n = r->score.size();
  if (n) {
    if (score) std::memcpy(score, r->score.data(), n * sizeof(int32_t));
    if (arange) std::memcpy(arange, r->arange.data(), n * sizeof(int32_t));
    if (brange) std::memcpy(brange, r->brange.data(), n * sizeof(int32_t));
  }
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  return IPUMA_OK;
}

int ipuma_server_get_stats(ipuma_server* s, ipuma_server_stats* out) {
  if (!s || !out) return fail(IPUMA_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  out->submitted = s->submitted.load();
  out->completed = s->completed.load();
  out->queued = s->n_queued;
  out->batches = s->batches;
  out->pairs = s->pairs_done;
  out->cells = s->cells_done;
  out->max_batch_pairs = s->max_batch_pairs_seen;
  out->pool_bytes = (int64_t)s->pool->size();
  out->pool_used = (int64_t)s->pool->used();
  out->max_pool_used = s->max_pool_used;
  out->busy_ms = s->busy_ms;
  return IPUMA_OK;
}

int ipuma_server_close(ipuma_server* s) {
  if (!s) return fail(IPUMA_ERR_INVALID_ARG, "null server");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->closing = true;
  }
  s->cv_work.notify_all();
  return IPUMA_OK;
}

void ipuma_server_destroy(ipuma_server* s) {
  if (!s) return;
  ipuma_server_close(s);
  for (auto& t : s->workers) t.join();
  for (auto& sh : s->shards) {
    {
      std::lock_guard<std::mutex> lk(sh.mu);
      for (auto& kv : sh.live)
        if (!kv.second->done) {
          kv.second->error.store(IPUMA_ERR_CLOSED);
          kv.second->message = "server closed";
          kv.second->done = true;
        }
    }
    sh.cv.notify_all();
  }
  cudaSetDevice(s->device);
  for (auto& row : s->engines)
    for (auto* e : row)
      if (e) ipuma_gpu_destroy(e);
  for (auto& rs : s->sets) {
    cudaFree(rs.d_codes);
    cudaFree(rs.d_packed2);
  }
  if (s->d_pool) cudaFree(s->d_pool);
  delete s;
}

}  // extern "C"
