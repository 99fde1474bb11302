// ipusw_b200 -- batch aligner front end with the command line, input formats,
// batching and JSON run logs of the reference's ipusw program
// (ipusw/main.cpp, ipusw/run_comparison.hpp, ipusw/batch.hpp,
// ipusw/ipuworker.hpp, ipusw/ipumultidriver.hpp), running on this library's
// drop-in SWAlgorithm (one per GPU).
//
//   ipusw_b200 [options] REFERENCE QUERY
//     REFERENCE, QUERY   sequences, one per line (.txt) or FASTA (any other
//                        name); reference i is aligned against query i
//     -c, --config FILE  JSON configuration with the reference's layout:
//                        {"sw": {gapInit, gapExtend, matchValue, ...},
//                         "ipu": {tilesUsed, maxAB, maxBatches, bufsize, ...},
//                         "numDevices", "numThreads", "duplicateDatasets",
//                         "duplicationFactor", "repeat"}
//     --KEY VALUE        any leaf key of that configuration (as the
//                        reference's options generated from it)
//     --output FILE      per-comparison results as TSV (index, score,
//                        reference start/end, query start/end); the
//                        reference program writes none
//     --dry-run          load and batch only (no GPU needed)
//     -h, --help
//
// As in the reference, duplicationFactor (or, under duplicateDatasets, the
// device count) submits every batch that many times, and "repeat" is read and
// logged but runs nothing more.  Results are received by numThreads/2
// threads, at least one (the reference starts none for numThreads = 1 and
// then times the submissions only).
//
// Log lines carry "IPUSWLOG" followed by one JSON object, tagged
// "run_comparison_setup", "batch_perf" (one per batch) and "final_log", as
// the reference writes them for its scripts/extract.py.
//
// Wire and result buffers are page-locked (--pinned 0: pageable), and each
// driver is tuned and its buffers allocated before the timed region, as the
// reference initialises its devices before starting its outer timer.  Batch times come
// from the device: time_inner = kernels, time_outer = upload + kernels,
// time_job = submit to join on the host.
#include <algorithm>
#include <atomic>
#include <cctype>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "driver.hpp"
#include "ipu_batch_affine.h"
#include "ipuma_b200.h"
#include "swatlib/fasta.h"

namespace {

// ---------------------------------------------------------------------------
// Minimal JSON reading: objects, strings, numbers, booleans.  The
// configuration is read into its leaf keys (the reference's option names).
// ---------------------------------------------------------------------------
class JsonLeaves {
 public:
  explicit JsonLeaves(const std::string& text) : t_(text) {
    skip();
    object();
    skip();
    if (i_ != t_.size()) fail("trailing characters");
  }
  std::map<std::string, std::string> leaves;

 private:
  const std::string& t_;
  size_t i_ = 0;
  [[noreturn]] void fail(const char* what) {
    throw std::runtime_error(std::string("config JSON: ") + what + " at offset " + std::to_string(i_));
  }
  void skip() {
    while (i_ < t_.size() && std::isspace((unsigned char)t_[i_])) ++i_;
  }
  std::string str() {
    if (i_ >= t_.size() || t_[i_] != '"') fail("expected a string");
    std::string s;
    for (++i_; i_ < t_.size() && t_[i_] != '"'; ++i_) {
      if (t_[i_] == '\\' && i_ + 1 < t_.size()) ++i_;
      s += t_[i_];
    }
    if (i_ >= t_.size()) fail("unterminated string");
    ++i_;
    return s;
  }
  void object() {
    if (i_ >= t_.size() || t_[i_] != '{') fail("expected an object");
    ++i_;
    skip();
    if (i_ < t_.size() && t_[i_] == '}') {
      ++i_;
      return;
    }
    while (true) {
      skip();
      const std::string key = str();
      skip();
      if (i_ >= t_.size() || t_[i_] != ':') fail("expected ':'");
      ++i_;
      skip();
      if (i_ < t_.size() && t_[i_] == '{') {
        object();
      } else if (i_ < t_.size() && t_[i_] == '"') {
        leaves[key] = str();
      } else {
        const size_t b = i_;
        while (i_ < t_.size() && t_[i_] != ',' && t_[i_] != '}' && !std::isspace((unsigned char)t_[i_])) ++i_;
        if (i_ == b) fail("expected a value");
        leaves[key] = t_.substr(b, i_ - b);
      }
      skip();
      if (i_ < t_.size() && t_[i_] == ',') {
        ++i_;
        continue;
      }
      if (i_ < t_.size() && t_[i_] == '}') {
        ++i_;
        return;
      }
      fail("expected ',' or '}'");
    }
  }
};

// The reference's IpuSwConfig (ipusw/ipuswconfig.hpp).
struct IpuSwConfig {
  ipu::SWConfig sw = SW_CONFIGURATION;
  ipu::IPUAlgoConfig ipu = ALGO_CONFIGURATION;
  int numDevices = 1;
  int numThreads = 1;
  bool duplicateDatasets = false;
  int duplicationFactor = 0;
  int repeat = 1;
};

int as_int(const std::string& v) {
  size_t used = 0;
  int x = 0;
  try {
    x = std::stoi(v, &used);
  } catch (const std::exception&) {
    used = 0;
  }
  if (used == 0 || used != v.size()) throw std::runtime_error("not an integer: " + v);
  return x;
}

bool as_bool(const std::string& v) {
  if (v == "true" || v == "1") return true;
  if (v == "false" || v == "0") return false;
  throw std::runtime_error("not a boolean: " + v);
}

// Sets one leaf key; false if the key is unknown.
bool set_key(IpuSwConfig& c, const std::string& k, const std::string& v) {
  if (k == "gapInit") c.sw.gapInit = as_int(v);
  else if (k == "gapExtend") c.sw.gapExtend = as_int(v);
  else if (k == "matchValue") c.sw.matchValue = as_int(v);
  else if (k == "mismatchValue") c.sw.mismatchValue = as_int(v);
  else if (k == "ambiguityValue") c.sw.ambiguityValue = as_int(v);
  else if (k == "similarity") c.sw.similarity = swatlib::strToSimilarity(v);
  else if (k == "datatype") c.sw.datatype = swatlib::strToDataType(v);
  else if (k == "tilesUsed") c.ipu.tilesUsed = as_int(v);
  else if (k == "maxAB") c.ipu.maxAB = as_int(v);
  else if (k == "maxBatches") c.ipu.maxBatches = as_int(v);
  else if (k == "bufsize") c.ipu.bufsize = as_int(v);
  else if (k == "vtype") c.ipu.vtype = ipu::strToVertexType(v);
  else if (k == "fillAlgo") c.ipu.fillAlgo = ipu::strToAlgorithm(v);
  else if (k == "forwardOnly") c.ipu.forwardOnly = as_bool(v);
  else if (k == "useRemoteBuffer") c.ipu.useRemoteBuffer = as_bool(v);
  else if (k == "transmissionPrograms") c.ipu.transmissionPrograms = as_int(v);
  else if (k == "ioTiles") c.ipu.ioTiles = as_int(v);
  else if (k == "numDevices") c.numDevices = as_int(v);
  else if (k == "numThreads") c.numThreads = as_int(v);
  else if (k == "duplicateDatasets") c.duplicateDatasets = as_bool(v);
  else if (k == "duplicationFactor") c.duplicationFactor = as_int(v);
  else if (k == "repeat") c.repeat = as_int(v);
  else return false;
  return true;
}

std::string to_json(const IpuSwConfig& c) {
  std::ostringstream o;
  o << "{\"sw\":" << ipu::toJsonString(c.sw) << ",\"ipu\":" << ipu::toJsonString(c.ipu)
    << ",\"numDevices\":" << c.numDevices << ",\"numThreads\":" << c.numThreads
    << ",\"duplicateDatasets\":" << (c.duplicateDatasets ? "true" : "false")
    << ",\"duplicationFactor\":" << c.duplicationFactor << ",\"repeat\":" << c.repeat << "}";
  return o.str();
}

std::string json_str(const std::string& s) {
  std::string o = "\"";
  for (char ch : s) {
    if (ch == '"' || ch == '\\') o += '\\';
    o += ch;
  }
  return o + "\"";
}

void log_json(const std::string& body) {
  std::printf("WARN  [ipusw] IPUSWLOG%s\n", body.c_str());
  std::fflush(stdout);
}

// run_comparison.hpp load_data: ".txt" = one sequence per line, otherwise
// FASTA records.
void load_data(const std::string& path, std::vector<std::string>& seqs, std::string* error) {
  std::ifstream is(path);
  if (!is.good()) {
    *error = "File not found: " + path;
    return;
  }
  if (path.size() >= 4 && path.compare(path.size() - 4, 4, ".txt") == 0) {
    std::string line;
    while (std::getline(is, line)) {
      if (!line.empty() && line.back() == '\r') line.pop_back();
      seqs.push_back(line);
    }
  } else {
    for (auto& f : swatlib::readFasta(is)) seqs.push_back(f.sequence);
  }
}

// A host buffer of int32 words, page-locked when requested and possible.
class HostBuf {
 public:
  HostBuf() = default;
  HostBuf(const HostBuf&) = delete;
  HostBuf& operator=(const HostBuf&) = delete;
  ~HostBuf() { ipuma_host_free(pinned_); }
  void assign(size_t n, bool pin) {
    ipuma_host_free(pinned_);
    pinned_ = nullptr;
    pageable_.clear();
    n_ = n;
    void* p = nullptr;
    if (pin && n && ipuma_host_alloc(n * sizeof(int32_t), &p) == IPUMA_OK) {
      pinned_ = static_cast<int32_t*>(p);
      std::memset(pinned_, 0, n * sizeof(int32_t));
    } else {
      pageable_.assign(n, 0);
    }
  }
  int32_t* data() { return pinned_ ? pinned_ : pageable_.data(); }
  const int32_t* data() const { return pinned_ ? pinned_ : pageable_.data(); }
  size_t size() const { return n_; }

 private:
  int32_t* pinned_ = nullptr;
  std::vector<int32_t> pageable_;
  size_t n_ = 0;
};

// batch.hpp: consecutive comparisons up to batchCmpLimit comparisons and
// batchDataLimit bytes of sequence per batch.
struct Batch {
  int startIndex, endIndex, numCmps, totalSize;
  std::shared_ptr<HostBuf> inputBuffer;
  std::vector<int32_t> mappingBuffer;
};

std::vector<Batch> createBatches(const std::vector<std::string>& A, const std::vector<std::string>& B,
                                 int batchCmpLimit, int batchDataLimit) {
  if (A.size() != B.size()) throw std::runtime_error("Sizes of A and B are not equal");
  std::vector<Batch> batches;
  int numCmps = 0, totalSize = 0, batchBegin = 0;
  for (size_t i = 0; i < A.size(); ++i) {
    const int alen = (int)A[i].size(), blen = (int)B[i].size();
    if (numCmps + 1 < batchCmpLimit && totalSize + alen + blen < batchDataLimit) {
      numCmps++;
      totalSize += alen + blen;
    } else {
      batches.push_back({batchBegin, batchBegin + numCmps, numCmps, totalSize, std::make_shared<HostBuf>(), {}});
      batchBegin += numCmps;
      numCmps = 1;
      totalSize = alen + blen;
    }
  }
  if (numCmps > 0)
    batches.push_back({batchBegin, batchBegin + numCmps, numCmps, totalSize, std::make_shared<HostBuf>(), {}});
  return batches;
}

void usage() {
  std::printf(
      "usage: ipusw_b200 [options] REFERENCE QUERY\n"
      "  -c, --config FILE   JSON configuration (sw, ipu, numDevices, numThreads,\n"
      "                      duplicateDatasets, duplicationFactor, repeat)\n"
      "  --KEY VALUE         override a configuration key (e.g. --gapInit -10 --maxAB 1000)\n"
      "  --output FILE       write per-comparison results as TSV\n"
      "  --pinned 0|1        page-locked wire and result buffers (default 1)\n"
      "  --dry-run           load and batch only\n");
}

int run(int argc, char** argv) {
  IpuSwConfig config;
  std::vector<std::string> positional;
  std::vector<std::pair<std::string, std::string>> overrides;
  std::string configPath, outputPath;
  bool dryRun = false;
  bool pinned = true;
  for (int a = 1; a < argc; ++a) {
    const std::string arg = argv[a];
    if (arg == "-h" || arg == "--help") {
      usage();
      return 0;
    } else if (arg == "--dry-run") {
      dryRun = true;
    } else if (arg == "--pinned") {
      if (a + 1 >= argc) throw std::runtime_error(arg + " needs a value");
      pinned = as_bool(argv[++a]);
    } else if (arg == "-c" || arg == "--config" || arg == "--output") {
      if (a + 1 >= argc) throw std::runtime_error(arg + " needs a value");
      (arg == "--output" ? outputPath : configPath) = argv[++a];
    } else if (arg.size() > 2 && arg.compare(0, 2, "--") == 0) {
      if (a + 1 >= argc) throw std::runtime_error(arg + " needs a value");
      overrides.emplace_back(arg.substr(2), argv[++a]);
    } else {
      positional.push_back(arg);
    }
  }
  if (positional.size() != 2) {
    usage();
    return 2;
  }
  if (!configPath.empty()) {
    std::ifstream cf(configPath);
    if (!cf.good()) throw std::runtime_error("cannot open config " + configPath);
    std::stringstream ss;
    ss << cf.rdbuf();
    JsonLeaves j(ss.str());
    for (const auto& kv : j.leaves)
      if (!set_key(config, kv.first, kv.second)) throw std::runtime_error("unknown config key " + kv.first);
  }
  for (const auto& kv : overrides)
    if (!set_key(config, kv.first, kv.second)) throw std::runtime_error("unknown option --" + kv.first);

  const std::string& refPath = positional[0];
  const std::string& queryPath = positional[1];
  int duplicationFactor = config.duplicateDatasets ? std::max(config.numDevices, 1) : 1;
  if (config.duplicationFactor > 0) duplicationFactor = config.duplicationFactor;
  log_json("{\"tag\":\"run_comparison_setup\",\"config\":" + to_json(config) + ",\"ref_path\":" +
           json_str(refPath) + ",\"query_path\":" + json_str(queryPath) +
           ",\"duplicationFactor\":" + std::to_string(duplicationFactor) + "}");

  std::vector<std::string> references, queries;
  std::string refErr, queryErr;
  std::thread refLoader(load_data, std::cref(refPath), std::ref(references), &refErr);
  std::thread queryLoader(load_data, std::cref(queryPath), std::ref(queries), &queryErr);
  refLoader.join();
  queryLoader.join();
  if (!refErr.empty()) throw std::runtime_error(refErr);
  if (!queryErr.empty()) throw std::runtime_error(queryErr);

  const auto& ic = config.ipu;
  const int batchCmpLimit = ic.getTotalNumberOfComparisons() - ic.maxBatches;
  const int batchDataLimit = ic.getTotalBufsize32b() * 4 - ic.bufsize * 100;
  auto batches = createBatches(references, queries, batchCmpLimit, batchDataLimit);
  std::printf("INFO  [ipusw] %zu comparisons in %zu batches (limits: %d comparisons, %d bytes)\n",
              references.size(), batches.size(), batchCmpLimit, batchDataLimit);
  if (dryRun) {
    for (const auto& b : batches)
      std::printf("batch %d %d %d %d\n", b.startIndex, b.endIndex, b.numCmps, b.totalSize);
    return 0;
  }

  // Workers fill the wire buffers of the batches (ipuworker.hpp runIpuWorker).
  const int numThreads = std::max(1, config.numThreads);
  const size_t inputWords = ic.getInputBufferSize32b();
  const size_t slots = ic.getTotalNumberOfComparisons();
  {
    std::vector<std::thread> workers;
    std::vector<std::string> errors(numThreads);
    for (int w = 0; w < numThreads; ++w)
      workers.emplace_back([&, w] {
        try {
          for (size_t i = w; i < batches.size(); i += numThreads) {
            Batch& b = batches[i];
            std::vector<std::string> aB(references.begin() + b.startIndex, references.begin() + b.endIndex);
            std::vector<std::string> bB(queries.begin() + b.startIndex, queries.begin() + b.endIndex);
            b.inputBuffer->assign(inputWords, pinned);
            b.mappingBuffer.assign(slots, 0);
            ipu::batchaffine::SWAlgorithm::prepare_remote(config.sw, ic, aB, bB, b.inputBuffer->data(),
                                                          b.inputBuffer->data() + inputWords,
                                                          b.mappingBuffer.data());
          }
        } catch (const std::exception& ex) {
          errors[w] = ex.what();
        }
      });
    for (auto& t : workers) t.join();
    for (const auto& e : errors)
      if (!e.empty()) throw std::runtime_error(e);
  }

  // One drop-in driver per device (ipumultidriver.hpp); batch i goes to
  // driver i % numDevices.
  const int numDevices = std::max(1, config.numDevices);
  std::vector<std::unique_ptr<ipu::batchaffine::SWAlgorithm>> drivers;
  for (int d = 0; d < numDevices; ++d)
    drivers.emplace_back(new ipu::batchaffine::SWAlgorithm(config.sw, ic, d, 1, 1, true));

  const size_t nJobs = batches.size() * (size_t)duplicationFactor;
  std::vector<HostBuf> results(nJobs);
  for (auto& r : results) r.assign(slots * 3, pinned);
  // Device set-up before the timed region, as the reference initialises its
  // devices before starting the outer timer: tuning, then one empty batch
  // per device buffer set (jobs alternate between two), which allocates the
  // wire buffers and streams.
  {
    HostBuf emptyIn, emptyOut;
    emptyIn.assign(inputWords, pinned);
    emptyOut.assign(slots * 3, pinned);
    for (auto& d : drivers) {
      if (ipuma_gpu_autotune(d->engine(), std::getenv("IPUMA_TUNE_CACHE")) != IPUMA_OK)
        throw std::runtime_error(std::string("autotune failed: ") + ipuma_last_error());
      for (int k = 0; k < 2; ++k) {
        std::unique_ptr<ipu::batchaffine::Job> job(d->async_submit_prepared_remote_compare(
            emptyIn.data(), emptyIn.data() + emptyIn.size(), emptyOut.data(), emptyOut.data() + emptyOut.size()));
        d->blocking_join_prepared_remote_compare(*job);
      }
    }
  }
  std::vector<int32_t> score(references.size()), arange(references.size()), brange(references.size());
  std::atomic<long> cmpsProcessed{0}, batchesProcessed{0};
  long cmpsSubmitted = 0, batchesSubmitted = 0;

  const auto t0 = std::chrono::steady_clock::now();
  {
    std::vector<ipu::batchaffine::Job*> jobs(nJobs, nullptr);
    std::vector<std::atomic<int>> ready(nJobs);
    std::atomic<bool> submitFailed{false};  // receivers stop waiting for jobs that never come
    for (auto& r : ready) r.store(0);
    const int receivers = std::max(1, numThreads / 2);
    std::vector<std::string> errors(receivers);
    std::vector<std::thread> recv;
    for (int w = 0; w < receivers; ++w)
      recv.emplace_back([&, w] {
        try {
          for (size_t i = w; i < nJobs; i += receivers) {
            while (!ready[i].load(std::memory_order_acquire)) {
              if (submitFailed.load(std::memory_order_acquire)) return;
              std::this_thread::yield();
            }
            ipu::batchaffine::Job* job = jobs[i];
            Batch& b = batches[i % batches.size()];
            drivers[i % numDevices]->blocking_join_prepared_remote_compare(*job);
            // GCUPS of the batch from its Meta (ipumultidriver.hpp wait()).
            const int32_t* meta = b.inputBuffer->data() + ic.getTotalBufsize32b();
            uint64_t cells = 0, data = 0;
            for (size_t s = 0; s < slots; ++s) {
              cells += (uint64_t)meta[4 * s] * (uint64_t)meta[4 * s + 2];
              data += (uint64_t)meta[4 * s] + (uint64_t)meta[4 * s + 2];
            }
            const double tInner = job->innerCycles * 1e-9, tOuter = job->h2dCycles * 1e-9;
            const double tJob = job->tick.accumulate_microseconds() * 1e-6;
            const double transfer = (double)inputWords * 4;
            const double tH2d = std::max(0.0, tOuter - tInner);
            char buf[1024];
            std::snprintf(buf, sizeof(buf),
                          "{\"tag\":\"batch_perf\",\"cycle_inner\":%llu,\"cycle_outer\":%llu,\"time_inner\":%.9g,"
                          "\"time_outer\":%.9g,\"time_job\":%.9g,\"cell_count\":%llu,\"gcups_inner\":%.6g,"
                          "\"gcups_outer\":%.6g,\"gcups_job\":%.6g,\"gcups_batch\":%.6g,"
                          "\"transfer_size_total\":%.0f,\"time_h2d\":%.9g,\"data_count\":%llu,"
                          "\"transfer_ratio\":%.6g,\"transfer_bandwidth\":%.6g,"
                          "\"transfer_bandwidth_per_vertex\":%.6g}",
                          (unsigned long long)job->innerCycles, (unsigned long long)job->h2dCycles, tInner, tOuter,
                          tJob, (unsigned long long)cells, tInner > 0 ? cells / tInner / 1e9 : 0.0,
                          tOuter > 0 ? cells / tOuter / 1e9 : 0.0, tJob > 0 ? cells / tJob / 1e9 : 0.0,
                          tJob > 0 ? cells / tJob / 1e9 : 0.0, transfer, tH2d, (unsigned long long)data,
                          transfer > 0 ? data / transfer * 100 : 0.0, tH2d > 0 ? transfer / tH2d / 1e6 : 0.0,
                          tH2d > 0 ? transfer / tH2d / 1e6 / std::max(1, ic.tilesUsed) : 0.0);
            log_json(buf);
            if (i < batches.size()) {
              // Results back in comparison order (transferResults).
              auto& r = results[i];
              const int n = b.numCmps;
              ipu::batchaffine::SWAlgorithm::transferResults(
                  r.data(), r.data() + r.size(), b.mappingBuffer.data(), b.mappingBuffer.data() + n,
                  score.data() + b.startIndex, score.data() + b.endIndex, arange.data() + b.startIndex,
                  arange.data() + b.endIndex, brange.data() + b.startIndex, brange.data() + b.endIndex, n);
            }
            delete job;
            batchesProcessed++;
            cmpsProcessed += b.numCmps;
          }
        } catch (const std::exception& ex) {
          errors[w] = ex.what();
        }
      });
    std::string submitError;
    try {
      for (size_t i = 0; i < nJobs; ++i) {
        Batch& b = batches[i % batches.size()];
        auto& r = results[i];
        jobs[i] = drivers[i % numDevices]->async_submit_prepared_remote_compare(
            b.inputBuffer->data(), b.inputBuffer->data() + b.inputBuffer->size(), r.data(), r.data() + r.size());
        ready[i].store(1, std::memory_order_release);
        cmpsSubmitted += b.numCmps;
        batchesSubmitted++;
      }
    } catch (const std::exception& ex) {
      // Jobs already submitted are still joined; the rest are not waited for.
      submitError = ex.what();
      submitFailed.store(true, std::memory_order_release);
    }
    for (auto& t : recv) t.join();
    if (!submitError.empty()) throw std::runtime_error(submitError);
    for (const auto& e : errors)
      if (!e.empty()) throw std::runtime_error(e);
  }
  const double outer = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  uint64_t cellCount = 0;
  for (size_t i = 0; i < references.size(); ++i) cellCount += (uint64_t)references[i].size() * queries[i].size();
  // Only the batches are duplicated; the reference counts the cells of the
  // duplicates only under duplicateDatasets (run_comparison.hpp:152-155).
  if (config.duplicateDatasets) cellCount *= (uint64_t)duplicationFactor;
  char buf[1024];
  std::snprintf(buf, sizeof(buf),
                "{\"tag\":\"final_log\",\"cells\":%llu,\"outer_time_s\":%.9g,\"outer_gcups\":%.6g,"
                "\"cmps_processed\":%ld,\"cmps_submitted\":%ld,\"cmps_orig\":%zu,\"batches_processed\":%ld,"
                "\"batches_submitted\":%ld,\"batches_orig\":%zu}",
                (unsigned long long)cellCount, outer, outer > 0 ? cellCount / outer / 1e9 : 0.0,
                cmpsProcessed.load(), cmpsSubmitted, references.size(), batchesProcessed.load(), batchesSubmitted,
                batches.size());
  log_json(buf);

  if (!outputPath.empty()) {
    std::ofstream out(outputPath);
    out << "index\tscore\tref_start\tref_end\tquery_start\tquery_end\n";
    for (size_t i = 0; i < references.size(); ++i)
      out << i << '\t' << score[i] << '\t' << (arange[i] & 0xffff) << '\t' << ((uint32_t)arange[i] >> 16) << '\t'
          << (brange[i] & 0xffff) << '\t' << ((uint32_t)brange[i] >> 16) << '\n';
    if (!out.good()) throw std::runtime_error("cannot write " + outputPath);
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    return run(argc, argv);
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "FATAL [ipusw] %s\n", ex.what());
    return 1;
  }
}
