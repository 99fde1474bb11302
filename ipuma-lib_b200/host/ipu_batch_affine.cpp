// SWAlgorithm on the B200 engine.  Host logic follows
// src/ipu_batch_affine.cpp (prepare_remote :891-950, fill_input_buffer
// :752-889, compare_local :564-663, compare_mn_local :697-750,
// transferResults :674-695, slots :952-990); device work goes through the
// C ABI (ipuma_gpu_*).
#include "ipu_batch_affine.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace ipu {
namespace batchaffine {

namespace {

ipuma_sw_config toC(const SWConfig& c) {
  return ipuma_sw_config{c.gapInit,
                         c.gapExtend,
                         c.matchValue,
                         c.mismatchValue,
                         c.ambiguityValue,
                         static_cast<int32_t>(c.similarity),
                         static_cast<int32_t>(c.datatype)};
}

ipuma_algo_config toC(const IPUAlgoConfig& a) {
  return ipuma_algo_config{a.tilesUsed,
                           a.maxAB,
                           a.maxBatches,
                           a.bufsize,
                           static_cast<int32_t>(a.vtype),
                           static_cast<int32_t>(a.fillAlgo),
                           a.forwardOnly ? 1 : 0,
                           a.useRemoteBuffer ? 1 : 0,
                           a.transmissionPrograms,
                           a.ioTiles};
}

[[noreturn]] void raise(const std::string& what) { throw std::runtime_error(what + ": " + ipuma_last_error()); }

void check(int rc, const char* what) {
  if (rc != IPUMA_OK) raise(what);
}

// Encodes one sequence into the bucket region.  Characters without a code
// (NA code 16, which has no row in the 16x16 matrix) are rejected.
void encodeInto(const std::vector<uint8_t>& table, swatlib::DataType dtype, const std::string& s, int8_t* out) {
  for (size_t j = 0; j < s.size(); ++j) {
    const unsigned char c = static_cast<unsigned char>(s[j]);
    const uint8_t v = c < 127 ? table[c] : table[0];
    if (dtype == swatlib::DataType::nucleicAcid && v == 16)
      throw std::runtime_error("Sequence contains a character that is not a nucleic-acid code.");
    out[j] = static_cast<int8_t>(v);
  }
}

}  // namespace

void Job::join() {
  if (joined) return;
  ipuma_stats st{};
  const int rc = ipuma_gpu_join_stats(engine, id, -1, &st);
  joined = true;
  tick.tock();
  if (rc != IPUMA_OK) raise("batch failed");
  h2dCycles = static_cast<uint64_t>(st.total_ms * 1e6);
  innerCycles = static_cast<uint64_t>(st.kernel_ms * 1e6);
}

SWAlgorithm::SWAlgorithm(SWConfig config, IPUAlgoConfig algoconfig, int thread_id, size_t slotCap, size_t ipuCount,
                         bool runExecutor)
    : thread_id(thread_id), ipus(static_cast<int>(ipuCount)), config(config), algoconfig(algoconfig) {
  const int total = algoconfig.getTotalNumberOfComparisons();
  slot_size = static_cast<int>(slotCap);
  const int programs = std::max(1, algoconfig.transmissionPrograms);
  slot_avail.assign(programs, slot_size);
  slots.assign(programs, std::vector<bool>(slot_size, false));
  scores.resize(total);
  a_range_result.resize(total);
  b_range_result.resize(total);

  const int ndev = std::max(1, ipuma_device_count());
  const auto sw = toC(config);
  const auto al = toC(algoconfig);
  check(ipuma_gpu_create(&sw, &al, thread_id % ndev, &engine_), "Could not acquire a device");
  (void)runExecutor;
}

SWAlgorithm::SWAlgorithm(SWConfig config, IPUAlgoConfig algoconfig) : SWAlgorithm(config, algoconfig, 0) {}

SWAlgorithm::~SWAlgorithm() {
  if (engine_) ipuma_gpu_destroy(engine_);
}

BlockAlignmentResults SWAlgorithm::get_result() { return {scores, a_range_result, b_range_result}; }

void SWAlgorithm::checkSequenceSizes(const IPUAlgoConfig& algoconfig, const std::vector<int>& SeqSizes) {
  if ((long)SeqSizes.size() > (long)algoconfig.maxBatches * algoconfig.tilesUsed)
    throw std::runtime_error("Input sequence (A) is over the max length.");
  for (const auto& s : SeqSizes)
    if (s > algoconfig.maxAB)
      throw std::runtime_error("Sequence size in seq " + std::to_string(s) + " > " + std::to_string(algoconfig.maxAB));
}

void SWAlgorithm::checkSequenceSizes(const IPUAlgoConfig& algoconfig, const RawSequences& Seqs) {
  std::vector<int> sizes;
  sizes.reserve(Seqs.size());
  for (const auto& s : Seqs) sizes.push_back(static_cast<int>(s.size()));
  checkSequenceSizes(algoconfig, sizes);
}

void SWAlgorithm::fillMNBuckets(Algorithm algo, partition::BucketMap& map, const RawSequences& Seqs,
                                const Comparisons& Cmps, int offset) {
  switch (algo) {
    case Algorithm::fillFirst: partition::fillFirst(map, Seqs, Cmps, offset); break;
    case Algorithm::roundRobin: partition::roundRobin(map, Seqs, Cmps, offset); break;
    case Algorithm::greedy: partition::greedy(map, Seqs, Cmps, offset); break;
  }
}

void SWAlgorithm::fillBuckets(Algorithm algo, partition::BucketMap& map, const RawSequences& A, const RawSequences& B,
                              int offset) {
  switch (algo) {
    case Algorithm::fillFirst: partition::fillFirst(map, A, B, offset); break;
    case Algorithm::roundRobin: partition::roundRobin(map, A, B, offset); break;
    case Algorithm::greedy: partition::greedy(map, A, B, offset); break;
  }
}

size_t SWAlgorithm::getSeqsOffset(const IPUAlgoConfig&) { return 0; }

size_t SWAlgorithm::getMetaOffset(const IPUAlgoConfig& config) { return config.getTotalBufsize32b(); }

void SWAlgorithm::refetch() { throw std::runtime_error("refetch is not implemented (results are final)"); }

std::tuple<int, slotToken> SWAlgorithm::unpack_slot(slotToken s) { return {(int)(s / slot_size), s % slot_size}; }

void SWAlgorithm::upload(int32_t*, int32_t*, slotToken) {
  throw std::runtime_error("upload (remote buffers) is not implemented");
}

std::string SWAlgorithm::printTensors() { return ""; }

void SWAlgorithm::prepared_remote_compare(int32_t* inputs_begin, int32_t* inputs_end, int32_t* results_begin,
                                          int32_t* results_end, slotToken slot_token) {
  if (algoconfig.useRemoteBuffer) release_slot(slot_token);
  auto job = std::unique_ptr<Job>(async_submit_prepared_remote_compare(inputs_begin, inputs_end, results_begin,
                                                                       results_end));
  blocking_join_prepared_remote_compare(*job);
}

Job* SWAlgorithm::async_submit_prepared_remote_compare(int32_t* inputs_begin, int32_t* inputs_end,
                                                       int32_t* results_begin, int32_t* results_end) {
  auto job = new Job();
  job->engine = engine_;
  job->tick.tick();
  const int rc = ipuma_gpu_submit_buffer(engine_, inputs_begin, (size_t)(inputs_end - inputs_begin), results_begin,
                                         (size_t)(results_end - results_begin), &job->id);
  if (rc != IPUMA_OK) {
    delete job;
    raise("submit failed");
  }
  return job;
}

void SWAlgorithm::blocking_join_prepared_remote_compare(Job& job) { job.join(); }

void SWAlgorithm::compare_local(const std::vector<std::string>& A, const std::vector<std::string>& B, bool errcheck) {
  if (A.size() != B.size()) throw std::runtime_error("A and B must hold the same number of sequences.");
  std::vector<int> mapping(A.size(), 0);
  const size_t inputs_size = algoconfig.getInputBufferSize32b();
  std::vector<int32_t> inputs(inputs_size + 4);
  const size_t results_size = scores.size() + a_range_result.size() + b_range_result.size();
  std::vector<int32_t> results(results_size + 4);

  const int32_t canaryBegin = (int32_t)0xDEADBEEF, canaryEnd = (int32_t)0xFEEBDAED;
  inputs[0] = inputs[1] = canaryBegin;
  inputs[inputs_size + 2] = inputs[inputs_size + 3] = canaryEnd;
  const int maxbucket =
      prepare_remote(config, algoconfig, A, B, inputs.data() + 2, inputs.data() + 2 + inputs_size, mapping.data());
  if (inputs[0] != canaryBegin || inputs[1] != canaryBegin || inputs[inputs_size + 2] != canaryEnd ||
      inputs[inputs_size + 3] != canaryEnd)
    throw std::runtime_error("Canary of the input buffer overwritten");

  results[0] = results[1] = canaryBegin;
  results[results_size + 2] = results[results_size + 3] = canaryEnd;
  slotToken slot = 0;
  if (algoconfig.useRemoteBuffer) slot = queue_slot(maxbucket);
  prepared_remote_compare(inputs.data() + 2, inputs.data() + 2 + inputs_size, results.data() + 2,
                          results.data() + 2 + results_size, slot);
  if (results[0] != canaryBegin || results[1] != canaryBegin || results[results_size + 2] != canaryEnd ||
      results[results_size + 3] != canaryEnd)
    throw std::runtime_error("Canary of the result buffer overwritten");

  // Reorder results by mapping (ipu_batch_affine.cpp:633-655).
  const size_t a_off = scores.size(), b_off = scores.size() + a_range_result.size();
  int nonzero = 0;
  for (size_t i = 0; i < mapping.size(); ++i) {
    const size_t m = mapping[i];
    scores[i] = results[m + 2];
    a_range_result[i] = results[a_off + m + 2];
    b_range_result[i] = results[b_off + m + 2];
    nonzero += scores[i] > 0;
    if (errcheck && scores[i] >= algoconfig.maxAB)
      throw std::runtime_error("errcheck: score " + std::to_string(scores[i]) + " of comparison " +
                               std::to_string(i) + " is not below maxAB");
  }
  if (errcheck && !A.empty() && (double)nonzero / A.size() < 0.5)
    throw std::runtime_error("errcheck: more than half of the scores are 0");
}

void SWAlgorithm::transferResults(int32_t* results_begin, int32_t* results_end, int* mapping_begin, int* mapping_end,
                                  int32_t* scores_begin, int32_t* scores_end, int32_t* arange_begin,
                                  int32_t* arange_end, int32_t* brange_begin, int32_t* brange_end) {
  transferResults(results_begin, results_end, mapping_begin, mapping_end, scores_begin, scores_end, arange_begin,
                  arange_end, brange_begin, brange_end, (int)(mapping_end - mapping_begin));
}

void SWAlgorithm::transferResults(int32_t* results_begin, int32_t* results_end, int* mapping_begin, int*,
                                  int32_t* scores_begin, int32_t*, int32_t* arange_begin, int32_t*,
                                  int32_t* brange_begin, int32_t*, int numComparisons) {
  const size_t results_size = results_end - results_begin;
  if (results_size % 3 != 0) throw std::runtime_error("Results buffer not 3 aligned.");
  const size_t part = results_size / 3;
  const int32_t* rs = results_begin;
  const int32_t* ra = results_begin + part;
  const int32_t* rb = results_begin + 2 * part;
  for (int i = 0; i < numComparisons; ++i) {
    const auto m = mapping_begin[i];
    scores_begin[i] = rs[m];
    arange_begin[i] = ra[m];
    brange_begin[i] = rb[m];
  }
}

void SWAlgorithm::compare_mn_local(const std::vector<std::string>& Seqs, const Comparisons& Cmps, bool errcheck) {
  (void)errcheck;
  const size_t inputs_size = algoconfig.getInputBufferSize32b();
  std::vector<int32_t> inputs(inputs_size);
  const size_t results_size = scores.size() + a_range_result.size() + b_range_result.size();
  std::vector<int32_t> results(results_size);
  if ((long)Cmps.size() > (long)algoconfig.getTotalNumberOfComparisons())
    throw std::runtime_error("Input sequence (A) is over the max length.");
  for (const auto& c : Cmps) {
    if (c.indexA < 0 || c.indexB < 0 || (size_t)c.indexA >= Seqs.size() || (size_t)c.indexB >= Seqs.size())
      throw std::runtime_error("Comparison index out of range.");
    if ((int)Seqs[c.indexA].size() > algoconfig.maxAB)
      throw std::runtime_error("Sequence size in seq " + std::to_string(Seqs[c.indexA].size()) + " > " +
                               std::to_string(algoconfig.maxAB));
  }
  std::vector<int> mapping(Cmps.size(), 0);
  partition::BucketMap map(algoconfig.tilesUsed, algoconfig.maxBatches, algoconfig.bufsize);
  fillMNBuckets(algoconfig.fillAlgo, map, Seqs, Cmps, 0);
  fill_input_buffer(map, config.datatype, algoconfig, Seqs, Cmps, inputs.data(), inputs.data() + inputs.size(),
                    mapping.data());
  int maxBucket = 0;
  for (const auto& b : map.buckets) maxBucket = std::max(maxBucket, b.seqSize);
  slotToken slot = 0;
  if (algoconfig.useRemoteBuffer) slot = queue_slot(maxBucket);
  prepared_remote_compare(inputs.data(), inputs.data() + inputs.size(), results.data(),
                          results.data() + results.size(), slot);
  transferResults(results.data(), results.data() + results.size(), mapping.data(), mapping.data() + mapping.size(),
                  scores.data(), scores.data() + scores.size(), a_range_result.data(),
                  a_range_result.data() + a_range_result.size(), b_range_result.data(),
                  b_range_result.data() + b_range_result.size());
}

// Wire layout (ipu_batch_affine.cpp:161-167,287): bucket b's sequences at
// byte b * 4*ceil(bufsize/4); Meta at word tilesUsed * ceil(bufsize/4), four
// words per slot; mapping[cmp] = bucket * maxBatches + slot.
static void writeBuckets(const partition::BucketMap& map, const swatlib::DataType dtype,
                         const IPUAlgoConfig& algoconfig, int32_t* inputs_begin, int32_t* inputs_end,
                         int32_t* mapping, const RawSequences* A, const RawSequences* B, const RawSequences* Seqs) {
  const size_t words = inputs_end - inputs_begin;
  if (words < (size_t)algoconfig.getInputBufferSize32b())
    throw std::runtime_error("Input buffer smaller than getInputBufferSize32b().");
  std::memset(inputs_begin, 0, words * sizeof(int32_t));
  const auto table = swatlib::getEncoder(dtype).getCodeTable();
  const size_t bucketBytes = (size_t)algoconfig.getBufsize32b() * 4;
  int8_t* seqs = reinterpret_cast<int8_t*>(inputs_begin);
  int32_t* meta = inputs_begin + algoconfig.getTotalBufsize32b();
  for (const auto& bm : map.buckets) {
    if (bm.bucketIndex >= algoconfig.tilesUsed) throw std::runtime_error("Bucket index out of range.");
    int8_t* bseq = seqs + (size_t)bm.bucketIndex * bucketBytes;
    int32_t* bmeta = meta + (size_t)bm.bucketIndex * algoconfig.maxBatches * 4;
    for (const auto& sm : bm.seqs) {
      const std::string* s = nullptr;
      switch (sm.origin) {
        case partition::SequenceOrigin::A:
          if (!A) throw std::runtime_error("Using A/B mapping with unordered comparison.");
          s = &(*A)[sm.index];
          break;
        case partition::SequenceOrigin::B:
          if (!B) throw std::runtime_error("Using A/B mapping with unordered comparison.");
          s = &(*B)[sm.index];
          break;
        case partition::SequenceOrigin::unordered:
          if (!Seqs) throw std::runtime_error("Using unordered mapping with A/B comparison.");
          s = &(*Seqs)[sm.index];
          break;
      }
      if ((size_t)sm.offset + s->size() > bucketBytes) throw std::runtime_error("Bucket overflow.");
      encodeInto(table, dtype, *s, bseq + sm.offset);
    }
    for (size_t i = 0; i < bm.cmps.size(); ++i) {
      const auto& c = bm.cmps[i];
      bmeta[i * 4 + 0] = c.sizeA;
      bmeta[i * 4 + 1] = c.offsetA;
      bmeta[i * 4 + 2] = c.sizeB;
      bmeta[i * 4 + 3] = c.offsetB;
      mapping[c.comparisonIndex] = map.cmpCapacity * bm.bucketIndex + (int)i;
    }
  }
}

void SWAlgorithm::fill_input_buffer(const partition::BucketMap& map, const swatlib::DataType dtype,
                                    const IPUAlgoConfig& algoconfig, const RawSequences& Seqs,
                                    const Comparisons& Cmps, int32_t* inputs_begin, int32_t* inputs_end,
                                    int32_t* mapping) {
  (void)Cmps;
  writeBuckets(map, dtype, algoconfig, inputs_begin, inputs_end, mapping, nullptr, nullptr, &Seqs);
}

void SWAlgorithm::fill_input_buffer(const partition::BucketMap& map, const swatlib::DataType dtype,
                                    const IPUAlgoConfig& algoconfig, const RawSequences& A, const RawSequences& B,
                                    int32_t* inputs_begin, int32_t* inputs_end, int32_t* mapping) {
  writeBuckets(map, dtype, algoconfig, inputs_begin, inputs_end, mapping, &A, &B, nullptr);
}

int SWAlgorithm::prepare_remote(const SWConfig& swconfig, const IPUAlgoConfig& algoconfig,
                                const std::vector<std::string>& A, const std::vector<std::string>& B,
                                int32_t* inputs_begin, int32_t* inputs_end, int* seqMapping) {
  if (A.size() != B.size()) throw std::runtime_error("A and B must hold the same number of sequences.");
  checkSequenceSizes(algoconfig, A);
  partition::BucketMap map(algoconfig.tilesUsed, algoconfig.maxBatches, algoconfig.bufsize);
  fillBuckets(algoconfig.fillAlgo, map, A, B, 0);
  fill_input_buffer(map, swconfig.datatype, algoconfig, A, B, inputs_begin, inputs_end, seqMapping);
  int maxBucket = 0;
  for (const auto& b : map.buckets) maxBucket = std::max(maxBucket, b.seqSize);
  return maxBucket;
}

slotToken SWAlgorithm::queue_slot(int max_bucket_size) {
  const int si = std::max(0, calculate_slot_region_index(max_bucket_size));
  if (si >= (int)slots.size()) throw std::runtime_error("No slot region for this buffer size.");
  int s = -1;
  for (int i = 0; i < (int)slots[si].size(); ++i)
    if (!slots[si][i]) {
      s = i;
      break;
    }
  if (s < 0) throw std::runtime_error("No free slot.");
  slots[si][s] = true;
  slot_avail[si]--;
  last_slot = s;
  return s + (long)si * slot_size;
}

void SWAlgorithm::release_slot(slotToken i) {
  auto [lot, sid] = unpack_slot(i);
  if (lot < 0 || lot >= (int)slots.size() || sid < 0 || sid >= (long)slots[lot].size()) return;
  if (slots[lot][sid]) {
    slots[lot][sid] = false;
    slot_avail[lot]++;
  }
}

bool SWAlgorithm::slot_available(int max_buffer_size) {
  const int si = calculate_slot_region_index(max_buffer_size);
  return si >= 0 && si < (int)slot_avail.size() && slot_avail[si] > 0;
}

int SWAlgorithm::calculate_slot_region_index(const IPUAlgoConfig& algoconfig, int max_buffer_size) {
  return (int)std::ceil((max_buffer_size / (double)algoconfig.bufsize) *
                        static_cast<double>(algoconfig.transmissionPrograms)) -
         1;
}

int SWAlgorithm::calculate_slot_region_index(int max_buffer_size) {
  return calculate_slot_region_index(algoconfig, max_buffer_size);
}

void SWAlgorithm::run_executor() {}

}  // namespace batchaffine
}  // namespace ipu
