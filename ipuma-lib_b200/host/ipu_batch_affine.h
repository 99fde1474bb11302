// ipu::batchaffine::SWAlgorithm -- the reference's batch driver API
// (src/ipu_batch_affine.h:18-120) on the B200 engine of include/ipuma_b200.h.
//
// Same class, method names, arguments, wire buffers and result layout, so
// callers of the reference compile and run unchanged.  Differences:
//   * the device is a CUDA GPU (thread_id selects device thread_id % count);
//   * conditions the reference ends with exit(1) (|A| > maxAB, overwritten
//     canaries) throw std::runtime_error instead;
//   * refetch/upload/printTensors, which the reference leaves unimplemented
//     (assert), throw std::runtime_error;
//   * a pair with an empty sequence scores 0 and does not stop the
//     comparisons after it in its bucket.
#ifndef IPUMA_B200_IPU_BATCH_AFFINE_H
#define IPUMA_B200_IPU_BATCH_AFFINE_H

#define WORK_QUEUE_SIZE 100'000

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "ipu_config.h"
#include "ipuma_b200.h"
#include "partition.h"

namespace ipu {
namespace batchaffine {

using slotToken = long;

struct BlockAlignmentResults {
  std::vector<int32_t> scores;
  std::vector<int32_t> a_range_result;
  std::vector<int32_t> b_range_result;
};

// Handle of an asynchronous batch (ipu_batch_affine.h:40-48).  Created by
// async_submit_prepared_remote_compare, deleted by the caller.
struct Job {
  Job() : tick({}) {}
  // Waits for the batch; throws std::runtime_error on failure.
  void join();
  uint64_t h2dCycles = 0;    // device time of the batch in ns (H2D + kernels)
  uint64_t innerCycles = 0;  // device time of the kernels in ns
  swatlib::TickTock tick;
  ipuma_engine* engine = nullptr;
  uint64_t id = 0;
  bool joined = false;
};

class SWAlgorithm {
 private:
  ipuma_engine* engine_ = nullptr;
  std::vector<int32_t> scores;
  std::vector<int32_t> a_range_result;
  std::vector<int32_t> b_range_result;

  int slot_size = 1;
  std::vector<int> slot_avail;
  int last_slot = 0;
  std::vector<std::vector<bool>> slots;

  static size_t getSeqsOffset(const IPUAlgoConfig& config);
  static size_t getMetaOffset(const IPUAlgoConfig& config);

  void release_slot(slotToken i);

 protected:
  int thread_id = 0;
  int ipus = 1;

 public:
  SWConfig config;
  IPUAlgoConfig algoconfig;

  SWAlgorithm(SWConfig config, IPUAlgoConfig algoconfig);
  SWAlgorithm(SWConfig config, IPUAlgoConfig algoconfig, int thread_id, size_t slotCap = 1, size_t ipuCount = 1,
              bool runExecutor = true);
  SWAlgorithm(const SWAlgorithm&) = delete;
  SWAlgorithm& operator=(const SWAlgorithm&) = delete;
  ~SWAlgorithm();

  std::string printTensors();

  static int calculate_slot_region_index(const IPUAlgoConfig& algoconfig, int max_buffer_size);
  int calculate_slot_region_index(int max_buffer_size);
  std::tuple<int, slotToken> unpack_slot(slotToken);
  bool slot_available(int max_buffer_size);
  slotToken queue_slot(int max_buffer_size);

  static void checkSequenceSizes(const IPUAlgoConfig& algoconfig, const std::vector<int>& SeqSizes);
  static void checkSequenceSizes(const IPUAlgoConfig& algoconfig, const RawSequences& Seqs);

  static void fillBuckets(Algorithm algo, partition::BucketMap& map, const RawSequences& A, const RawSequences& B,
                          int offset = 0);
  static void fillMNBuckets(Algorithm algo, partition::BucketMap& map, const RawSequences& Seqs,
                            const Comparisons& Cmps, int offset = 0);

  static void fill_input_buffer(const partition::BucketMap& map, const swatlib::DataType dtype,
                                const IPUAlgoConfig& algoconfig, const RawSequences& Seqs, const Comparisons& Cmps,
                                int32_t* inputs_begin, int32_t* inputs_end, int32_t* mapping);
  static void fill_input_buffer(const partition::BucketMap& map, const swatlib::DataType dtype,
                                const IPUAlgoConfig& algoconfig, const RawSequences& A, const RawSequences& B,
                                int32_t* inputs_begin, int32_t* inputs_end, int32_t* mapping);

  BlockAlignmentResults get_result();

  // Local buffers
  void compare_local(const std::vector<std::string>& A, const std::vector<std::string>& B, bool errcheck = false);
  void compare_mn_local(const std::vector<std::string>& Seqs, const Comparisons& Cmps, bool errcheck = false);

  void refetch();

  // Prepared ("remote") buffers
  void prepared_remote_compare(int32_t* inputs_begin, int32_t* inputs_end, int32_t* results_begin,
                               int32_t* results_end, slotToken slot_token = 0);
  Job* async_submit_prepared_remote_compare(int32_t* inputs_begin, int32_t* inputs_end, int32_t* results_begin,
                                            int32_t* results_end);
  void blocking_join_prepared_remote_compare(Job& job);

  void upload(int32_t* inputs_begin, int32_t* inputs_end, slotToken slot);

  void run_executor();
  static int prepare_remote(const SWConfig& swconfig, const IPUAlgoConfig& algoconfig,
                            const std::vector<std::string>& A, const std::vector<std::string>& B,
                            int32_t* inputs_begin, int32_t* inputs_end, int* deviceMapping);
  static void transferResults(int32_t* results_begin, int32_t* results_end, int* mapping_begin, int* mapping_end,
                              int32_t* scores_begin, int32_t* scores_end, int32_t* arange_begin,
                              int32_t* arange_end, int32_t* brange_begin, int32_t* brange_end);
  static void transferResults(int32_t* results_begin, int32_t* results_end, int* mapping_begin, int* mapping_end,
                              int32_t* scores_begin, int32_t* scores_end, int32_t* arange_begin,
                              int32_t* arange_end, int32_t* brange_begin, int32_t* brange_end,
                              int numComparisons);

  // The underlying engine (C ABI handle), e.g. for ipuma_gpu_set_option.
  ipuma_engine* engine() const { return engine_; }
};

}  // namespace batchaffine
}  // namespace ipu
#endif
