// Host-side bucket partitioning of comparisons (src/partition.h:1-80).
//
// Keeps the reference's contract: `numBuckets` buckets (one per IPU tile in
// the reference, one wire-buffer region here), each holding at most
// `cmpCapacity` comparisons and `sequenceCapacity` bytes of sequence.
// Policies fillFirst / roundRobin / greedy and their M x N variants (which
// store a sequence shared by several comparisons of a bucket only once)
// produce the same assignment as the reference for inputs that fit.
#ifndef IPUMA_B200_PARTITION_H
#define IPUMA_B200_PARTITION_H

#include <deque>
#include <functional>
#include <queue>
#include <string>
#include <vector>

#include "types.h"

namespace ipu {
namespace partition {

enum class SequenceOrigin { unordered, A, B };
std::string sequenceOriginToString(SequenceOrigin o);

struct ComparisonMapping {
  int comparisonIndex;  // index in the comparison input list
  int sizeA;
  int offsetA;
  int sizeB;
  int offsetB;
  std::string toString();
};

struct SequenceMapping {
  int index;  // index in the sequence input list
  int offset;
  SequenceOrigin origin = SequenceOrigin::unordered;
  std::string toString();
};

struct BucketMapping {
  int bucketIndex = 0;
  int maxLen = 0;   // length of the longest sequence
  int seqSize = 0;  // bytes of sequence stored
  int weight[6] = {};  // cost per slot group (roundRobin / greedy)
  std::vector<SequenceMapping> seqs;
  std::vector<ComparisonMapping> cmps;
  std::string toString();
};

// Heap order of the greedy policy: by the smallest of the six weights.
bool operator<(const BucketMapping& b1, const BucketMapping& b2);
bool operator>(const BucketMapping& b1, const BucketMapping& b2);

struct BucketMap {
  std::vector<BucketMapping> buckets;
  int numBuckets;
  int cmpCapacity;
  int sequenceCapacity;

  BucketMap();
  BucketMap(int nB, int nC, int sC);
  std::string toString();
};

struct BucketData {
  int count;
  int lenSeq;
  int weight;
};

using BucketHeap = std::priority_queue<std::reference_wrapper<BucketMapping>,
                                       std::deque<std::reference_wrapper<BucketMapping>>,
                                       std::greater<std::reference_wrapper<BucketMapping>>>;

bool fillFirst(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset, int& curBucket);
bool roundRobin(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset, int& curBucket);
bool greedy(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset, BucketHeap& heap);

void fillFirst(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset = 0);
void roundRobin(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset = 0);
void greedy(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset = 0);

void fillFirst(BucketMap& map, const RawSequences& Seqs, const Comparisons& Cmps, int indexOffset = 0);
void roundRobin(BucketMap& map, const RawSequences& Seqs, const Comparisons& Cmps, int indexOffset = 0);
void greedy(BucketMap& map, const RawSequences& Seqs, const Comparisons& Cmps, int indexOffset = 0);

bool fillBuckets(Algorithm algo, BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset,
                 int& curBucket, BucketHeap& heap);

}  // namespace partition
}  // namespace ipu

#endif
