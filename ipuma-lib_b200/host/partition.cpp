// Bucket policies of src/partition.cpp, restated.
//
//   fillFirst   (:197-223)  first bucket from the current one (wrapping) with
//                           room for the comparison; stays there
//   roundRobin  (:241-289)  same search, then moves to the next bucket
//   greedy      (:378-462)  comparisons by descending |A|*|B| (std::sort),
//                           each to the top of a min-heap on the bucket's
//                           smallest slot-group weight, skipping full buckets
//   M x N forms (:105-172, :225-239, :291-376) reuse a sequence already
//                           stored in the bucket (it costs no bytes there)
//
// One deviation: when greedy meets a full bucket at the top of the heap the
// reference assigns the next heap entry *into* the full bucket object
// (`bucket = q.top().get()` through a reference, :337/:408), which overwrites
// that bucket's contents.  Here the next bucket is taken instead.  Results
// are identical whenever no full bucket reaches the top of the heap.
#include "partition.h"

#include <algorithm>
#include <climits>
#include <sstream>
#include <stdexcept>
#include <utility>

namespace ipu {
namespace partition {

std::string sequenceOriginToString(SequenceOrigin o) {
  switch (o) {
    case SequenceOrigin::A: return "SequenceOrigin::A";
    case SequenceOrigin::B: return "SequenceOrigin::B";
    case SequenceOrigin::unordered: return "SequenceOrigin::unordered";
  }
  throw std::runtime_error("Unhandled sequence type.");
}

std::string ComparisonMapping::toString() {
  std::stringstream ss;
  ss << "CM[" << comparisonIndex << ": a(l" << sizeA << " o" << offsetA << ") b(l" << sizeB << " o" << offsetB << ")]";
  return ss.str();
}

std::string SequenceMapping::toString() {
  std::stringstream ss;
  ss << "SM[" << index << ": o" << offset << " t" << sequenceOriginToString(origin) << "]";
  return ss.str();
}

std::string BucketMapping::toString() {
  std::stringstream ss;
  ss << "BMapping[" << bucketIndex << ": cmps(" << cmps.size() << ") maxLen(" << maxLen << ") seqSize(" << seqSize
     << ")]";
  return ss.str();
}

std::string BucketMap::toString() {
  std::stringstream ss;
  ss << "BMap[" << numBuckets << ": maxCmps(" << cmpCapacity << ") bufsize(" << sequenceCapacity << ")]";
  return ss.str();
}

BucketMap::BucketMap() : numBuckets(0), cmpCapacity(0), sequenceCapacity(0) {}

BucketMap::BucketMap(int nB, int cC, int sC) : numBuckets(nB), cmpCapacity(cC), sequenceCapacity(sC) {
  buckets.resize(nB);
  for (int i = 0; i < nB; ++i) buckets[i].bucketIndex = i;
}

static inline int minWeight(const int z[6]) { return *std::min_element(z, z + 6); }

bool operator>(const BucketMapping& b1, const BucketMapping& b2) { return minWeight(b1.weight) > minWeight(b2.weight); }
bool operator<(const BucketMapping& b1, const BucketMapping& b2) { return minWeight(b1.weight) < minWeight(b2.weight); }

namespace {

bool fits(const BucketMap& map, const BucketMapping& b, long bytes) {
  return (long)b.cmps.size() + 1 <= map.cmpCapacity && (long)b.seqSize + bytes <= map.sequenceCapacity;
}

// Appends one A/B comparison (both sequences stored) to a bucket.
void addPair(BucketMapping& bucket, int ci, int aLen, int bLen) {
  bucket.maxLen = std::max(bucket.maxLen, std::max(aLen, bLen));
  const int offsetA = bucket.seqSize;
  const int offsetB = bucket.seqSize + aLen;
  bucket.seqs.push_back({ci, offsetA, SequenceOrigin::A});
  bucket.seqs.push_back({ci, offsetB, SequenceOrigin::B});
  bucket.cmps.push_back({ci, aLen, offsetA, bLen, offsetB});
  bucket.seqSize += aLen + bLen;
}

// Where a comparison of the M x N form would go in `bucket`: bytes it costs
// and the offsets of sequences the bucket already holds.
struct MNPlacement {
  int effA, effB, offA, offB;
};

MNPlacement placeMN(const BucketMapping& bucket, int ai, int bi, int aLen, int bLen) {
  MNPlacement pl{aLen, bLen, 0, 0};
  for (const auto& s : bucket.seqs) {
    if (s.index == ai) {
      pl.effA = 0;
      pl.offA = s.offset;
    }
    if (s.index == bi) {
      pl.effB = 0;
      pl.offB = s.offset;
    }
  }
  return pl;
}

void addMN(BucketMapping& bucket, MNPlacement pl, int ai, int bi, int ci, int aLen, int bLen) {
  bucket.maxLen = std::max(bucket.maxLen, std::max(aLen, bLen));
  if (pl.effA) {
    pl.offA = bucket.seqSize;
    bucket.seqs.push_back({ai, pl.offA, SequenceOrigin::unordered});
  }
  if (pl.effB) {
    pl.offB = bucket.seqSize + pl.effA;
    bucket.seqs.push_back({bi, pl.offB, SequenceOrigin::unordered});
  }
  bucket.cmps.push_back({ci, aLen, pl.offA, bLen, pl.offB});
  bucket.seqSize += pl.effA + pl.effB;
}

// M x N search from `start` (wrapping) for the first bucket with room.
BucketMapping& nextMNBucket(BucketMap& map, int start, int ai, int bi, int aLen, int bLen, MNPlacement& pl) {
  for (int off = 0; off < map.numBuckets; ++off) {
    auto& bucket = map.buckets[(start + off) % map.numBuckets];
    pl = placeMN(bucket, ai, bi, aLen, bLen);
    if (fits(map, bucket, (long)pl.effA + pl.effB)) return bucket;
  }
  throw std::runtime_error("Out of buckets.");
}

void logBucketWeights(const BucketMap&) {}

}  // namespace

bool fillFirst(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset, int& curBucket) {
  for (size_t i = 0; i < A.size(); ++i) {
    const int aLen = (int)A[i].size(), bLen = (int)B[i].size();
    int off = 0;
    for (; off < map.numBuckets; ++off)
      if (fits(map, map.buckets[(curBucket + off) % map.numBuckets], (long)aLen + bLen)) break;
    if (off >= map.numBuckets) return false;
    curBucket = (curBucket + off) % map.numBuckets;
    addPair(map.buckets[curBucket], indexOffset + (int)i, aLen, bLen);
  }
  return true;
}

bool roundRobin(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset, int& curBucket) {
  for (size_t i = 0; i < A.size(); ++i) {
    const int aLen = (int)A[i].size(), bLen = (int)B[i].size();
    int off = 0;
    for (; off < map.numBuckets; ++off)
      if (fits(map, map.buckets[(curBucket + off) % map.numBuckets], (long)aLen + bLen)) break;
    if (off >= map.numBuckets) return false;
    curBucket = (curBucket + off) % map.numBuckets;
    auto& bucket = map.buckets[curBucket];
    addPair(bucket, indexOffset + (int)i, aLen, bLen);
    bucket.weight[(bucket.cmps.size() - 1) % 6] += aLen * bLen;
    curBucket++;
  }
  logBucketWeights(map);
  return true;
}

bool greedy(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset, BucketHeap& q) {
  std::vector<std::pair<int, int>> order(A.size());
  for (size_t i = 0; i < A.size(); ++i) order[i] = {(int)(A[i].size() * B[i].size()), (int)i};
  std::sort(order.begin(), order.end(),
            [](std::pair<int, int>& a, std::pair<int, int>& b) { return a.first > b.first; });
  for (size_t k = 0; k < order.size(); ++k) {
    const int idx = order[k].second;
    const int aLen = (int)A[idx].size(), bLen = (int)B[idx].size();
    std::deque<std::reference_wrapper<BucketMapping>> skipped;
    BucketMapping* bucket = nullptr;
    int tries = 0;
    while (tries < map.numBuckets && !q.empty()) {
      BucketMapping& top = q.top().get();
      q.pop();
      if (fits(map, top, (long)aLen + bLen)) {
        bucket = &top;
        break;
      }
      skipped.push_back(std::ref(top));
      tries++;
    }
    for (auto b : skipped) q.push(b);
    if (!bucket) return false;
    addPair(*bucket, indexOffset + idx, aLen, bLen);
    bucket->weight[(bucket->cmps.size() - 1) % 6] += aLen * bLen;
    q.push(std::ref(*bucket));
  }
  logBucketWeights(map);
  return true;
}

void fillFirst(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset) {
  int cur = 0;
  if (!fillFirst(map, A, B, indexOffset, cur)) throw std::runtime_error("Out of buckets.");
}

void roundRobin(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset) {
  int cur = 0;
  if (!roundRobin(map, A, B, indexOffset, cur)) throw std::runtime_error("Out of buckets.");
}

void greedy(BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset) {
  BucketHeap q;
  for (auto& b : map.buckets) q.push(std::ref(b));
  if (!greedy(map, A, B, indexOffset, q)) throw std::runtime_error("Out of buckets.");
}

void fillFirst(BucketMap& map, const RawSequences& Seqs, const Comparisons& Cmps, int indexOffset) {
  int cur = 0;
  for (size_t i = 0; i < Cmps.size(); ++i) {
    const auto& c = Cmps[i];
    const int aLen = (int)Seqs[c.indexA].size(), bLen = (int)Seqs[c.indexB].size();
    MNPlacement pl;
    auto& bucket = nextMNBucket(map, cur, indexOffset + c.indexA, indexOffset + c.indexB, aLen, bLen, pl);
    cur = bucket.bucketIndex;
    addMN(bucket, pl, indexOffset + c.indexA, indexOffset + c.indexB, indexOffset + (int)i, aLen, bLen);
  }
}

void roundRobin(BucketMap& map, const RawSequences& Seqs, const Comparisons& Cmps, int indexOffset) {
  int cur = 0;
  for (size_t i = 0; i < Cmps.size(); ++i) {
    const auto& c = Cmps[i];
    const int aLen = (int)Seqs[c.indexA].size(), bLen = (int)Seqs[c.indexB].size();
    MNPlacement pl;
    auto& bucket = nextMNBucket(map, cur, indexOffset + c.indexA, indexOffset + c.indexB, aLen, bLen, pl);
    addMN(bucket, pl, indexOffset + c.indexA, indexOffset + c.indexB, indexOffset + (int)i, aLen, bLen);
    cur = bucket.bucketIndex + 1;
  }
}

void greedy(BucketMap& map, const RawSequences& Seqs, const Comparisons& Cmps, int indexOffset) {
  BucketHeap q;
  for (auto& b : map.buckets) q.push(std::ref(b));
  std::vector<std::pair<int, int>> order(Cmps.size());
  for (size_t i = 0; i < Cmps.size(); ++i)
    order[i] = {(int)(Seqs[Cmps[i].indexA].size() * Seqs[Cmps[i].indexB].size()), (int)i};
  std::sort(order.begin(), order.end(),
            [](std::pair<int, int>& a, std::pair<int, int>& b) { return a.first > b.first; });
  for (size_t k = 0; k < order.size(); ++k) {
    const int ci = order[k].second;
    const auto& c = Cmps[ci];
    const int aLen = (int)Seqs[c.indexA].size(), bLen = (int)Seqs[c.indexB].size();
    const int ai = indexOffset + c.indexA, bi = indexOffset + c.indexB;
    std::deque<std::reference_wrapper<BucketMapping>> skipped;
    BucketMapping* bucket = nullptr;
    MNPlacement pl{};
    int tries = 0;
    while (tries < map.numBuckets && !q.empty()) {
      BucketMapping& top = q.top().get();
      q.pop();
      pl = placeMN(top, ai, bi, aLen, bLen);
      if (fits(map, top, (long)pl.effA + pl.effB)) {
        bucket = &top;
        break;
      }
      skipped.push_back(std::ref(top));
      tries++;
    }
    for (auto b : skipped) q.push(b);
    if (!bucket) throw std::runtime_error("Out of buckets");
    addMN(*bucket, pl, ai, bi, indexOffset + ci, aLen, bLen);
    bucket->weight[(bucket->cmps.size() - 1) % 6] += aLen * bLen;
    q.push(std::ref(*bucket));
  }
}

bool fillBuckets(Algorithm algo, BucketMap& map, const RawSequences& A, const RawSequences& B, int indexOffset,
                 int& curBucket, BucketHeap& heap) {
  switch (algo) {
    case Algorithm::fillFirst: return fillFirst(map, A, B, indexOffset, curBucket);
    case Algorithm::roundRobin: return roundRobin(map, A, B, indexOffset, curBucket);
    case Algorithm::greedy: return greedy(map, A, B, indexOffset, heap);
  }
  return false;
}

}  // namespace partition
}  // namespace ipu
