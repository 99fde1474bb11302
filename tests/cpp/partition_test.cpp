// Host-only tests of the drop-in layer, mirroring the reference's
// test/partition-test.cpp, test/mn_cmp-test.cpp:6-26 and
// test/simple-test.cpp:195-225 (PrepareTest).  No GPU needed.
#include <cstring>
#include <string>
#include <vector>

#include "ipu_batch_affine.h"
#include "mini_test.h"

namespace {
struct PartitioningFixture {
  int tilesUsed = 10;
  int maxBatches = 2;
  int maxAB = 10;
  int bufsize = 2 * 10 * 2;
  std::vector<std::string> a, b;
  ipu::partition::BucketMap map{10, 2, 40};
  void genFull() {
    for (int i = 0; i < tilesUsed * maxBatches; ++i) {
      a.push_back(std::string(maxAB, 'A'));
      b.push_back(std::string(maxAB, 'A'));
    }
  }
  void checkBucketIndices() {
    EXPECT_EQ((int)map.buckets.size(), tilesUsed);
    for (int i = 0; i < tilesUsed; ++i) EXPECT_EQ(map.buckets[i].bucketIndex, i);
  }
  void checkFull() {
    checkBucketIndices();
    for (int i = 0; i < tilesUsed; ++i) {
      EXPECT_EQ(map.buckets[i].maxLen, maxAB);
      EXPECT_EQ(map.buckets[i].seqSize, maxAB * maxBatches * 2);
    }
  }
};
}  // namespace

TEST(PartitioningTest, fullFillFirst) {
  PartitioningFixture f;
  f.genFull();
  ipu::batchaffine::SWAlgorithm::fillBuckets(ipu::Algorithm::fillFirst, f.map, f.a, f.b, 0);
  f.checkFull();
}

TEST(PartitioningTest, fullRoundRobin) {
  PartitioningFixture f;
  f.genFull();
  ipu::batchaffine::SWAlgorithm::fillBuckets(ipu::Algorithm::roundRobin, f.map, f.a, f.b, 0);
  f.checkFull();
}

TEST(PartitioningTest, fullGreedy) {
  PartitioningFixture f;
  f.genFull();
  ipu::batchaffine::SWAlgorithm::fillBuckets(ipu::Algorithm::greedy, f.map, f.a, f.b, 0);
  f.checkFull();
}

TEST(PartitioningTest, partialFillFirst) {
  PartitioningFixture f;
  f.a = {"AAAAAA", "AA"};
  f.b = {"AAAAAA", "AAA"};
  ipu::batchaffine::SWAlgorithm::fillBuckets(ipu::Algorithm::fillFirst, f.map, f.a, f.b, 0);
  f.checkBucketIndices();
  for (int i = 0; i < f.tilesUsed; ++i) {
    EXPECT_EQ(f.map.buckets[i].maxLen, i == 0 ? 6 : 0);
    EXPECT_EQ(f.map.buckets[i].seqSize, i == 0 ? 17 : 0);
  }
}

TEST(PartitioningTest, partialRoundRobin) {
  PartitioningFixture f;
  f.a = {"AAAAAA", "AA"};
  f.b = {"AAAAAA", "AAA"};
  ipu::batchaffine::SWAlgorithm::fillBuckets(ipu::Algorithm::roundRobin, f.map, f.a, f.b, 0);
  f.checkBucketIndices();
  for (int i = 0; i < f.tilesUsed; ++i) {
    const int ml = i == 0 ? 6 : (i == 1 ? 3 : 0);
    const int ss = i == 0 ? 12 : (i == 1 ? 5 : 0);
    EXPECT_EQ(f.map.buckets[i].maxLen, ml);
    EXPECT_EQ(f.map.buckets[i].seqSize, ss);
  }
}

TEST(PartitioningTest, outOfBuckets) {
  ipu::partition::BucketMap map(2, 1, 10);
  std::vector<std::string> a = {"AAAA", "AAAA", "AAAA"}, b = {"AAAA", "AAAA", "AAAA"};
  for (auto algo : {ipu::Algorithm::fillFirst, ipu::Algorithm::roundRobin, ipu::Algorithm::greedy}) {
    ipu::partition::BucketMap m(2, 1, 10);
    EXPECT_THROW(ipu::batchaffine::SWAlgorithm::fillBuckets(algo, m, a, b, 0));
  }
}

TEST(PartitionMNTest, compression) {
  for (auto algo : {ipu::Algorithm::fillFirst, ipu::Algorithm::roundRobin, ipu::Algorithm::greedy}) {
    ipu::RawSequences Seqs = {"AAAA", "AAAA", "AAAA"};
    ipu::Comparisons Cmps = {{0, 1}, {0, 2}, {0, 2}};
    ipu::partition::BucketMap map(1, 5, 100);
    ipu::batchaffine::SWAlgorithm::fillMNBuckets(algo, map, Seqs, Cmps);
    EXPECT_EQ(map.buckets[0].seqSize, 12);
    EXPECT_EQ((int)map.buckets[0].cmps.size(), 3);
  }
}

TEST(MN_Partitioning, checkMappingSimple) {
  ipu::IPUAlgoConfig algoconfig = {2, 30, 10, 1000};
  std::vector<std::string> seqs = {"AAAA", "TTTT", "GGGG", "CCCC"};
  ipu::Comparisons comparisons = {{0, 1}};
  ipu::partition::BucketMap map(algoconfig.tilesUsed, algoconfig.maxBatches, algoconfig.bufsize);
  ipu::batchaffine::SWAlgorithm::fillMNBuckets(algoconfig.fillAlgo, map, seqs, comparisons);
  EXPECT_EQ(map.numBuckets, 2);
  EXPECT_EQ((int)map.buckets[0].cmps.size(), 1);
  EXPECT_EQ((int)map.buckets[1].cmps.size(), 0);
  EXPECT_EQ(map.buckets[0].cmps[0].comparisonIndex, 0);
  EXPECT_EQ(map.buckets[0].cmps[0].offsetA, 0);
  EXPECT_EQ(map.buckets[0].cmps[0].offsetB, 4);
}

TEST(PrepareTest, simple) {
  const int tilesUsed = 10, maxBatches = 2, maxAB = 10, bufsize = maxBatches * maxAB * 2;
  ipu::SWConfig swconfig = {};
  ipu::IPUAlgoConfig config = {tilesUsed, maxAB, maxBatches, bufsize, ipu::VertexType::cpp,
                               ipu::Algorithm::fillFirst};
  std::vector<std::string> A, B;
  for (int i = 0; i < tilesUsed * maxBatches; ++i) {
    A.push_back(std::string(maxAB, 'A'));
    B.push_back(std::string(maxAB, 'A'));
  }
  std::vector<int32_t> inputs(config.getInputBufferSize32b() + 2);
  std::vector<int> mapping(A.size(), 0);
  inputs[0] = (int32_t)0xDEADBEEF;
  inputs[inputs.size() - 1] = (int32_t)0xDEADBEEF;
  ipu::batchaffine::SWAlgorithm::prepare_remote(swconfig, config, A, B, inputs.data() + 1,
                                                inputs.data() + inputs.size() - 1, mapping.data());
  EXPECT_EQ(inputs[0], (int32_t)0xDEADBEEF);
  EXPECT_EQ(inputs[inputs.size() - 1], (int32_t)0xDEADBEEF);
  // Layout: bucket t's sequences at byte t * 40, Meta after tilesUsed * 10 words.
  const int32_t* meta = inputs.data() + 1 + config.getTotalBufsize32b();
  for (int i = 0; i < tilesUsed * maxBatches; ++i) {
    EXPECT_EQ(meta[4 * mapping[i] + 0], maxAB);
    EXPECT_EQ(meta[4 * mapping[i] + 2], maxAB);
  }
  const uint8_t* seq = reinterpret_cast<const uint8_t*>(inputs.data() + 1);
  EXPECT_EQ((int)seq[0], 1);  // 'A' -> code 1
}

TEST(PrepareTest, mappingFollowsBuckets) {
  ipu::IPUAlgoConfig config = {3, 20, 4, 64, ipu::VertexType::cpp, ipu::Algorithm::roundRobin};
  std::vector<std::string> A = {"ACGT", "TTTTT", "GG", "ACGTACGT", "C"};
  std::vector<std::string> B = {"ACG", "TTTT", "GGGG", "ACGT", "CCCCCC"};
  std::vector<int32_t> inputs(config.getInputBufferSize32b());
  std::vector<int> mapping(A.size(), -1);
  ipu::batchaffine::SWAlgorithm::prepare_remote({}, config, A, B, inputs.data(), inputs.data() + inputs.size(),
                                                mapping.data());
  const uint8_t* seqs = reinterpret_cast<const uint8_t*>(inputs.data());
  const int32_t* meta = inputs.data() + config.getTotalBufsize32b();
  const auto enc = swatlib::getEncoder(swatlib::DataType::nucleicAcid);
  for (size_t i = 0; i < A.size(); ++i) {
    const int g = mapping[i];
    const int tile = g / config.maxBatches;
    const uint8_t* base = seqs + tile * config.getBufsize32b() * 4;
    EXPECT_EQ(meta[4 * g], (int)A[i].size());
    EXPECT_EQ(meta[4 * g + 2], (int)B[i].size());
    for (size_t j = 0; j < A[i].size(); ++j) EXPECT_EQ(base[meta[4 * g + 1] + j], enc.encode(A[i][j]));
    for (size_t j = 0; j < B[i].size(); ++j) EXPECT_EQ(base[meta[4 * g + 3] + j], enc.encode(B[i][j]));
  }
}

TEST(PrepareTest, rejectsTooLongA) {
  ipu::IPUAlgoConfig config = {1, 4, 4, 64};
  std::vector<int32_t> inputs(config.getInputBufferSize32b());
  std::vector<int> mapping(1);
  EXPECT_THROW(ipu::batchaffine::SWAlgorithm::prepare_remote({}, config, {"ACGTA"}, {"A"}, inputs.data(),
                                                             inputs.data() + inputs.size(), mapping.data()));
}

TEST(PrepareTest, rejectsUnknownNucleotide) {
  ipu::IPUAlgoConfig config = {1, 10, 4, 64};
  std::vector<int32_t> inputs(config.getInputBufferSize32b());
  std::vector<int> mapping(1);
  EXPECT_THROW(ipu::batchaffine::SWAlgorithm::prepare_remote({}, config, {"ACXT"}, {"A"}, inputs.data(),
                                                             inputs.data() + inputs.size(), mapping.data()));
}

TEST(Config, jsonRoundTrip) {
  ipu::SWConfig sw = {-10, -1, 2, -3, -4, swatlib::Similarity::blosum62, swatlib::DataType::aminoAcid};
  auto sw2 = ipu::swConfigFromJson(ipu::toJsonString(sw));
  EXPECT_EQ(sw2.gapInit, -10);
  EXPECT_EQ(sw2.mismatchValue, -3);
  EXPECT_EQ(sw2.ambiguityValue, -4);
  EXPECT_TRUE(sw2.similarity == swatlib::Similarity::blosum62);
  ipu::IPUAlgoConfig al = {7, 123, 9, 4000, ipu::VertexType::multiasm, ipu::Algorithm::greedy, true};
  auto al2 = ipu::algoConfigFromJson(ipu::toJsonString(al));
  EXPECT_EQ(al2.tilesUsed, 7);
  EXPECT_EQ(al2.maxAB, 123);
  EXPECT_EQ(al2.bufsize, 4000);
  EXPECT_TRUE(al2.vtype == ipu::VertexType::multiasm);
  EXPECT_TRUE(al2.fillAlgo == ipu::Algorithm::greedy);
  EXPECT_TRUE(al2.forwardOnly);
  EXPECT_EQ(al.getInputBufferSize32b(), 7 * 1000 + 7 * 9 * 4);
}

TEST(Swatlib, encoders) {
  auto na = swatlib::getEncoder(swatlib::DataType::nucleicAcid);
  EXPECT_EQ((int)na.encode('A'), 1);
  EXPECT_EQ((int)na.encode('a'), 1);
  EXPECT_EQ((int)na.encode('N'), 0);
  EXPECT_EQ((int)na.encode('X'), 16);
  auto aa = swatlib::getEncoder(swatlib::DataType::aminoAcid);
  EXPECT_EQ((int)aa.encode('W'), 17);
  EXPECT_EQ((int)aa.encode('*'), 23);
  EXPECT_EQ((int)aa.encode('?'), 24);
  auto m = swatlib::selectMatrix(swatlib::Similarity::nucleicAcid, 2, -3, -1);
  EXPECT_EQ((int)m(1, 1), 2);
  EXPECT_EQ((int)m(1, 2), -3);
  EXPECT_EQ((int)m(0, 4), -1);
  EXPECT_EQ((int)m(4, 0), -1);
}

int main(int argc, char** argv) { return mini_main(argc, argv); }
