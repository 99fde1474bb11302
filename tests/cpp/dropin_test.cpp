// GPU tests of the drop-in SWAlgorithm API, mirroring the reference's
// test/simple-test.cpp (known answers through compare_local and
// compare_mn_local under each vertex type and fill policy) and
// test/mn_cmp-test.cpp:29-117 (M x N scores under the three policies).
// The known answers are read from tests/golden/known_answers.txt, which
// tests/golden/make_golden.py extracts from those reference test files.
#include <array>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "driver.hpp"
#include "ipu_batch_affine.h"
#include "mini_test.h"

namespace {

struct Known {
  std::string ref, query;
  int qstart, qend, rstart, rend, score;
};
struct KnownSet {
  std::vector<Known> simple;
  std::vector<std::string> mnseqs;
  std::vector<std::array<int, 3>> mncmps;
};

const KnownSet& known() {
  static KnownSet k = [] {
    KnownSet ks;
    const char* env = std::getenv("IPUMA_GOLDEN_DIR");
    std::string dir = env ? env : "tests/golden";
    std::ifstream f(dir + "/known_answers.txt");
    if (!f) throw std::runtime_error("cannot open " + dir + "/known_answers.txt");
    std::string line;
    while (std::getline(f, line)) {
      std::istringstream ss(line);
      std::string tag;
      ss >> tag;
      if (tag == "simple") {
        Known c;
        ss >> c.ref >> c.query >> c.qstart >> c.qend >> c.rstart >> c.rend >> c.score;
        ks.simple.push_back(c);
      } else if (tag == "mnseq") {
        std::string s;
        ss >> s;
        ks.mnseqs.push_back(s);
      } else if (tag == "mncmp") {
        std::array<int, 3> c;
        ss >> c[0] >> c[1] >> c[2];
        ks.mncmps.push_back(c);
      }
    }
    return ks;
  }();
  return k;
}

void checkResults(const ipu::batchaffine::BlockAlignmentResults& results, bool withStarts = true) {
  const auto& data = known().simple;
  for (size_t i = 0; i < data.size(); ++i) {
    const auto& t = data[i];
    const auto uda = results.a_range_result[i];
    const int16_t query_begin = uda & 0xffff;
    const int16_t query_end = uda >> 16;
    const auto udb = results.b_range_result[i];
    const int16_t ref_begin = udb & 0xffff;
    const int16_t ref_end = udb >> 16;
    EXPECT_EQ(results.scores[i], t.score);
    EXPECT_EQ((int)ref_end, t.rend);
    EXPECT_EQ((int)query_end, t.qend);
    if (withStarts) {
      EXPECT_EQ((int)ref_begin, t.rstart);
      EXPECT_EQ((int)query_begin, t.qstart);
    }
  }
}

std::vector<std::string> queries() {
  std::vector<std::string> q;
  for (const auto& t : known().simple) q.push_back(t.query);
  return q;
}
std::vector<std::string> refs() {
  std::vector<std::string> r;
  for (const auto& t : known().simple) r.push_back(t.ref);
  return r;
}

void runSimple(ipu::IPUAlgoConfig algo, ipu::SWConfig sw = {}) {
  ipu::batchaffine::SWAlgorithm driver(sw, algo);
  driver.compare_local(queries(), refs());
  checkResults(driver.get_result(), !algo.forwardOnly);
}

}  // namespace

TEST(SimpleCorrectnessTest, UseAssemblyVertex) {
  ipu::SWConfig sw = {0, -ALN_GAP_EXTENDING_COST, ALN_MATCH_SCORE, -ALN_MISMATCH_COST, -ALN_AMBIGUITY_COST,
                      swatlib::Similarity::nucleicAcid, swatlib::DataType::nucleicAcid};
  runSimple({1, 20, 30, 1000, ipu::VertexType::assembly}, sw);
}

TEST(SimpleCorrectnessTest, UseCppVertex) {
  runSimple({2, 300, 20, 3000, ipu::VertexType::cpp, ipu::Algorithm::roundRobin});
}

TEST(SimpleCorrectnessTest, UseCppMultiVertex) {
  runSimple({2, 300, 20, 3000, ipu::VertexType::multi, ipu::Algorithm::roundRobin});
}

TEST(SimpleCorrectnessTest, UseAsmMultiVertex) {
  runSimple({2, 300, 20, 3000, ipu::VertexType::multiasm, ipu::Algorithm::roundRobin});
}

TEST(SimpleCorrectnessTest, UseGreedy) { runSimple({4, 300, 6, 3000, ipu::VertexType::cpp, ipu::Algorithm::greedy}); }

TEST(SimpleCorrectnessTest, ForwardOnly) {
  ipu::IPUAlgoConfig algo = {2, 300, 20, 3000, ipu::VertexType::cpp, ipu::Algorithm::fillFirst};
  algo.forwardOnly = true;
  runSimple(algo);
}

TEST(SimpleCorrectnessTest, PlainScheduler) {
  ipu::batchaffine::SWAlgorithm driver({}, {2, 300, 20, 3000, ipu::VertexType::cpp, ipu::Algorithm::roundRobin});
  EXPECT_EQ(ipuma_gpu_set_option(driver.engine(), "scheduler", 1), IPUMA_OK);
  driver.compare_local(queries(), refs());
  checkResults(driver.get_result());
}

TEST(SimpleCorrectnessTest, useMNComparisons) {
  ipu::batchaffine::SWAlgorithm driver({}, {4, 300, 5, 3000, ipu::VertexType::cpp, ipu::Algorithm::roundRobin});
  std::vector<std::string> seqs;
  ipu::Comparisons comparisons;
  const auto q = queries(), r = refs();
  for (size_t i = 0; i < q.size(); ++i) {
    seqs.push_back(q[i]);
    seqs.push_back(r[i]);
    comparisons.push_back({(int32_t)(2 * i), (int32_t)(2 * i + 1)});
  }
  driver.compare_mn_local(seqs, comparisons);
  checkResults(driver.get_result());
}

TEST(SimpleCorrectnessTest, asyncSubmitJoin) {
  ipu::IPUAlgoConfig algo = {2, 300, 20, 3000, ipu::VertexType::cpp, ipu::Algorithm::fillFirst};
  ipu::batchaffine::SWAlgorithm driver({}, algo);
  const auto q = queries(), r = refs();
  std::vector<int32_t> inputs(algo.getInputBufferSize32b());
  std::vector<int> mapping(q.size());
  ipu::batchaffine::SWAlgorithm::prepare_remote({}, algo, q, r, inputs.data(), inputs.data() + inputs.size(),
                                                mapping.data());
  std::vector<int32_t> results(3 * algo.getTotalNumberOfComparisons());
  std::unique_ptr<ipu::batchaffine::Job> job(driver.async_submit_prepared_remote_compare(
      inputs.data(), inputs.data() + inputs.size(), results.data(), results.data() + results.size()));
  driver.blocking_join_prepared_remote_compare(*job);
  ipu::batchaffine::BlockAlignmentResults res;
  res.scores.resize(q.size());
  res.a_range_result.resize(q.size());
  res.b_range_result.resize(q.size());
  ipu::batchaffine::SWAlgorithm::transferResults(
      results.data(), results.data() + results.size(), mapping.data(), mapping.data() + mapping.size(),
      res.scores.data(), res.scores.data() + res.scores.size(), res.a_range_result.data(),
      res.a_range_result.data() + res.a_range_result.size(), res.b_range_result.data(),
      res.b_range_result.data() + res.b_range_result.size());
  checkResults(res);
}

static void mnCompare(ipu::Algorithm algo) {
  ipu::SWConfig sw = {0, -1, 1, -1, -1, swatlib::Similarity::nucleicAcid, swatlib::DataType::nucleicAcid};
  ipu::batchaffine::SWAlgorithm driver(sw, {1, 20, 30, 1000, ipu::VertexType::assembly, algo});
  ipu::Comparisons cmps;
  for (const auto& c : known().mncmps) cmps.push_back({c[0], c[1]});
  driver.compare_mn_local(known().mnseqs, cmps);
  const auto result = driver.get_result();
  for (size_t i = 0; i < known().mncmps.size(); ++i) EXPECT_EQ(result.scores[i], known().mncmps[i][2]);
}

TEST(MN_Test, CompareAll) { mnCompare(ipu::Algorithm::fillFirst); }
TEST(MN_Test, CompareAllRR) { mnCompare(ipu::Algorithm::roundRobin); }
TEST(MN_Test, CompareAllGreedy) { mnCompare(ipu::Algorithm::greedy); }

TEST(LargerTest, simple) {
  ipu::IPUAlgoConfig config = {10, 10, 2, 40, ipu::VertexType::assembly, ipu::Algorithm::fillFirst};
  std::vector<std::string> A, B;
  for (int i = 0; i < 2; ++i) {
    A.push_back(std::string(10, 'A'));
    B.push_back("TTTT" + std::string(10, 'A'));
  }
  ipu::batchaffine::SWAlgorithm driver({}, config);
  driver.compare_local(A, B);
  const auto result = driver.get_result();
  EXPECT_EQ(result.scores[0], 10);
  EXPECT_EQ(result.scores[1], 10);
}

TEST(Driver, globalSingleton) {
  init_single_ipu(SW_CONFIGURATION, {2, 300, 20, 3000});
  auto* d = getDriver();
  d->compare_local(queries(), refs());
  checkResults(d->get_result());
}

int main(int argc, char** argv) { return mini_main(argc, argv); }
