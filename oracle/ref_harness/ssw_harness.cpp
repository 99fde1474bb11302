// Host harness over the reference's vendored StripedSmithWaterman C API
// (extern/include/ssw/ssw_core.hpp:76,116), driven the way the reference's
// CPU benchmark drives it (cpusw/aligners.hpp:128-152,212-226): worker w
// takes pairs w, w+T, ...; the query profile is built with ssw_init inside
// the timed loop; score_size 2 (byte pass with word rerun).  Sequences and
// the substitution matrix are passed as ipuma's own integer codes and
// matrix, so A is SSW's "read" (query) and B its "ref".
// Built by oracle/Makefile into oracle/_ref/.  TEST INFRASTRUCTURE ONLY.
#include <cstdint>
#include <thread>
#include <vector>
#include <algorithm>

#include "ssw_core.hpp"

extern "C" int ref_ssw_pairs(const uint8_t* codes, const int64_t* a_off, const int32_t* a_len,
                             const int64_t* b_off, const int32_t* b_len, int64_t n,
                             const int8_t* sim, int simN, int gapO, int gapE, int reportBegin,
                             int nthreads, int32_t* score, int32_t* a_end, int32_t* b_end,
                             int32_t* a_begin, int32_t* b_begin) {
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  auto worker = [&](int w) {
    for (int64_t c = w; c < n; c += nthreads) {
      if (a_len[c] <= 0 || b_len[c] <= 0) {
        score[c] = 0;
        a_end[c] = b_end[c] = a_begin[c] = b_begin[c] = 0;
        continue;
      }
      const int8_t* q = reinterpret_cast<const int8_t*>(codes + a_off[c]);
      const int8_t* r = reinterpret_cast<const int8_t*>(codes + b_off[c]);
      s_profile* prof = ssw_init(q, a_len[c], sim, simN, 2);
      const uint8_t flag = reportBegin ? 0x08 : 0;
      const int32_t maskLen = std::max(b_len[c] / 2, 15);
      s_align* al = ssw_align(prof, r, b_len[c], (uint8_t)gapO, (uint8_t)gapE, flag, 0, 32767,
                              maskLen);
      score[c] = al->score1;
      a_end[c] = al->read_end1;
      b_end[c] = al->ref_end1;
      a_begin[c] = al->read_begin1;
      b_begin[c] = al->ref_begin1;
      align_destroy(al);
      init_destroy(prof);
    }
  };
  std::vector<std::thread> ts;
  for (int w = 0; w < nthreads; ++w) ts.emplace_back(worker, w);
  for (auto& t : ts) t.join();
  return 0;
}
