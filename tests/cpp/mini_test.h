// Minimal test registry for the C++ drop-in tests: TEST(group, name) bodies
// use EXPECT_EQ / ASSERT_* like googletest; main() runs the tests whose
// "group.name" contains any command-line filter and exits non-zero on failure.
#pragma once
#include <cstdio>
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace mini {
struct Case {
  std::string name;
  std::function<void()> fn;
};
inline std::vector<Case>& registry() {
  static std::vector<Case> r;
  return r;
}
inline int& failures() {
  static int f = 0;
  return f;
}
struct Reg {
  Reg(const char* g, const char* n, std::function<void()> fn) {
    registry().push_back({std::string(g) + "." + n, std::move(fn)});
  }
};
struct Fatal {};
}  // namespace mini

#define TEST(G, N)                                            \
  static void G##_##N##_body();                               \
  static mini::Reg G##_##N##_reg(#G, #N, G##_##N##_body);     \
  static void G##_##N##_body()

#define EXPECT_EQ(a, b)                                                                         \
  do {                                                                                          \
    auto _va = (a);                                                                             \
    auto _vb = (b);                                                                             \
    if (!(_va == _vb)) {                                                                        \
      std::ostringstream _os;                                                                   \
      _os << __FILE__ << ":" << __LINE__ << ": " #a " == " #b " failed: " << +_va << " vs " << +_vb; \
      std::cerr << _os.str() << "\n";                                                           \
      mini::failures()++;                                                                       \
    }                                                                                           \
  } while (0)

#define EXPECT_TRUE(c)                                                          \
  do {                                                                          \
    if (!(c)) {                                                                 \
      std::cerr << __FILE__ << ":" << __LINE__ << ": " #c " is false\n";        \
      mini::failures()++;                                                       \
    }                                                                           \
  } while (0)

#define EXPECT_THROW(stmt)                                                      \
  do {                                                                          \
    bool _t = false;                                                            \
    try {                                                                       \
      stmt;                                                                     \
    } catch (const std::exception&) {                                           \
      _t = true;                                                                \
    }                                                                           \
    if (!_t) {                                                                  \
      std::cerr << __FILE__ << ":" << __LINE__ << ": " #stmt " did not throw\n"; \
      mini::failures()++;                                                       \
    }                                                                           \
  } while (0)

inline int mini_main(int argc, char** argv) {
  int ran = 0;
  for (auto& c : mini::registry()) {
    bool sel = argc <= 1;
    for (int i = 1; i < argc; ++i)
      if (c.name.find(argv[i]) != std::string::npos) sel = true;
    if (!sel) continue;
    const int before = mini::failures();
    try {
      c.fn();
    } catch (const std::exception& e) {
      std::cerr << c.name << ": exception: " << e.what() << "\n";
      mini::failures()++;
    }
    std::cout << (mini::failures() == before ? "[ OK ] " : "[FAIL] ") << c.name << "\n";
    ++ran;
  }
  std::cout << ran << " tests, " << mini::failures() << " failures\n";
  return mini::failures() ? 1 : (ran ? 0 : 2);
}
