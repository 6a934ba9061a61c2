// ORACLE / TEST INFRASTRUCTURE — a minimal googletest-compatible header (my own code) so that the reference's own test
// files (tests/test_kspace.cpp, tests/test_nbnxm.cpp) compile unmodified against the oracle library without the
// googletest download their CMake fetches. Supports TEST, EXPECT_/ASSERT_ comparisons with streamed messages,
// EXPECT_NEAR, EXPECT_THROW / EXPECT_NO_THROW, and provides main().
#pragma once
#include <cmath>
#include <cstdio>
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace gshim {

struct Registry {
  struct Entry { std::string suite, name; std::function<void()> fn; };
  std::vector<Entry> tests;
  int failures = 0;
  static Registry& get() { static Registry r; return r; }
};

struct Add {
  Add(const char* s, const char* n, void (*fn)()) { Registry::get().tests.push_back({s, n, fn}); }
};

struct Msg {
  std::ostringstream os;
  template <class T> Msg& operator<<(const T& v) { os << v; return *this; }
};

struct Fail {
  const char* file; int line; std::string what;
  Fail(const char* f, int l, std::string w) : file(f), line(l), what(std::move(w)) {}
  void operator=(const Msg& m) const {
    ++Registry::get().failures;
    std::cerr << file << ":" << line << ": Failure: " << what << " " << m.os.str() << "\n";
  }
};

template <class A, class B> bool near(const A& a, const B& b, double tol) { return std::fabs(double(a) - double(b)) <= tol; }
inline bool dbl_eq(double a, double b) {
  if (a == b) return true;
  const double d = std::fabs(a - b), m = std::max(std::fabs(a), std::fabs(b));
  return d <= 4 * 2.220446049250313e-16 * m;
}

template <class A, class B> std::string pair_text(const A& a, const B& b) {
  std::ostringstream os;
  os.precision(17);
  os << "(" << a << " vs " << b << ")";
  return os.str();
}

}  // namespace gshim

#define GSHIM_CAT2(a, b) a##b
#define GSHIM_CAT(a, b) GSHIM_CAT2(a, b)
#define TEST(suite, name)                                                                       \
  static void GSHIM_CAT(gshim_test_, GSHIM_CAT(suite, GSHIM_CAT(_, name)))();                    \
  static ::gshim::Add GSHIM_CAT(gshim_add_, GSHIM_CAT(suite, GSHIM_CAT(_, name)))(#suite, #name, \
      GSHIM_CAT(gshim_test_, GSHIM_CAT(suite, GSHIM_CAT(_, name))));                              \
  static void GSHIM_CAT(gshim_test_, GSHIM_CAT(suite, GSHIM_CAT(_, name)))()

#define GSHIM_CHECK(cond, text, fatal) \
  if (cond) {                          \
  } else fatal ::gshim::Fail(__FILE__, __LINE__, text) = ::gshim::Msg()

#define GSHIM_BIN(a, b, op, fatal) GSHIM_CHECK(((a)op(b)), std::string(#a " " #op " " #b " ") + ::gshim::pair_text((a), (b)), fatal)

#define EXPECT_TRUE(c) GSHIM_CHECK(bool(c), "EXPECT_TRUE(" #c ")", )
#define EXPECT_FALSE(c) GSHIM_CHECK(!bool(c), "EXPECT_FALSE(" #c ")", )
#define ASSERT_TRUE(c) GSHIM_CHECK(bool(c), "ASSERT_TRUE(" #c ")", return)
#define ASSERT_FALSE(c) GSHIM_CHECK(!bool(c), "ASSERT_FALSE(" #c ")", return)
#define EXPECT_EQ(a, b) GSHIM_BIN(a, b, ==, )
#define EXPECT_NE(a, b) GSHIM_BIN(a, b, !=, )
#define EXPECT_LT(a, b) GSHIM_BIN(a, b, <, )
#define EXPECT_LE(a, b) GSHIM_BIN(a, b, <=, )
#define EXPECT_GT(a, b) GSHIM_BIN(a, b, >, )
#define EXPECT_GE(a, b) GSHIM_BIN(a, b, >=, )
#define ASSERT_EQ(a, b) GSHIM_BIN(a, b, ==, return)
#define ASSERT_NE(a, b) GSHIM_BIN(a, b, !=, return)
#define ASSERT_LT(a, b) GSHIM_BIN(a, b, <, return)
#define ASSERT_LE(a, b) GSHIM_BIN(a, b, <=, return)
#define ASSERT_GT(a, b) GSHIM_BIN(a, b, >, return)
#define ASSERT_GE(a, b) GSHIM_BIN(a, b, >=, return)
#define EXPECT_NEAR(a, b, tol) GSHIM_CHECK(::gshim::near((a), (b), (tol)), "EXPECT_NEAR(" #a ", " #b ") " + ::gshim::pair_text((a), (b)), )
#define ASSERT_NEAR(a, b, tol) GSHIM_CHECK(::gshim::near((a), (b), (tol)), "ASSERT_NEAR(" #a ", " #b ") " + ::gshim::pair_text((a), (b)), return)
#define EXPECT_DOUBLE_EQ(a, b) GSHIM_CHECK(::gshim::dbl_eq((a), (b)), "EXPECT_DOUBLE_EQ(" #a ", " #b ") " + ::gshim::pair_text((a), (b)), )
#define EXPECT_THROW(stmt, exc)                                \
  {                                                            \
    bool gshim_ok = false;                                     \
    try { stmt; } catch (const exc&) { gshim_ok = true; } catch (...) {} \
    GSHIM_CHECK(gshim_ok, "EXPECT_THROW(" #stmt ")", );        \
  }
#define EXPECT_NO_THROW(stmt)                                  \
  {                                                            \
    bool gshim_ok = true;                                      \
    try { stmt; } catch (...) { gshim_ok = false; }            \
    GSHIM_CHECK(gshim_ok, "EXPECT_NO_THROW(" #stmt ")", );     \
  }
#define ASSERT_NO_THROW(stmt)                                  \
  {                                                            \
    bool gshim_ok = true;                                      \
    try { stmt; } catch (...) { gshim_ok = false; }            \
    GSHIM_CHECK(gshim_ok, "ASSERT_NO_THROW(" #stmt ")", return); \
  }

int main(int argc, char** argv) {
  const std::string only = argc > 1 ? argv[1] : "";
  auto& R = ::gshim::Registry::get();
  int run = 0;
  for (auto& t : R.tests) {
    const std::string full = t.suite + "." + t.name;
    if (!only.empty() && full.find(only) == std::string::npos) continue;
    const int before = R.failures;
    std::cout << "[ RUN      ] " << full << std::endl;
    try {
      t.fn();
    } catch (const std::exception& e) {
      ++R.failures;
      std::cerr << "exception: " << e.what() << "\n";
    }
    std::cout << (R.failures == before ? "[       OK ] " : "[  FAILED  ] ") << full << std::endl;
    ++run;
  }
  std::cout << run << " tests, " << R.failures << " failed checks" << std::endl;
  return R.failures == 0 ? 0 : 1;
}
