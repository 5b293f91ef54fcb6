// gtest.h -- TEST INFRASTRUCTURE: the small part of the GoogleTest interface that the reference's unit tests use
// (TEST, ASSERT_EQ / ASSERT_NE / ASSERT_TRUE / ASSERT_FALSE, testing::AssertionResult), so that those test files
// compile unchanged against this repository's include/dt headers (GoogleTest itself is not installed here).
// A failed assertion prints where and why and returns from the test body, as ASSERT_* does in GoogleTest.
#pragma once

#include <cstdio>
#include <functional>
#include <sstream>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace testing
{
  class AssertionResult
  {
  public:
    explicit AssertionResult(bool ok) : m_ok(ok) {}
    explicit operator bool() const { return m_ok; }
    const std::string& message() const { return m_msg; }
    template <typename T>
    AssertionResult& operator<<(const T& v)
    {
      std::ostringstream os;
      os << v;
      m_msg += os.str();
      return *this;
    }

  private:
    bool        m_ok;
    std::string m_msg;
  };

  inline AssertionResult AssertionSuccess() { return AssertionResult(true); }
  inline AssertionResult AssertionFailure() { return AssertionResult(false); }

  namespace shim
  {
    struct test_case
    {
      const char*           suite;
      const char*           name;
      std::function<void()> body;
    };
    inline std::vector<test_case>& registry()
    {
      static std::vector<test_case> r;
      return r;
    }
    inline bool& current_failed()
    {
      static bool f = false;
      return f;
    }
    struct registrar
    {
      registrar(const char* suite, const char* name, void (*fn)()) { registry().push_back({suite, name, fn}); }
    };

    template <typename T>
    std::string show(const T& v)
    {
      if constexpr (requires(std::ostream& os) { os << v; })
      {
        std::ostringstream os;
        if constexpr (sizeof(T) == 1 && std::is_integral_v<T>)
          os << static_cast<int>(v);
        else
          os << v;
        return os.str();
      }
      else
        return "<value>";
    }

    inline void report(const char* file, int line, const std::string& what)
    {
      std::fprintf(stderr, "%s:%d: Failure\n%s\n", file, line, what.c_str());
      current_failed() = true;
    }

    inline std::string message_of(const AssertionResult& r) { return r.message(); }
    template <typename T>
    std::string message_of(const T&)
    {
      return std::string();
    }
  } // namespace shim
} // namespace testing

#define DTB_GTEST_CONCAT_(a, b) a##b
#define DTB_GTEST_CONCAT(a, b) DTB_GTEST_CONCAT_(a, b)

#define TEST(suite, name)                                                                                             \
  static void DTB_GTEST_CONCAT(suite##_##name, _body)();                                                             \
  static ::testing::shim::registrar DTB_GTEST_CONCAT(suite##_##name, _reg)(#suite, #name,                            \
                                                                           &DTB_GTEST_CONCAT(suite##_##name, _body)); \
  static void DTB_GTEST_CONCAT(suite##_##name, _body)()

#define ASSERT_TRUE(cond)                                                                                      \
  do                                                                                                           \
  {                                                                                                            \
    const auto& dtb_gtest_v = (cond);                                                                          \
    if (!static_cast<bool>(dtb_gtest_v))                                                                       \
    {                                                                                                          \
      ::testing::shim::report(__FILE__, __LINE__,                                                              \
                              std::string("Value of: " #cond "\n  Actual: false\n") +                          \
                                  ::testing::shim::message_of(dtb_gtest_v));                                   \
      return;                                                                                                  \
    }                                                                                                          \
  } while (0)

#define ASSERT_FALSE(cond)                                                                                            \
  do                                                                                                                  \
  {                                                                                                                   \
    if (static_cast<bool>(cond))                                                                                      \
    {                                                                                                                 \
      ::testing::shim::report(__FILE__, __LINE__, std::string("Value of: " #cond "\n  Actual: true"));                \
      return;                                                                                                         \
    }                                                                                                                 \
  } while (0)

#define DTB_GTEST_CMP(a, b, op)                                                                                       \
  do                                                                                                                  \
  {                                                                                                                   \
    const auto& dtb_gtest_a = (a);                                                                                    \
    const auto& dtb_gtest_b = (b);                                                                                    \
    if (!(dtb_gtest_a op dtb_gtest_b))                                                                                \
    {                                                                                                                 \
      ::testing::shim::report(__FILE__, __LINE__,                                                                     \
                              std::string("Expected: (" #a ") " #op " (" #b "), actual: ") +                          \
                                  ::testing::shim::show(dtb_gtest_a) + " vs " + ::testing::shim::show(dtb_gtest_b)); \
      return;                                                                                                         \
    }                                                                                                                 \
  } while (0)

#define ASSERT_EQ(a, b) DTB_GTEST_CMP(a, b, ==)
#define ASSERT_NE(a, b) DTB_GTEST_CMP(a, b, !=)
