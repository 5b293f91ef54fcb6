// gtest_main.cpp -- TEST INFRASTRUCTURE: runs every TEST registered through gtest_shim/gtest/gtest.h and prints
// one line per test; exit status 1 if any failed.  An optional argument selects tests whose "suite.name"
// contains it.
#include <gtest/gtest.h>

#include <cstring>
#include <exception>

int main(int argc, char** argv)
{
  const char* filter = argc > 1 ? argv[1] : nullptr;
  int         failed = 0, run = 0;
  for (auto& t : testing::shim::registry())
  {
    const std::string full = std::string(t.suite) + "." + t.name;
    if (filter && full.find(filter) == std::string::npos)
      continue;
    testing::shim::current_failed() = false;
    try
    {
      t.body();
    }
    catch (const std::exception& e)
    {
      std::fprintf(stderr, "%s: uncaught exception: %s\n", full.c_str(), e.what());
      testing::shim::current_failed() = true;
    }
    ++run;
    const bool f = testing::shim::current_failed();
    failed += f;
    std::printf("[%s] %s\n", f ? "  FAILED  " : "       OK ", full.c_str());
  }
  std::printf("%d tests, %d failed\n", run, failed);
  return failed ? 1 : 0;
}
