/* Stand-in for <re2/re2.h> so that the reference's plan.h -> statement.h
 * compiles without RE2. Only the LIKE evaluation of scan filters uses RE2,
 * and scan filters run before execute(); nothing on the join path calls it.
 * Any use at run time reports "no match". TEST INFRASTRUCTURE. */
#pragma once
#include <string>
#include <string_view>

class RE2 {
  public:
    struct Options {};
    RE2(const std::string &, const Options &) {}
    bool ok() const { return false; }
    const std::string &error() const { static const std::string e("re2 unavailable"); return e; }
    static bool FullMatch(std::string_view, const RE2 &) { return false; }
};
