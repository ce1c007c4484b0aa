/* Stand-in for <range/v3/all.hpp> (range-v3 is absent here) so that the
 * reference's src/build_table.cpp and include/data_access/table.h compile
 * for the `.tbl` cache check: C++23's std::ranges provides the few views
 * they use, plus a small ranges::to. TEST INFRASTRUCTURE. */
#pragma once
#include <ranges>
#include <string>

namespace ranges {
namespace views {
using std::views::enumerate;
using std::views::transform;
inline constexpr auto join = [](auto delim) { return std::views::join_with(delim); };
} // namespace views
template <class C> struct to_adaptor {};
template <class C> to_adaptor<C> to() { return {}; }
template <std::ranges::input_range R, class C> C operator|(R &&r, to_adaptor<C>) {
    C c;
    for (auto &&x : r) c.push_back(x);
    return c;
}
} // namespace ranges
