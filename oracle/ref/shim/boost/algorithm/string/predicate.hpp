// Stand-in for the one boost string predicate the reference's argument parser
// uses (prefix test), so its loader compiles without boost.  Test
// infrastructure only.
#pragma once
#include <string>
#include <string_view>

namespace boost {
inline bool starts_with(std::string_view s, std::string_view prefix) {
    return s.size() >= prefix.size() && s.compare(0, prefix.size(), prefix) == 0;
}
}  // namespace boost
