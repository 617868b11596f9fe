// Test infrastructure only (the oracle). Stand-in for ips2ra (absent): a stable sort by the
// extracted radix key. ips2ra itself leaves the order of equal keys unspecified; this stand-in
// orders them by input position.
#pragma once
#include <algorithm>
#include <cassert>
#include <cstddef>

namespace ips2ra {
template <typename It, typename Extractor> void sort(It begin, It end, Extractor ex) {
    std::stable_sort(begin, end, [&](const auto &a, const auto &b) { return ex(a) < ex(b); });
}
namespace parallel {
template <typename It, typename Extractor> void sort(It begin, It end, Extractor ex, size_t) {
    ::ips2ra::sort(begin, end, ex);
}
} // namespace parallel
} // namespace ips2ra
