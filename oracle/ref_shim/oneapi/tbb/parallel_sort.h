// Test-infrastructure shim (see parallel_for.h): tbb::parallel_sort as a
// serial std::sort (only reachable with the reference's
// deterministic_behaviour macro, which it leaves off).
#pragma once
#include <algorithm>

namespace tbb {
template <typename It, typename Cmp>
void parallel_sort(It first, It last, const Cmp& cmp) { std::sort(first, last, cmp); }
template <typename It>
void parallel_sort(It first, It last) { std::sort(first, last); }
} // namespace tbb

namespace oneapi { namespace tbb { using ::tbb::parallel_sort; } }
