// Test-infrastructure shim (see parallel_for.h): tbb::concurrent_vector as a
// plain std::vector (the reference only sizes it once and indexes it).
#pragma once
#include <vector>
#include <memory>

namespace tbb {
template <typename T, typename A = std::allocator<T>>
using concurrent_vector = std::vector<T, A>;
} // namespace tbb

namespace oneapi { namespace tbb { using ::tbb::concurrent_vector; } }
