// Test-infrastructure shim (see parallel_for.h): tbb::scalable_allocator as
// std::allocator.
#pragma once
#include <memory>

namespace tbb {
template <typename T>
using scalable_allocator = std::allocator<T>;
} // namespace tbb

namespace oneapi { namespace tbb { using ::tbb::scalable_allocator; } }
