// Test-infrastructure shim (see parallel_for.h): tbb::concurrent_unordered_map
// as std::unordered_map (the reference only includes the header).
#pragma once
#include <unordered_map>

namespace tbb {
template <typename K, typename V, typename H = std::hash<K>, typename E = std::equal_to<K>>
using concurrent_unordered_map = std::unordered_map<K, V, H, E>;
} // namespace tbb

namespace oneapi { namespace tbb { using ::tbb::concurrent_unordered_map; } }
