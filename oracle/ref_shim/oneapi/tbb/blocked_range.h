// Test-infrastructure shim (see parallel_for.h): tbb::blocked_range.
#pragma once
#include <cstddef>

namespace tbb {

template <typename Value>
class blocked_range
{
public:
	blocked_range(Value b, Value e, size_t grain = 1) : b_(b), e_(e), g_(grain) {}
	Value begin() const { return b_; }
	Value end() const { return e_; }
	size_t size() const { return size_t(e_ - b_); }
	size_t grainsize() const { return g_; }
	bool empty() const { return !(b_ < e_); }
private:
	Value b_, e_;
	size_t g_;
};

} // namespace tbb

namespace oneapi { namespace tbb { using ::tbb::blocked_range; } }
