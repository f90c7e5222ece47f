// Test-infrastructure shim (see parallel_for.h): tbb::enumerable_thread_specific.
// One slot per OpenMP thread, all constructed up front as copies of the
// exemplar, so iterating over the slots visits every thread's copy (unused
// slots still hold the exemplar, which the reference only ever sums or
// min/maxes, so they do not change its results).
#pragma once
#include <omp.h>
#include <vector>
#include <utility>
#include <memory>

namespace tbb {

template <typename T>
class enumerable_thread_specific
{
public:
	enumerable_thread_specific() : slots_(nthreads()) {}
	explicit enumerable_thread_specific(const T& exemplar) : slots_(nthreads(), exemplar) {}
	enumerable_thread_specific(const enumerable_thread_specific&) = default;
	enumerable_thread_specific(enumerable_thread_specific&&) = default;
	enumerable_thread_specific& operator=(const enumerable_thread_specific&) = default;
	enumerable_thread_specific& operator=(enumerable_thread_specific&&) = default;

	T& local() { return slots_[omp_get_thread_num()]; }

	using iterator = typename std::vector<T>::iterator;
	using const_iterator = typename std::vector<T>::const_iterator;
	iterator begin() { return slots_.begin(); }
	iterator end() { return slots_.end(); }
	const_iterator begin() const { return slots_.begin(); }
	const_iterator end() const { return slots_.end(); }
	size_t size() const { return slots_.size(); }

private:
	static size_t nthreads() { return size_t(omp_get_max_threads()); }
	std::vector<T> slots_;
};

} // namespace tbb

namespace oneapi { namespace tbb { using ::tbb::enumerable_thread_specific; } }
