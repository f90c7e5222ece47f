// Test-infrastructure shim (see parallel_for.h): tbb::parallel_for_each over
// random-access ranges.
#pragma once
#include <omp.h>
#include <iterator>
#include "parallel_for.h"

namespace tbb {

template <typename It, typename Body>
void parallel_for_each(It first, It last, const Body& body)
{
	long long n = (long long)std::distance(first, last);
#pragma omp parallel for schedule(dynamic, 64)
	for (long long i = 0; i < n; ++i)
		body(*(first + i));
}

} // namespace tbb

namespace oneapi { namespace tbb { using ::tbb::parallel_for_each; } }
