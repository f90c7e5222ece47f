// Test-infrastructure shim: the subset of oneTBB that the reference CPU FMM
// uses, implemented over OpenMP so the unmodified reference sources compile
// here without TBB.  Used only to build the oracle library under oracle/_ref.
#pragma once
#include <omp.h>
#include <cstddef>
#include <iterator>
#include <type_traits>
#include "blocked_range.h"

namespace tbb {

template <typename Index, typename Body>
void parallel_for(Index first, Index last, const Body& body)
{
	using S = long long;
	S n = (S)last - (S)first;
#pragma omp parallel for schedule(dynamic, 16)
	for (S i = 0; i < n; ++i)
		body((Index)((S)first + i));
}

template <typename Value, typename Body>
void parallel_for(const blocked_range<Value>& range, const Body& body)
{
	using S = long long;
	S b = (S)range.begin(), e = (S)range.end();
	S n = e - b;
	if (n <= 0) return;
	S chunk = (S)range.grainsize();
	int nt = omp_get_max_threads();
	S target = (n + 8 * nt - 1) / (8 * nt);
	if (chunk < target) chunk = target;
	if (chunk < 1) chunk = 1;
	S nchunks = (n + chunk - 1) / chunk;
#pragma omp parallel for schedule(dynamic, 1)
	for (S c = 0; c < nchunks; ++c)
	{
		S lo = b + c * chunk;
		S hi = lo + chunk < e ? lo + chunk : e;
		body(blocked_range<Value>((Value)lo, (Value)hi));
	}
}

} // namespace tbb

namespace oneapi { namespace tbb { using ::tbb::parallel_for; } }
