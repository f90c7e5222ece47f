// Test-infrastructure shim (see oneapi/tbb/parallel_for.h).  Deliberately no
// tbb/tbb.h: libstdc++'s parallel algorithms would then pick a TBB backend.
#pragma once
#include "../oneapi/tbb/parallel_for.h"
