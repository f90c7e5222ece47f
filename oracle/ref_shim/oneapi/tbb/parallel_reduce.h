// Test-infrastructure shim (see parallel_for.h): the reference includes this
// header but never calls parallel_reduce.
#pragma once
#include "blocked_range.h"
