// Stand-in header (test infrastructure): the reference includes
// <oneapi/tbb/concurrent_vector.h> (src/SolutionKmeans.hpp:24, src/ann.hpp:21)
// but never uses tbb::concurrent_vector on the compiled path.
#pragma once
#include "../tbb.h"
