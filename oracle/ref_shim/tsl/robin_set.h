// Stand-in for tsl::robin_set (test infrastructure).  The reference uses it
// only in topUpSingle (src/SolutionKmeans.hpp:513-537) to deduplicate candidate
// ids: insert, erase, clear and iteration.  The real container iterates in
// hash-table order, which the reference does not rely on.
//
// Serial build (parity): an ordered set, so the refinement pass offers
// candidates in ascending id order and the oracle can be pinned to it.
// Threaded build (CPU timing): a hash set, closer to the real container's cost.
#pragma once

#ifndef KNNG_SHIM_THREADS
#define KNNG_SHIM_THREADS 0
#endif

#if KNNG_SHIM_THREADS == 0
#include <set>
namespace tsl {
template <class Key>
class robin_set : public std::set<Key> {};
}  // namespace tsl
#else
#include <unordered_set>
namespace tsl {
template <class Key>
class robin_set : public std::unordered_set<Key> {
public:
    robin_set() { this->reserve(16384); }
};
}  // namespace tsl
#endif
