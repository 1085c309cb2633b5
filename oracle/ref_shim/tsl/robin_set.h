// Stand-in for tsl::robin_set (test infrastructure).  The reference uses it
// only in topUpSingle (src/SolutionKmeans.hpp:513-537) to deduplicate candidate
// ids: insert, erase, clear and iteration.  The real container iterates in
// hash-table order, which the reference does not rely on; this stand-in
// iterates in ascending id order so that the refinement pass is deterministic
// and the oracle can be pinned to it.
#pragma once
#include <set>

namespace tsl {

template <class Key>
class robin_set : public std::set<Key> {};

}  // namespace tsl
