// Stand-in for Boost's unordered_flat_map (Boost is absent here): an alias of std::unordered_map.
// The reference uses it only for its initial-operator side map, off the per-gate path.
#pragma once
#include <functional>
#include <unordered_map>

namespace boost {
template <class K, class V, class H = std::hash<K>, class E = std::equal_to<K>,
          class A = std::allocator<std::pair<const K, V>>>
using unordered_flat_map = std::unordered_map<K, V, H, E, A>;
} // namespace boost
