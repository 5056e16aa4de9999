// Topology stand-ins for the reference's hwloc-backed CpuTopology.cpp (hwloc is absent here).
// With no topology the reference sizes partitions from hardware_concurrency()/2; the oracle
// driver always passes an explicit partition count. Pinning is a no-op.
#include <cstddef>
#include <cstdint>
#include <vector>

#include "monoprop/detail/partition/CpuTopology.h"

namespace monoprop::detail::partition {
namespace topo_detail {
auto placement_order(const std::vector<PhysicalCore> &, size_t n, size_t, size_t) -> std::vector<int> {
    return std::vector<int>(n, -1);
}
} // namespace topo_detail
auto enumerate_physical_cores() -> std::vector<PhysicalCore> { return {}; }
auto affinity_mask_words(uint64_t *out, size_t nwords) -> bool {
    for (size_t i = 0; i < nwords; ++i) out[i] = 0;
    return false;
}
auto masks_are_pairwise_disjoint(const uint64_t *, size_t, size_t) -> bool { return false; }
auto partition_cpusets(size_t n, size_t, size_t, NodeMask) -> std::vector<CpuSet> { return std::vector<CpuSet>(n); }
auto pin_this_thread(const CpuSet &) -> void {}
} // namespace monoprop::detail::partition
