// Tier "std": int32 ordinals, int32 offsets, int32 weights.
#include "api_impl.cuh"

namespace jetb {
TierOps ops_i32() { return make_ops<int32_t, int32_t, int32_t>(); }
}  // namespace jetb

extern "C" int jet_partition_i32(const jet_config_c* config, int32_t n, const int32_t* row_map, const int32_t* entries,
                                 const int32_t* values, const int32_t* vweights, int uniform_ew, int mem, uint64_t seed,
                                 void* stream, int32_t* part_out, int32_t* edge_cut, jet_stats_c* stats) {
    return jetb::partition_impl<int32_t, int32_t, int32_t>(config, n, row_map, entries, values, vweights, uniform_ew, mem, seed,
                                                           stream, part_out, edge_cut, stats);
}
