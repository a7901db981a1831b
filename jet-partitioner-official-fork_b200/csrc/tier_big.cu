// Tier "big": int32 ordinals, int64 offsets, int64 weights.
#include "api_impl.cuh"

namespace jetb {
TierOps ops_big() { return make_ops<int32_t, int64_t, int64_t>(); }
}  // namespace jetb

extern "C" int jet_partition_big(const jet_config_c* config, int32_t n, const int64_t* row_map, const int32_t* entries,
                                 const int64_t* values, const int64_t* vweights, int uniform_ew, int mem, uint64_t seed,
                                 void* stream, int32_t* part_out, int64_t* edge_cut, jet_stats_c* stats) {
    return jetb::partition_impl<int32_t, int64_t, int64_t>(config, n, row_map, entries, values, vweights, uniform_ew, mem, seed,
                                                           stream, part_out, edge_cut, stats);
}
