// Autotuner: chooses tier, warp pre-aggregation, block shape, tile size and
// shared-cache size for an aggregate, keyed on the spec's shape, the batch
// size and the estimated cardinality (both bucketed by powers of two).
#pragma once
#include <cstdint>

#include "vrgpu.h"

namespace vr {
bool tune_lookup_internal(const vr_agg_spec& spec, int64_t rows, vr_tune_choice* out);
uint64_t spec_signature(const vr_agg_spec& spec);
}  // namespace vr
