// Spec compiler: vr_agg_spec -> device Program + EmitProgram.
// This is the GPU gate of the reference's planner (VectorAggregatePlanner.plan,
// spark/src/main/scala/org/apache/spark/sql/vecruntime/VectorHashAggregateExec.scala:1288-1380):
// a spec outside it is refused with VR_ERR_UNSUPPORTED and a reason, and the
// caller keeps the Vector API iterator (then Spark) for that aggregate.
#pragma once
#include <string>
#include <vector>

#include "vr_internal.h"

namespace vr {

struct Plan {
    Program prog;
    EmitProgram emit;
    std::vector<int> staged_of_spec;  // spec column -> staged column (-1: unused)
    std::vector<int> spec_of_staged;  // staged column -> spec column
    std::vector<vr_column_type> out_types;
    bool direct_ok = false;           // dictionary / boolean keys (or no keys)
    std::string reason;               // why the spec was refused
};

// Returns VR_OK or VR_ERR_INVALID / VR_ERR_UNSUPPORTED with plan.reason set.
int compile_plan(const vr_agg_spec& spec, Plan& plan);

}  // namespace vr
