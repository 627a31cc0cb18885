// Candidate fused plans and seeded random fused passes, with their features
// and (optionally) measured device times, as JSON text.
#pragma once

#include <string>

#include "simulator.hpp"

namespace dq {

class CostModel;

// Every candidate fused plan of the circuit's unitary prefix (the default
// portfolio, or with `wide` the learned planner's), each distinct pass's
// features, its measured device milliseconds when `measure` (one complex64
// state of the circuit's size on the simulator's device) and a pass-cost
// model's predicted milliseconds when `model` is given.
std::string fused_portfolio_json(Simulator& sim, const char* json, size_t len, bool wide, bool measure,
                                 const CostModel* model);
// `count` seeded random fused passes over n qubits, with features and, when
// `measure`, device milliseconds.
std::string fused_random_passes_json(Simulator& sim, int n, uint64_t count, uint64_t seed, bool measure);

}  // namespace dq
