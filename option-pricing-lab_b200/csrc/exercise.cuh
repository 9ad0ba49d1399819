// The issuer's Longstaff-Schwartz policy fitted on the device from a pilot record that is already in device memory
// (the backward regression of packages/structured/src/optlab/structured/exercise.py:212-252 with the basis of
// :125-140). Used by ob_script_pilot_fit (csrc/script.cu), which runs the pilot and hands its record over.
#pragma once

#include "common.cuh"

namespace ob {

// The pilot's record: n_paths rows of stride doubles, per event k its discounted flows before and after the call
// statement (2 k, 2 k + 1), then per call c its mask, alive mass, amount and n_state state values (at
// 2 n_events + c (3 + n_state)). call_event[c]: the event of call c; pay_discount[k]: the discount factor of event
// k's payment (0: none counted). rules receives n_calls rows of OB_RULE_STRIDE doubles (a call that no path reaches
// gets a row of zeros), in_sample the pilot's value under its own policy. False: a regression's basis was (nearly)
// rank-deficient and the least squares of the normal equations cannot stand in for the reference's SVD solve.
bool fit_policy_on_device(const double* record, long long n_paths, int stride, int n_events, int n_calls, int n_state,
                          const int* call_event, const double* pay_discount, double* rules, double* in_sample,
                          DeviceArena& arena);

}  // namespace ob
