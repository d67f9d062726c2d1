// The bookkeeping of the reference's clocked time loop on a thx_time_loop
// record, shared by the host entry points and the device loop kernels.
//   TimeEventTolerance / TimeEventReached / TimeToNextEvent /
//   LimitTimeStepToEvents: include/TimeStepControl.hpp:15-49
//   StepLimitReached: include/RunControl.hpp:11-14
//   the cycle: src/Simulation.cpp:1241-1335 (step shortened to the events,
//   t += step, ti++, new nominal step from the stability estimate when dt is
//   variable, done test, output and checkpoint events)
// Every product and sum is written as its own rounded operation; the file is
// compiled without FMA contraction on both sides.
#pragma once

#include "theseus_b200.h"

#ifdef __CUDACC__
#define THX_HD __host__ __device__ inline
#else
#define THX_HD inline
#endif

namespace thx {

THX_HD double time_abs(double x) { return x < 0.0 ? -x : x; }
THX_HD bool time_finite(double x) { return x - x == 0.0; }

THX_HD double time_event_tolerance(double t) {
  const double m = time_abs(t) > 1.0 ? time_abs(t) : 1.0;
  return 16.0 * 2.220446049250313080847e-16 * m;
}

THX_HD bool time_event_reached(double t, double event_time) {
  return t + time_event_tolerance(t) >= event_time;
}

THX_HD double limit_step_to_events(double step, double t, const double *events, int n) {
  const double tol = time_event_tolerance(t);
  double r = step;
  for (int i = 0; i < n; ++i) {
    const double d = events[i] - t;
    if (time_finite(events[i]) && d > tol && d < r) r = d;
  }
  return r;
}

THX_HD bool step_limit_reached(long long cycle, long long max_cycles) {
  return max_cycles > 0 && cycle >= max_cycles;
}

// The step of the next cycle: 0 once the loop is done.
THX_HD double time_loop_begin(thx_time_loop &L) {
  if (L.done) {
    L.last_dt = 0.0;
    return 0.0;
  }
  const double ev[3] = {L.t_final, L.next_output, L.next_checkpoint};
  const double s = limit_step_to_events(L.dt, L.t, ev, 3);
  L.last_dt = s;
  return s;
}

// After the cycle's step: total_rate is TotalRate of the new state (read
// only when cfl > 0).  Returns false when the rate is not positive.
THX_HD bool time_loop_end(thx_time_loop &L, double taken, double total_rate, double cfl) {
  if (L.done) return true;
  bool ok = true;
  L.t = L.t + taken;
  L.cycle += 1;
  if (cfl > 0.0) {
    if (total_rate > 0.0) {
      const double est = cfl / total_rate;
      const double grown = L.max_dt_growth * L.dt;
      L.dt = est < grown ? est : grown;
    } else {
      ok = false;
    }
  }
  const double margin = 1e-8 * L.dt;
  const bool done = L.t >= L.t_final - margin || step_limit_reached(L.cycle, L.max_cycles);
  if (time_finite(L.next_output) &&
      (done || time_event_reached(L.t, L.next_output) ||
       (L.output_cycles > 0 && L.cycle % L.output_cycles == 0))) {
    L.next_output = L.next_output + (L.t < L.refine_time ? L.output_dt : L.refined_output_dt);
    L.outputs += 1;
  }
  if (time_finite(L.next_checkpoint) && (done || time_event_reached(L.t, L.next_checkpoint))) {
    L.next_checkpoint = L.next_checkpoint + L.checkpoint_dt;
    L.checkpoints += 1;
  }
  if (done) L.done = 1;
  return ok;
}

}  // namespace thx
