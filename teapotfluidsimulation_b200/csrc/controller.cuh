// Target-volume pour controller (src/sim/motion.ts:21-159), evaluated on the device at the start of
// every substep so that the discharge measured by the previous substep's advection feeds it with no
// host round trip and no lag (solver3d.ts:289-290).
#pragma once

#include "common.cuh"

namespace pl {

__device__ __forceinline__ double pour_target(const pl_motion& c, const DevController& s) {
  int reps = c.repeats > 1 ? c.repeats : 1;
  return (c.target_volume * (s.pour + 1)) / reps;  // motion.ts:53-56
}

__device__ __forceinline__ void ctl_enter(DevController& s, int phase, double t) {  // motion.ts:62-68
  s.phase = phase;
  s.phase_start = t;
  s.start_angle = s.angle;
  s.start_rate = s.last_rate;
}

__device__ __forceinline__ bool ctl_should_return(const pl_motion& c, const DevController& s, double t,
                                                  double discharged) {  // motion.ts:145-154
  if (c.kind == PL_MOTION_TILT) return s.phase == PL_PHASE_HOLD && t - s.phase_start >= c.hold_time;
  if (s.phase == PL_PHASE_HOLD && t - s.phase_start >= c.max_hold) return true;
  if (c.target_volume <= 0) return false;
  double in_transit = dmax(0.0, s.flow_rate) * c.anticipation * c.return_duration;
  return discharged + in_transit >= pour_target(c, s);
}

// PourController.advance(t, dt, discharged) (motion.ts:74-143): returns the tilt at t (rad).
__device__ double ctl_advance(const pl_motion& c, DevController& s, double t, double dt, double discharged) {
  if (dt > 0) {
    double inst = (discharged - s.last_discharged) / dt;
    double k = dmin(1.0, dt / 0.25);
    s.flow_rate += (inst - s.flow_rate) * k;
  }
  s.last_discharged = discharged;
  double prev = s.angle;
  if (s.phase == PL_PHASE_MANUAL) {
    if (dt > 0) {
      double desired = dmax(-90 * DEG, dmin(90 * DEG, (s.target - s.angle) / 0.15));
      double max_change = 600 * DEG * dt;
      s.manual_rate += dmax(-max_change, dmin(max_change, desired - s.manual_rate));
      s.angle += s.manual_rate * dt;
      s.last_rate = (s.angle - prev) / dt;
    }
    return s.angle;
  }
  double hold = c.hold_angle_deg * DEG;
  double max_a = c.max_angle_deg * DEG;
  int reps = c.repeats > 1 ? c.repeats : 1;
  for (int guard = 0; guard < 4; guard++) {
    double el = t - s.phase_start;
    if (s.phase == PL_PHASE_WAIT && t >= c.start_delay) {
      ctl_enter(s, PL_PHASE_TILT_IN, c.start_delay);
    } else if ((s.phase == PL_PHASE_TILT_IN || s.phase == PL_PHASE_HOLD) && ctl_should_return(c, s, t, discharged)) {
      ctl_enter(s, PL_PHASE_RETURN, t);
    } else if (s.phase == PL_PHASE_TILT_IN && el >= c.tilt_duration) {
      s.angle = hold;
      ctl_enter(s, PL_PHASE_HOLD, s.phase_start + c.tilt_duration);
    } else if (s.phase == PL_PHASE_RETURN && el >= c.return_duration) {
      s.angle = 0;
      s.pour++;
      ctl_enter(s, PL_PHASE_REST, s.phase_start + c.return_duration);
    } else if (s.phase == PL_PHASE_REST && s.pour < reps && el >= c.repeat_gap) {
      ctl_enter(s, PL_PHASE_TILT_IN, s.phase_start + c.repeat_gap);
    } else if (s.phase == PL_PHASE_REST && s.pour >= reps) {
      ctl_enter(s, PL_PHASE_DONE, t);
    } else {
      break;
    }
  }
  double el = t - s.phase_start;
  switch (s.phase) {
    case PL_PHASE_TILT_IN: {
      double u = dmin(1.0, el / c.tilt_duration);
      s.angle = s.start_angle + (hold - s.start_angle) * 0.5 * (1 - cos(PI * u));
      break;
    }
    case PL_PHASE_HOLD:
      s.angle = dmin(max_a, s.start_angle + c.hold_tilt_rate * DEG * el);
      break;
    case PL_PHASE_RETURN: {
      double T = c.return_duration;
      double u = dmin(1.0, el / T);
      double u3 = pow(u, 3.0);
      double h00 = 2 * u3 - 3 * (u * u) + 1;
      double h10 = u3 - 2 * (u * u) + u;
      s.angle = h00 * s.start_angle + h10 * T * s.start_rate;
      break;
    }
    default:
      s.angle = 0;
  }
  if (dt > 0) s.last_rate = (s.angle - prev) / dt;
  return s.angle;
}

}  // namespace pl
