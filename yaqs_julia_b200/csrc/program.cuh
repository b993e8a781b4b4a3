// program.cuh — the per-trajectory TJM program and the unit scheduler of
// the persistent trajectory kernels (shared by the kernels of engine.cu and
// the tensor-core kernel of engine_tc.cu).
#pragma once
#include "tjm.cuh"

// ---------------------------------------------------------------------------
// Device program
// ---------------------------------------------------------------------------
static __device__ void copy_state(Ctx& c, const DState& dst, const DState& src) {
  ProfScope prof_scope_(PF_COPY);
  cta_copy(dst.a, src.a, c.P.mps_size);
  for (int b = ltid(); b <= c.P.L; b += NT) dst.chi[b] = src.chi[b];
  if (ltid() == 0) *dst.oc = *src.oc;
  cta_sync();
}

static __device__ void sample(Ctx& c, const DState& phi, const DState& psi, int col) {
  copy_state(c, psi, phi);
  tdvp_sweep(c, psi);
  if (c.sm.fail) return;
  apply_dissipation(c, psi, false, c.P.dt / 2);
  if (c.sm.fail) return;
  if (c.P.noise_present) stochastic_process(c, psi, c.P.dt);
  if (c.sm.fail) return;
  evaluate(c, psi, col);
}

static __device__ void run_step(Ctx& c, int j) {
  ProfScope prof_scope_(PF_STEP);
  const DevParams& P = c.P;
  const int L = P.L;
  DState phi{P.phi + (long long)c.traj * P.mps_size, P.phi_chi + (long long)c.traj * (L + 1), P.phi_oc + c.traj};
  DState psi{c.ws + P.lay.psi, c.wsi + P.lay.i_chi, c.wsi + P.lay.i_oc};
  if (j == 0) {
    cta_copy(phi.a, P.psi0, P.mps_size);
    for (int b = ltid(); b <= L; b += NT) phi.chi[b] = P.chi0[b];
    if (ltid() == 0) *phi.oc = 0;
    cta_sync();
    normalize_state(c, phi);  // Simulator.jl:128
    if (P.sample_ts) evaluate(c, phi, 0);
    if (P.order == 2) {
      apply_dissipation(c, phi, false, P.dt / 2);  // initialize, AnalogTJM.jl:21-33
      if (c.sm.fail) return;
      if (P.noise_present) stochastic_process(c, phi, P.dt);
      if (c.sm.fail) return;
      if (P.sample_ts && P.n_times > 1) sample(c, phi, psi, 1);
    }
    return;
  }
  tdvp_sweep(c, phi);
  if (c.sm.fail) return;
  if (P.order == 2) {
    apply_dissipation(c, phi, true, P.dt);  // step_through, AnalogTJM.jl:40-55
    if (c.sm.fail) return;
    if (P.noise_present) stochastic_process(c, phi, P.dt);
    if (c.sm.fail) return;
    if (P.sample_ts || j == P.n_times - 1) sample(c, phi, psi, P.sample_ts ? j : 0);
  } else {
    if (P.noise_present) {  // AnalogTJM.jl:160-173
      apply_dissipation(c, phi, true, P.dt);
      if (c.sm.fail) return;
      stochastic_process(c, phi, P.dt);
      if (c.sm.fail) return;
    }
    if (P.sample_ts)
      evaluate(c, phi, j);
    else if (j == P.n_times - 1)
      evaluate(c, phi, 0);
  }
}

// Work units of a launch are (position, trajectory) pairs in position-major
// order, where the positions first .. first+count-1 index P.jlist.  Each CTA
// pulls the next unit from an atomic counter, so work is balanced at the
// granularity of one time index (or circuit layer) of one trajectory, not of
// whole trajectories.  A unit runs only after the same trajectory's previous
// position has finished: that unit was pulled earlier by a CTA that is
// executing it, so the wait always ends; it is still bounded (about 100 s)
// and gives up with ST_TIMEOUT.
#define DONE_WAIT_POLLS 100000000LL
static __device__ bool wait_done(const DevParams& P, int t, int need, CtaSmem& sm) {
  if (ltid() == 0) {
    volatile int* d = P.done + t;
    int ok = 0;
    for (long long it = 0; it < DONE_WAIT_POLLS; ++it) {
      if (*d >= need) {
        ok = 1;
        break;
      }
      __nanosleep(1000);
    }
    __threadfence();
    sm.bcast_i[6] = ok;
  }
  cta_sync();
  const int ok = sm.bcast_i[6];
  cta_sync();
  return ok != 0;
}

template <class StepFn>
static __device__ void run_units(const DevParams& P, CtaSmem& sm, int first, int count, StepFn step) {
  const int slot = cta_slot();
  cplx* ws = P.ws + (long long)slot * P.lay.total;
  int* wsi = P.wsi + (long long)slot * P.lay.itotal;
  const int nt = P.num_traj;
  const int total = count * nt;
  for (;;) {
    if (ltid() == 0) sm.bcast_i[7] = atomicAdd(&P.queue[first], 1);
    cta_sync();
    const int u = sm.bcast_i[7];
    cta_sync();
    if (u >= total) break;
    const int k = u / nt, t = u - k * nt, pos = first + k;
    bool ready = true;
    if (k > 0) ready = wait_done(P, t, pos - 1, sm);
    if (ltid() == 0) sm.fail = ready ? 0 : ST_TIMEOUT;
    cta_sync();
    if (ready && P.status[t] == 0) {
      Ctx c{P, sm, ws, wsi, slot, t, P.counters + (long long)slot * 8, P.flops + slot};
      step(c, P.jlist[pos]);
    }
    cta_sync();
    const bool tc_dead = P.tc && sm.e.tc.fatal;  // a tensor-core wait gave up: stop pulling units
    if (ltid() == 0) {
      if (tc_dead) sm.fail = ST_TIMEOUT;
      if (sm.fail && P.status[t] == 0) P.status[t] = sm.fail;
      __threadfence();
      atomicExch(P.done + t, pos);
    }
    cta_sync();
    if (tc_dead) break;
  }
}

