// serve.cuh — the device loop of the request server (yaqs_server_*): one
// launch runs a batch, a list of runs each advancing positions
// [first, first + count) of its launch list.  Work units are (run, position,
// trajectory) triples, run-major and position-major within a run; each
// trajectory program pulls the next unit from an atomic counter, copies that
// run's parameters into shared memory and runs one time index (or circuit
// layer) of one trajectory in its pool slot, with the same per-trajectory
// ordering flags as the single-run kernels.  Shared by the server's kernel
// (server.cuh) and its two-program tensor-core kernel (engine_tc.cu).
#pragma once
#include "digital.cuh"
#include "program.cuh"

struct BatchRun {
  DevParams P;
  DigParams D;
  int digital;
  int first, count;
  int unit_begin;
};

static __device__ void serve_units(const BatchRun* runs, int nruns, int total_units, int* counter, CtaSmem& sm,
                                   BatchRun& br) {
  const int slot = cta_slot();
  for (;;) {
    if (ltid() == 0) {
      const int u = atomicAdd(counter, 1);
      int r = 0;
      while (r + 1 < nruns && runs[r + 1].unit_begin <= u) ++r;
      sm.bcast_i[7] = u;
      sm.bcast_i[5] = r;
    }
    cta_sync();
    const int u = sm.bcast_i[7], r = sm.bcast_i[5];
    cta_sync();
    if (u >= total_units) break;
    {
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(runs + r);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(&br);
      for (int e = ltid(); e < (int)(sizeof(BatchRun) / 8); e += NT) dst[e] = src[e];
    }
    cta_sync();
    const DevParams& P = br.P;
    const int nt = P.num_traj;
    const int local = u - br.unit_begin, k = local / nt, t = local - k * nt, pos = br.first + k;
    cplx* ws = P.ws + (long long)slot * P.lay.total;
    int* wsi = P.wsi + (long long)slot * P.lay.itotal;
    bool ready = true;
    if (k > 0) ready = wait_done(P, t, pos - 1, sm);
    if (ltid() == 0) sm.fail = ready ? 0 : ST_TIMEOUT;
    cta_sync();
    if (ready && P.status[t] == 0) {
      Ctx c{P, sm, ws, wsi, slot, t, P.counters + (long long)slot * 8, P.flops + slot};
      if (br.digital)
        run_digital_step(c, br.D, P.jlist[pos]);
      else
        run_step(c, P.jlist[pos]);
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
