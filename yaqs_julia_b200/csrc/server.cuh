// server.cuh — request loop serving many simulations on one GPU
// (yaqs_server_*).  Included at the end of engine.cu.
//
// Device side (serve.cuh): serve_kernel, or its two-program tensor-core
// form when the server admits mixed-precision runs (engine_tc.cu), runs one
// batch of every admitted run.
//
// Host side: one thread per server admits queued requests (first come,
// first served, while their footprint fits the HBM budget), builds a batch
// of every admitted run, launches it, and retires runs whose launch list is
// exhausted.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>

#include "serve.cuh"

__global__ void __launch_bounds__(NT, 2) serve_kernel(const BatchRun* runs, int nruns, int total_units,
                                                      int* counter) {
  extern __shared__ __align__(16) unsigned char smraw[];
  CtaSmem& sm = *reinterpret_cast<CtaSmem*>(align_smem_1024(smraw));
  __shared__ __align__(16) BatchRun br;
  serve_units(runs, nruns, total_units, counter, sm, br);
}

namespace {

using Clock = std::chrono::steady_clock;

// Owned copy of one request's descriptors (submit returns before the
// request is admitted, so nothing may point into caller memory).
struct ReqCopy {
  int digital = 0;
  int L = 0;
  std::vector<int32_t> chi, w;
  std::vector<std::vector<double>> mps, mpo;
  std::vector<const double*> mps_ptrs, mpo_ptrs;
  yaqs_mps_desc mps_desc{};
  yaqs_mpo_desc mpo_desc{};
  std::vector<yaqs_noise_proc> procs;
  yaqs_noise_desc noise{};
  bool has_noise = false;
  std::vector<yaqs_obs_desc> obs;
  yaqs_tev_config tcfg{};
  yaqs_circuit_config ccfg{};
  std::vector<yaqs_gate_desc> gates;
  std::vector<double> uniforms;
  yaqs_rng_desc rng{};
};

struct Request {
  int64_t id = 0;
  ReqCopy in;
  int state = YAQS_REQ_QUEUED;
  int status = YAQS_OK;
  std::string err;
  size_t footprint = 0;
  int num_traj = 0, n_obs = 0, ncols = 0;
  yaqs_run* run = nullptr;
  Clock::time_point t_submit, t_admit, t_done;
  std::vector<double> traj, mean;
  std::vector<int32_t> maxchi;
  yaqs_run_stats stats{};
};

bool copy_common(ReqCopy& r, const yaqs_mps_desc* psi0, const yaqs_noise_desc* noise, const yaqs_obs_desc* obs,
                 int32_t n_obs, const yaqs_rng_desc* rng, int num_traj, std::string& err) {
  if (!psi0 || !rng || (n_obs > 0 && !obs) || n_obs < 0 || psi0->L < 2 || psi0->L > MAX_L || !psi0->chi ||
      !psi0->tensors) {
    err = "null or malformed descriptor";
    return false;
  }
  const int L = psi0->L;
  r.L = L;
  r.chi.assign(psi0->chi, psi0->chi + L + 1);
  r.mps.resize(L);
  for (int i = 0; i < L; ++i) {
    if (!psi0->tensors[i] || r.chi[i] < 1 || r.chi[i + 1] < 1 || r.chi[i] > 4096 || r.chi[i + 1] > 4096) {
      err = "null MPS tensor or bad bond dimension";
      return false;
    }
    const size_t n = (size_t)r.chi[i] * 2 * r.chi[i + 1] * 2;
    r.mps[i].assign(psi0->tensors[i], psi0->tensors[i] + n);
  }
  for (auto& t : r.mps) r.mps_ptrs.push_back(t.data());
  r.mps_desc = {L, r.chi.data(), r.mps_ptrs.data()};
  r.has_noise = noise && noise->present;
  if (r.has_noise) {
    if (noise->n < 0 || noise->n > MAX_PROCS || (noise->n > 0 && !noise->procs)) {
      err = "bad noise descriptor";
      return false;
    }
    r.procs.assign(noise->procs, noise->procs + noise->n);
    if (has_long_range(noise, noise->n)) {  // slots carry no long-range work buffers
      err = "UNSUPPORTED: long-range noise processes are served by yaqs_analog_run / yaqs_digital_run only";
      return false;
    }
  }
  r.noise = {r.has_noise ? 1 : 0, (int32_t)r.procs.size(), r.procs.empty() ? nullptr : r.procs.data()};
  if (n_obs > 0) r.obs.assign(obs, obs + n_obs);
  r.rng = *rng;
  if (rng->mode == YAQS_RNG_INJECTED) {
    if (!rng->uniforms || rng->stride < 1) {
      err = "injected uniforms need a buffer and stride >= 1";
      return false;
    }
    r.uniforms.assign(rng->uniforms, rng->uniforms + (size_t)num_traj * rng->stride);
    r.rng.uniforms = r.uniforms.data();
  }
  return true;
}

}  // namespace

struct yaqs_server {
  yaqs_ctx* ctx = nullptr;  // the caller's context (device)
  yaqs_ctx ictx;            // the server thread's own context (errors, lock)
  yaqs_server_config cfg{};
  ServePool pool;
  DevMem pool_mem;
  size_t smem = 0;
  size_t budget = 0, in_use = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread th;
  bool stop = false;
  int64_t next_id = 1;
  std::deque<Request*> pending;
  std::vector<Request*> active;
  std::map<int64_t, Request*> all;
  int64_t submitted = 0, completed = 0, failed = 0, launches = 0;
  double busy_s = 0;
  std::vector<double> lat, qlat;
  std::string err;
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  BatchRun* d_batch = nullptr;
  int batch_cap = 0;
  int* d_counter = nullptr;

  void loop();
  void fail_request(Request* r, int st, const std::string& msg) {
    r->state = YAQS_REQ_FAILED;
    r->status = st;
    r->err = msg;
    r->t_done = Clock::now();
    ++failed;
  }
};

void yaqs_server::loop() {
  cudaSetDevice(ictx.device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    cv_work.wait(lk, [&] { return stop || !pending.empty() || !active.empty(); });
    if (stop) break;
    // ---- admission: arrival order, while the footprint fits ----
    while (!pending.empty()) {
      Request* r = pending.front();
      if (!active.empty() && in_use + r->footprint > budget) break;
      pending.pop_front();
      lk.unlock();
      yaqs_run* run = nullptr;
      int st;
      ReqCopy& in = r->in;
      if (in.digital)
        st = digital_begin(&ictx, &in.mps_desc, in.gates.empty() ? nullptr : in.gates.data(), (int32_t)in.gates.size(),
                           &in.noise, in.obs.empty() ? nullptr : in.obs.data(), (int32_t)in.obs.size(), &in.ccfg,
                           &in.rng, &run, &pool);
      else
        st = analog_begin_impl(&ictx, &in.mps_desc, &in.mpo_desc, &in.noise, in.obs.empty() ? nullptr : in.obs.data(),
                               (int32_t)in.obs.size(), &in.tcfg, &in.rng, &run, &pool);
      std::string msg = ictx.err;
      lk.lock();
      if (st != YAQS_OK) {
        fail_request(r, st, msg);
        cv_done.notify_all();
        continue;
      }
      r->run = run;
      r->state = YAQS_REQ_RUNNING;
      r->t_admit = Clock::now();
      qlat.push_back(std::chrono::duration<double>(r->t_admit - r->t_submit).count());
      in_use += r->footprint;
      active.push_back(r);
    }
    if (active.empty()) continue;
    // ---- one batch: every admitted run advances by up to `chunk` positions ----
    std::vector<BatchRun> batch;
    int units = 0;
    for (Request* r : active) {
      yaqs_run* run = r->run;
      const int rem = (int)(run->launches.size() - run->next);
      const int cnt = std::min(rem, std::max(1, cfg.chunk));
      if (cnt <= 0) continue;
      const long long add = (long long)cnt * run->P.num_traj;
      if (!batch.empty() && (long long)units + add > (1LL << 30)) break;
      BatchRun b;
      memset(&b, 0, sizeof(b));
      b.P = run->P;
      b.D = run->D;
      b.digital = run->digital;
      b.first = (int)run->next;
      b.count = cnt;
      b.unit_begin = units;
      units += (int)add;
      run->next += cnt;
      batch.push_back(b);
    }
    lk.unlock();
    int st = YAQS_OK;
    std::string msg;
    float ms = 0.f;
    auto cuda_fail = [&](cudaError_t e, const char* what) {
      st = YAQS_E_CUDA;
      msg = std::string(what) + ": " + cudaGetErrorString(e);
    };
    if ((int)batch.size() > batch_cap) {
      if (d_batch) cudaFree(d_batch);
      batch_cap = (int)batch.size() * 2;
      cudaError_t e = cudaMalloc(&d_batch, batch_cap * sizeof(BatchRun));
      if (e != cudaSuccess) {
        d_batch = nullptr;
        batch_cap = 0;
        cuda_fail(e, "batch allocation");
      }
    }
    if (st == YAQS_OK && !batch.empty()) {
      cudaError_t e = cudaMemcpyAsync(d_batch, batch.data(), batch.size() * sizeof(BatchRun), cudaMemcpyHostToDevice,
                                      stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(d_counter, 0, sizeof(int), stream);
      if (e == cudaSuccess) e = cudaEventRecord(e0, stream);
      if (e == cudaSuccess) {
        if (pool.tc) {
          e = tc_serve_launch(pool.slots, smem, stream, d_batch, (int)batch.size(), units, d_counter);
        } else {
          serve_kernel<<<pool.slots, NT, smem, stream>>>(d_batch, (int)batch.size(), units, d_counter);
          e = cudaGetLastError();
        }
      }
      if (e == cudaSuccess) e = cudaEventRecord(e1, stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) cuda_fail(e, "served launch");
    }
    lk.lock();
    ++launches;
    busy_s += ms / 1e3;
    // ---- retire finished runs (and every run if the launch failed) ----
    std::vector<Request*> keep;
    for (Request* r : active) {
      yaqs_run* run = r->run;
      const bool finished = st != YAQS_OK || run->next >= run->launches.size();
      if (!finished) {
        keep.push_back(r);
        continue;
      }
      r->run = nullptr;
      lk.unlock();
      r->traj.assign((size_t)r->num_traj * std::max(r->n_obs, 1) * r->ncols, 0.0);
      r->mean.assign((size_t)std::max(r->n_obs, 1) * r->ncols, 0.0);
      r->maxchi.assign((size_t)r->num_traj * r->ncols, 0);
      int fst = st;
      if (st == YAQS_OK)
        fst = yaqs_analog_finish(run, r->traj.data(), r->mean.data(), r->maxchi.data(), &r->stats);
      else
        yaqs_analog_finish(run, nullptr, nullptr, nullptr, nullptr);
      std::string fmsg = st == YAQS_OK ? ictx.err : msg;
      lk.lock();
      in_use -= r->footprint;
      if (fst != YAQS_OK) {
        fail_request(r, fst, fmsg);
      } else {
        r->state = YAQS_REQ_DONE;
        r->t_done = Clock::now();
        lat.push_back(std::chrono::duration<double>(r->t_done - r->t_submit).count());
        ++completed;
      }
    }
    active.swap(keep);
    cv_done.notify_all();
  }
  // shutdown: fail what is left
  for (Request* r : active) {
    yaqs_run* run = r->run;
    r->run = nullptr;
    lk.unlock();
    yaqs_analog_finish(run, nullptr, nullptr, nullptr, nullptr);
    lk.lock();
    fail_request(r, YAQS_E_ARG, "server destroyed");
  }
  active.clear();
  for (Request* r : pending) fail_request(r, YAQS_E_ARG, "server destroyed");
  pending.clear();
  cv_done.notify_all();
}

namespace {
double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - i;
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

// Device bytes a request's run allocates besides the shared slot pool.
size_t request_footprint(const ReqCopy& in, int num_traj, int n_obs, int ncols, int max_bond) {
  std::vector<int> w(in.L + 1, 1);
  if (!in.digital) w = std::vector<int>(in.w.begin(), in.w.end());
  Caps c;
  if (!plan_caps(in.L, in.chi.data(), w.data(), max_bond, c)) return 0;
  const size_t per_traj = (size_t)c.mps_size * sizeof(cplx) + (in.L + 4) * sizeof(int) + 64 +
                          (size_t)std::max(n_obs, 1) * ncols * sizeof(double) + ncols * sizeof(int) + 8;
  return (size_t)num_traj * per_traj + (size_t)c.mps_size * sizeof(cplx) + in.uniforms.size() * sizeof(double) +
         (1u << 20);
}

int submit(yaqs_server* srv, Request* r, int64_t* id) {
  std::lock_guard<std::mutex> lk(srv->mu);
  if (srv->stop) {
    delete r;
    return YAQS_E_ARG;
  }
  r->id = srv->next_id++;
  r->t_submit = Clock::now();
  srv->all[r->id] = r;
  srv->pending.push_back(r);
  ++srv->submitted;
  *id = r->id;
  srv->cv_work.notify_all();
  return YAQS_OK;
}
}  // namespace

extern "C" {

int yaqs_server_create(yaqs_ctx* ctx, const yaqs_server_config* cfg, yaqs_server** out) {
  if (!ctx || !cfg || !out) return set_err(ctx, YAQS_E_ARG, "null argument");
  *out = nullptr;
  if (cfg->max_L < 2 || cfg->max_L > MAX_L || cfg->max_bond_dim < 1 || cfg->max_bond_dim > SVD_MAX_COLS / 2 ||
      cfg->max_mpo_width < 1 || cfg->max_mpo_width > 8 || cfg->krylov_dim < 1 || cfg->krylov_dim > KRYLOV_MAX ||
      cfg->chunk < 1 || cfg->hbm_budget < 0)
    return set_err(ctx, YAQS_E_ARG, "bad server config");
  std::unique_ptr<yaqs_server> srv(new yaqs_server());
  srv->ctx = ctx;
  srv->cfg = *cfg;
  srv->ictx.device = ctx->device;
  srv->ictx.sms = ctx->sms;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  // slot shape: the largest analog and digital layouts the config admits
  const int L = cfg->max_L;
  std::vector<int> wmax(L + 1, cfg->max_mpo_width), wone(L + 1, 1);
  wmax[0] = wmax[L] = 1;
  Caps ca, cd;
  plan_caps(L, nullptr, wmax.data(), cfg->max_bond_dim, ca);
  plan_caps(L, nullptr, wone.data(), cfg->max_bond_dim, cd);
  const WsLayout la = plan_layout(L, ca, wmax.data(), true, cfg->krylov_dim, cfg->mixed != 0);
  const WsLayout ld = plan_layout(L, cd, wone.data(), false, 0, false);
  long long stride = std::max(la.total, ld.total);
  srv->pool.wsi_stride = std::max(la.itotal, ld.itotal);
  // a server that admits mixed runs serves every batch with the two-program
  // tensor-core kernel; the tcgen05 operands of every slot sit at its end
  srv->pool.tc = cfg->mixed != 0;
  if (srv->pool.tc) {
    const WsLayout lt = plan_layout(L, ca, wmax.data(), true, cfg->krylov_dim, true, false, true);
    WsLayout g = lt;  // the staged operands are the last buffers plan_layout takes
    g.sL = stride + (lt.sL - lt.sL);
    g.sx = stride + (lt.sx - lt.sL);
    g.sT2 = stride + (lt.sT2 - lt.sL);
    g.sR = stride + (lt.sR - lt.sL);
    srv->pool.stage = g;
    stride += lt.total - lt.sL;
  }
  srv->pool.ws_stride = stride;
  int per_sm = 0;
  if (srv->pool.tc) {
    CUDA_TRY(ctx, tc_serve_prepare(&per_sm, &srv->smem));
    per_sm = std::min(per_sm, TMEM_PROGRAMS_PER_SM);
  } else {
    srv->smem = cta_smem_bytes();
    CUDA_TRY(ctx, cudaFuncSetAttribute(serve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)srv->smem));
    CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_kernel, NT, srv->smem));
  }
  if (per_sm < 1) return set_err(ctx, YAQS_E_CUDA, "served kernel does not fit on an SM");
  srv->pool.slots = ctx->sms * per_sm;
  CUDA_TRY(ctx, srv->pool_mem.alloc(&srv->pool.ws, (size_t)srv->pool.slots * srv->pool.ws_stride));
  CUDA_TRY(ctx, srv->pool_mem.alloc(&srv->pool.wsi, (size_t)srv->pool.slots * srv->pool.wsi_stride));
  if (srv->pool.tc) {  // four tensor maps per slot
    std::vector<CUtensorMap> maps(4 * (size_t)srv->pool.slots);
    const WsLayout& g = srv->pool.stage;
    for (int sl = 0; sl < srv->pool.slots; ++sl) {
      const cplx* base = srv->pool.ws + (long long)sl * stride;
      if (!make_tc_map(&maps[4 * sl + 0], base + g.sL, g.pL, g.rL, TC_A_MN) ||
          !make_tc_map(&maps[4 * sl + 1], base + g.sx, g.px, g.rx, TC_B_K) ||
          !make_tc_map(&maps[4 * sl + 2], base + g.sT2, g.pT2, g.rT2, TC_A_MN) ||
          !make_tc_map(&maps[4 * sl + 3], base + g.sR, g.pR, g.rR, TC_B_MN))
        return set_err(ctx, YAQS_E_CUDA, "cuTensorMapEncodeTiled refused a staged H_eff operand");
    }
    CUtensorMap* d_maps;
    CUDA_TRY(ctx, srv->pool_mem.alloc(&d_maps, maps.size()));
    CUDA_TRY(ctx, cudaMemcpy(d_maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    srv->pool.tmaps = d_maps;
  }
  CUDA_TRY(ctx, srv->pool_mem.alloc(&srv->d_counter, 1));
  size_t free_b = 0, total_b = 0;
  CUDA_TRY(ctx, cudaMemGetInfo(&free_b, &total_b));
  srv->budget = cfg->hbm_budget > 0 ? (size_t)cfg->hbm_budget : (size_t)(0.9 * (double)free_b);
  CUDA_TRY(ctx, cudaStreamCreateWithFlags(&srv->stream, cudaStreamNonBlocking));
  CUDA_TRY(ctx, cudaEventCreate(&srv->e0));
  CUDA_TRY(ctx, cudaEventCreate(&srv->e1));
  yaqs_server* s = srv.release();
  s->th = std::thread([s] { s->loop(); });
  *out = s;
  return YAQS_OK;
}

int yaqs_server_submit_analog(yaqs_server* srv, const yaqs_mps_desc* psi0, const yaqs_mpo_desc* H,
                              const yaqs_noise_desc* noise, const yaqs_obs_desc* obs, int32_t n_obs,
                              const yaqs_tev_config* cfg, const yaqs_rng_desc* rng, int64_t* id) {
  if (!srv || !id || !cfg || !H || !psi0) return set_err(nullptr, YAQS_E_ARG, "null argument");
  std::unique_ptr<Request> r(new Request());
  ReqCopy& in = r->in;
  std::string err;
  if (cfg->num_traj < 1 || cfg->n_times < 1) return set_err(nullptr, YAQS_E_ARG, "bad config");
  if (!copy_common(in, psi0, noise, obs, n_obs, rng, cfg->num_traj, err))
    return set_err(nullptr, err.rfind("UNSUPPORTED", 0) == 0 ? YAQS_E_UNSUPPORTED : YAQS_E_ARG, err);
  if (H->L != psi0->L || !H->w || !H->tensors) return set_err(nullptr, YAQS_E_ARG, "bad MPO descriptor");
  in.w.assign(H->w, H->w + H->L + 1);
  in.mpo.resize(H->L);
  for (int i = 0; i < H->L; ++i) {
    if (!H->tensors[i] || in.w[i] < 1 || in.w[i + 1] < 1 || in.w[i] > 8 || in.w[i + 1] > 8)
      return set_err(nullptr, YAQS_E_ARG, "bad MPO tensor");
    in.mpo[i].assign(H->tensors[i], H->tensors[i] + (size_t)in.w[i] * 4 * in.w[i + 1] * 2);
  }
  for (auto& t : in.mpo) in.mpo_ptrs.push_back(t.data());
  in.mpo_desc = {H->L, in.w.data(), in.mpo_ptrs.data()};
  in.tcfg = *cfg;
  r->num_traj = cfg->num_traj;
  r->n_obs = n_obs;
  r->ncols = cfg->sample_timesteps ? cfg->n_times : 1;
  r->footprint = request_footprint(in, r->num_traj, n_obs, r->ncols, cfg->max_bond_dim);
  return submit(srv, r.release(), id);
}

int yaqs_server_submit_digital(yaqs_server* srv, const yaqs_mps_desc* psi0, const yaqs_gate_desc* gates,
                               int32_t n_gates, const yaqs_noise_desc* noise, const yaqs_obs_desc* obs,
                               int32_t n_obs, const yaqs_circuit_config* cfg, const yaqs_rng_desc* rng,
                               int64_t* id) {
  if (!srv || !id || !cfg || !psi0 || n_gates < 0 || (n_gates > 0 && !gates))
    return set_err(nullptr, YAQS_E_ARG, "null argument");
  std::unique_ptr<Request> r(new Request());
  ReqCopy& in = r->in;
  std::string err;
  if (cfg->num_traj < 1) return set_err(nullptr, YAQS_E_ARG, "bad config");
  if (!copy_common(in, psi0, noise, obs, n_obs, rng, cfg->num_traj, err))
    return set_err(nullptr, err.rfind("UNSUPPORTED", 0) == 0 ? YAQS_E_UNSUPPORTED : YAQS_E_ARG, err);
  in.digital = 1;
  in.gates.assign(gates, gates + n_gates);
  in.ccfg = *cfg;
  HostCircuit C;
  int st = plan_circuit(nullptr, gates, n_gates, psi0->L, C);
  if (st != YAQS_OK) return st;
  r->num_traj = cfg->num_traj;
  r->n_obs = n_obs;
  r->ncols = C.n_samples;
  r->footprint = request_footprint(in, r->num_traj, n_obs, r->ncols, cfg->max_bond_dim);
  return submit(srv, r.release(), id);
}

int yaqs_server_poll(yaqs_server* srv, int64_t id, int32_t* state) {
  if (!srv || !state) return set_err(nullptr, YAQS_E_ARG, "null argument");
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->all.find(id);
  if (it == srv->all.end()) return set_err(nullptr, YAQS_E_ARG, "unknown request id");
  *state = it->second->state;
  return YAQS_OK;
}

int yaqs_server_wait(yaqs_server* srv, int64_t id, double timeout_s) {
  if (!srv) return set_err(nullptr, YAQS_E_ARG, "null server");
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->all.find(id);
  if (it == srv->all.end()) return set_err(nullptr, YAQS_E_ARG, "unknown request id");
  Request* r = it->second;
  auto done = [&] { return r->state == YAQS_REQ_DONE || r->state == YAQS_REQ_FAILED; };
  if (timeout_s < 0) {
    srv->cv_done.wait(lk, done);
  } else if (!srv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
    return set_err(nullptr, YAQS_E_TIMEOUT, "request not finished in time");
  }
  return YAQS_OK;
}

int yaqs_server_take(yaqs_server* srv, int64_t id, double* traj_out, double* mean_out, int32_t* maxchi_out,
                     yaqs_run_stats* stats, double* times_s) {
  if (!srv) return set_err(nullptr, YAQS_E_ARG, "null server");
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->all.find(id);
  if (it == srv->all.end()) return set_err(nullptr, YAQS_E_ARG, "unknown request id");
  Request* r = it->second;
  if (r->state != YAQS_REQ_DONE && r->state != YAQS_REQ_FAILED)
    return set_err(nullptr, YAQS_E_ARG, "request not finished (wait for it first)");
  srv->all.erase(it);
  std::unique_ptr<Request> guard(r);
  if (r->state == YAQS_REQ_FAILED) {
    srv->err = r->err;
    return r->status;
  }
  const size_t nt = r->num_traj, no = r->n_obs, nc = r->ncols;
  if (traj_out) memcpy(traj_out, r->traj.data(), nt * no * nc * sizeof(double));
  if (mean_out) memcpy(mean_out, r->mean.data(), no * nc * sizeof(double));
  if (maxchi_out) memcpy(maxchi_out, r->maxchi.data(), nt * nc * sizeof(int32_t));
  if (stats) *stats = r->stats;
  if (times_s) {
    times_s[0] = std::chrono::duration<double>(r->t_admit - r->t_submit).count();
    times_s[1] = std::chrono::duration<double>(r->t_done - r->t_admit).count();
    times_s[2] = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  }
  return YAQS_OK;
}

const char* yaqs_server_last_error(yaqs_server* srv) { return srv ? srv->err.c_str() : g_static_err.c_str(); }

int yaqs_server_stats_get(yaqs_server* srv, yaqs_server_stats* out) {
  if (!srv || !out) return set_err(nullptr, YAQS_E_ARG, "null argument");
  std::lock_guard<std::mutex> lk(srv->mu);
  memset(out, 0, sizeof(*out));
  out->submitted = srv->submitted;
  out->completed = srv->completed;
  out->failed = srv->failed;
  out->launches = srv->launches;
  out->queued_now = (int64_t)srv->pending.size();
  out->running_now = (int64_t)srv->active.size();
  out->bytes_in_use = (int64_t)srv->in_use;
  out->hbm_budget = (int64_t)srv->budget;
  out->slots = srv->pool.slots;
  out->latency_p50_s = percentile(srv->lat, 0.50);
  out->latency_p99_s = percentile(srv->lat, 0.99);
  out->queue_p50_s = percentile(srv->qlat, 0.50);
  out->queue_p99_s = percentile(srv->qlat, 0.99);
  out->busy_s = srv->busy_s;
  return YAQS_OK;
}

int yaqs_server_destroy(yaqs_server* srv) {
  if (!srv) return YAQS_OK;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
  }
  srv->cv_work.notify_all();
  if (srv->th.joinable()) srv->th.join();
  for (auto& kv : srv->all) delete kv.second;
  if (srv->d_batch) cudaFree(srv->d_batch);
  if (srv->stream) {
    cudaStreamSynchronize(srv->stream);
    cudaStreamDestroy(srv->stream);
  }
  if (srv->e0) cudaEventDestroy(srv->e0);
  if (srv->e1) cudaEventDestroy(srv->e1);
  delete srv;
  return YAQS_OK;
}

}  // extern "C"
