// tjm.cuh — per-trajectory TJM program executed by one CTA.
//
// Restates, for one trajectory held in HBM, the analog TJM step of
// AnalogTJM.jl:21-176: the symmetric two-site TDVP sweep
// (Algorithms.jl:580-819), apply_dissipation (Dissipation.jl:37-159),
// stochastic_process! (StochasticProcess.jl:35-38, 89-330) and the
// observables (SimulationConfigs.jl:42-56, MPS.jl:608-651), together with
// the MPS gauge moves they rely on (MPS.jl:182-311, 528-585).
#pragma once
#include "common.cuh"
#include "gemm.cuh"
#include "krylov.cuh"
#include "linalg.cuh"

#define MAX_L 256
#define MAX_PROCS 512
#define MAX_OBS 512

enum { OBS_LOCAL1 = 1, OBS_LOCAL2 = 2, OBS_ENTROPY = 3 };
enum { ST_OK = 0, ST_ARG = 1, ST_NONFINITE = 3, ST_TIMEOUT = 5, ST_RNG = 7, ST_UNSUPPORTED = 8 };

struct DevProc {
  int nsites, s0, s1;
  int pauli_name, pauli_proc;
  int unitary;  // matrix^dag matrix = 1 (a jump then keeps every tensor's gauge)
  // Long-range process (s1 > s0 + 1): operator alpha*1 + beta*(sig at s0)
  // (tau at s1), mat[0..3] = sig, mat[4..7] = tau, mat[8] = alpha,
  // mat[9] = beta; pauli_proc marks the "pauli_long_range" candidate.
  int lr;
  double gamma;
  double drate;  // rate of the scalar decay exp(-dt/2 * drate) when pauli_name
  cplx mat[16];
  cplx diss_half[16];
  cplx diss_full[16];
};

struct DevObs {
  int kind, s0, s1;
  cplx mat[16];
};

// Offsets (in cplx elements) of the parts of one slot's workspace.
struct WsLayout {
  long long psi, EL, ER, Q, T1, T2, tA, tB, tC, th, B, X, Yo, Zo, y, dbl;
  // mixed form (FP32 buffers, offsets in complex-double units)
  long long Lf, Rf, xf, T1f, T2f, Af;
  // long-range jumps: right-canonical tensors of the operator applied to
  // the state (4 x the MPS arena) and work buffers
  long long lrQ, lrPhi, lrM, lrH, lrQh, lrL, lrR, lrC0, lrC1;
  // mixed form on tcgen05: TMA-staged FP32 operands of the H_eff products
  // (offsets in complex-double units, pitches and row counts in complex
  // FP32 values): SL = L as [k][a + chil m], Sx = x as [p + D c][k],
  // ST2 = T2 as [m' + wr c][a + chil p'], SR = R as [m' + wr c][b]
  long long sL, sx, sT2, sR;
  int pL, px, pT2, pR, rL, rx, rT2, rR;
  long long total;
  // int workspace (per slot)
  long long i_chi, i_oc, i_ord, i_cand, i_lr, itotal;
};

struct DevParams {
  int L, n_times, order, sample_ts, max_bond, nobs, nprocs, noise_present, all_zero, rng_mode, num_traj,
      traj_offset, ncols;
  int mixed;  // H_eff and environment contractions in complex FP32 on the tensor cores
  int tc;     // mixed H_eff products on tcgen05 (the tensor-core kernel, engine_tc.cu)
  const CUtensorMap* tmaps;  // [slots][4]: SL, Sx, ST2, SR of each slot
  const unsigned char* tune;  // [TUNE_ENTRIES] autotuned product form per bucket (null: tcgen05)
  int tdvp_mode;  // YAQS_TDVP_2SITE / _1SITE / _DYNAMIC
  double dt, thr;
  KrylovCfg kc;
  unsigned long long seed;
  long long stride;
  const int* cap;            // [L+1]
  const long long* mps_off;  // [L]
  long long mps_size;
  const int* w;              // [L+1]
  const WMat* wm_heff1;      // [L]
  const WMat* wm_heff2;      // [L-1]
  const WMat* wm_envL;       // [L]
  const WMat* wm_envR;       // [L]
  const WMat* wm_bond;       // [L+1] identity on the MPO bond (project_bond as a D = 1 H_eff)
  const long long* env_off;  // [L+1]
  long long kry_n;
  const DevProc* procs;
  const DevObs* obs;
  const cplx* psi0;  // arena layout, compact tensors
  const int* chi0;   // [L+1]
  cplx* phi;         // [num_traj][mps_size]
  int* phi_chi;      // [num_traj][L+1]
  int* phi_oc;       // [num_traj]
  cplx* ws;
  int* wsi;
  WsLayout lay;
  const double* uniforms;
  long long* rng_pos;  // [num_traj]
  double* traj_out;    // [num_traj][nobs][ncols]
  int* chi_out;        // [num_traj][ncols]
  int* status;         // [num_traj]
  unsigned long long* counters;  // [num_slots][8]
  double* flops;                 // [num_slots]
  int* queue;                    // [n_times] unit counter of the launch starting at each position
  int* done;                     // [num_traj] last launch-list position completed by each trajectory
  const int* jlist;              // [n_positions] time index (or layer) run at each launch-list position
};

struct CtaSmem {
  EngineSmem e;
  LinalgSmem la;
  int bcast_i[8];
  double bcast_d[8];
  int fail;
  int canon;  // the state is in mixed canonical form around its centre
};

// Dynamic shared memory of one trajectory program, with 1024 bytes of slack
// for aligning the base (the tensor-core buffers want 1024-byte alignment).
constexpr size_t cta_smem_bytes() { return sizeof(CtaSmem) + 1024; }
static __device__ __forceinline__ unsigned char* align_smem_1024(unsigned char* p) {
  const unsigned off = smem_u32(p);
  return p + ((1024u - (off & 1023u)) & 1023u);
}

struct Ctx {  // per-CTA view
  const DevParams& P;
  CtaSmem& sm;
  cplx* ws;
  int* wsi;
  int slot;
  int traj;
  unsigned long long* cnt;
  double* fl;
};

struct DState {
  cplx* a;
  int* chi;
  int* oc;
};

static __device__ __forceinline__ cplx* site_ptr(const Ctx& c, const DState& s, int i) { return s.a + c.P.mps_off[i]; }

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon et al., SC'11), one 53-bit double per counter.
// ---------------------------------------------------------------------------
static __device__ __forceinline__ double philox_uniform(unsigned long long seed, unsigned long long stream,
                                                 unsigned long long draw) {
  unsigned int c0 = (unsigned int)draw, c1 = (unsigned int)(draw >> 32), c2 = (unsigned int)stream,
               c3 = (unsigned int)(stream >> 32);
  unsigned int k0 = (unsigned int)seed, k1 = (unsigned int)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    unsigned int hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    unsigned int hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    unsigned int n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
    if (r < 9) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
  }
  unsigned long long bits = ((unsigned long long)c1 << 32) | c0;
  return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
}

// Next uniform of this trajectory (CTA-collective; broadcast).
static __device__ double draw_uniform(Ctx& c) {
  if (ltid() == 0) {
    long long pos = c.P.rng_pos[c.traj];
    double u;
    if (c.P.rng_mode == 1) {
      if (pos >= c.P.stride) {
        u = 1.0;
        c.sm.fail = ST_RNG;
      } else {
        u = c.P.uniforms[(long long)c.traj * c.P.stride + pos];
      }
    } else {
      u = philox_uniform(c.P.seed, (unsigned long long)(c.P.traj_offset + c.traj), (unsigned long long)pos);
    }
    c.P.rng_pos[c.traj] = pos + 1;
    c.sm.bcast_d[0] = u;
  }
  cta_sync();
  double u = c.sm.bcast_d[0];
  cta_sync();
  return u;
}

// ---------------------------------------------------------------------------
// Gauge moves (MPS.jl:182-311)
// ---------------------------------------------------------------------------
static __device__ void set_chi(Ctx& c, const DState& s, int b, int v) {
  cta_sync();
  if (ltid() == 0) {
    if (v > c.P.cap[b]) c.sm.fail = ST_UNSUPPORTED;
    else s.chi[b] = v;
  }
  cta_sync();
}

// site i: A = Q R, Q -> site i, R absorbed into site i+1.
static __device__ void qr_right(Ctx& c, const DState& s, int i) {
  const int l = s.chi[i], r = s.chi[i + 1], m = 2 * l, rn = min(m, r);
  const int r2 = s.chi[i + 2];
  cplx* A = site_ptr(c, s, i);
  cplx* An = site_ptr(c, s, i + 1);
  cplx* H = c.ws + c.P.lay.tA;
  cplx* Rb = c.ws + c.P.lay.tB;
  cplx* T = c.ws + c.P.lay.tC;
  cta_copy(H, A, (long long)m * r);
  cta_sync();
  dev_qr_factor(H, m, r, c.sm.la, c.sm.e.r);
  dev_qr_formq(H, m, r, A, c.sm.la);
  dev_qr_extract_r(H, m, r, Rb);
  cta_gemm(gemm_args(rn, 2 * r2, r, Rb, 1, rn, An, 1, r, T, 1, rn), c.sm.e.u.gw.g);
  cta_copy(An, T, (long long)rn * 2 * r2);
  set_chi(c, s, i + 1, rn);
}

// site i: A = L Q, Q -> site i, L absorbed into site i-1.
static __device__ void lq_left(Ctx& c, const DState& s, int i) {
  const int l = s.chi[i], r = s.chi[i + 1], n2 = 2 * r, rn = min(l, n2);
  const int lp = s.chi[i - 1];
  cplx* A = site_ptr(c, s, i);
  cplx* Ap = site_ptr(c, s, i - 1);
  cplx* H = c.ws + c.P.lay.tA;
  cplx* Qh = c.ws + c.P.lay.tB;
  cplx* Rb = c.ws + c.P.lay.tC;
  for (int e = ltid(); e < n2 * l; e += NT) {
    int cc = (int)(e % n2), ii = (int)(e / n2);
    H[e] = cconj(A[ii + (long long)l * cc]);
  }
  cta_sync();
  dev_qr_factor(H, n2, l, c.sm.la, c.sm.e.r);
  dev_qr_formq(H, n2, l, Qh, c.sm.la);
  dev_qr_extract_r(H, n2, l, Rb);
  for (int e = ltid(); e < rn * n2; e += NT) {
    int k = (int)(e % rn), cc = (int)(e / rn);
    A[e] = cconj(Qh[cc + (long long)n2 * k]);
  }
  cta_sync();
  cta_gemm(gemm_args(2 * lp, rn, l, Ap, 1, 2 * lp, Rb, rn, 1, H, 1, 2 * lp, false, true), c.sm.e.u.gw.g);
  cta_copy(Ap, H, (long long)2 * lp * rn);
  set_chi(c, s, i, rn);
}

static __device__ void shift_oc(Ctx& c, const DState& s, int nc) {
  int oc = *s.oc;
  cta_sync();
  if (oc == nc) return;
  if (nc > oc) {
    for (int i = oc; i < nc && !c.sm.fail; ++i) qr_right(c, s, i);
  } else {
    for (int i = oc; i > nc && !c.sm.fail; --i) lq_left(c, s, i);
  }
  cta_sync();
  if (ltid() == 0) *s.oc = nc;
  cta_sync();
}

static __device__ void normalize_state(Ctx& c, const DState& s) {
  for (int i = c.P.L - 1; i >= 1 && !c.sm.fail; --i) lq_left(c, s, i);
  cplx* A = site_ptr(c, s, 0);
  const long long n = (long long)s.chi[0] * 2 * s.chi[1];
  double nr = sqrt(cta_norm2(A, n, c.sm.e.r));
  if (nr > 1e-13) cta_scale(A, n, 1.0 / nr);
  cta_sync();
  if (ltid() == 0) *s.oc = 0;
  cta_sync();
}

// Scale the orthogonality-centre tensor to unit norm (normalize!, MPS.jl:274-311).
static __device__ void normalize_center(Ctx& c, const DState& s) {
  const int oc = *s.oc;
  cplx* A = site_ptr(c, s, oc);
  const long long n = (long long)s.chi[oc] * 2 * s.chi[oc + 1];
  double nr = sqrt(cta_norm2(A, n, c.sm.e.r));
  if (nr > 1e-13) cta_scale(A, n, 1.0 / nr);
  cta_sync();
}

// True when every bond satisfies chi[b] <= 2 chi[b-1] and chi[b] <= 2 chi[b+1]:
// then the thin QR / LQ factorisations of a gauge sweep keep every shape, so
// a sweep is a pure gauge move.  Uniform across the CTA.
static __device__ bool chain_tight(const Ctx& c, const DState& s) {
  bool ok = true;
  for (int b = 1; b < c.P.L; ++b) {
    const int x = s.chi[b];
    if (x > 2 * s.chi[b - 1] || x > 2 * s.chi[b + 1]) ok = false;
  }
  return ok;
}

// normalize! of a state in mixed canonical form around its centre: on a
// tight chain the full sweep only rescales the centre tensor; otherwise run
// the sweep.
static __device__ void finish_normalize(Ctx& c, const DState& s) {
  if (chain_tight(c, s))
    normalize_center(c, s);
  else
    normalize_state(c, s);
}

// Re <psi|psi> by full contraction (scalar_product, MPS.jl:528-585).
static __device__ double scalar_product(Ctx& c, const DState& s) {
  ProfScope prof_scope_(PF_SCALAR);
  cplx* Ea = c.ws + c.P.lay.tA;
  cplx* Eb = c.ws + c.P.lay.tB;
  cplx* T = c.ws + c.P.lay.tC;
  if (ltid() == 0) Ea[0] = make_double2(1.0, 0.0);
  cta_sync();
  for (int i = 0; i < c.P.L; ++i) {
    const int l = s.chi[i], r = s.chi[i + 1];
    const cplx* A = site_ptr(c, s, i);
    cta_gemm(gemm_args(l, 2 * r, l, Ea, l, 1, A, 1, l, T, 1, l), c.sm.e.u.gw.g);
    cta_gemm(gemm_args(r, r, 2 * l, T, 2 * l, 1, A, 1, 2 * l, Eb, 1, r, false, true), c.sm.e.u.gw.g);
    cplx* t = Ea;
    Ea = Eb;
    Eb = t;
  }
  double v = Ea[0].x;
  cta_sync();
  return v;
}

// ---------------------------------------------------------------------------
// Environments (Algorithms.jl:191-211)
// ---------------------------------------------------------------------------
static __device__ __forceinline__ cplx* envL(const Ctx& c, int b) { return c.ws + c.P.lay.EL + c.P.env_off[b]; }
static __device__ __forceinline__ cplx* envR(const Ctx& c, int b) { return c.ws + c.P.lay.ER + c.P.env_off[b]; }

static __device__ void identity_env(Ctx& c, cplx* E, int dim, int w) {
  for (int e = ltid(); e < dim * w * dim; e += NT) {
    long long a = e % dim, rest = e / dim;
    long long m = rest % w, k = rest / w;
    E[e] = make_double2((m == 0 && a == k) ? 1.0 : 0.0, 0.0);
  }
  cta_sync();
}

// EL[i+1] from EL[i], A_i and the map Wenv of W_i (update_left_environment)
static __device__ void update_left_w(Ctx& c, const DState& s, int i, const WMat& Wenv) {
  ProfScope prof_scope_(PF_ENV);
  const int l = s.chi[i], r = s.chi[i + 1], wl = c.P.w[i], wr = c.P.w[i + 1];
  const cplx* A = site_ptr(c, s, i);
  cplx* T1 = c.ws + c.P.lay.T1;
  cplx* T2 = c.ws + c.P.lay.T2;
  cflt* Af = reinterpret_cast<cflt*>(c.ws + c.P.lay.Af);
  cflt* Ef = reinterpret_cast<cflt*>(c.ws + c.P.lay.Lf);
  cflt* T1f = reinterpret_cast<cflt*>(c.ws + c.P.lay.T1f);
  cflt* T2f = reinterpret_cast<cflt*>(c.ws + c.P.lay.T2f);
  GemmSmemF& gf = reinterpret_cast<GemmSmemF&>(c.sm.e.u.gw.g);
  if (c.P.mixed) {
    cta_to_f32(Af, A, (long long)l * 2 * r);
    cta_to_f32(Ef, envL(c, i), (long long)l * wl * l);
    cta_gemm_tf32<cflt>(gemm_args_f(l * wl, 2 * r, l, Ef, 1, (long long)l * wl, Af, 1, l, T1f, 1, (long long)l * wl),
                        gf);
  } else {
    cta_gemm(gemm_args(l * wl, 2 * r, l, envL(c, i), 1, (long long)l * wl, A, 1, l, T1, 1, (long long)l * wl),
             c.sm.e.u.gw.g);
  }
  WApplyGeom g;
  g.n0 = l;
  g.n1 = r;
  g.is0 = 1;
  g.is1 = (long long)l * wl * 2;
  g.ni1 = wl;
  g.ii1 = l;
  g.ii2 = (long long)l * wl;
  g.os0 = 1;
  g.os1 = (long long)l * 2 * wr;
  g.no1 = 2;
  g.oo1 = l;
  g.oo2 = 2 * l;
  if (c.P.mixed) {
    dev_wapply<cflt>(T1f, T2f, Wenv, g, c.sm.e.u.gw.w);
    cta_gemm_tf32<cplx>(gemm_args_f(r, wr * r, 2 * l, Af, 2 * l, 1, T2f, 1, 2 * l, envL(c, i + 1), 1, r, true, false),
                        gf);
  } else {
    dev_wapply<cplx>(T1, T2, Wenv, g, c.sm.e.u.gw.w);
    cta_gemm(gemm_args(r, wr * r, 2 * l, A, 2 * l, 1, T2, 1, 2 * l, envL(c, i + 1), 1, r, true, false),
             c.sm.e.u.gw.g);
  }
}

static __device__ void update_left(Ctx& c, const DState& s, int i) { update_left_w(c, s, i, c.P.wm_envL[i]); }

// ER[i] from ER[i+1], A_i and the map Wenv of W_i (update_right_environment)
static __device__ void update_right_w(Ctx& c, const DState& s, int i, const WMat& Wenv) {
  ProfScope prof_scope_(PF_ENV);
  const int l = s.chi[i], r = s.chi[i + 1], wl = c.P.w[i], wr = c.P.w[i + 1];
  const cplx* A = site_ptr(c, s, i);
  cplx* T1 = c.ws + c.P.lay.T1;
  cplx* T2 = c.ws + c.P.lay.T2;
  cflt* Af = reinterpret_cast<cflt*>(c.ws + c.P.lay.Af);
  cflt* Ef = reinterpret_cast<cflt*>(c.ws + c.P.lay.Rf);
  cflt* T1f = reinterpret_cast<cflt*>(c.ws + c.P.lay.T1f);
  cflt* T2f = reinterpret_cast<cflt*>(c.ws + c.P.lay.T2f);
  GemmSmemF& gf = reinterpret_cast<GemmSmemF&>(c.sm.e.u.gw.g);
  if (c.P.mixed) {
    cta_to_f32(Af, A, (long long)l * 2 * r);
    cta_to_f32(Ef, envR(c, i + 1), (long long)r * wr * r);
    cta_gemm_tf32<cflt>(gemm_args_f(2 * l, r * wr, r, Af, 1, 2 * l, Ef, (long long)r * wr, 1, T1f, 1, 2 * l), gf);
  } else {
    cta_gemm(gemm_args(2 * l, r * wr, r, A, 1, 2 * l, envR(c, i + 1), (long long)r * wr, 1, T1, 1, 2 * l),
             c.sm.e.u.gw.g);
  }
  WApplyGeom g;
  g.n0 = l;
  g.n1 = r;
  g.is0 = 1;
  g.is1 = 2 * l;
  g.ni1 = 2;
  g.ii1 = l;
  g.ii2 = (long long)2 * l * r;
  g.os0 = (long long)2 * r * wl;
  g.os1 = 2;
  g.no1 = 2;
  g.oo1 = 1;
  g.oo2 = 2 * r;
  if (c.P.mixed) {
    dev_wapply<cflt>(T1f, T2f, Wenv, g, c.sm.e.u.gw.w);
    cta_gemm_tf32<cplx>(gemm_args_f(l, wl * l, 2 * r, Af, 1, l, T2f, 1, 2 * r, envR(c, i), 1, l, true, false), gf);
  } else {
    dev_wapply<cplx>(T1, T2, Wenv, g, c.sm.e.u.gw.w);
    cta_gemm(gemm_args(l, wl * l, 2 * r, A, 1, l, T2, 1, 2 * r, envR(c, i), 1, l, true, false), c.sm.e.u.gw.g);
  }
}

static __device__ void update_right(Ctx& c, const DState& s, int i) { update_right_w(c, s, i, c.P.wm_envR[i]); }

// ---------------------------------------------------------------------------
// Two-site TDVP (Algorithms.jl:580-760)
// ---------------------------------------------------------------------------
// Autotuned choice of the mixed H_eff products per shape bucket
// (tune_index): 0 = tcgen05 (128 x 64 tiles, TMA-fed), 1 = mma.sync 3xTF32
// (64 x 64 tiles).  Buckets: ceil(log2 chi_l), ceil(log2 chi_r) in 0..7 and
// D in {1, 2, 4}.
#define TUNE_ENTRIES (8 * 8 * 3)
__host__ __device__ __forceinline__ int tune_log2(int v) {
  int e = 0;
  while ((1 << e) < v && e < 7) ++e;
  return e;
}
__host__ __device__ __forceinline__ int tune_index(int chil, int D, int chir) {
  return (tune_log2(chil) * 8 + tune_log2(chir)) * 3 + (D == 1 ? 0 : D == 2 ? 1 : 2);
}

// The H_eff operator of a Krylov solve on (l, D, r) between environments bl
// and br, with its operands staged for the product form chosen for the
// bucket.  CTA-collective.
static __device__ HeffOp make_heff(Ctx& c, int l, int D, int r, int bl, int br, const WMat& W) {
  HeffOp h;
  h.L = envL(c, bl);
  h.R = envR(c, br);
  h.W = W;
  h.chil = l;
  h.D = D;
  h.chir = r;
  h.wl = c.P.w[bl];
  h.wr = c.P.w[br];
  h.T1 = c.ws + c.P.lay.T1;
  h.T2 = c.ws + c.P.lay.T2;
  h.mixed = c.P.mixed;
  const bool tc = c.P.tc && !(c.P.tune && c.P.tune[tune_index(l, D, r)] == 1);
  if (tc) {  // environments staged once per Krylov solve as the TMA operands
    const WsLayout& y = c.P.lay;
    h.tc = 1;
    h.maps = c.P.tmaps + 4 * c.slot;
    h.SL = reinterpret_cast<cflt*>(c.ws + y.sL);
    h.Sx = reinterpret_cast<cflt*>(c.ws + y.sx);
    h.ST2 = reinterpret_cast<cflt*>(c.ws + y.sT2);
    h.SR = reinterpret_cast<cflt*>(c.ws + y.sR);
    h.pL = y.pL;
    h.px = y.px;
    h.pT2 = y.pT2;
    h.pR = y.pR;
    h.T1f = reinterpret_cast<cflt*>(c.ws + y.T1f);
    const long long ml = (long long)l * h.wl;
    for (long long e = ltid(); e < ml * l; e += NT) {  // SL[k pL + i] = L[i + ml k]
      const cplx v = h.L[e];
      h.SL[(e / ml) * h.pL + e % ml] = make_float2((float)v.x, (float)v.y);
    }
    for (long long e = ltid(); e < (long long)r * h.wr * r; e += NT) {  // SR[k pR + b] = R[b + r k]
      const cplx v = h.R[e];
      h.SR[(e / r) * h.pR + e % r] = make_float2((float)v.x, (float)v.y);
    }
  } else if (c.P.mixed) {  // FP32 environments for the whole Krylov solve
    cflt* Lf = reinterpret_cast<cflt*>(c.ws + c.P.lay.Lf);
    cflt* Rf = reinterpret_cast<cflt*>(c.ws + c.P.lay.Rf);
    cta_to_f32(Lf, h.L, (long long)l * h.wl * l);
    cta_to_f32(Rf, h.R, (long long)r * h.wr * r);
    h.Lf = Lf;
    h.Rf = Rf;
    h.xf = reinterpret_cast<cflt*>(c.ws + c.P.lay.xf);
    h.T1f = reinterpret_cast<cflt*>(c.ws + c.P.lay.T1f);
    h.T2f = reinterpret_cast<cflt*>(c.ws + c.P.lay.T2f);
  }
  return h;
}

static __device__ void evolve(Ctx& c, cplx* x, int l, int D, int r, int bl, int br, const WMat& W, double dt) {
  const HeffOp h = make_heff(c, l, D, r, bl, br, W);
  int mv = dev_expm_krylov(h, x, dt, c.P.kc, c.ws + c.P.lay.Q, c.P.kry_n, c.sm.e);
  if (ltid() == 0) {
    c.cnt[0] += mv;
    c.cnt[1] += (mv > 0);
    *c.fl += mv * heff_flops(l, h.wl, D, r, h.wr);
  }
}

// Theta (l,4,r) of sites i,i+1 into buffer th.
static __device__ void merge(Ctx& c, const DState& s, int i, cplx* th) {
  const int l = s.chi[i], m = s.chi[i + 1], r = s.chi[i + 2];
  cta_gemm(gemm_args(2 * l, 2 * r, m, site_ptr(c, s, i), 1, 2 * l, site_ptr(c, s, i + 1), 1, m, th, 1, 2 * l),
           c.sm.e.u.gw.g);
}

static __device__ SvdWork svd_work(const Ctx& c) {
  SvdWork w;
  w.B = c.ws + c.P.lay.B;
  w.X = c.ws + c.P.lay.X;
  w.Yo = c.ws + c.P.lay.Yo;
  w.Zo = c.ws + c.P.lay.Zo;
  w.y = c.ws + c.P.lay.y;
  w.sig = reinterpret_cast<double*>(c.ws + c.P.lay.dbl);
  w.ord = c.wsi + c.P.lay.i_ord;
  return w;
}

// NaN/Inf -> 0 before the SVD (Algorithms.jl:414-417).
static __device__ void fix_nonfinite(Ctx& c, cplx* th, long long n) {
  int bad = 0;
  for (int e = ltid(); e < (int)n; e += NT) {
    cplx v = th[e];
    if (!isfinite(v.x) || !isfinite(v.y)) {
      th[e] = make_double2(0.0, 0.0);
      bad = 1;
    }
  }
  double b = block_sum((double)bad, c.sm.e.r);
  if (b > 0 && ltid() == 0) c.cnt[4] += 1;
}

// SVD split of theta (2l x 2r) into sites i (l,2,keep) and i+1 (keep,2,r).
// rule 0: TDVP (absolute, min 2); 1: relative; 2: TEBD.  With s_left the
// singular values go left (U S | Vt, Vt orthonormal, Algorithms.jl:701-708),
// otherwise right (U | S Vt, U orthonormal, Algorithms.jl:656-663).  The
// scaled factor is computed as a product with theta and is exactly zero for
// null singular values.
static __device__ void split(Ctx& c, const DState& s, int i, cplx* th, int l, int r, int rule, bool s_left) {
  const int m = 2 * l, n = 2 * r;
  fix_nonfinite(c, th, (long long)m * n);
  SvdWork w = svd_work(c);
  SvdResult res = dev_svd(th, m, n, s_left ? SVD_RIGHT : SVD_LEFT, w, c.sm.la, c.sm.e.r, c.sm.e.u.svd);
  if (ltid() == 0) {
    int keep = rule == 0   ? keep_tdvp(w.sig, res.p, c.P.thr, c.P.max_bond)
               : rule == 1 ? keep_relative(w.sig, res.p, c.P.thr, c.P.max_bond)
               : rule == 2 ? keep_tebd(w.sig, res.p, c.P.thr, c.P.max_bond)
                           : max(1, min(res.p, c.P.max_bond));  // dynamic TDVP split (tdvp.py:144-152)
    c.sm.bcast_i[0] = keep;
    c.cnt[2] += 1;
    c.cnt[5] += res.sweeps;
  }
  cta_sync();
  const int keep = c.sm.bcast_i[0];
  cta_sync();
  if (keep > c.P.cap[i + 1]) {
    if (ltid() == 0) c.sm.fail = ST_UNSUPPORTED;
    cta_sync();
    return;
  }
  dev_svd_vectors(res, keep, w, c.sm.e.r);
  cplx* Lt = site_ptr(c, s, i);
  cplx* Rt = site_ptr(c, s, i + 1);
  if (!s_left) {
    cta_copy(Lt, w.Yo, (long long)m * keep);
    cta_sync();
    cta_gemm(gemm_args(keep, n, m, w.Yo, m, 1, th, 1, m, Rt, 1, keep, true, false), c.sm.e.u.gw.g);
    for (int e = ltid(); e < keep * n; e += NT)
      if ((int)(e % keep) >= res.rank) Rt[e] = make_double2(0.0, 0.0);
  } else {
    for (int e = ltid(); e < keep * n; e += NT) {
      int k = (int)(e % keep), cc = (int)(e / keep);
      Rt[e] = cconj(w.Yo[cc + (long long)n * k]);
    }
    cta_gemm(gemm_args(m, keep, n, th, 1, m, w.Yo, 1, n, Lt, 1, m), c.sm.e.u.gw.g);
    for (int e = ltid(); e < m * keep; e += NT)
      if ((int)(e / m) >= res.rank) Lt[e] = make_double2(0.0, 0.0);
  }
  cta_sync();
  set_chi(c, s, i + 1, keep);
  if (ltid() == 0) *s.oc = s_left ? i : i + 1;  // the scaled factor holds the centre
  cta_sync();
}

// _init_envs (Algorithms.jl:802-819) after moving the centre to site 0.
static __device__ void init_envs(Ctx& c, const DState& s) {
  const int L = c.P.L;
  shift_oc(c, s, 0);
  identity_env(c, envR(c, L), s.chi[L], c.P.w[L]);
  for (int i = L - 1; i >= 1; --i) update_right(c, s, i);
  identity_env(c, envL(c, 0), s.chi[0], c.P.w[0]);
}

// exp(-i dtb H_bond) C on bond b (project_bond, Algorithms.jl:222-226), C (k x r).
static __device__ void evolve_bond(Ctx& c, cplx* C, int k, int r, int b, double dtb) {
  evolve(c, C, k, 1, r, b, b, c.P.wm_bond[b], dtb);
}

// Site i = Q R (thin QR): Q -> site i, EL[i+1] from it, R evolved by dtb on
// bond i+1 and absorbed into site i+1 (Algorithms.jl:491-505).
static __device__ void qr_bond_forward(Ctx& c, const DState& s, int i, double dtb) {
  const int l = s.chi[i], r = s.chi[i + 1], m = 2 * l, rn = min(m, r);
  const int r2 = s.chi[i + 2];
  cplx* A = site_ptr(c, s, i);
  cplx* An = site_ptr(c, s, i + 1);
  cplx* H = c.ws + c.P.lay.tA;
  cplx* Rb = c.ws + c.P.lay.tB;
  cplx* T = c.ws + c.P.lay.tC;
  cta_copy(H, A, (long long)m * r);
  cta_sync();
  dev_qr_factor(H, m, r, c.sm.la, c.sm.e.r);
  dev_qr_formq(H, m, r, A, c.sm.la);
  dev_qr_extract_r(H, m, r, Rb);
  set_chi(c, s, i + 1, rn);
  if (c.sm.fail) return;
  update_left(c, s, i);
  evolve_bond(c, Rb, rn, r, i + 1, dtb);
  cta_gemm(gemm_args(rn, 2 * r2, r, Rb, 1, rn, An, 1, r, T, 1, rn), c.sm.e.u.gw.g);
  cta_copy(An, T, (long long)rn * 2 * r2);
  cta_sync();
}

// Site i = L Q (thin LQ): Q -> site i, ER[i] from it, L evolved by dtb on
// bond i and absorbed into site i-1 (Algorithms.jl:515-529).
static __device__ void lq_bond_backward(Ctx& c, const DState& s, int i, double dtb) {
  const int l = s.chi[i], r = s.chi[i + 1], n2 = 2 * r, rn = min(l, n2);
  const int lp = s.chi[i - 1];
  cplx* A = site_ptr(c, s, i);
  cplx* Ap = site_ptr(c, s, i - 1);
  cplx* H = c.ws + c.P.lay.tA;
  cplx* Qh = c.ws + c.P.lay.tB;
  cplx* Rb = c.ws + c.P.lay.tC;
  for (int e = ltid(); e < n2 * l; e += NT) {
    int cc = (int)(e % n2), ii = (int)(e / n2);
    H[e] = cconj(A[ii + (long long)l * cc]);
  }
  cta_sync();
  dev_qr_factor(H, n2, l, c.sm.la, c.sm.e.r);
  dev_qr_formq(H, n2, l, Qh, c.sm.la);
  dev_qr_extract_r(H, n2, l, Rb);
  for (int e = ltid(); e < rn * n2; e += NT) {
    int k = (int)(e % rn), cc = (int)(e / rn);
    A[e] = cconj(Qh[cc + (long long)n2 * k]);
  }
  cplx* Lm = H;  // L = R^H (l x rn)
  for (int e = ltid(); e < l * rn; e += NT) {
    int a = (int)(e % l), k = (int)(e / l);
    Lm[e] = cconj(Rb[k + (long long)rn * a]);
  }
  set_chi(c, s, i, rn);
  if (c.sm.fail) return;
  update_right(c, s, i);
  evolve_bond(c, Lm, l, rn, i, dtb);
  cta_gemm(gemm_args(2 * lp, rn, l, Ap, 1, 2 * lp, Lm, 1, l, Rb, 1, 2 * lp), c.sm.e.u.gw.g);
  cta_copy(Ap, Rb, (long long)2 * lp * rn);
  cta_sync();
}

static __device__ void evolve_site1(Ctx& c, const DState& s, int i, double dts) {
  evolve(c, site_ptr(c, s, i), s.chi[i], 2, s.chi[i + 1], i, i + 1, c.P.wm_heff1[i], dts);
}

// _tdvp_sweep_hamiltonian_1site! (Algorithms.jl:472-533).
static __device__ void tdvp_sweep_1site(Ctx& c, const DState& s) {
  const int L = c.P.L;
  const double dt = c.P.dt;
  init_envs(c, s);
  for (int i = 0; i < L && !c.sm.fail; ++i) {
    evolve_site1(c, s, i, dt / 2);
    if (i < L - 1) qr_bond_forward(c, s, i, -dt / 2);
  }
  for (int i = L - 1; i >= 0 && !c.sm.fail; --i) {
    evolve_site1(c, s, i, dt / 2);
    if (i > 0) lq_bond_backward(c, s, i, -dt / 2);
  }
  cta_sync();
  if (ltid() == 0) *s.oc = 0;
  cta_sync();
}

// local_dynamic_tdvp (mqt-yaqs/src/mqt/yaqs/core/methods/tdvp.py:667-855):
// per bond a 2-site update while the bond is below max_bond_dim (split
// keeping min(rank, max_bond_dim) values), a 1-site update with bond
// back-evolution once it has reached it; once a 1-site step reaches the
// last bond the last site (first site on the way back) is updated alone.
static __device__ void tdvp_sweep_dynamic(Ctx& c, const DState& s) {
  const int L = c.P.L;
  const double dt = c.P.dt;
  cplx* th = c.ws + c.P.lay.th;
  init_envs(c, s);
  bool lock = false;
  for (int i = 0; i < L && !c.sm.fail; ++i) {
    if (s.chi[i + 1] >= c.P.max_bond || lock) {
      evolve_site1(c, s, i, dt / 2);
      if (i != L - 1) qr_bond_forward(c, s, i, -dt / 2);
      if (i == L - 2) lock = true;
    } else if (i == L - 1) {
      continue;
    } else {
      const int l = s.chi[i], r = s.chi[i + 2];
      merge(c, s, i, th);
      evolve(c, th, l, 4, r, i, i + 2, c.P.wm_heff2[i], dt / 2);
      split(c, s, i, th, l, r, 3, false);
      if (c.sm.fail) break;
      update_left(c, s, i);
      if (i != L - 2)
        evolve(c, site_ptr(c, s, i + 1), s.chi[i + 1], 2, r, i + 1, i + 2, c.P.wm_heff1[i + 1], -dt / 2);
    }
  }
  lock = false;
  for (int i = L - 1; i >= 0 && !c.sm.fail; --i) {
    if (s.chi[i] >= c.P.max_bond || lock) {
      evolve_site1(c, s, i, dt / 2);
      if (i != 0) {
        lq_bond_backward(c, s, i, -dt / 2);
        if (i == 1) lock = true;
      }
    } else if (i == 0) {
      continue;
    } else {
      const int l = s.chi[i - 1], r = s.chi[i + 1];
      merge(c, s, i - 1, th);
      evolve(c, th, l, 4, r, i - 1, i + 1, c.P.wm_heff2[i - 1], dt / 2);
      split(c, s, i - 1, th, l, r, 3, true);
      if (c.sm.fail) break;
      update_right(c, s, i);
      if (i != 1) evolve(c, site_ptr(c, s, i - 1), s.chi[i - 1], 2, s.chi[i], i - 1, i, c.P.wm_heff1[i - 1], -dt / 2);
    }
  }
  cta_sync();
  if (ltid() == 0) *s.oc = 0;
  cta_sync();
}

static __device__ void tdvp_sweep_2site(Ctx& c, const DState& s) {
  const int L = c.P.L;
  const double dt = c.P.dt;
  cplx* th = c.ws + c.P.lay.th;
  init_envs(c, s);
  // forward (Algorithms.jl:631-672)
  for (int i = 0; i <= L - 3 && !c.sm.fail; ++i) {
    const int l = s.chi[i], r = s.chi[i + 2];
    merge(c, s, i, th);
    evolve(c, th, l, 4, r, i, i + 2, c.P.wm_heff2[i], dt / 2);
    split(c, s, i, th, l, r, 0, false);
    if (c.sm.fail) break;
    update_left(c, s, i);
    evolve(c, site_ptr(c, s, i + 1), s.chi[i + 1], 2, r, i + 1, i + 2, c.P.wm_heff1[i + 1], -dt / 2);
  }
  // edge (Algorithms.jl:674-711) and backward (:713-760)
  for (int i = L - 2; i >= 0 && !c.sm.fail; --i) {
    const double dts = (i == L - 2) ? dt : dt / 2;
    if (i < L - 2)
      evolve(c, site_ptr(c, s, i + 1), s.chi[i + 1], 2, s.chi[i + 2], i + 1, i + 2, c.P.wm_heff1[i + 1], -dts);
    const int l = s.chi[i], r = s.chi[i + 2];
    merge(c, s, i, th);
    evolve(c, th, l, 4, r, i, i + 2, c.P.wm_heff2[i], dts);
    split(c, s, i, th, l, r, 0, true);
    if (c.sm.fail) break;
    update_right(c, s, i + 1);
  }
}

static __device__ void tdvp_sweep(Ctx& c, const DState& s) {
  ProfScope prof_scope_(PF_SWEEP);
  if (c.P.tdvp_mode == 1)
    tdvp_sweep_1site(c, s);
  else if (c.P.tdvp_mode == 2)
    tdvp_sweep_dynamic(c, s);
  else
    tdvp_sweep_2site(c, s);
}

// ---------------------------------------------------------------------------
// Local operators
// ---------------------------------------------------------------------------
// A[l,p,r] <- sum_k op[p,k] A[l,k,r] for a d x d op (d = 2 or 4), in place.
static __device__ void apply_local(cplx* A, int l, int d, int r, const cplx* op) {
  for (int e = ltid(); e < l * r; e += NT) {
    long long a = e % l, b = e / l;
    cplx v[4], o[4];
    for (int p = 0; p < d; ++p) v[p] = A[a + (long long)l * (p + (long long)d * b)];
    for (int p = 0; p < d; ++p) {
      cplx acc = make_double2(0.0, 0.0);
      for (int k = 0; k < d; ++k) cfma(acc, op[p + d * k], v[k]);
      o[p] = acc;
    }
    for (int p = 0; p < d; ++p) A[a + (long long)l * (p + (long long)d * b)] = o[p];
  }
  cta_sync();
}

// sum |op . A|^2 (or sum |A|^2 when op == nullptr), d = 2 or 4.
static __device__ double local_norm2(Ctx& c, const cplx* A, int l, int d, int r, const cplx* op) {
  double sacc = 0.0;
  for (int e = ltid(); e < l * r; e += NT) {
    long long a = e % l, b = e / l;
    cplx v[4];
    for (int p = 0; p < d; ++p) v[p] = A[a + (long long)l * (p + (long long)d * b)];
    for (int p = 0; p < d; ++p) {
      if (op) {
        cplx acc = make_double2(0.0, 0.0);
        for (int k = 0; k < d; ++k) cfma(acc, op[p + d * k], v[k]);
        sacc += cabs2(acc);
      } else {
        sacc += cabs2(v[p]);
      }
    }
  }
  return block_sum(sacc, c.sm.e.r);
}

// Re sum conj(A) (op A)
static __device__ double local_expect(Ctx& c, const cplx* A, int l, int d, int r, const cplx* op) {
  double sacc = 0.0;
  for (int e = ltid(); e < l * r; e += NT) {
    long long a = e % l, b = e / l;
    cplx v[4];
    for (int p = 0; p < d; ++p) v[p] = A[a + (long long)l * (p + (long long)d * b)];
    for (int p = 0; p < d; ++p) {
      cplx acc = make_double2(0.0, 0.0);
      for (int k = 0; k < d; ++k) cfma(acc, op[p + d * k], v[k]);
      sacc += v[p].x * acc.x + v[p].y * acc.y;
    }
  }
  return block_sum(sacc, c.sm.e.r);
}

// ---------------------------------------------------------------------------
// Dissipation (Dissipation.jl:37-159)
// ---------------------------------------------------------------------------
// Processes taken by a noise step: all of them (f1 < 0), or the local noise
// model of a gate on sites (f1, f2) (create_local_noise_model,
// DigitalTJM.jl:172-188): 1-site processes on either site and 2-site
// processes on exactly that pair.
static __device__ __forceinline__ bool proc_on(const DevProc& pr, int f1, int f2) {
  if (f1 < 0) return true;
  return pr.nsites == 1 ? (pr.s0 == f1 || pr.s0 == f2) : ((pr.s0 == f1 && pr.s1 == f2) || (pr.s0 == f2 && pr.s1 == f1));
}

static __device__ void apply_dissipation(Ctx& c, const DState& s, bool full, double dt, int f1 = -1, int f2 = -1) {
  ProfScope prof_scope_(PF_DISS);
  const int L = c.P.L;
  bool all_zero = c.P.all_zero != 0;
  if (f1 >= 0) {
    all_zero = true;
    for (int k = 0; k < c.P.nprocs; ++k)
      if (proc_on(c.P.procs[k], f1, f2) && c.P.procs[k].gamma != 0.0) all_zero = false;
  }
  // Every dissipator a scalar (Pauli names, Dissipation.jl:14-21, 57-60, 88-91)
  // on a tight chain: the sweep only multiplies the state by their product
  // and moves the centre to site 0 by shape-preserving gauge steps.
  bool scalar_only = true;
  double fscal = 1.0;
  for (int k = 0; k < c.P.nprocs; ++k) {
    const DevProc& pr = c.P.procs[k];
    if (!proc_on(pr, f1, f2)) continue;
    if (!pr.pauli_name) scalar_only = false;
    fscal *= exp(-0.5 * dt * pr.drate);
  }
  if ((!c.P.noise_present || all_zero || scalar_only) && chain_tight(c, s)) {
    shift_oc(c, s, 0);
    if (c.P.noise_present && !all_zero) {
      cplx* A = site_ptr(c, s, 0);
      cta_scale(A, (long long)s.chi[0] * 2 * s.chi[1], fscal);
      cta_sync();
    }
    if (ltid() == 0) c.sm.canon = 1;
    cta_sync();
    return;
  }
  // The reference sweep applies its first dissipators to site L while the
  // centre sits elsewhere, so the chain is not canonical afterwards.
  if (ltid() == 0) c.sm.canon = 0;
  cta_sync();
  if (!c.P.noise_present || all_zero) {
    for (int i = L - 1; i >= 1 && !c.sm.fail; --i) shift_oc(c, s, i - 1);
    return;
  }
  cplx* th = c.ws + c.P.lay.th;
  for (int i = L - 1; i >= 0 && !c.sm.fail; --i) {
    for (int k = 0; k < c.P.nprocs; ++k) {
      const DevProc& pr = c.P.procs[k];
      if (pr.nsites == 1 && pr.s0 == i && proc_on(pr, f1, f2)) {
        cplx* A = site_ptr(c, s, i);
        const long long n = (long long)s.chi[i] * 2 * s.chi[i + 1];
        if (pr.pauli_name) {
          cta_scale(A, n, exp(-0.5 * dt * pr.gamma));
          cta_sync();
        } else {
          apply_local(A, s.chi[i], 2, s.chi[i + 1], full ? pr.diss_full : pr.diss_half);
        }
      }
    }
    if (i > 0) {
      for (int k = 0; k < c.P.nprocs && !c.sm.fail; ++k) {
        const DevProc& pr = c.P.procs[k];
        if (pr.nsites == 2 && pr.s1 == i && proc_on(pr, f1, f2)) {
          if (pr.pauli_name) {  // Pauli names and long-range processes: a scalar at the right site
            cta_scale(site_ptr(c, s, i), (long long)s.chi[i] * 2 * s.chi[i + 1], exp(-0.5 * dt * pr.drate));
            cta_sync();
          } else {
            const int l = s.chi[i - 1], r = s.chi[i + 1];
            merge(c, s, i - 1, th);
            apply_local(th, l, 4, r, full ? pr.diss_full : pr.diss_half);
            split(c, s, i - 1, th, l, r, 1, false);
          }
        }
      }
      shift_oc(c, s, i - 1);
    }
  }
}

#include "longrange.cuh"

// ---------------------------------------------------------------------------
// Stochastic process (StochasticProcess.jl:219-330)
// ---------------------------------------------------------------------------
static __device__ void stochastic_process(Ctx& c, const DState& s, double dt, int f1 = -1, int f2 = -1) {
  ProfScope prof_scope_(PF_STOCH);
  const int L = c.P.L;
  const double dp = 1.0 - scalar_product(c, s);
  bool jump = false;
  int ntake = 0;
  for (int k = 0; k < c.P.nprocs; ++k) ntake += proc_on(c.P.procs[k], f1, f2) ? 1 : 0;
  if (ntake > 0) {
    double u1 = draw_uniform(c);
    jump = u1 < dp;
  }
  if (!jump) {
    if (c.sm.canon)
      finish_normalize(c, s);
    else
      normalize_state(c, s);
    return;
  }
  double* cand = reinterpret_cast<double*>(c.ws + c.P.lay.dbl) + SVD_MAX_COLS;
  int* candp = c.wsi + c.P.lay.i_cand;
  int nc = 0;
  cplx* th = c.ws + c.P.lay.th;
  for (int site = 0; site < L && !c.sm.fail; ++site) {
    shift_oc(c, s, site);
    for (int k = 0; k < c.P.nprocs; ++k) {
      const DevProc& pr = c.P.procs[k];
      if (pr.nsites == 1 && pr.s0 == site && proc_on(pr, f1, f2)) {
        double nr = local_norm2(c, site_ptr(c, s, site), s.chi[site], 2, s.chi[site + 1],
                                pr.pauli_proc ? nullptr : pr.mat);
        if (ltid() == 0) {
          cand[nc] = dt * pr.gamma * nr;
          candp[nc] = k;
        }
        ++nc;
      }
    }
    if (site < L - 1) {
      for (int k = 0; k < c.P.nprocs; ++k) {
        const DevProc& pr = c.P.procs[k];
        if (pr.nsites == 2 && !pr.lr && pr.s0 == site && proc_on(pr, f1, f2)) {
          double nr;
          if (pr.pauli_proc) {
            nr = local_norm2(c, site_ptr(c, s, site), s.chi[site], 2, s.chi[site + 1], nullptr);
          } else {
            merge(c, s, site, th);
            nr = local_norm2(c, th, s.chi[site], 4, s.chi[site + 2], pr.mat);
          }
          if (ltid() == 0) {
            cand[nc] = dt * pr.gamma * nr;
            candp[nc] = k;
          }
          ++nc;
        }
      }
    }
  }
  // long-range processes after every local candidate (StochasticProcess.jl:169-202);
  // the centre is at site L-1
  for (int k = 0; k < c.P.nprocs && !c.sm.fail; ++k) {
    const DevProc& pr = c.P.procs[k];
    if (!pr.lr || !proc_on(pr, f1, f2)) continue;
    const double nr = pr.pauli_proc ? local_norm2(c, site_ptr(c, s, L - 1), s.chi[L - 1], 2, s.chi[L], nullptr)
                                    : lr_weight(c, s, pr);
    if (ltid() == 0) {
      cand[nc] = dt * pr.gamma * nr;
      candp[nc] = k;
    }
    ++nc;
  }
  cta_sync();
  double total = 0.0;
  for (int e = 0; e < nc; ++e) total += cand[e];
  if (total == 0.0) {
    finish_normalize(c, s);  // the candidate scan moved the centre through every site
    return;
  }
  const double r = draw_uniform(c);
  double acc = 0.0;
  int chosen = 0;
  for (int e = 0; e < nc; ++e) {
    acc += cand[e] / total;
    if (r <= acc) {
      chosen = e;
      break;
    }
  }
  const DevProc& pr = c.P.procs[candp[chosen]];
  cta_sync();
  if (pr.lr) {
    // "pauli_long_range" has no branch of its own in the reference
    // (StochasticProcess.jl:311 tests "mpo_pauli"): only the normalisation acts
    if (!pr.pauli_proc) lr_apply(c, s, pr);
  } else if (pr.nsites == 1) {
    shift_oc(c, s, pr.s0);
    apply_local(site_ptr(c, s, pr.s0), s.chi[pr.s0], 2, s.chi[pr.s0 + 1], pr.mat);
  } else {
    shift_oc(c, s, pr.s0);
    const int l = s.chi[pr.s0], rr = s.chi[pr.s0 + 2];
    merge(c, s, pr.s0, th);
    apply_local(th, l, 4, rr, pr.mat);
    split(c, s, pr.s0, th, l, rr, 1, false);
  }
  if (ltid() == 0) c.cnt[3] += 1;
  finish_normalize(c, s);
}

// ---------------------------------------------------------------------------
// Observables
// ---------------------------------------------------------------------------
// Re sum_{a,p,q,b} conj(A[a,p,b]) op[p,q] T[a,q,b] for two (l, 2, r) tensors.
// CTA-collective.
static __device__ double env_expect(Ctx& c, const cplx* A, const cplx* T, int l, int r, const cplx* op) {
  double sacc = 0.0;
  for (int e = ltid(); e < l * r; e += NT) {
    const long long a = e % l, b = e / l;
    const cplx a0 = A[a + (long long)l * (2 * b)], a1 = A[a + (long long)l * (1 + 2 * b)];
    const cplx t0 = T[a + (long long)l * (2 * b)], t1 = T[a + (long long)l * (1 + 2 * b)];
    cplx u0 = make_double2(0.0, 0.0), u1 = make_double2(0.0, 0.0);
    cfma(u0, op[0], t0);
    cfma(u0, op[2], t1);
    cfma(u1, op[1], t0);
    cfma(u1, op[3], t1);
    sacc += a0.x * u0.x + a0.y * u0.y + a1.x * u1.x + a1.y * u1.y;
  }
  return block_sum(sacc, c.sm.e.r);
}

// The 1-site observables of a state whose bonds are all tight.  The
// reference (expect -> local_expect, MPS.jl:608-651) moves the orthogonality
// centre to each observable's site and contracts the centre tensor; on a
// tight chain those QR / LQ steps change no shape and are pure gauge moves.
// Here the state is left as it is and each <O_i> is contracted with transfer
// matrices, which holds in any gauge:
//   R_L = 1,  R_b = sum_p A_b^p R_{b+1} A_b^p^dag          (right to left)
//   E_0 = 1,  <O_i> = sum E_i[a,a'] A_i[a,q,r] O[p,q] conj(A_i[a',p,r']) R_{i+1}[r,r'],
//   E_{i+1} = sum_p A_i^p^T E_i conj(A_i^p)                (left to right)
// six small GEMMs a site instead of a QR step a site in each direction.  The
// right environments go in the slot's environment arena (free between
// sweeps) or else in the SVD scratch (B, X, Yo, Zo, adjacent); returns false,
// having written nothing, when no observable is 1-site, the chain is not
// tight, or neither region holds them.  CTA-collective.
static __device__ bool local_by_envs(Ctx& c, const DState& s, int col) {
  const DevParams& P = c.P;
  const int L = P.L;
  bool any1 = false;
  for (int k = 0; k < P.nobs; ++k) any1 |= P.obs[k].kind == OBS_LOCAL1;
  if (!any1 || !chain_tight(c, s)) return false;
  long long need = 0;
  for (int b = 1; b <= L; ++b) need += (long long)s.chi[b] * s.chi[b];
  cplx* Rs;
  if (P.lay.ER - P.lay.EL >= need)
    Rs = c.ws + P.lay.EL;  // R_b at offset sum_{b' > b} chi_b'^2
  else if (P.lay.Zo + (P.lay.Zo - P.lay.Yo) - P.lay.B >= need)
    Rs = c.ws + P.lay.B;
  else
    return false;
  cplx* E0 = c.ws + P.lay.tA;
  cplx* E1 = c.ws + P.lay.tB;
  cplx* T1 = c.ws + P.lay.tC;
  cplx* T3 = c.ws + P.lay.th;
  GemmSmem& gs = c.sm.e.u.gw.g;
  cta_sync();
  if (ltid() == 0) {
    Rs[0] = make_double2(1.0, 0.0);  // R_L (chi_L = 1)
    E0[0] = make_double2(1.0, 0.0);  // E_0 (chi_0 = 1)
  }
  cta_sync();
  long long off = 0;  // offset of R_{b+1}
  for (int b = L - 1; b >= 1; --b) {
    const int l = s.chi[b], r = s.chi[b + 1];
    const cplx* A = site_ptr(c, s, b);
    // X[(a,p), r'] = sum_r A[a,p,r] R_{b+1}[r, r']
    cta_gemm(gemm_args(2 * l, r, r, A, 1, 2 * l, Rs + off, 1, r, T1, 1, 2 * l), gs);
    off += (long long)r * r;
    // R_b[x, y] = sum_{p,r'} X[x,p,r'] conj(A[y,p,r'])
    cta_gemm(gemm_args(l, l, 2 * r, T1, 1, l, A, l, 1, Rs + off, 1, l, false, true), gs);
  }
  double* vals = reinterpret_cast<double*>(c.ws + P.lay.dbl) + SVD_MAX_COLS;  // one value per observable
  off = need;  // R_{i+1} at off - chi_{i+1}^2
  for (int i = 0; i < L; ++i) {
    const int l = s.chi[i], r = s.chi[i + 1];
    const cplx* A = site_ptr(c, s, i);
    off -= (long long)r * r;
    bool here = false;
    for (int k = 0; k < P.nobs; ++k) here |= P.obs[k].kind == OBS_LOCAL1 && P.obs[k].s0 == i;
    if (here) {
      // T1[a,q,r'] = sum_r A[a,q,r] R_{i+1}[r,r'];  T3[a',q,r'] = sum_a E_i[a,a'] T1[a,q,r']
      cta_gemm(gemm_args(2 * l, r, r, A, 1, 2 * l, Rs + off, 1, r, T1, 1, 2 * l), gs);
      cta_gemm(gemm_args(l, 2 * r, l, E0, l, 1, T1, 1, l, T3, 1, l), gs);
      for (int k = 0; k < P.nobs; ++k) {
        if (P.obs[k].kind != OBS_LOCAL1 || P.obs[k].s0 != i) continue;
        const double v = env_expect(c, A, T3, l, r, P.obs[k].mat);
        if (ltid() == 0) vals[k] = v;
      }
    }
    if (i + 1 < L) {
      // V[a',p,r] = sum_a E_i[a,a'] A[a,p,r];  E_{i+1}[r,r'] = sum_{a',p} V[a',p,r] conj(A[a',p,r'])
      cta_gemm(gemm_args(l, 2 * r, l, E0, l, 1, A, 1, l, T1, 1, l), gs);
      cta_gemm(gemm_args(r, r, 2 * l, T1, 2 * l, 1, A, 1, 2 * l, E1, 1, r, false, true), gs);
      cplx* t = E0;
      E0 = E1;
      E1 = t;
    }
  }
  cta_sync();
  if (ltid() == 0)
    for (int k = 0; k < P.nobs; ++k)
      if (P.obs[k].kind == OBS_LOCAL1) P.traj_out[((long long)c.traj * P.nobs + k) * P.ncols + col] = vals[k];
  cta_sync();
  return true;
}

static __device__ void evaluate(Ctx& c, const DState& s, int col) {
  ProfScope prof_scope_(PF_EVAL);
  const int ncols = c.P.ncols;
  const bool local_done = local_by_envs(c, s, col);
  for (int k = 0; k < c.P.nobs && !c.sm.fail; ++k) {
    const DevObs& o = c.P.obs[k];
    if (local_done && o.kind == OBS_LOCAL1) continue;
    double val = 0.0;
    if (o.kind == OBS_LOCAL1) {
      shift_oc(c, s, o.s0);
      val = local_expect(c, site_ptr(c, s, o.s0), s.chi[o.s0], 2, s.chi[o.s0 + 1], o.mat);
    } else if (o.kind == OBS_LOCAL2) {
      shift_oc(c, s, o.s0);
      cplx* th = c.ws + c.P.lay.th;
      merge(c, s, o.s0, th);
      val = local_expect(c, th, s.chi[o.s0], 4, s.chi[o.s0 + 2], o.mat);
    } else {
      shift_oc(c, s, o.s0);
      const int l = s.chi[o.s0], r = s.chi[o.s0 + 1];
      SvdWork w = svd_work(c);
      SvdResult res = dev_svd(site_ptr(c, s, o.s0), 2 * l, r, SVD_LEFT, w, c.sm.la, c.sm.e.r, c.sm.e.u.svd);
      if (ltid() == 0) {
        double nsq = 0.0;
        for (int e = 0; e < res.p; ++e) nsq += w.sig[e] * w.sig[e];
        double ent = 0.0;
        for (int e = 0; e < res.p; ++e) {
          double p = w.sig[e] * w.sig[e] / nsq;
          if (p > 0.0) ent -= p * log(p);
        }
        c.sm.bcast_d[1] = ent;
      }
      cta_sync();
      val = c.sm.bcast_d[1];
      cta_sync();
    }
    if (ltid() == 0) c.P.traj_out[((long long)c.traj * c.P.nobs + k) * ncols + col] = val;
  }
  if (ltid() == 0) {
    int mx = 0;
    for (int b = 0; b <= c.P.L; ++b) mx = max(mx, s.chi[b]);
    if (c.P.chi_out) c.P.chi_out[(long long)c.traj * ncols + col] = mx;
  }
  cta_sync();
}
