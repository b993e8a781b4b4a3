// krylov.cuh — effective-Hamiltonian product and Lanczos exponential.
//
// dev_heff restates project_site (Algorithms.jl:215-220, :330-361):
//   T1[a,m,p,c]   = sum_k L[a,m,k] x[k,p,c]                    (GEMM)
//   T2[a,p',m',c] = sum_{m,p} W[m,p',p,m'] T1[a,m,p,c]         (sparse MPO apply)
//   y[a,p',b]     = sum_{m',c} T2[a,p',m',c] R[b,m',c]         (GEMM)
// dev_expm_krylov restates expm_krylov (Algorithms.jl:144-187) / KrylovKit
// exponentiate: Lanczos with classical Gram-Schmidt against the whole basis,
// refined by a second pass when the first kept less than 1/sqrt(2) of the
// norm (DGKS), stopping at krylov_dim, at breakdown (beta <= |dt| tol), or
// once prod(beta_i |dt|)/k! <= exit_tol; the small tridiagonal exponential
// is taken on one warp by Taylor series over substeps of norm <= 1/2.
#pragma once
#include "common.cuh"
#include "gemm_tf32.cuh"
#include "tcgemm.cuh"

#define WAPPLY_IN_CPLX 2560  // staged inputs: ni x PT values, PT = 256, 128 or 64 by what fits
#define WAPPLY_MAXI 32
#define WAPPLY_MAXNNZ 512
#define WAPPLY_LB 8  // inputs a thread loads back to back
#define KRYLOV_MAX 32

// Sparse MPO matrix M[o, i] in CSR form (rows are outputs).
struct WMat {
  int no, ni, nnz;
  int ident;  // identity map with a physical dimension of 1 (bond): T2 is T1
  const int* rowp;  // no+1
  const int* col;   // nnz
  const cplx* val;  // nnz
};

struct WApplyGeom {
  int n0, n1;
  long long is0, is1, ii1, ii2;
  int ni1;
  long long os0, os1, oo1, oo2;
  int no1;
};

struct WApplySmem {
  cplx in[WAPPLY_IN_CPLX];
  cplx val[WAPPLY_MAXNNZ];
  int col[WAPPLY_MAXNNZ];
  int rowp[WAPPLY_MAXI + 1];
  int in_off[WAPPLY_MAXI];
  int out_off[WAPPLY_MAXI];
};

// out[q0,q1,o] = sum_i M[o,i] in[q0,q1,i].  CTA-collective.  A tile holds PT
// pairs (the largest of 256, 128, 64 whose ni inputs fit the staging
// buffer); each thread owns pair slot tid % PT of every tile and
// input/output rows tid / PT + k NT / PT, so index arithmetic is per tile,
// not per element, and with PT = NT a thread issues all ni loads of its pair
// back to back.  T is cplx (FP64 form) or float2 (mixed form, FP32 products).
// in and out may be the same buffer when every pair's inputs and outputs
// occupy the same addresses (a tile reads all its inputs before it writes).
static __device__ __forceinline__ void wfma(cplx& acc, cplx v, cplx x) { cfma(acc, v, x); }
static __device__ __forceinline__ void wfma(float2& acc, cplx v, float2 x) {
  const float vr = (float)v.x, vi = (float)v.y;
  acc.x = fmaf(vr, x.x, fmaf(-vi, x.y, acc.x));
  acc.y = fmaf(vr, x.y, fmaf(vi, x.x, acc.y));
}
static __device__ __forceinline__ void wzero(cplx& z) { z = make_double2(0.0, 0.0); }
static __device__ __forceinline__ void wzero(float2& z) { z = make_float2(0.f, 0.f); }

template <class T>
static __device__ __noinline__ void dev_wapply(const T* in, T* out, const WMat W,
                                        const WApplyGeom g, WApplySmem& ws) {
  ProfScope prof_scope_(PF_WAPPLY);
  T* sin = reinterpret_cast<T*>(&ws.in[0]);
  const int cap = (int)(WAPPLY_IN_CPLX * sizeof(cplx) / sizeof(T));
  const int PT = W.ni * NT <= cap ? NT : (W.ni * (NT / 2) <= cap ? NT / 2 : NT / 4);
  const int tid = ltid();
  for (int e = tid; e < W.nnz; e += NT) {
    ws.val[e] = W.val[e];
    ws.col[e] = W.col[e];
  }
  for (int e = tid; e <= W.no; e += NT) ws.rowp[e] = W.rowp[e];
  for (int i = tid; i < W.ni; i += NT) ws.in_off[i] = (int)((i % g.ni1) * g.ii1 + (i / g.ni1) * g.ii2);
  for (int o = tid; o < W.no; o += NT) ws.out_off[o] = (int)((o % g.no1) * g.oo1 + (o / g.no1) * g.oo2);
  const int npair = g.n0 * g.n1;
  const int pl = tid % PT, r0 = tid / PT;
  const int RS = NT / PT;
  T zero;
  wzero(zero);
  for (int base = 0; base < npair; base += PT) {
    const int pair = base + pl;
    const bool live = pair < npair;
    const int q0 = live ? pair % g.n0 : 0, q1 = live ? pair / g.n0 : 0;
    const long long ib = q0 * g.is0 + q1 * g.is1, ob = q0 * g.os0 + q1 * g.os1;
    cta_sync();
    // batches of WAPPLY_LB loads issued before their stores: `in` may alias
    // the staging buffer as far as the compiler knows, so a plain loop would
    // wait out one L2 latency per input
    for (int i0 = r0; i0 < W.ni; i0 += RS * WAPPLY_LB) {
      T v[WAPPLY_LB];
#pragma unroll
      for (int k = 0; k < WAPPLY_LB; ++k) {
        const int i = i0 + k * RS;
        v[k] = (live && i < W.ni) ? in[ib + ws.in_off[i]] : zero;
      }
#pragma unroll
      for (int k = 0; k < WAPPLY_LB; ++k) {
        const int i = i0 + k * RS;
        if (i < W.ni) sin[i * PT + pl] = v[k];
      }
    }
    cta_sync();
    if (live) {
      for (int o = r0; o < W.no; o += RS) {
        T acc = zero;
        for (int z = ws.rowp[o]; z < ws.rowp[o + 1]; ++z) wfma(acc, ws.val[z], sin[ws.col[z] * PT + pl]);
        out[ob + ws.out_off[o]] = acc;
      }
    }
  }
  cta_sync();
}

struct HeffOp {
  const cplx* L;  // (chil, wl, chil)
  const cplx* R;  // (chir, wr, chir)
  WMat W;         // rows p'+D m', cols m + wl p
  int chil, D, chir, wl, wr;
  cplx* T1;
  cplx* T2;
  // mixed form: FP32 copies of the environments and FP32 intermediates
  int mixed = 0;
  const cflt* Lf = nullptr;
  const cflt* Rf = nullptr;
  cflt* xf = nullptr;
  cflt* T1f = nullptr;
  cflt* T2f = nullptr;
  // mixed form on tcgen05 (tc = 1): TMA-staged operands of the two products,
  // tensor maps maps[0..3] = SL (A, MN-major), Sx (B, K-major), ST2 (A,
  // MN-major), SR (B, MN-major); pitches in complex FP32 values
  int tc = 0;
  const CUtensorMap* maps = nullptr;
  cflt* SL = nullptr;
  cflt* Sx = nullptr;
  cflt* ST2 = nullptr;
  cflt* SR = nullptr;
  int pL = 0, px = 0, pT2 = 0, pR = 0;
};

struct KrySmem {
  double alpha[KRYLOV_MAX + 1];
  double beta[KRYLOV_MAX + 1];
  cplx h[KRYLOV_MAX + 1];
  cplx y[KRYLOV_MAX + 1];
  int m;
};

// Shared memory of one CTA.  The GEMM / MPO-apply staging and the SVD block
// buffer are never live at the same time and share storage.
#define SVD_SMEM_CPLX_K 4096
union EngineSmemU {
  union {  // the GEMM and the MPO apply run one after the other, never together
    GemmSmem g;
    WApplySmem w;
  } gw;
  cplx svd[SVD_SMEM_CPLX_K];
  TcSmem t;  // the tensor-core pipeline (mixed form), no larger than the GEMM staging
};
struct EngineSmem {
  RedScratch r;
  KrySmem k;
  TcState tc;
  EngineSmemU u;
};
#if !YAQS_TC
static_assert(sizeof(TcSmem) <= sizeof(GemmSmem), "the default pipeline must not grow the CTA's shared memory");
#endif

#if YAQS_TC
// Mixed form on tcgen05 (compiled only into the tensor-core kernel,
// engine_tc.cu: a kernel that contains tcgen05 code is given one CTA per
// SM).  x is staged as the K-major B operand of the first product, the MPO
// apply writes T2 straight into the MN-major A operand of the second
// product, and both products run in tc_gemm; the environments were staged
// once per Krylov solve.
static __device__ void dev_heff_tc(const HeffOp& h, const cplx* x, cplx* y, EngineSmem& sm) {
  const int chil = h.chil, D = h.D, chir = h.chir, wl = h.wl, wr = h.wr;
  const long long n = (long long)chil * D * chir;
  // Sx[nn px + k] = x[k + chil nn], 8 loads in flight per thread
  for (long long e0 = ltid(); e0 < n; e0 += 8 * NT) {
    cplx v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = e0 + u * NT < n ? x[e0 + u * NT] : make_double2(0.0, 0.0);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const long long e = e0 + u * NT;
      if (e < n) h.Sx[(e / chil) * h.px + e % chil] = make_float2((float)v[u].x, (float)v[u].y);
    }
  }
  const TcOp A1{h.maps + 0, 1, 0}, B1{h.maps + 1, 0, 0}, A2{h.maps + 2, 1, 0}, B2{h.maps + 3, 1, 0};
  tc_gemm<cflt>(chil * wl, D * chir, chil, A1, B1, h.T1f, 1, (long long)chil * wl, false, sm.u.t, sm.tc);
  if (h.W.ident) {  // bond (D = 1, wl = wr): T2 is T1 re-laid into ST2
    const long long nt1 = (long long)chil * wl * chir;
    for (long long e0 = ltid(); e0 < nt1; e0 += 8 * NT) {
      cflt v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = e0 + u * NT < nt1 ? h.T1f[e0 + u * NT] : make_float2(0.f, 0.f);
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const long long e = e0 + u * NT;
        if (e >= nt1) continue;
        const long long a = e % chil, m = (e / chil) % wl, c = e / ((long long)chil * wl);
        h.ST2[(m + (long long)wr * c) * h.pT2 + a] = v[u];
      }
    }
  } else {
    WApplyGeom g;
    g.n0 = chil;
    g.n1 = chir;
    g.is0 = 1;
    g.is1 = (long long)chil * wl * D;
    g.ni1 = wl;
    g.ii1 = chil;
    g.ii2 = (long long)chil * wl;
    g.os0 = 1;                      // a
    g.os1 = (long long)h.pT2 * wr;  // c: rows m' + wr c of ST2
    g.no1 = D;
    g.oo1 = chil;   // p'
    g.oo2 = h.pT2;  // m'
    dev_wapply<cflt>(h.T1f, h.ST2, h.W, g, sm.u.gw.w);
  }
  tc_gemm<cplx>(chil * D, chir, wr * chir, A2, B2, y, 1, (long long)chil * D, false, sm.u.t, sm.tc);
}
#endif

// y = H_eff x.  CTA-collective.  In the mixed form x is rounded to FP32, the
// three contractions run in FP32 (tensor cores for the two GEMMs) and y is
// written back in FP64.
static __device__ __noinline__ void dev_heff(const HeffOp& h, const cplx* x, cplx* y, EngineSmem& sm) {
  const int chil = h.chil, D = h.D, chir = h.chir, wl = h.wl, wr = h.wr;
#if YAQS_TC
  if (h.tc) {
    dev_heff_tc(h, x, y, sm);
    return;
  }
#endif
  if (h.mixed) {
    GemmSmemF& gf = reinterpret_cast<GemmSmemF&>(sm.u.gw.g);
    cta_to_f32(h.xf, x, (long long)chil * D * chir);
    cta_gemm_tf32<cflt>(gemm_args_f(chil * wl, D * chir, chil, h.Lf, 1, (long long)chil * wl, h.xf, 1, chil, h.T1f,
                                    1, (long long)chil * wl),
                        gf);
  } else {
    cta_gemm(gemm_args(chil * wl, D * chir, chil, h.L, 1, (long long)chil * wl, x, 1, chil, h.T1, 1,
                       (long long)chil * wl),
             sm.u.gw.g);
  }
  WApplyGeom g;
  g.n0 = chil;
  g.n1 = chir;
  g.is0 = 1;
  g.is1 = (long long)chil * wl * D;
  g.ni1 = wl;
  g.ii1 = chil;
  g.ii2 = (long long)chil * wl;
  g.os0 = 1;
  g.os1 = (long long)chil * D * wr;
  g.no1 = D;
  g.oo1 = chil;
  g.oo2 = (long long)chil * D;
  // an identity W with D = 1 (the bond operator) leaves T1 in T2's layout.
  // With wl == wr the pair (a, b) holds its wl*D inputs and its wr*D outputs
  // at the same addresses (a + chil * j within the block of b), so the MPO
  // apply runs in place: T2's stores land on the lines T1 just left in L2
  // and one buffer per slot is written back instead of two.
  const bool inplace = wl == wr;
  if (h.mixed) {
    GemmSmemF& gf = reinterpret_cast<GemmSmemF&>(sm.u.gw.g);
    const cflt* T2 = h.T1f;
    if (!h.W.ident) {
      dev_wapply<cflt>(h.T1f, inplace ? h.T1f : h.T2f, h.W, g, sm.u.gw.w);
      T2 = inplace ? h.T1f : h.T2f;
    }
    cta_gemm_tf32<cplx>(gemm_args_f(chil * D, chir, wr * chir, T2, 1, (long long)chil * D, h.Rf, chir, 1, y, 1,
                                    (long long)chil * D),
                        gf);
  } else {
    const cplx* T2 = h.T1;
    if (!h.W.ident) {
      dev_wapply<cplx>(h.T1, inplace ? h.T1 : h.T2, h.W, g, sm.u.gw.w);
      T2 = inplace ? h.T1 : h.T2;
    }
    cta_gemm(gemm_args(chil * D, chir, wr * chir, T2, 1, (long long)chil * D, h.R, chir, 1, y, 1,
                       (long long)chil * D),
             sm.u.gw.g);
  }
}

static __device__ __forceinline__ double heff_flops(int chil, int wl, int D, int chir, int wr) {
  return 8.0 * ((double)chil * chil * wl * D * chir + (double)chil * chir * D * D * wl * wr +
                (double)chil * D * chir * chir * wr);
}

struct KrylovCfg {
  int kdim;
  double tol;
  double exit_tol;
};

// Warp 0: y = exp(-i dt T) e_1 for the m x m Lanczos matrix in ks.
static __device__ void dev_tridiag_expm(int m, double dt, KrySmem& ks) {
  ProfScope prof_scope_(PF_TRIDIAG);
  if (ltid() >= 32) return;
  const int j = ltid();
  const bool on = j < m;
  const double a = on ? ks.alpha[j] : 0.0;
  const double bl = (on && j > 0) ? ks.beta[j - 1] : 0.0;
  const double br = (on && j + 1 < m) ? ks.beta[j] : 0.0;
  double rowsum = on ? fabs(a) + bl + br : 0.0;
  const double tn = warp_max(rowsum) * fabs(dt);
  int ns = (int)ceil(tn / 0.5);
  if (ns < 1) ns = 1;
  const double h = dt / ns;
  cplx v = make_double2(j == 0 ? 1.0 : 0.0, 0.0);
  for (int s = 0; s < ns; ++s) {
    cplx term = v, acc = v;
    for (int n = 1; n < 60; ++n) {
      // term <- (-i h T) term / n
      cplx tl = make_double2(__shfl_up_sync(0xffffffffu, term.x, 1), __shfl_up_sync(0xffffffffu, term.y, 1));
      cplx tr = make_double2(__shfl_down_sync(0xffffffffu, term.x, 1), __shfl_down_sync(0xffffffffu, term.y, 1));
      cplx tt = make_double2(a * term.x + bl * tl.x + br * tr.x, a * term.y + bl * tl.y + br * tr.y);
      if (!on) tt = make_double2(0.0, 0.0);
      // multiply by -i h / n:  (x + i y) * (-i c) = c y - i c x
      const double c = h / n;
      term = make_double2(c * tt.y, -c * tt.x);
      acc = cadd(acc, term);
      double tnorm = warp_sum(cabs2(term));
      if (tnorm < 1e-40) break;
    }
    v = acc;
  }
  if (on) ks.y[j] = v;
}

// h_j = <q_j, w> (j < k) into ks.h and |w|^2 in the same pass over w: the
// first group takes seven vectors and the norm, later groups eight.  Each
// thread takes two elements per iteration so that up to 18 independent
// loads are in flight (the pass is bound by memory latency).
static __device__ double lanczos_dots(const cplx* Q, long long qs, const cplx* w, long long n, int k, EngineSmem& sm) {
  const int tid = ltid();
  double nw2 = 0.0;
  for (int j0 = 0, first = 1; j0 < k || first; first = 0) {
    const int G = first ? 7 : 8;
    double d[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) d[e] = 0.0;
    for (long long i0 = tid; i0 < n; i0 += 2 * NT) {
      const long long i1 = i0 + NT;
      const bool two = i1 < n;
      const cplx w0 = w[i0];
      const cplx w1 = two ? w[i1] : make_double2(0.0, 0.0);
      cplx a0[8], a1[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const bool live = e < G && j0 + e < k;
        a0[e] = live ? Q[qs * (j0 + e) + i0] : make_double2(0.0, 0.0);
        a1[e] = (live && two) ? Q[qs * (j0 + e) + i1] : make_double2(0.0, 0.0);
      }
      if (first) d[15] += cabs2(w0) + cabs2(w1);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        if (e == 7 && first) continue;
        const cplx p = cadd(cmulc(a0[e], w0), cmulc(a1[e], w1));
        d[2 * e] += p.x;
        d[2 * e + 1] += p.y;
      }
    }
    block_sum_n<16>(d, sm.r);
    if (tid < G && j0 + tid < k) sm.k.h[j0 + tid] = make_double2(d[2 * tid], d[2 * tid + 1]);
    if (first) nw2 = d[15];
    j0 += G;
  }
  cta_sync();
  return nw2;
}

// out_i = s (w_i - sum_{j<k} c_j q_j[i]) for i < n (w null: w_i = 0; out may
// be w), c in shared memory; returns the CTA sum of |out_i|^2 when norm.
// Basis vectors go in groups of eight, two elements per thread, so the loads
// of a group are in flight together.  CTA-collective.
static __device__ double basis_combine(const cplx* Q, long long qs, const cplx* w, cplx* out, long long n, int k,
                                       const cplx* c, double s, bool norm, EngineSmem& sm) {
  double part = 0.0;
  for (long long i0 = ltid(); i0 < n; i0 += 2 * NT) {
    const long long i1 = i0 + NT;
    const bool two = i1 < n;
    cplx v0 = w ? w[i0] : make_double2(0.0, 0.0);
    cplx v1 = (w && two) ? w[i1] : make_double2(0.0, 0.0);
    for (int j0 = 0; j0 < k; j0 += 8) {
      cplx a0[8], a1[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const bool live = j0 + e < k;
        a0[e] = live ? Q[qs * (j0 + e) + i0] : make_double2(0.0, 0.0);
        a1[e] = (live && two) ? Q[qs * (j0 + e) + i1] : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        if (j0 + e < k) {
          const cplx ce = c[j0 + e];
          v0 = csub(v0, cmul(ce, a0[e]));
          v1 = csub(v1, cmul(ce, a1[e]));
        }
      }
    }
    v0 = cscale(v0, s);
    v1 = cscale(v1, s);
    out[i0] = v0;
    if (two) out[i1] = v1;
    part += cabs2(v0) + cabs2(v1);
  }
  if (!norm) {
    cta_sync();
    return 0.0;
  }
  return block_sum(part, sm.r);
}

// w <- w - sum_j h_j q_j (j < k); with norm, returns |w|^2 after the update.
static __device__ double lanczos_subtract(const cplx* Q, long long qs, cplx* w, long long n, int k, EngineSmem& sm,
                                          bool norm) {
  return basis_combine(Q, qs, w, w, n, k, sm.k.h, 1.0, norm, sm);
}

// In place: x <- exp(-i dt H_eff) x.  Q holds kdim+1 vectors of stride qs.
// Returns the number of H_eff products.  CTA-collective.
static __device__ __noinline__ int dev_expm_krylov(const HeffOp& h, cplx* x, double dt, const KrylovCfg& kc, cplx* Q,
                                            long long qs, EngineSmem& sm) {
  const int tid = ltid();
  const long long n = (long long)h.chil * h.D * h.chir;
  const double beta0 = sqrt(cta_norm2(x, n, sm.r));
  if (beta0 == 0.0) return 0;
  const double tau = fabs(dt);
  for (long long i = tid; i < n; i += NT) Q[i] = cscale(x[i], 1.0 / beta0);
  cta_sync();
  double bound = 1.0;
  int m = 0;
  int mv = 0;
  for (int k = 1; k <= kc.kdim; ++k) {
    cplx* w = Q + qs * k;
    dev_heff(h, Q + qs * (k - 1), w, sm);
    ++mv;
    ProfScope orth_scope_(PF_ORTH);
    // classical Gram-Schmidt.  One pass gives h_j = <q_j, w> and |w|^2; when
    // the projection keeps at least 1/sqrt(2) of the norm (DGKS criterion,
    // |w - Q h|^2 = |w|^2 - |h|^2 >= |w|^2 / 2) the residual norm follows from
    // Pythagoras and one more pass forms q_k = (w - Q h) / b_k; otherwise a
    // refinement pass projects again and the norm is taken directly.
    const double nw2 = lanczos_dots(Q, qs, w, n, k, sm);
    double hh = 0.0;
    for (int j = 0; j < k; ++j) hh += cabs2(sm.k.h[j]);
    double a_k = sm.k.h[k - 1].x;
    const double r2 = nw2 - hh;
    const bool accept = r2 >= 0.5 * nw2;
    double b_k;
    if (accept) {
      b_k = sqrt(r2);
    } else {
      lanczos_subtract(Q, qs, w, n, k, sm, false);
      lanczos_dots(Q, qs, w, n, k, sm);
      a_k += sm.k.h[k - 1].x;
      b_k = sqrt(lanczos_subtract(Q, qs, w, n, k, sm, true));
    }
    if (tid == 0) sm.k.alpha[k - 1] = a_k;
    m = k;
    if (b_k <= tau * kc.tol) break;
    if (k == kc.kdim) break;
    bound *= b_k * tau / k;
    if (kc.exit_tol > 0.0 && bound <= kc.exit_tol) break;
    if (tid == 0) sm.k.beta[k - 1] = b_k;
    const double inv = 1.0 / b_k;
    if (accept) {
      basis_combine(Q, qs, w, w, n, k, sm.k.h, inv, false, sm);
    } else {
      for (long long i = tid; i < n; i += NT) w[i] = cscale(w[i], inv);
      cta_sync();
    }
  }
  cta_sync();
  dev_tridiag_expm(m, dt, sm.k);
  cta_sync();
  if (tid < m) sm.k.h[tid] = make_double2(-sm.k.y[tid].x, -sm.k.y[tid].y);  // x = beta0 sum_j y_j q_j
  cta_sync();
  basis_combine(Q, qs, nullptr, x, n, m, sm.k.h, beta0, false, sm);
  return mv;
}
