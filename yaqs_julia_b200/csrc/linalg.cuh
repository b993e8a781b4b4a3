// linalg.cuh — CTA-level Householder QR/LQ and one-sided Jacobi SVD (FP64).
//
// Restates the LAPACK factorizations the reference calls through Julia's
// LinearAlgebra (Decompositions.jl:18-73, MPS.jl:182-311 for QR/LQ;
// Algorithms.jl:420, Dissipation.jl:281, StochasticProcess.jl:280 for SVD).
// The conventions (zlarfg reflectors with real R diagonal; round-robin
// Jacobi pair order; stable descending sort; deterministic completion of
// null singular vectors) are identical to the CPU oracle so both produce the
// same gauge up to rounding.
#pragma once
#include "common.cuh"

#define QR_NULL_TOL 1e-14
#define SVD_NULL_TOL 1e-14
#define JACOBI_MAX_SWEEPS 60
#define SVD_MAX_COLS 256

struct LinalgSmem {
  cplx tau[SVD_MAX_COLS];
  int rot_count;
  int flag;
};

// ---------------------------------------------------------------------------
// Householder QR
// ---------------------------------------------------------------------------
// Factor H (m x n, col-major, ld m) in place: R in the upper triangle,
// reflector vectors below, scalars in ls.tau.  CTA-collective.
__device__ __noinline__ void dev_qr_factor(cplx* H, int m, int n, LinalgSmem& ls, RedScratch& rs) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int kq = min(m, n);
  double fro2 = cta_norm2(H, (long long)m * n, rs);
  const double null_abs = QR_NULL_TOL * sqrt(fro2);
  for (int j = 0; j < kq; ++j) {
    cplx* col = H + (long long)m * j;
    double s = 0.0;
    for (int i = j + 1 + tid; i < m; i += NT) s += cabs2(col[i]);
    const double xn2 = block_sum(s, rs);
    const cplx alpha = col[j];
    const double full = sqrt(cabs2(alpha) + xn2);
    __syncthreads();
    if (full <= null_abs || (xn2 == 0.0 && alpha.y == 0.0)) {
      for (int i = j + 1 + tid; i < m; i += NT) col[i] = make_double2(0.0, 0.0);
      if (tid == 0) ls.tau[j] = make_double2(0.0, 0.0);
      __syncthreads();
      continue;
    }
    const double beta = (alpha.x >= 0.0) ? -full : full;
    const cplx t = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
    const cplx amb = make_double2(alpha.x - beta, alpha.y);
    const double d = cabs2(amb);
    const cplx scale = make_double2(amb.x / d, -amb.y / d);
    for (int i = j + 1 + tid; i < m; i += NT) col[i] = cmul(col[i], scale);
    __syncthreads();
    if (tid == 0) {
      col[j] = make_double2(beta, 0.0);
      ls.tau[j] = t;
    }
    const cplx ct = cconj(t);
    for (int c = j + 1 + wid; c < n; c += NW) {
      cplx* x = H + (long long)m * c;
      cplx acc = make_double2(0.0, 0.0);
      if (lane == 0) acc = x[j];
      for (int i = j + 1 + lane; i < m; i += 32) cfmac(acc, col[i], x[i]);
      acc.x = warp_sum(acc.x);
      acc.y = warp_sum(acc.y);
      acc = cmul(acc, ct);
      for (int i = j + 1 + lane; i < m; i += 32) x[i] = csub(x[i], cmul(acc, col[i]));
      if (lane == 0) x[j] = csub(x[j], acc);
    }
    __syncthreads();
  }
}

// Q (m x kq) of a factored H.  CTA-collective.
__device__ __noinline__ void dev_qr_formq(const cplx* H, int m, int n, cplx* Q, LinalgSmem& ls) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int kq = min(m, n);
  for (long long e = tid; e < (long long)m * kq; e += NT) {
    int r = (int)(e % m), c = (int)(e / m);
    Q[e] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  for (int j = kq - 1; j >= 0; --j) {
    const cplx t = ls.tau[j];
    if (t.x == 0.0 && t.y == 0.0) continue;
    const cplx* v = H + (long long)m * j;
    for (int c = j + wid; c < kq; c += NW) {
      cplx* q = Q + (long long)m * c;
      cplx acc = make_double2(0.0, 0.0);
      if (lane == 0) acc = q[j];
      for (int i = j + 1 + lane; i < m; i += 32) cfmac(acc, v[i], q[i]);
      acc.x = warp_sum(acc.x);
      acc.y = warp_sum(acc.y);
      acc = cmul(acc, t);
      for (int i = j + 1 + lane; i < m; i += 32) q[i] = csub(q[i], cmul(acc, v[i]));
      if (lane == 0) q[j] = csub(q[j], acc);
    }
    __syncthreads();
  }
}

// R (kq x n) of a factored H into Rout (ld kq), zero below the diagonal.
__device__ __forceinline__ void dev_qr_extract_r(const cplx* H, int m, int n, cplx* Rout) {
  const int kq = min(m, n);
  for (long long e = threadIdx.x; e < (long long)kq * n; e += NT) {
    int r = (int)(e % kq), c = (int)(e / kq);
    Rout[e] = (r <= c) ? H[r + (long long)m * c] : make_double2(0.0, 0.0);
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// One-sided Jacobi SVD
// ---------------------------------------------------------------------------
struct SvdWork {
  cplx* B;      // q x p
  cplx* X;      // p x p
  cplx* Yo;     // q x p (sorted, normalised left vectors of B)
  cplx* Zo;     // p x p (sorted right vectors)
  cplx* y;      // q (completion scratch)
  double* sig;  // p
  int* ord;     // p
};

struct SvdResult {
  bool tr;
  int q, p, rank;  // rank = number of non-null singular values
};

// Orthonormal completion of column k of Y (rows x *) against columns 0..k-1.
__device__ void dev_complete_column(cplx* Y, int rows, int k, cplx* y, RedScratch& rs) {
  for (int c = 0; c < rows; ++c) {
    // pass 1: y = e_c - sum_h conj(Y_h[c]) Y_h
    for (int i = threadIdx.x; i < rows; i += NT) {
      cplx v = make_double2(i == c ? 1.0 : 0.0, 0.0);
      for (int h = 0; h < k; ++h) {
        cplx yc = Y[c + (long long)rows * h];
        cplx yi = Y[i + (long long)rows * h];
        v = csub(v, cmulc(yc, yi));
      }
      y[i] = v;
    }
    __syncthreads();
    // pass 2: y -= sum_h (Y_h^H y) Y_h, dot products in chunks of 8
    for (int h0 = 0; h0 < k; h0 += 8) {
      double d[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) d[e] = 0.0;
      for (int i = threadIdx.x; i < rows; i += NT) {
        cplx yi = y[i];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          if (h0 + e < k) {
            cplx a = Y[i + (long long)rows * (h0 + e)];
            cplx p = cmulc(a, yi);
            d[2 * e] += p.x;
            d[2 * e + 1] += p.y;
          }
        }
      }
      block_sum_n<16>(d, rs);
      for (int i = threadIdx.x; i < rows; i += NT) {
        cplx v = y[i];
#pragma unroll
        for (int e = 0; e < 8; ++e)
          if (h0 + e < k) v = csub(v, cmul(make_double2(d[2 * e], d[2 * e + 1]), Y[i + (long long)rows * (h0 + e)]));
        y[i] = v;
      }
      __syncthreads();
    }
    double nr = sqrt(cta_norm2(y, rows, rs));
    if (nr > 0.5) {
      for (int i = threadIdx.x; i < rows; i += NT) Y[i + (long long)rows * k] = cscale(y[i], 1.0 / nr);
      __syncthreads();
      return;
    }
  }
}

// SVD of M (m x n, col-major ld m), phase 1: Jacobi sweeps, sorting and
// the sorted singular values in w.sig (null values set to 0).
// CTA-collective.  Returns metadata (uniform in all threads).
__device__ __noinline__ SvdResult dev_svd(const cplx* M, int m, int n, SvdWork& w, LinalgSmem& ls, RedScratch& rs) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  SvdResult res;
  res.tr = m < n;
  const int q = res.tr ? n : m;
  const int p = res.tr ? m : n;
  res.q = q;
  res.p = p;
  for (long long e = tid; e < (long long)q * p; e += NT) {
    int r = (int)(e % q), c = (int)(e / q);
    w.B[e] = res.tr ? cconj(M[c + (long long)m * r]) : M[e];
  }
  for (long long e = tid; e < (long long)p * p; e += NT) {
    int r = (int)(e % p), c = (int)(e / p);
    w.X[e] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  const double tol = 2.220446049250313e-16 * q;
  const int pe = p + (p & 1);
  for (int sweep = 0; sweep < JACOBI_MAX_SWEEPS && pe > 1; ++sweep) {
    if (tid == 0) ls.rot_count = 0;
    __syncthreads();
    for (int round = 0; round < pe - 1; ++round) {
      for (int pr = wid; pr < pe / 2; pr += NW) {
        int ta = pr, tb = pe - 1 - pr;
        int a = ta == 0 ? 0 : ((ta - 1 - round + 2 * (pe - 1)) % (pe - 1)) + 1;
        int b = tb == 0 ? 0 : ((tb - 1 - round + 2 * (pe - 1)) % (pe - 1)) + 1;
        int i = min(a, b), j = max(a, b);
        if (j >= p) continue;
        cplx* bi = w.B + (long long)q * i;
        cplx* bj = w.B + (long long)q * j;
        double al = 0.0, be = 0.0, gx = 0.0, gy = 0.0;
        for (int r = lane; r < q; r += 32) {
          cplx x = bi[r], y = bj[r];
          al += cabs2(x);
          be += cabs2(y);
          gx += x.x * y.x + x.y * y.y;
          gy += x.x * y.y - x.y * y.x;
        }
        al = warp_sum(al);
        be = warp_sum(be);
        gx = warp_sum(gx);
        gy = warp_sum(gy);
        double ag = sqrt(gx * gx + gy * gy);
        if (!(ag > tol * sqrt(al * be))) continue;
        if (lane == 0) atomicAdd(&ls.rot_count, 1);
        double zeta = (be - al) / (2.0 * ag);
        double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        double c = 1.0 / sqrt(1.0 + t * t);
        double s = c * t;
        cplx e = make_double2(gx / ag, gy / ag);
        cplx se = cscale(e, s), sec = cscale(cconj(e), s);
        for (int r = lane; r < q; r += 32) {
          cplx x = bi[r], y = bj[r];
          bi[r] = csub(cscale(x, c), cmul(sec, y));
          bj[r] = cadd(cmul(se, x), cscale(y, c));
        }
        cplx* xi = w.X + (long long)p * i;
        cplx* xj = w.X + (long long)p * j;
        for (int r = lane; r < p; r += 32) {
          cplx x = xi[r], y = xj[r];
          xi[r] = csub(cscale(x, c), cmul(sec, y));
          xj[r] = cadd(cmul(se, x), cscale(y, c));
        }
      }
      __syncthreads();
    }
    int rc = ls.rot_count;
    __syncthreads();
    if (rc == 0) break;
  }
  // singular values
  for (int c = wid; c < p; c += NW) {
    const cplx* bc = w.B + (long long)q * c;
    double s = 0.0;
    for (int r = lane; r < q; r += 32) s += cabs2(bc[r]);
    s = warp_sum(s);
    if (lane == 0) w.sig[c] = sqrt(s);
  }
  __syncthreads();
  // stable descending order
  for (int c = tid; c < p; c += NT) {
    double sc = w.sig[c];
    int rank = 0;
    for (int c2 = 0; c2 < p; ++c2) {
      double s2 = w.sig[c2];
      if (s2 > sc || (s2 == sc && c2 < c)) ++rank;
    }
    w.ord[rank] = c;
  }
  __syncthreads();
  const double smax = p > 0 ? w.sig[w.ord[0]] : 0.0;
  // rank of non-null values (sorted prefix)
  int cnt = 0;
  for (int k = tid; k < p; k += NT) {
    double s = w.sig[w.ord[k]];
    if (smax > 0.0 && s > SVD_NULL_TOL * smax) ++cnt;
  }
  res.rank = (int)block_sum((double)cnt, rs);
  // sorted singular values into sig (nulls zeroed)
  double sk = 0.0;
  int myk = tid;
  if (myk < p) {
    double s = w.sig[w.ord[myk]];
    sk = (smax > 0.0 && s > SVD_NULL_TOL * smax) ? s : 0.0;
  }
  __syncthreads();
  if (myk < p) w.sig[myk] = sk;
  __syncthreads();
  return res;
}

// Phase 2: sorted left/right vectors Yo (q x need), Zo (p x need):
// Yo = B[:,ord[k]]/sigma_k, Zo = X[:,ord[k]] for non-null k, orthonormal
// completions for null k < need.  CTA-collective.
__device__ __noinline__ void dev_svd_vectors(const SvdResult& res, int need, SvdWork& w, RedScratch& rs) {
  const int tid = threadIdx.x, q = res.q, p = res.p;
  need = min(need, p);
  const int ng = min(need, res.rank);
  for (long long e = tid; e < (long long)q * ng; e += NT) {
    int r = (int)(e % q), k = (int)(e / q);
    w.Yo[e] = cscale(w.B[r + (long long)q * w.ord[k]], 1.0 / w.sig[k]);
  }
  for (long long e = tid; e < (long long)p * ng; e += NT) {
    int r = (int)(e % p), k = (int)(e / p);
    w.Zo[e] = w.X[r + (long long)p * w.ord[k]];
  }
  __syncthreads();
  for (int k = res.rank; k < need; ++k) {
    dev_complete_column(w.Yo, q, k, w.y, rs);
    dev_complete_column(w.Zo, p, k, w.y, rs);
  }
}

// Truncation ranks (see the oracle for the reference lines they restate).
// split_mps_tensor_svd / two_site_svd: absolute, keep crossing value, min 2.
__device__ __forceinline__ int keep_tdvp(const double* S, int n, double thr, int max_bond) {
  double disc = 0.0;
  int keep = n;
  for (int k = n; k >= 1; --k) {
    disc += S[k - 1] * S[k - 1];
    if (disc >= thr) {
      keep = max(k, 2);
      break;
    }
  }
  return max(1, min(keep, max_bond));
}
// Dissipation / jump split: relative, min 1.
__device__ __forceinline__ int keep_relative(const double* S, int n, double thr, int max_bond) {
  double nsq = 0.0;
  for (int k = 0; k < n; ++k) nsq += S[k] * S[k];
  double cur = 0.0;
  int rank = n;
  for (int k = n; k >= 1; --k) {
    cur += S[k - 1] * S[k - 1];
    if (cur > thr * nsq) {
      rank = k;
      break;
    }
  }
  return max(1, min(rank, max_bond));
}

// Write the truncated factors of an SVD: U (m x keep, ld m) and
// Vt (keep x n, ld keep).  scaleU / scaleV multiply the columns of U or
// the rows of Vt by S.  CTA-collective.
__device__ __forceinline__ void dev_svd_write(const SvdResult& r, const SvdWork& w, int m, int n, int keep,
                                              cplx* U, bool scaleU, cplx* Vt, bool scaleV) {
  for (long long e = threadIdx.x; e < (long long)m * keep; e += NT) {
    int i = (int)(e % m), k = (int)(e / m);
    cplx v = r.tr ? w.Zo[i + (long long)r.p * k] : w.Yo[i + (long long)r.q * k];
    if (scaleU) v = cscale(v, w.sig[k]);
    U[e] = v;
  }
  for (long long e = threadIdx.x; e < (long long)keep * n; e += NT) {
    int k = (int)(e % keep), c = (int)(e / keep);
    cplx v = r.tr ? cconj(w.Yo[c + (long long)r.q * k]) : cconj(w.Zo[c + (long long)r.p * k]);
    if (scaleV) v = cscale(v, w.sig[k]);
    Vt[e] = v;
  }
  __syncthreads();
}
