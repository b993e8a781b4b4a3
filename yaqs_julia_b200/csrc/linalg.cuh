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
#define QR_REG_ROWS 4  // Householder rows per lane kept in registers (m - j - 1 <= 128)
// The register-held reflector pays off from about this many rows; smaller
// factorisations (the short bonds of a growing chain) keep the plain column
// loop, which measured 10 % faster on the digital workload.
#define QR_REG_MIN_ROWS 48

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
static __device__ __noinline__ void dev_qr_factor(cplx* H, int m, int n, LinalgSmem& ls, RedScratch& rs) {
  ProfScope prof_scope_(PF_QR);
  const int tid = ltid(), lane = tid & 31, wid = tid >> 5;
  const int kq = min(m, n);
  double fro2 = cta_norm2(H, (long long)m * n, rs);
  const double null_abs = QR_NULL_TOL * sqrt(fro2);
  for (int j = 0; j < kq; ++j) {
    cplx* col = H + (long long)m * j;
    double s = 0.0;
    for (int i = j + 1 + tid; i < m; i += NT) s += cabs2(col[i]);
    const double xn2 = block_sum(s, rs);
    // col[j] is rewritten (by thread 0) only after the barrier that follows
    // the scaling below, so no barrier is needed between this read and it
    const cplx alpha = col[j];
    const double full = sqrt(cabs2(alpha) + xn2);
    if (full <= null_abs || (xn2 == 0.0 && alpha.y == 0.0)) {
      for (int i = j + 1 + tid; i < m; i += NT) col[i] = make_double2(0.0, 0.0);
      if (tid == 0) ls.tau[j] = make_double2(0.0, 0.0);
      cta_sync();
      continue;
    }
    const double beta = (alpha.x >= 0.0) ? -full : full;
    const cplx t = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
    const cplx amb = make_double2(alpha.x - beta, alpha.y);
    const double d = cabs2(amb);
    const cplx scale = make_double2(amb.x / d, -amb.y / d);
    for (int i = j + 1 + tid; i < m; i += NT) col[i] = cmul(col[i], scale);
    cta_sync();
    if (tid == 0) {
      col[j] = make_double2(beta, 0.0);
      ls.tau[j] = t;
    }
    const cplx ct = cconj(t);
    if (m >= QR_REG_MIN_ROWS && m <= 32 * QR_REG_ROWS + 1) {
      // reflector rows held in registers; two trailing columns per warp pass
      cplx v[QR_REG_ROWS];
#pragma unroll
      for (int q = 0; q < QR_REG_ROWS; ++q) {
        const int i = j + 1 + lane + 32 * q;
        v[q] = i < m ? col[i] : make_double2(0.0, 0.0);
      }
      for (int c0 = j + 1 + wid; c0 < n; c0 += 2 * NW) {
        const int c1 = c0 + NW;
        const bool two = c1 < n;
        cplx* x0 = H + (long long)m * c0;
        cplx* x1 = H + (long long)m * (two ? c1 : c0);
        cplx a0 = make_double2(0.0, 0.0), a1 = make_double2(0.0, 0.0);
        if (lane == 0) {
          a0 = x0[j];
          a1 = x1[j];
        }
        cplx y0[QR_REG_ROWS], y1[QR_REG_ROWS];
#pragma unroll
        for (int q = 0; q < QR_REG_ROWS; ++q) {
          const int i = j + 1 + lane + 32 * q;
          y0[q] = i < m ? x0[i] : make_double2(0.0, 0.0);
          y1[q] = i < m ? x1[i] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int q = 0; q < QR_REG_ROWS; ++q) {
          cfmac(a0, v[q], y0[q]);
          cfmac(a1, v[q], y1[q]);
        }
        a0.x = warp_sum(a0.x);
        a0.y = warp_sum(a0.y);
        a1.x = warp_sum(a1.x);
        a1.y = warp_sum(a1.y);
        a0 = cmul(a0, ct);
        a1 = cmul(a1, ct);
#pragma unroll
        for (int q = 0; q < QR_REG_ROWS; ++q) {
          const int i = j + 1 + lane + 32 * q;
          if (i < m) {
            x0[i] = csub(y0[q], cmul(a0, v[q]));
            if (two) x1[i] = csub(y1[q], cmul(a1, v[q]));
          }
        }
        if (lane == 0) {
          x0[j] = csub(x0[j], a0);
          if (two) x1[j] = csub(x1[j], a1);
        }
      }
    } else {
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
    }
    cta_sync();
  }
}

// Q (m x kq) of a factored H.  CTA-collective.
static __device__ __noinline__ void dev_qr_formq(const cplx* H, int m, int n, cplx* Q, LinalgSmem& ls) {
  ProfScope prof_scope_(PF_QRQ);
  const int tid = ltid(), lane = tid & 31, wid = tid >> 5;
  const int kq = min(m, n);
  for (int e = tid; e < m * kq; e += NT) {
    int r = (int)(e % m), c = (int)(e / m);
    Q[e] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  cta_sync();
  for (int j = kq - 1; j >= 0; --j) {
    const cplx t = ls.tau[j];
    if (t.x == 0.0 && t.y == 0.0) continue;
    const cplx* v = H + (long long)m * j;
    if (m >= QR_REG_MIN_ROWS && m <= 32 * QR_REG_ROWS + 1) {
      cplx vr[QR_REG_ROWS];
#pragma unroll
      for (int qq = 0; qq < QR_REG_ROWS; ++qq) {
        const int i = j + 1 + lane + 32 * qq;
        vr[qq] = i < m ? v[i] : make_double2(0.0, 0.0);
      }
      for (int c0 = j + wid; c0 < kq; c0 += 2 * NW) {
        const int c1 = c0 + NW;
        const bool two = c1 < kq;
        cplx* q0 = Q + (long long)m * c0;
        cplx* q1 = Q + (long long)m * (two ? c1 : c0);
        cplx a0 = make_double2(0.0, 0.0), a1 = make_double2(0.0, 0.0);
        if (lane == 0) {
          a0 = q0[j];
          a1 = q1[j];
        }
        cplx y0[QR_REG_ROWS], y1[QR_REG_ROWS];
#pragma unroll
        for (int qq = 0; qq < QR_REG_ROWS; ++qq) {
          const int i = j + 1 + lane + 32 * qq;
          y0[qq] = i < m ? q0[i] : make_double2(0.0, 0.0);
          y1[qq] = i < m ? q1[i] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int qq = 0; qq < QR_REG_ROWS; ++qq) {
          cfmac(a0, vr[qq], y0[qq]);
          cfmac(a1, vr[qq], y1[qq]);
        }
        a0.x = warp_sum(a0.x);
        a0.y = warp_sum(a0.y);
        a1.x = warp_sum(a1.x);
        a1.y = warp_sum(a1.y);
        a0 = cmul(a0, t);
        a1 = cmul(a1, t);
#pragma unroll
        for (int qq = 0; qq < QR_REG_ROWS; ++qq) {
          const int i = j + 1 + lane + 32 * qq;
          if (i < m) {
            q0[i] = csub(y0[qq], cmul(a0, vr[qq]));
            if (two) q1[i] = csub(y1[qq], cmul(a1, vr[qq]));
          }
        }
        if (lane == 0) {
          q0[j] = csub(q0[j], a0);
          if (two) q1[j] = csub(q1[j], a1);
        }
      }
    } else {
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
    }
    cta_sync();
  }
}

// R (kq x n) of a factored H into Rout (ld kq), zero below the diagonal.
static __device__ __forceinline__ void dev_qr_extract_r(const cplx* H, int m, int n, cplx* Rout) {
  const int kq = min(m, n);
  for (int e = ltid(); e < kq * n; e += NT) {
    int r = (int)(e % kq), c = (int)(e / kq);
    Rout[e] = (r <= c) ? H[r + (long long)m * c] : make_double2(0.0, 0.0);
  }
  cta_sync();
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
  int sweeps;
};

// Orthonormal completion of column k of Y (rows x *) against columns 0..k-1.
static __device__ void dev_complete_column(cplx* Y, int rows, int k, cplx* y, RedScratch& rs) {
  for (int c = 0; c < rows; ++c) {
    // pass 1: y = e_c - sum_h conj(Y_h[c]) Y_h
    for (int i = ltid(); i < rows; i += NT) {
      cplx v = make_double2(i == c ? 1.0 : 0.0, 0.0);
      for (int h = 0; h < k; ++h) {
        cplx yc = Y[c + (long long)rows * h];
        cplx yi = Y[i + (long long)rows * h];
        v = csub(v, cmulc(yc, yi));
      }
      y[i] = v;
    }
    cta_sync();
    // pass 2: y -= sum_h (Y_h^H y) Y_h, dot products in chunks of 8
    for (int h0 = 0; h0 < k; h0 += 8) {
      double d[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) d[e] = 0.0;
      for (int i = ltid(); i < rows; i += NT) {
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
      for (int i = ltid(); i < rows; i += NT) {
        cplx v = y[i];
#pragma unroll
        for (int e = 0; e < 8; ++e)
          if (h0 + e < k) v = csub(v, cmul(make_double2(d[2 * e], d[2 * e + 1]), Y[i + (long long)rows * (h0 + e)]));
        y[i] = v;
      }
      cta_sync();
    }
    double nr = sqrt(cta_norm2(y, rows, rs));
    if (nr > 0.5) {
      for (int i = ltid(); i < rows; i += NT) Y[i + (long long)rows * k] = cscale(y[i], 1.0 / nr);
      cta_sync();
      return;
    }
  }
}

// Block size of the block-cyclic Jacobi ordering: blocks of b columns of B
// (q rows) so that a pair of blocks fits the SVD_SMEM_CPLX shared buffer.
// The CPU oracle uses the same rule.
#define SVD_SMEM_CPLX 4096
__host__ __device__ __forceinline__ int svd_block_size(int q, int p) {
  int b = SVD_SMEM_CPLX / (2 * q);
  if (b > 32) b = 32;
  if (b > p) b = p;
  if (b < 1) b = 1;
  return b;
}

// Jacobi rotation parameters for columns with |b_i|^2 = al, |b_j|^2 = be,
// b_i^H b_j = (gx, gy).  Same rotation as the oracle's
//   zeta = (be-al)/(2|g|), t = sign(zeta)/(|zeta| + sqrt(1+zeta^2)),
//   c = 1/sqrt(1+t^2), s = c t, e = g/|g|,
// written with fewer dependent divisions/square roots:
//   t = sign(d) 2|g| / (|d| + sqrt(d^2 + 4|g|^2)),  d = be - al.
// Returns false when the pair is already orthogonal to tolerance.
static __device__ __forceinline__ bool jacobi_params(double al, double be, double gx, double gy, double tol, double& c,
                                              cplx& se, cplx& sec) {
  const double g2 = gx * gx + gy * gy;
  if (!(g2 > tol * tol * (al * be))) return false;
  const double rag = rsqrt(g2);
  const double ag = g2 * rag;
  const double d = be - al;
  const double R = sqrt(fma(d, d, 4.0 * g2));
  double t = 2.0 * ag / (fabs(d) + R);
  if (d < 0.0) t = -t;
  c = rsqrt(fma(t, t, 1.0));
  const double f = c * t * rag;
  se = make_double2(f * gx, f * gy);
  sec = make_double2(f * gx, -f * gy);
  return true;
}

// One Jacobi rotation pass over disjoint column pairs held in shared memory
// (columns c of the stacked [B; X] block at sb + c*ld).  pairs(k) gives the
// k-th pair as (i, j) local column indices, -1 to skip.  Each half-warp
// takes one pair.
template <class PairFn>
static __device__ __forceinline__ void smem_rotate_round(cplx* sb, int ld, int q, int rows, int npairs, PairFn pairs,
                                                  double tol, int* rot) {
  const int hl = ltid() & 15, hw = ltid() >> 4;
  const unsigned mask = (ltid() & 16) ? 0xffff0000u : 0x0000ffffu;
  for (int k = hw; k < npairs; k += NT / 16) {
    int i, j;
    pairs(k, i, j);
    if (i < 0 || j < 0) continue;
    cplx* bi = sb + (long long)ld * i;
    cplx* bj = sb + (long long)ld * j;
    double al = 0.0, be = 0.0, gx = 0.0, gy = 0.0;
    for (int r = hl; r < q; r += 16) {
      cplx x = bi[r], y = bj[r];
      al += cabs2(x);
      be += cabs2(y);
      gx += x.x * y.x + x.y * y.y;
      gy += x.x * y.y - x.y * y.x;
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      al += __shfl_xor_sync(mask, al, o);
      be += __shfl_xor_sync(mask, be, o);
      gx += __shfl_xor_sync(mask, gx, o);
      gy += __shfl_xor_sync(mask, gy, o);
    }
    double c;
    cplx se, sec;
    if (!jacobi_params(al, be, gx, gy, tol, c, se, sec)) continue;
    if (hl == 0) atomicAdd(rot, 1);
    for (int r = hl; r < rows; r += 16) {
      cplx x = bi[r], y = bj[r];
      bi[r] = csub(cscale(x, c), cmul(sec, y));
      bj[r] = cadd(cmul(se, x), cscale(y, c));
    }
  }
  cta_sync();
}

// Stage columns [c0, c0+nc0) and [c1, c1+nc1) of B into sb (ld = q), or
// write them back.
static __device__ __forceinline__ void svd_stage(cplx* sb, int ld, const SvdWork& w, int q, int c0, int nc0, int c1, int nc1,
                                          bool store) {
  const int nc = nc0 + nc1;
  for (int e = ltid(); e < nc * ld; e += NT) {
    int r = (int)(e % ld), lc = (int)(e / ld);
    int col = lc < nc0 ? c0 + lc : c1 + (lc - nc0);
    cplx* g = w.B + (long long)q * col + r;
    if (store) *g = sb[e];
    else sb[e] = *g;
  }
  cta_sync();
}

// SVD of M (m x n, col-major ld m), phase 1.  side LEFT asks for the left
// singular vectors (orthonormal U, m-vectors), side RIGHT for the right ones
// (orthonormal V, n-vectors).  QR-preconditioned one-sided Jacobi
// (Drmac-Veselic): LEFT factors M^H = Q R and orthogonalises the columns of
// B = R^H (m x k); RIGHT factors M = Q R and orthogonalises B = R^H
// (n x k); k = min(m, n).  Either way B's columns converge to (vectors) x
// Sigma.  Jacobi runs in the block-cyclic order (per sweep: every diagonal
// block with a round-robin pass, then every pair of blocks in round-robin
// order with b rounds of disjoint cross pairs) on blocks staged in the
// shared buffer sb (SVD_SMEM_CPLX elements).  Leaves the sorted singular
// values in w.sig (nulls set to 0).  CTA-collective; returns metadata.
enum { SVD_LEFT = 0, SVD_RIGHT = 1 };
static __device__ __noinline__ SvdResult dev_svd(const cplx* M, int m, int n, int side, SvdWork& w, LinalgSmem& ls,
                                          RedScratch& rs, cplx* sb) {
  ProfScope prof_scope_(PF_SVD);
  const int tid = ltid();
  SvdResult res;
  res.tr = side == SVD_RIGHT;
  const int mm = res.tr ? m : n;  // rows of the factored matrix H
  const int nn = res.tr ? n : m;
  const int k = min(m, n);
  const int q = nn, p = k;
  res.q = q;
  res.p = p;
  res.sweeps = 0;
  cplx* H = w.X;
  for (int e = tid; e < mm * nn; e += NT) {
    int r = (int)(e % mm), c = (int)(e / mm);
    H[e] = res.tr ? M[e] : cconj(M[c + (long long)m * r]);
  }
  cta_sync();
  dev_qr_factor(H, mm, nn, ls, rs);
  // B = R^H (nn x k): B[r, c] = conj(R[c, r]) for c <= r
  for (int e = tid; e < q * p; e += NT) {
    int r = (int)(e % q), c = (int)(e / q);
    w.B[e] = (c <= r) ? cconj(H[c + (long long)mm * r]) : make_double2(0.0, 0.0);
  }
  cta_sync();
  const double tol = 2.220446049250313e-16 * q;
  const int ld = q;
  const int b = svd_block_size(q, p);
  const int nb = (p + b - 1) / b;
  const int nbe = nb + (nb & 1);
  const int be2 = b + (b & 1);
  for (int sweep = 0; sweep < JACOBI_MAX_SWEEPS; ++sweep) {
    if (tid == 0) ls.rot_count = 0;
    cta_sync();
    for (int I = 0; I < nb; ++I) {
      const int c0 = I * b, nc = min(b, p - c0);
      svd_stage(sb, ld, w, q, c0, nc, 0, 0, false);
      for (int round = 0; round < be2 - 1; ++round) {
        smem_rotate_round(sb, ld, q, q, be2 / 2,
                          [&](int pr, int& i, int& j) {
                            int ta = pr, tb = be2 - 1 - pr;
                            int a = ta == 0 ? 0 : ((ta - 1 - round + 2 * (be2 - 1)) % (be2 - 1)) + 1;
                            int c = tb == 0 ? 0 : ((tb - 1 - round + 2 * (be2 - 1)) % (be2 - 1)) + 1;
                            i = min(a, c);
                            j = max(a, c);
                            if (j >= nc) i = j = -1;
                          },
                          tol, &ls.rot_count);
      }
      svd_stage(sb, ld, w, q, c0, nc, 0, 0, true);
    }
    for (int round = 0; round < nbe - 1; ++round) {
      for (int pr = 0; pr < nbe / 2; ++pr) {
        int ta = pr, tb = nbe - 1 - pr;
        int A = ta == 0 ? 0 : ((ta - 1 - round + 2 * (nbe - 1)) % (nbe - 1)) + 1;
        int Bk = tb == 0 ? 0 : ((tb - 1 - round + 2 * (nbe - 1)) % (nbe - 1)) + 1;
        int I = min(A, Bk), J = max(A, Bk);
        if (J >= nb) continue;
        const int c0 = I * b, n0 = min(b, p - c0), c1 = J * b, n1 = min(b, p - c1);
        svd_stage(sb, ld, w, q, c0, n0, c1, n1, false);
        for (int t = 0; t < b; ++t) {
          smem_rotate_round(sb, ld, q, q, b,
                            [&](int kk, int& i, int& j) {
                              int jj = (kk + t) % b;
                              if (kk >= n0 || jj >= n1) {
                                i = j = -1;
                              } else {
                                i = kk;
                                j = n0 + jj;
                              }
                            },
                            tol, &ls.rot_count);
        }
        svd_stage(sb, ld, w, q, c0, n0, c1, n1, true);
      }
    }
    int rc = ls.rot_count;
    cta_sync();
    res.sweeps = sweep + 1;
    if (rc == 0) break;
  }
  // singular values
  const int lane = tid & 31, wid = tid >> 5;
  for (int c = wid; c < p; c += NW) {
    const cplx* bc = w.B + (long long)q * c;
    double s = 0.0;
    for (int r = lane; r < q; r += 32) s += cabs2(bc[r]);
    s = warp_sum(s);
    if (lane == 0) w.sig[c] = sqrt(s);
  }
  cta_sync();
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
  cta_sync();
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
  cta_sync();
  if (myk < p) w.sig[myk] = sk;
  cta_sync();
  return res;
}

// Phase 2: the requested orthonormal vectors Yo (q x need): column k is
// B[:, ord[k]] / sigma_k for non-null k and an orthonormal completion for
// null k < need.  CTA-collective.
static __device__ __noinline__ void dev_svd_vectors(const SvdResult& res, int need, SvdWork& w, RedScratch& rs) {
  ProfScope prof_scope_(PF_SVDVEC);
  const int tid = ltid(), q = res.q, p = res.p;
  need = min(need, p);
  const int ng = min(need, res.rank);
  for (int e = tid; e < q * ng; e += NT) {
    int r = (int)(e % q), k = (int)(e / q);
    w.Yo[e] = cscale(w.B[r + (long long)q * w.ord[k]], 1.0 / w.sig[k]);
  }
  cta_sync();
  for (int k = res.rank; k < need; ++k) dev_complete_column(w.Yo, q, k, w.y, rs);
}

// Truncation ranks (see the oracle for the reference lines they restate).
// split_mps_tensor_svd / two_site_svd: absolute, keep crossing value, min 2.
static __device__ __forceinline__ int keep_tdvp(const double* S, int n, double thr, int max_bond) {
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
static __device__ __forceinline__ int keep_relative(const double* S, int n, double thr, int max_bond) {
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

// apply_local_gate_exact! (DigitalTJM.jl:282-292): absolute, drop while the
// running sum plus s^2 stays <= thr, no minimum.
static __device__ __forceinline__ int keep_tebd(const double* S, int n, double thr, int max_bond) {
  double cur = 0.0;
  int keep = n;
  for (int k = n; k >= 1; --k) {
    if (cur + S[k - 1] * S[k - 1] > thr) break;
    cur += S[k - 1] * S[k - 1];
    --keep;
  }
  return max(1, min(keep, max_bond));
}
