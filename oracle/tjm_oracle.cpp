// tjm_oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of the analog tensor-jump-method path of Yaqs.jl
// (MaxFroehlich1410/yaqs-julia).  It is the checker for the CUDA engine and
// the timed CPU baseline; nothing in the product links or calls it.  Only
// tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
//
// Each routine names the reference file:line it restates.  Three pieces of
// arithmetic live in third-party Julia packages that are not in the
// reference tree and are restated from their published methods:
//   * KrylovKit 0.10.2 `exponentiate` (Algorithms.jl:185): Lanczos with
//     full (classical Gram-Schmidt, two pass) re-orthogonalisation, then the
//     exact exponential of the small tridiagonal matrix through its
//     eigendecomposition (Hochbruck-Lubich Krylov exponential).
//   * LAPACK QR/LQ (Decompositions.jl:18-73, MPS.jl:182-311): Householder
//     reflections in the zlarfg convention (real R diagonal, beta =
//     -sign(Re alpha)*|x|).
//   * LAPACK SVD (Algorithms.jl:420): one-sided (Hestenes) Jacobi.
// QR and SVD factors are unique only up to phases and, for zero singular
// values, up to the choice of null vectors.  The restatement fixes that
// choice deterministically (see null_tol below) so the CUDA engine can
// reproduce it bit-for-bit up to rounding.
//
// Layouts follow the reference (column-major): MPS tensor (l, p, r)
// (MPS.jl:22), MPO tensor (wl, p_out, p_in, wr) (MPO.jl:19-24), environment
// (bra, mpo, ket) (Algorithms.jl:191-211).  Sites are 0-based.

#include "../include/yaqs_tjm.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using cd = std::complex<double>;
using std::vector;

// Relative thresholds that make null directions deterministic.
constexpr double kQrNullTol = 1e-14;    // trailing column treated as exactly zero
constexpr double kSvdNullTol = 1e-14;   // singular value treated as exactly zero
constexpr int kJacobiMaxSweeps = 60;

inline double nrm2(const cd* x, long n) {
  double s = 0;
  for (long i = 0; i < n; ++i) s += std::norm(x[i]);
  return std::sqrt(s);
}

// ---------------------------------------------------------------------------
// Tensors
// ---------------------------------------------------------------------------
struct Ten {  // MPS-like rank-3 tensor (l, d, r), column-major
  int l = 1, d = 2, r = 1;
  vector<cd> v;
  Ten() {}
  Ten(int l_, int d_, int r_) : l(l_), d(d_), r(r_), v((size_t)l_ * d_ * r_) {}
  cd& at(int a, int p, int b) { return v[a + (size_t)l * (p + (size_t)d * b)]; }
  cd at(int a, int p, int b) const { return v[a + (size_t)l * (p + (size_t)d * b)]; }
};

struct Wt {  // MPO tensor (wl, d, d, wr)
  int wl = 1, d = 2, wr = 1;
  vector<cd> v;
  Wt() {}
  Wt(int wl_, int d_, int wr_) : wl(wl_), d(d_), wr(wr_), v((size_t)wl_ * d_ * d_ * wr_) {}
  cd at(int m, int po, int pi, int mr) const {
    return v[m + (size_t)wl * (po + (size_t)d * (pi + (size_t)d * mr))];
  }
  cd& at(int m, int po, int pi, int mr) {
    return v[m + (size_t)wl * (po + (size_t)d * (pi + (size_t)d * mr))];
  }
};

struct Env {  // (bra, w, ket)
  int b = 1, w = 1, k = 1;
  vector<cd> v;
  Env() {}
  Env(int b_, int w_, int k_) : b(b_), w(w_), k(k_), v((size_t)b_ * w_ * k_) {}
  cd at(int x, int m, int y) const { return v[x + (size_t)b * (m + (size_t)w * y)]; }
  cd& at(int x, int m, int y) { return v[x + (size_t)b * (m + (size_t)w * y)]; }
};

struct State {
  int L = 0;
  vector<Ten> t;
  int oc = 0;  // orth_center (0-based)
};

// Optional optimised BLAS for the timed CPU baseline: a CBLAS zgemm (the
// reference's contractions run on OpenBLAS ZGEMM through TensorOperations,
// Manifest.toml).  Installed by orc_set_zgemm; null (the default, and what
// every test uses) keeps the plain loops below.  Column-major only.
typedef void (*cblas_zgemm_t)(int order, int transa, int transb, int m, int n, int k, const void* alpha,
                              const void* A, int lda, const void* B, int ldb, const void* beta, void* C, int ldc);
static cblas_zgemm_t g_zgemm = nullptr;
enum { CB_COLMAJOR = 102, CB_NOTRANS = 111, CB_TRANS = 112, CB_CONJTRANS = 113 };
inline void blas_gemm(int ta, int tb, int m, int n, int k, const cd* A, int lda, const cd* B, int ldb, cd* C,
                      int ldc) {
  const cd one(1.0, 0.0), zero(0.0, 0.0);
  g_zgemm(CB_COLMAJOR, ta, tb, m, n, k, &one, A, lda, B, ldb, &zero, C, ldc);
}

// C(m x n) = A(m x k) * B(k x n), column-major with leading dims = rows.
void matmul(int m, int n, int k, const cd* A, const cd* B, cd* C) {
  if (g_zgemm) {
    blas_gemm(CB_NOTRANS, CB_NOTRANS, m, n, k, A, m, B, k, C, m);
    return;
  }
  for (long i = 0; i < (long)m * n; ++i) C[i] = 0;
  for (int j = 0; j < n; ++j)
    for (int p = 0; p < k; ++p) {
      cd b = B[p + (size_t)k * j];
      if (b == cd(0)) continue;
      const cd* a = A + (size_t)m * p;
      cd* c = C + (size_t)m * j;
      for (int i = 0; i < m; ++i) c[i] += a[i] * b;
    }
}

// ---------------------------------------------------------------------------
// Householder QR / LQ (restates LAPACK geqrf/orgqr as used by
// Decompositions.jl:18-73 and MPS.jl:182-311).
// ---------------------------------------------------------------------------
// Thin QR of M (m x n): Q (m x kq), R (kq x n), kq = min(m, n).
void house_qr(int m, int n, const cd* M, vector<cd>& Q, vector<cd>& R) {
  const int kq = std::min(m, n);
  vector<cd> A(M, M + (size_t)m * n);
  vector<cd> tau(kq, 0.0);
  const double fro = nrm2(M, (long)m * n);
  const double null_abs = kQrNullTol * fro;
  for (int j = 0; j < kq; ++j) {
    cd* col = &A[(size_t)m * j];
    cd alpha = col[j];
    double xn2 = 0;
    for (int i = j + 1; i < m; ++i) xn2 += std::norm(col[i]);
    double full = std::sqrt(std::norm(alpha) + xn2);
    if (full <= null_abs || (xn2 == 0.0 && alpha.imag() == 0.0)) {
      tau[j] = 0.0;
      for (int i = j + 1; i < m; ++i) col[i] = 0.0;
      continue;
    }
    double beta = (alpha.real() >= 0.0) ? -full : full;
    tau[j] = (cd(beta) - alpha) / beta;
    cd scale = 1.0 / (alpha - beta);
    for (int i = j + 1; i < m; ++i) col[i] *= scale;
    col[j] = beta;
    cd ct = std::conj(tau[j]);
    for (int c = j + 1; c < n; ++c) {
      cd* x = &A[(size_t)m * c];
      cd s = x[j];
      for (int i = j + 1; i < m; ++i) s += std::conj(col[i]) * x[i];
      s *= ct;
      x[j] -= s;
      for (int i = j + 1; i < m; ++i) x[i] -= s * col[i];
    }
  }
  R.assign((size_t)kq * n, 0.0);
  for (int c = 0; c < n; ++c)
    for (int i = 0; i <= std::min(c, kq - 1); ++i) R[i + (size_t)kq * c] = A[i + (size_t)m * c];
  Q.assign((size_t)m * kq, 0.0);
  for (int c = 0; c < kq; ++c) Q[c + (size_t)m * c] = 1.0;
  for (int j = kq - 1; j >= 0; --j) {
    if (tau[j] == cd(0)) continue;
    const cd* v = &A[(size_t)m * j];
    for (int c = j; c < kq; ++c) {
      cd* q = &Q[(size_t)m * c];
      cd s = q[j];
      for (int i = j + 1; i < m; ++i) s += std::conj(v[i]) * q[i];
      s *= tau[j];
      q[j] -= s;
      for (int i = j + 1; i < m; ++i) q[i] -= s * v[i];
    }
  }
}

// Thin LQ of M (m x n) = Lm (m x k) * Qm (k x n), via QR of M^H.
void house_lq(int m, int n, const cd* M, vector<cd>& Lm, vector<cd>& Qm) {
  vector<cd> MH((size_t)n * m);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) MH[j + (size_t)n * i] = std::conj(M[i + (size_t)m * j]);
  vector<cd> Q, R;
  house_qr(n, m, MH.data(), Q, R);  // Q (n x k), R (k x m)
  const int k = std::min(m, n);
  Lm.assign((size_t)m * k, 0.0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < k; ++j) Lm[i + (size_t)m * j] = std::conj(R[j + (size_t)k * i]);
  Qm.assign((size_t)k * n, 0.0);
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < n; ++j) Qm[i + (size_t)k * j] = std::conj(Q[j + (size_t)n * i]);
}

// ---------------------------------------------------------------------------
// One-sided Jacobi SVD (restates the `svd` of Algorithms.jl:420,
// Decompositions.jl:105, Dissipation.jl:281, StochasticProcess.jl:280).
// QR-preconditioned (Drmac-Veselic): side LEFT (orthonormal left vectors of
// M, m x n) factors M^H = Q R and orthogonalises the columns of B = R^H
// (m x k); side RIGHT factors M = Q R and orthogonalises B = R^H (n x k).
// The columns of B converge to (requested singular vectors) x Sigma.
// ---------------------------------------------------------------------------
// Orthonormal completion: fills column `slot` of X (rows x *) with the
// first unit vector e_c whose component orthogonal to columns `have` exceeds
// 1/2 in norm (two Gram-Schmidt passes), normalised.
void complete_column(int rows, vector<cd>& X, const vector<int>& have, int slot) {
  vector<cd> y(rows);
  for (int c = 0; c < rows; ++c) {
    std::fill(y.begin(), y.end(), cd(0));
    y[c] = 1.0;
    for (int pass = 0; pass < 2; ++pass)
      for (int h : have) {
        const cd* x = &X[(size_t)rows * h];
        cd s = 0;
        for (int i = 0; i < rows; ++i) s += std::conj(x[i]) * y[i];
        for (int i = 0; i < rows; ++i) y[i] -= s * x[i];
      }
    double nr = nrm2(y.data(), rows);
    if (nr > 0.5) {
      for (int i = 0; i < rows; ++i) X[(size_t)rows * slot + i] = y[i] / nr;
      return;
    }
  }
}

// Block size of the block-cyclic Jacobi order (same rule as the GPU engine:
// a pair of b-column blocks of B (q rows) fits 4096 complex values).
int svd_block_size(int q, int p) {
  int b = 4096 / (2 * q);
  if (b > 32) b = 32;
  if (b > p) b = p;
  if (b < 1) b = 1;
  return b;
}

enum { SVD_LEFT = 0, SVD_RIGHT = 1 };

struct SvdOut {
  int q = 0, p = 0, rank = 0;
  vector<double> S;  // sorted descending, nulls zeroed (length p)
  vector<cd> B;      // q x p after Jacobi
  vector<int> ord;   // sorted column order
};

SvdOut svd_side(int m, int n, const cd* M, int side) {
  SvdOut o;
  const bool right = side == SVD_RIGHT;
  const int mm = right ? m : n, nn = right ? n : m, k = std::min(m, n);
  vector<cd> H((size_t)mm * nn);
  for (int r = 0; r < mm; ++r)
    for (int c = 0; c < nn; ++c)
      H[r + (size_t)mm * c] = right ? M[r + (size_t)m * c] : std::conj(M[c + (size_t)m * r]);
  vector<cd> Q, R;
  house_qr(mm, nn, H.data(), Q, R);  // R (k x nn)
  const int q = nn, p = k;
  o.q = q;
  o.p = p;
  vector<cd>& B = o.B;
  B.assign((size_t)q * p, 0.0);
  for (int r = 0; r < q; ++r)
    for (int c = 0; c <= std::min(r, p - 1); ++c) B[r + (size_t)q * c] = std::conj(R[c + (size_t)k * r]);
  const double tol = 2.220446049250313e-16 * q;
  auto rotate = [&](int i, int j, int& rotations) {
    cd* bi = &B[(size_t)q * i];
    cd* bj = &B[(size_t)q * j];
    double al = 0, be = 0;
    cd g = 0;
    for (int r = 0; r < q; ++r) {
      al += std::norm(bi[r]);
      be += std::norm(bj[r]);
      g += std::conj(bi[r]) * bj[r];
    }
    double ag = std::abs(g);
    if (!(ag > tol * std::sqrt(al * be))) return;
    ++rotations;
    double zeta = (be - al) / (2.0 * ag);
    double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
    double c = 1.0 / std::sqrt(1.0 + t * t);
    double s = c * t;
    cd e = g / ag;
    cd se = s * e, sec = s * std::conj(e);
    for (int r = 0; r < q; ++r) {
      cd x = bi[r], y = bj[r];
      bi[r] = c * x - sec * y;
      bj[r] = se * x + c * y;
    }
  };
  // Round-robin (tournament) slot of position t in round `round` of n players.
  auto slot = [](int t, int round, int n) { return t == 0 ? 0 : ((t - 1 - round + 2 * (n - 1)) % (n - 1)) + 1; };
  // Block-cyclic order: per sweep every diagonal block gets a round-robin
  // pass, then every pair of blocks (round-robin over blocks) gets b rounds
  // of disjoint cross pairs (k, (k + t) mod b).
  const int b = svd_block_size(q, p);
  const int nb = (p + b - 1) / b, nbe = nb + (nb & 1), be2 = b + (b & 1);
  for (int sweep = 0; sweep < kJacobiMaxSweeps; ++sweep) {
    int rotations = 0;
    for (int I = 0; I < nb; ++I) {
      const int c0 = I * b, nc = std::min(b, p - c0);
      for (int round = 0; round < be2 - 1; ++round)
        for (int pr = 0; pr < be2 / 2; ++pr) {
          int a = slot(pr, round, be2), cc = slot(be2 - 1 - pr, round, be2);
          int i = std::min(a, cc), j = std::max(a, cc);
          if (j >= nc) continue;
          rotate(c0 + i, c0 + j, rotations);
        }
    }
    for (int round = 0; round < nbe - 1; ++round)
      for (int pr = 0; pr < nbe / 2; ++pr) {
        int A = slot(pr, round, nbe), Bk = slot(nbe - 1 - pr, round, nbe);
        int I = std::min(A, Bk), J = std::max(A, Bk);
        if (J >= nb) continue;
        const int c0 = I * b, n0 = std::min(b, p - c0), c1 = J * b, n1 = std::min(b, p - c1);
        for (int t = 0; t < b; ++t)
          for (int kk = 0; kk < b; ++kk) {
            int jj = (kk + t) % b;
            if (kk >= n0 || jj >= n1) continue;
            rotate(c0 + kk, c1 + jj, rotations);
          }
      }
    if (rotations == 0) break;
  }
  vector<double> sig(p);
  for (int c = 0; c < p; ++c) sig[c] = nrm2(&B[(size_t)q * c], q);
  o.ord.resize(p);
  for (int i = 0; i < p; ++i) o.ord[i] = i;
  std::stable_sort(o.ord.begin(), o.ord.end(), [&](int a, int b2) { return sig[a] > sig[b2]; });
  const double smax = p > 0 ? sig[o.ord[0]] : 0.0;
  o.S.assign(p, 0.0);
  o.rank = 0;
  for (int kk = 0; kk < p; ++kk) {
    double sv = sig[o.ord[kk]];
    if (smax > 0 && sv > kSvdNullTol * smax) {
      o.S[kk] = sv;
      ++o.rank;
    }
  }
  return o;
}

// Requested orthonormal vectors Y (q x need): B[:, ord[k]] / S[k], with
// orthonormal completions for the null columns.
vector<cd> svd_vectors(const SvdOut& o, int need) {
  need = std::min(need, o.p);
  vector<cd> Y((size_t)o.q * need, 0.0);
  vector<int> have;
  for (int kk = 0; kk < std::min(need, o.rank); ++kk) {
    const cd* bc = &o.B[(size_t)o.q * o.ord[kk]];
    for (int r = 0; r < o.q; ++r) Y[(size_t)o.q * kk + r] = bc[r] / o.S[kk];
    have.push_back(kk);
  }
  for (int kk = o.rank; kk < need; ++kk) {
    complete_column(o.q, Y, have, kk);
    have.push_back(kk);
  }
  return Y;
}

// Component form used by the tests: U (m x k), S (k), SVt = U^H M (k x n).
void jacobi_svd(int m, int n, const cd* M, vector<cd>& U, vector<double>& S, vector<cd>& SVt) {
  SvdOut o = svd_side(m, n, M, SVD_LEFT);
  const int k = o.p;
  U = svd_vectors(o, k);
  S = o.S;
  SVt.assign((size_t)k * n, 0.0);
  for (int c = 0; c < n; ++c)
    for (int kk = 0; kk < k; ++kk) {
      if (kk >= o.rank) continue;
      cd sacc = 0;
      for (int r = 0; r < m; ++r) sacc += std::conj(U[r + (size_t)m * kk]) * M[r + (size_t)m * c];
      SVt[kk + (size_t)k * c] = sacc;
    }
}

// Truncation rules (each restates one call site).
// split_mps_tensor_svd (Algorithms.jl:423-438) and two_site_svd
// (Decompositions.jl:121-149): absolute, keep the crossing value, min 2.
int keep_tdvp(const vector<double>& S, double thr, int max_bond) {
  int n = (int)S.size();
  double disc = 0;
  int keep = n;
  for (int k = n; k >= 1; --k) {
    disc += S[k - 1] * S[k - 1];
    if (disc >= thr) {
      keep = std::max(k, 2);
      break;
    }
  }
  return std::max(1, std::min(keep, max_bond));
}
// Dissipation.jl:290-303 and StochasticProcess.jl:288-300: relative, min 1.
int keep_relative(const vector<double>& S, double thr, int max_bond) {
  int n = (int)S.size();
  double nsq = 0;
  for (double s : S) nsq += s * s;
  double cur = 0;
  int rank = n;
  for (int k = n; k >= 1; --k) {
    cur += S[k - 1] * S[k - 1];
    if (cur > thr * nsq) {
      rank = k;
      break;
    }
  }
  return std::max(1, std::min(rank, max_bond));
}

// apply_local_gate_exact! (DigitalTJM.jl:282-292): absolute, drop while the
// running sum plus s^2 stays <= thr, no minimum.
int keep_tebd(const vector<double>& S, double thr, int max_bond) {
  int n = (int)S.size();
  double cur = 0;
  int keep = n;
  for (int k = n; k >= 1; --k) {
    if (cur + S[k - 1] * S[k - 1] > thr) break;
    cur += S[k - 1] * S[k - 1];
    --keep;
  }
  return std::max(1, std::min(keep, max_bond));
}

// ---------------------------------------------------------------------------
// Small symmetric eigensolver (cyclic Jacobi) for the Lanczos matrix.
// ---------------------------------------------------------------------------
void sym_eig(int n, vector<double>& A, vector<double>& V) {  // A (n x n) -> diag, V eigenvectors
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[i + (size_t)n * i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0, tot = 0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double x = A[i + (size_t)n * j] * A[i + (size_t)n * j];
        tot += x;
        if (i != j) off += x;
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p + (size_t)n * q];
        if (apq == 0.0) continue;
        double app = A[p + (size_t)n * p], aqq = A[q + (size_t)n * q];
        double zeta = (aqq - app) / (2.0 * apq);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
        for (int k = 0; k < n; ++k) {  // columns p,q
          double akp = A[k + (size_t)n * p], akq = A[k + (size_t)n * q];
          A[k + (size_t)n * p] = c * akp - s * akq;
          A[k + (size_t)n * q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p,q
          double apk = A[p + (size_t)n * k], aqk = A[q + (size_t)n * k];
          A[p + (size_t)n * k] = c * apk - s * aqk;
          A[q + (size_t)n * k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = V[k + (size_t)n * p], vkq = V[k + (size_t)n * q];
          V[k + (size_t)n * p] = c * vkp - s * vkq;
          V[k + (size_t)n * q] = s * vkp + c * vkq;
        }
      }
  }
}

// ---------------------------------------------------------------------------
// Krylov exponential (restates expm_krylov, Algorithms.jl:144-187, and the
// KrylovKit exponentiate call at :185): returns exp(-i*dt*H) v.
// ---------------------------------------------------------------------------
struct KrylovParams {
  int kdim = 25;
  double tol = 1e-10;
  double exit_tol = 0.0;
};

struct Counters {
  long long matvecs = 0, solves = 0, svds = 0, jumps = 0, nonfinite = 0;
  double flops = 0;
};

template <class Op>
vector<cd> expm_krylov(Op&& op, const vector<cd>& v, double dt, const KrylovParams& kp, Counters& cnt) {
  const long n = (long)v.size();
  const double beta0 = nrm2(v.data(), n);
  if (beta0 == 0.0) return v;
  cnt.solves++;
  const double tau = std::fabs(dt);
  vector<vector<cd>> Q;
  Q.reserve(kp.kdim + 1);
  vector<cd> q0(n);
  for (long i = 0; i < n; ++i) q0[i] = v[i] / beta0;
  Q.push_back(std::move(q0));
  vector<double> alpha, beta;
  double bound = 1.0;
  int m = 0;
  vector<cd> w(n);
  for (int k = 1; k <= kp.kdim; ++k) {
    op(Q[k - 1], w);
    cnt.matvecs++;
    // classical Gram-Schmidt against q_1..q_k.  h_j = <q_j, w> and |w|^2 come
    // from one pass; when the projection keeps at least 1/sqrt(2) of the norm
    // (DGKS criterion, the eta of KrylovKit's iteratively refined
    // Gram-Schmidt, tested as |w|^2 - |h|^2 >= |w|^2 / 2) the residual norm
    // is sqrt(|w|^2 - |h|^2) and q_k = (w - Q h) / b_k; otherwise one
    // refinement pass projects again and the norm is taken directly.
    auto dots = [&](vector<cd>& h) {
      for (int j = 0; j < k; ++j) {
        cd sacc = 0;
        const cd* qj = Q[j].data();
        for (long i = 0; i < n; ++i) sacc += std::conj(qj[i]) * w[i];
        h[j] = sacc;
      }
    };
    auto subtract = [&](const vector<cd>& h) {
      for (long i = 0; i < n; ++i) {
        cd v = w[i];
        for (int j = 0; j < k; ++j) v -= h[j] * Q[j][i];
        w[i] = v;
      }
    };
    vector<cd> h(k);
    dots(h);
    double nw2 = 0.0, hh = 0.0;
    for (long i = 0; i < n; ++i) nw2 += std::norm(w[i]);
    for (int j = 0; j < k; ++j) hh += std::norm(h[j]);
    double a_k = h[k - 1].real(), b_k;
    const double r2 = nw2 - hh;
    const bool accept = r2 >= 0.5 * nw2;
    if (accept) {
      b_k = std::sqrt(r2);
    } else {
      subtract(h);
      dots(h);
      a_k += h[k - 1].real();
      subtract(h);
      b_k = nrm2(w.data(), n);
    }
    alpha.push_back(a_k);
    m = k;
    if (b_k <= tau * kp.tol) break;  // invariant subspace (KrylovKit normres test)
    if (k == kp.kdim) break;
    bound *= b_k * tau / k;
    if (kp.exit_tol > 0.0 && bound <= kp.exit_tol) break;
    beta.push_back(b_k);
    if (accept) subtract(h);
    vector<cd> qn(n);
    for (long i = 0; i < n; ++i) qn[i] = w[i] / b_k;
    Q.push_back(std::move(qn));
  }
  // T (m x m) symmetric tridiagonal
  vector<double> T((size_t)m * m, 0.0), V;
  for (int i = 0; i < m; ++i) T[i + (size_t)m * i] = alpha[i];
  for (int i = 0; i + 1 < m; ++i) {
    T[i + (size_t)m * (i + 1)] = beta[i];
    T[(i + 1) + (size_t)m * i] = beta[i];
  }
  sym_eig(m, T, V);
  vector<cd> y(m, 0.0);
  for (int e = 0; e < m; ++e) {
    double lam = T[e + (size_t)m * e];
    cd ph = std::exp(cd(0.0, -dt * lam)) * V[0 + (size_t)m * e];
    for (int j = 0; j < m; ++j) y[j] += V[j + (size_t)m * e] * ph;
  }
  vector<cd> out(n, 0.0);
  for (int j = 0; j < m; ++j) {
    cd c = y[j] * beta0;
    const cd* qj = Q[j].data();
    for (long i = 0; i < n; ++i) out[i] += c * qj[i];
  }
  return out;
}

// ---------------------------------------------------------------------------
// Environments and projected operators (Algorithms.jl:191-226)
// ---------------------------------------------------------------------------
Env identity_env(int dim, int w) {  // make_identity_env, Algorithms.jl:191-197
  Env E(dim, w, dim);
  for (int i = 0; i < dim; ++i) E.at(i, 0, i) = 1.0;
  return E;
}

// update_left_environment (Algorithms.jl:199-204)
Env update_left(const Ten& A, const Wt& W, const Env& E) {
  const int bl = A.l, d = A.d, br = A.r, wl = W.wl, wr = W.wr;
  // T1[bra_l, ml, pin, ket_r] = sum_k E[bra_l, ml, k] A[k, pin, ket_r]
  vector<cd> T1((size_t)bl * wl * d * br);
  matmul(bl * wl, d * br, bl, E.v.data(), A.v.data(), T1.data());
  if (g_zgemm) {  // T2 as [bra_l, pout, ket_r, mr], then E'_mr = A^H T2_mr
    vector<cd> T2((size_t)bl * d * br * wr, 0.0);
    for (int kr = 0; kr < br; ++kr)
      for (int mr = 0; mr < wr; ++mr)
        for (int po = 0; po < d; ++po)
          for (int ml = 0; ml < wl; ++ml)
            for (int pi = 0; pi < d; ++pi) {
              cd w = W.at(ml, po, pi, mr);
              if (w == cd(0)) continue;
              const cd* t1 = &T1[(size_t)bl * (ml + (size_t)wl * (pi + (size_t)d * kr))];
              cd* t2 = &T2[(size_t)bl * (po + (size_t)d * (kr + (size_t)br * mr))];
              for (int a = 0; a < bl; ++a) t2[a] += t1[a] * w;
            }
    Env En(br, wr, br);
    for (int mr = 0; mr < wr; ++mr)
      blas_gemm(CB_CONJTRANS, CB_NOTRANS, br, br, bl * d, A.v.data(), bl * d, &T2[(size_t)bl * d * br * mr], bl * d,
                &En.v[(size_t)br * mr], br * wr);
    return En;
  }
  // T2[bra_l, ket_r, pout, mr] = sum T1[bra_l, ml, pin, ket_r] W[ml, pout, pin, mr]
  vector<cd> T2((size_t)bl * br * d * wr, 0.0);
  for (int kr = 0; kr < br; ++kr)
    for (int mr = 0; mr < wr; ++mr)
      for (int po = 0; po < d; ++po)
        for (int ml = 0; ml < wl; ++ml)
          for (int pi = 0; pi < d; ++pi) {
            cd w = W.at(ml, po, pi, mr);
            if (w == cd(0)) continue;
            const cd* t1 = &T1[(size_t)bl * (ml + (size_t)wl * (pi + (size_t)d * kr))];
            cd* t2 = &T2[(size_t)bl * (kr + (size_t)br * (po + (size_t)d * mr))];
            for (int a = 0; a < bl; ++a) t2[a] += t1[a] * w;
          }
  // E'[bra_r, mr, ket_r] = sum T2[bl, ket_r, pout, mr] conj(A[bl, pout, bra_r])
  Env En(br, wr, br);
  for (int kr = 0; kr < br; ++kr)
    for (int mr = 0; mr < wr; ++mr)
      for (int b = 0; b < br; ++b) {
        cd s = 0;
        for (int po = 0; po < d; ++po) {
          const cd* t2 = &T2[(size_t)bl * (kr + (size_t)br * (po + (size_t)d * mr))];
          for (int a = 0; a < bl; ++a) s += t2[a] * std::conj(A.at(a, po, b));
        }
        En.at(b, mr, kr) = s;
      }
  return En;
}

// update_right_environment (Algorithms.jl:206-211)
Env update_right(const Ten& A, const Wt& W, const Env& E) {
  const int kl = A.l, d = A.d, kr = A.r, wl = W.wl, wr = W.wr;
  if (g_zgemm) {  // T1 = A E^T, T2 as [pout, br, ket_l, ml] conjugated, E'_ml = conj(A conj(T2_ml))
    vector<cd> T1((size_t)kl * d * kr * wr);
    blas_gemm(CB_NOTRANS, CB_TRANS, kl * d, kr * wr, kr, A.v.data(), kl * d, E.v.data(), kr * wr, T1.data(), kl * d);
    vector<cd> T2((size_t)d * kr * kl * wl, 0.0);
    for (int b = 0; b < kr; ++b)
      for (int a = 0; a < kl; ++a)
        for (int ml = 0; ml < wl; ++ml)
          for (int po = 0; po < d; ++po) {
            cd sum = 0;
            for (int mr = 0; mr < wr; ++mr)
              for (int pi = 0; pi < d; ++pi) {
                cd w = W.at(ml, po, pi, mr);
                if (w == cd(0)) continue;
                sum += w * T1[a + (size_t)kl * (pi + (size_t)d * (b + (size_t)kr * mr))];
              }
            T2[po + (size_t)d * (b + (size_t)kr * (a + (size_t)kl * ml))] = std::conj(sum);
          }
    Env En(kl, wl, kl);
    for (int ml = 0; ml < wl; ++ml)
      blas_gemm(CB_NOTRANS, CB_NOTRANS, kl, kl, d * kr, A.v.data(), kl, &T2[(size_t)d * kr * kl * ml], d * kr,
                &En.v[(size_t)kl * ml], kl * wl);
    for (auto& v : En.v) v = std::conj(v);
    return En;
  }
  // T1[ket_l, pin, bra_r, mr] = sum_k A[ket_l, pin, k] E[bra_r, mr, k]
  vector<cd> T1((size_t)kl * d * kr * wr, 0.0);
  for (int k = 0; k < kr; ++k)
    for (int mr = 0; mr < wr; ++mr)
      for (int b = 0; b < kr; ++b) {
        cd e = E.at(b, mr, k);
        if (e == cd(0)) continue;
        for (int pi = 0; pi < d; ++pi) {
          cd* t1 = &T1[(size_t)kl * (pi + (size_t)d * (b + (size_t)kr * mr))];
          for (int a = 0; a < kl; ++a) t1[a] += A.at(a, pi, k) * e;
        }
      }
  // T2[ml, pout, ket_l, bra_r] = sum W[ml, pout, pin, mr] T1[ket_l, pin, bra_r, mr]
  vector<cd> T2((size_t)wl * d * kl * kr, 0.0);
  for (int b = 0; b < kr; ++b)
    for (int a = 0; a < kl; ++a)
      for (int ml = 0; ml < wl; ++ml)
        for (int po = 0; po < d; ++po) {
          cd s = 0;
          for (int mr = 0; mr < wr; ++mr)
            for (int pi = 0; pi < d; ++pi) {
              cd w = W.at(ml, po, pi, mr);
              if (w == cd(0)) continue;
              s += w * T1[a + (size_t)kl * (pi + (size_t)d * (b + (size_t)kr * mr))];
            }
          T2[ml + (size_t)wl * (po + (size_t)d * (a + (size_t)kl * b))] = s;
        }
  // E'[bra_l, ml, ket_l] = sum T2[ml, pout, ket_l, br] conj(A[bra_l, pout, br])
  Env En(kl, wl, kl);
  for (int a = 0; a < kl; ++a)
    for (int ml = 0; ml < wl; ++ml)
      for (int x = 0; x < kl; ++x) {
        cd s = 0;
        for (int b = 0; b < kr; ++b)
          for (int po = 0; po < d; ++po)
            s += T2[ml + (size_t)wl * (po + (size_t)d * (a + (size_t)kl * b))] * std::conj(A.at(x, po, b));
        En.at(x, ml, a) = s;
      }
  return En;
}

// project_site (Algorithms.jl:215-220, workspace form :330-361).
// x is (chil, D, chir); out is (chil, D, chir).
void project_site(const Env& Le, const Env& Re, const Wt& W, int chil, int D, int chir, const vector<cd>& x,
                  vector<cd>& out) {
  const int wl = W.wl, wr = W.wr;
  // T1[a, ml, pin, c] = sum_k L[a, ml, k] x[k, pin, c]
  vector<cd> T1((size_t)chil * wl * D * chir);
  matmul(chil * wl, D * chir, chil, Le.v.data(), x.data(), T1.data());
  if (g_zgemm) {  // T2 as [a, mr, c, pout]; out_po = T2_po R^T with R as (chir x wr chir)
    vector<cd> T2((size_t)chil * wr * chir * D, 0.0);
    for (int c = 0; c < chir; ++c)
      for (int mr = 0; mr < wr; ++mr)
        for (int po = 0; po < D; ++po)
          for (int ml = 0; ml < wl; ++ml)
            for (int pi = 0; pi < D; ++pi) {
              cd w = W.at(ml, po, pi, mr);
              if (w == cd(0)) continue;
              const cd* t1 = &T1[(size_t)chil * (ml + (size_t)wl * (pi + (size_t)D * c))];
              cd* t2 = &T2[(size_t)chil * (mr + (size_t)wr * (c + (size_t)chir * po))];
              for (int a = 0; a < chil; ++a) t2[a] += t1[a] * w;
            }
    out.assign((size_t)chil * D * chir, 0.0);
    for (int po = 0; po < D; ++po)
      blas_gemm(CB_NOTRANS, CB_TRANS, chil, chir, wr * chir, &T2[(size_t)chil * wr * chir * po], chil, Re.v.data(),
                chir, &out[(size_t)chil * po], chil * D);
    return;
  }
  // T2[a, c, pout, mr] = sum T1[a, ml, pin, c] W[ml, pout, pin, mr]
  vector<cd> T2((size_t)chil * chir * D * wr, 0.0);
  for (int c = 0; c < chir; ++c)
    for (int mr = 0; mr < wr; ++mr)
      for (int po = 0; po < D; ++po)
        for (int ml = 0; ml < wl; ++ml)
          for (int pi = 0; pi < D; ++pi) {
            cd w = W.at(ml, po, pi, mr);
            if (w == cd(0)) continue;
            const cd* t1 = &T1[(size_t)chil * (ml + (size_t)wl * (pi + (size_t)D * c))];
            cd* t2 = &T2[(size_t)chil * (c + (size_t)chir * (po + (size_t)D * mr))];
            for (int a = 0; a < chil; ++a) t2[a] += t1[a] * w;
          }
  // out[a, pout, b] = sum T2[a, c, pout, mr] R[b, mr, c]
  out.assign((size_t)chil * D * chir, 0.0);
  for (int b = 0; b < chir; ++b)
    for (int po = 0; po < D; ++po) {
      cd* o = &out[(size_t)chil * (po + (size_t)D * b)];
      for (int mr = 0; mr < wr; ++mr)
        for (int c = 0; c < chir; ++c) {
          cd r = Re.at(b, mr, c);
          if (r == cd(0)) continue;
          const cd* t2 = &T2[(size_t)chil * (c + (size_t)chir * (po + (size_t)D * mr))];
          for (int a = 0; a < chil; ++a) o[a] += t2[a] * r;
        }
    }
}

inline double heff_flops(int chil, int wl, int D, int chir, int wr) {
  return 8.0 * ((double)chil * chil * wl * D * chir + (double)chil * chir * D * D * wl * wr +
                (double)chil * D * chir * chir * wr);
}

// ---------------------------------------------------------------------------
// MPS gauge operations (MPS.jl:182-311)
// ---------------------------------------------------------------------------
void shift_oc(State& s, int nc) {  // shift_orthogonality_center!, MPS.jl:182-266
  int oc = s.oc;
  if (oc == nc) return;
  if (nc > oc) {
    for (int i = oc; i < nc; ++i) {
      Ten& A = s.t[i];
      vector<cd> Q, R;
      house_qr(A.l * A.d, A.r, A.v.data(), Q, R);
      int rn = std::min(A.l * A.d, A.r);
      Ten An(A.l, A.d, rn);
      An.v = Q;
      Ten& N = s.t[i + 1];
      Ten Nn(rn, N.d, N.r);
      matmul(rn, N.d * N.r, A.r, R.data(), N.v.data(), Nn.v.data());
      A = std::move(An);
      N = std::move(Nn);
    }
  } else {
    for (int i = oc; i > nc; --i) {
      Ten& A = s.t[i];
      vector<cd> Lm, Qm;
      house_lq(A.l, A.d * A.r, A.v.data(), Lm, Qm);
      int rn = std::min(A.l, A.d * A.r);
      Ten An(rn, A.d, A.r);
      An.v = Qm;
      Ten& P = s.t[i - 1];
      Ten Pn(P.l, P.d, rn);
      matmul(P.l * P.d, rn, P.r, P.v.data(), Lm.data(), Pn.v.data());
      A = std::move(An);
      P = std::move(Pn);
    }
  }
  s.oc = nc;
}

void normalize_mps(State& s) {  // normalize!, MPS.jl:274-311
  for (int i = s.L - 1; i >= 1; --i) {
    Ten& A = s.t[i];
    vector<cd> Lm, Qm;
    house_lq(A.l, A.d * A.r, A.v.data(), Lm, Qm);
    int rn = std::min(A.l, A.d * A.r);
    Ten An(rn, A.d, A.r);
    An.v = Qm;
    Ten& P = s.t[i - 1];
    Ten Pn(P.l, P.d, rn);
    matmul(P.l * P.d, rn, P.r, P.v.data(), Lm.data(), Pn.v.data());
    A = std::move(An);
    P = std::move(Pn);
  }
  Ten& A1 = s.t[0];
  double nr = nrm2(A1.v.data(), (long)A1.v.size());
  if (nr > 1e-13)
    for (auto& x : A1.v) x *= (1.0 / nr);
  s.oc = 0;
}

cd scalar_product(const State& s) {  // scalar_product(psi, psi), MPS.jl:528-585
  vector<cd> E(1, 1.0);
  int eb = 1;
  for (int i = 0; i < s.L; ++i) {
    const Ten& A = s.t[i];
    // E'[ra, rb] = sum E[la, lb] A[la, p, ra] conj(A[lb, p, rb])
    vector<cd> T1((size_t)A.l * A.d * A.r, 0.0);  // T1[lb, p, ra] = sum_la E[la, lb] A[la, p, ra]
    for (int ra = 0; ra < A.r; ++ra)
      for (int p = 0; p < A.d; ++p)
        for (int lb = 0; lb < A.l; ++lb) {
          cd sacc = 0;
          for (int la = 0; la < A.l; ++la) sacc += E[la + (size_t)eb * lb] * A.at(la, p, ra);
          T1[lb + (size_t)A.l * (p + (size_t)A.d * ra)] = sacc;
        }
    vector<cd> En((size_t)A.r * A.r, 0.0);
    for (int rb = 0; rb < A.r; ++rb)
      for (int ra = 0; ra < A.r; ++ra) {
        cd sacc = 0;
        for (int p = 0; p < A.d; ++p)
          for (int lb = 0; lb < A.l; ++lb)
            sacc += T1[lb + (size_t)A.l * (p + (size_t)A.d * ra)] * std::conj(A.at(lb, p, rb));
        En[ra + (size_t)A.r * rb] = sacc;
      }
    E.swap(En);
    eb = A.r;
  }
  return E[0];
}

// scalar_product(psi, phi) of MPS.jl:528-585 for two states: the code
// contracts psi with conj(phi), so this is sum psi * conj(phi) = <phi|psi>.
cd scalar_product(const State& psi, const State& phi) {
  vector<cd> E(1, 1.0);  // E[la, lb], leading dimension ea
  int ea = 1;
  for (int i = 0; i < psi.L; ++i) {
    const Ten& A = psi.t[i];
    const Ten& B = phi.t[i];
    vector<cd> En((size_t)A.r * B.r, 0.0);
    for (int rb = 0; rb < B.r; ++rb)
      for (int ra = 0; ra < A.r; ++ra) {
        cd acc = 0;
        for (int p = 0; p < A.d; ++p)
          for (int lb = 0; lb < B.l; ++lb)
            for (int la = 0; la < A.l; ++la)
              acc += E[la + (size_t)ea * lb] * A.at(la, p, ra) * std::conj(B.at(lb, p, rb));
        En[ra + (size_t)A.r * rb] = acc;
      }
    E.swap(En);
    ea = A.r;
  }
  return E[0];
}

void apply_1site(Ten& A, const cd* op) {  // T[l,p,r] <- sum_k op[p,k] T[l,k,r]
  Ten B(A.l, A.d, A.r);
  for (int r = 0; r < A.r; ++r)
    for (int p = 0; p < A.d; ++p)
      for (int l = 0; l < A.l; ++l) {
        cd sacc = 0;
        for (int k = 0; k < A.d; ++k) sacc += op[p + A.d * k] * A.at(l, k, r);
        B.at(l, p, r) = sacc;
      }
  A = std::move(B);
}

Ten merge(const Ten& A1, const Ten& A2) {  // Theta[l, p1, p2, r] as (l, 4, r), p = p1 + 2 p2
  Ten T(A1.l, A1.d * A2.d, A2.r);
  matmul(A1.l * A1.d, A2.d * A2.r, A1.r, A1.v.data(), A2.v.data(), T.v.data());
  return T;
}

void apply_2site(Ten& T, const cd* op) {  // op (4x4) on the merged index p1 + 2 p2
  Ten B(T.l, T.d, T.r);
  for (int r = 0; r < T.r; ++r)
    for (int p = 0; p < T.d; ++p)
      for (int l = 0; l < T.l; ++l) {
        cd sacc = 0;
        for (int k = 0; k < T.d; ++k) sacc += op[p + T.d * k] * T.at(l, k, r);
        B.at(l, p, r) = sacc;
      }
  T = std::move(B);
}

double tnorm2(const Ten& A) {
  double s = 0;
  for (auto& x : A.v) s += std::norm(x);
  return s;
}

// Split Theta (l, 4, r) by SVD into left (l,2,keep) and right (keep,2,r)
// tensors; rule 0 = TDVP (absolute, min 2), 1 = relative.  With s_left the
// singular values go left (U S | Vt, Vt orthonormal); otherwise right
// (U | S Vt, U orthonormal).  The scaled factor is the product with M,
// exactly zero for null singular values.
void split_theta(const Ten& Th, int rule, double thr, int max_bond, bool s_left, Ten& Lo, Ten& Ro, Counters& cnt) {
  const int m = Th.l * 2, n = 2 * Th.r;
  vector<cd> M = Th.v;
  bool bad = false;
  for (auto& x : M)
    if (!std::isfinite(x.real()) || !std::isfinite(x.imag())) {
      x = 0.0;
      bad = true;
    }
  if (bad) cnt.nonfinite++;
  SvdOut o = svd_side(m, n, M.data(), s_left ? SVD_RIGHT : SVD_LEFT);
  cnt.svds++;
  const int keep = rule == 0   ? keep_tdvp(o.S, thr, max_bond)
                   : rule == 1 ? keep_relative(o.S, thr, max_bond)
                   : rule == 2 ? keep_tebd(o.S, thr, max_bond)
                               : std::max(1, std::min((int)o.S.size(), max_bond));  // dynamic TDVP split
  vector<cd> Y = svd_vectors(o, keep);
  Lo = Ten(Th.l, 2, keep);
  Ro = Ten(keep, 2, Th.r);
  if (!s_left) {  // U = Y (m x keep), S Vt = Y^H M
    for (int j = 0; j < keep; ++j)
      for (int i = 0; i < m; ++i) Lo.v[i + (size_t)m * j] = Y[i + (size_t)m * j];
    for (int c = 0; c < n; ++c)
      for (int kk = 0; kk < keep; ++kk) {
        if (kk >= o.rank) continue;
        cd sacc = 0;
        for (int r = 0; r < m; ++r) sacc += std::conj(Y[r + (size_t)m * kk]) * M[r + (size_t)m * c];
        Ro.v[kk + (size_t)keep * c] = sacc;
      }
  } else {  // Vt = Y^H (keep x n), U S = M Y
    for (int c = 0; c < n; ++c)
      for (int kk = 0; kk < keep; ++kk) Ro.v[kk + (size_t)keep * c] = std::conj(Y[c + (size_t)n * kk]);
    for (int kk = 0; kk < keep; ++kk) {
      if (kk >= o.rank) continue;
      for (int i = 0; i < m; ++i) {
        cd sacc = 0;
        for (int c = 0; c < n; ++c) sacc += M[i + (size_t)m * c] * Y[c + (size_t)n * kk];
        Lo.v[i + (size_t)m * kk] = sacc;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Problem definition (host copies of the C-ABI descriptors)
// ---------------------------------------------------------------------------
struct NoiseProc {
  int nsites;
  int s0, s1;
  double gamma;
  cd mat[16];
  bool pauli_name, pauli_proc;
  cd diss_half[16];  // expm(-0.5*dt*gamma*L^dag L) for dt/2 (computed per run)
  cd diss_full[16];  // ... for dt
  // Long-range process (MPONoiseProcess, Noise.jl:22-33) on s0 < s1 - 1:
  // O = alpha*1 + beta*(sig at s0)(tau at s1) (build_mpo_phys, Noise.jl:71-131).
  // pauli_proc marks the "pauli_long_range" candidate (StochasticProcess.jl:
  // 176-185), otherwise "mpo_general"; diss_rate is the scalar decay rate of
  // handle_longrange_scalar! (Dissipation.jl:161-204).
  bool lr = false;
  cd sig[4], tau[4], alpha, beta;
  double diss_rate = 0.0;
};

struct Obs {
  int kind;
  int s0, s1;
  cd mat[16];
};

struct NoiseSet {  // a NoiseModel: `present` == false means `nothing`
  bool present = false;
  bool all_zero = true;
  vector<NoiseProc> procs;
};

// W_group of two neighbouring MPO tensors (Algorithms.jl:639-643).
Wt merge_wt(const Wt& W1, const Wt& Wn) {
  Wt G(W1.wl, 4, Wn.wr);
  for (int l = 0; l < W1.wl; ++l)
    for (int r = 0; r < Wn.wr; ++r)
      for (int p1o = 0; p1o < 2; ++p1o)
        for (int p2o = 0; p2o < 2; ++p2o)
          for (int p1i = 0; p1i < 2; ++p1i)
            for (int p2i = 0; p2i < 2; ++p2i) {
              cd sacc = 0;
              for (int k = 0; k < W1.wr; ++k) sacc += W1.at(l, p1o, p1i, k) * Wn.at(k, p2o, p2i, r);
              G.at(l, p1o + 2 * p2o, p1i + 2 * p2i, r) = sacc;
            }
  return G;
}

struct Problem {
  int L;
  vector<Wt> W;
  vector<Wt> W2;  // merged two-site W_group (Algorithms.jl:639-643), index i for sites (i, i+1)
  State psi0;
  NoiseSet noise;
  vector<Obs> obs;
  double dt;
  int n_times, num_traj, max_bond, order;
  double thr;
  bool sample_timesteps;
  KrylovParams kp;
  int rng_mode;
  uint64_t seed;
  const double* uniforms;
  long long stride;
  int traj_offset;
  int tdvp_mode = YAQS_TDVP_2SITE;
  int local_method = YAQS_METHOD_TEBD, long_range_method = YAQS_METHOD_TEBD;  // digital
};

// Hermitian matrix exponential exp(c * H) for small H (n<=4) via Jacobi on
// the 2n x 2n real embedding-free approach: eigendecompose Hermitian H with
// complex Jacobi rotations.
void herm_expm(int n, const cd* H, double c, cd* out) {
  vector<cd> A(H, H + n * n), V(n * n, 0.0);
  for (int i = 0; i < n; ++i) V[i + n * i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        if (i != j) off += std::norm(A[i + n * j]);
    if (off < 1e-34) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        cd apq = A[p + n * q];
        double ag = std::abs(apq);
        if (ag == 0.0) continue;
        double app = A[p + n * p].real(), aqq = A[q + n * q].real();
        double zeta = (aqq - app) / (2.0 * ag);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        double cc = 1.0 / std::sqrt(1.0 + t * t), s = cc * t;
        cd e = apq / ag;
        // J = [[cc, s e],[-s conj(e), cc]] acting on columns p,q: A <- J^H A J
        for (int k = 0; k < n; ++k) {
          cd x = A[k + n * p], y = A[k + n * q];
          A[k + n * p] = cc * x - s * std::conj(e) * y;
          A[k + n * q] = s * e * x + cc * y;
        }
        for (int k = 0; k < n; ++k) {
          cd x = A[p + n * k], y = A[q + n * k];
          A[p + n * k] = cc * x - s * e * y;
          A[q + n * k] = s * std::conj(e) * x + cc * y;
        }
        for (int k = 0; k < n; ++k) {
          cd x = V[k + n * p], y = V[k + n * q];
          V[k + n * p] = cc * x - s * std::conj(e) * y;
          V[k + n * q] = s * e * x + cc * y;
        }
      }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      cd sacc = 0;
      for (int k = 0; k < n; ++k) sacc += V[i + n * k] * std::exp(c * A[k + n * k].real()) * std::conj(V[j + n * k]);
      out[i + n * j] = sacc;
    }
}

// ---------------------------------------------------------------------------
// Uniform draws
// ---------------------------------------------------------------------------
inline void philox_round(uint32_t* c, const uint32_t* k) {
  const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
  const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
  uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
  uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
  uint32_t n0 = hi1 ^ c[1] ^ k[0];
  uint32_t n1 = lo1;
  uint32_t n2 = hi0 ^ c[3] ^ k[1];
  uint32_t n3 = lo0;
  c[0] = n0;
  c[1] = n1;
  c[2] = n2;
  c[3] = n3;
}

// Philox-4x32-10 (Salmon et al., SC'11).  Counter = (draw lo, draw hi,
// stream lo, stream hi), key = seed.  Returns a 53-bit double in [0,1).
double philox_uniform(uint64_t seed, uint64_t stream, uint64_t draw) {
  uint32_t c[4] = {(uint32_t)draw, (uint32_t)(draw >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
  uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int r = 0; r < 10; ++r) {
    philox_round(c, k);
    if (r < 9) {
      k[0] += 0x9E3779B9u;
      k[1] += 0xBB67AE85u;
    }
  }
  uint64_t bits = ((uint64_t)c[1] << 32) | c[0];
  return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
}

struct Draws {
  const Problem* P;
  long long traj;
  long long pos = 0;
  bool exhausted = false;
  double next() {
    if (P->rng_mode == YAQS_RNG_INJECTED) {
      if (pos >= P->stride) {
        exhausted = true;
        return 1.0;
      }
      return P->uniforms[traj * P->stride + pos++];
    }
    return philox_uniform(P->seed, (uint64_t)(P->traj_offset + traj), (uint64_t)pos++);
  }
};

// ---------------------------------------------------------------------------
// Two-site TDVP, Hamiltonian symmetric sweep (Algorithms.jl:580-603, 631-760)
// ---------------------------------------------------------------------------
struct Sweeper {
  const Problem& P;
  Counters& cnt;
  vector<Env> EL, ER;

  Sweeper(const Problem& p, Counters& c) : P(p), cnt(c) {}

  vector<cd> evolve(const Env& Le, const Env& Re, const Wt& W, const Ten& x, double dt) {
    auto op = [&](const vector<cd>& in, vector<cd>& out) {
      project_site(Le, Re, W, x.l, x.d, x.r, in, out);
      cnt.flops += heff_flops(x.l, W.wl, x.d, x.r, W.wr);
    };
    return expm_krylov(op, x.v, dt, P.kp, cnt);
  }

  void init_envs(State& s) {  // _init_envs, Algorithms.jl:802-819
    const int L = s.L;
    ER.assign(L + 1, Env());
    EL.assign(L + 1, Env());
    ER[L] = identity_env(s.t[L - 1].r, P.W[L - 1].wr);
    for (int i = L - 1; i >= 1; --i) ER[i] = update_right(s.t[i], P.W[i], ER[i + 1]);
    EL[0] = identity_env(s.t[0].l, P.W[0].wl);
  }

  // _two_site_update_forward! (Algorithms.jl:631-672), evolve_back = true
  void forward(State& s, int i, double dts) {
    Ten Th = merge(s.t[i], s.t[i + 1]);
    Th.v = evolve(EL[i], ER[i + 2], P.W2[i], Th, dts);
    Ten U, V;
    split_theta(Th, 0, P.thr, P.max_bond, false, U, V, cnt);
    s.t[i] = U;
    EL[i + 1] = update_left(s.t[i], P.W[i], EL[i]);
    V.v = evolve(EL[i + 1], ER[i + 2], P.W[i + 1], V, -dts);
    s.t[i + 1] = V;
  }

  // _two_site_update_edge_hamiltonian! (Algorithms.jl:674-711) and the
  // second half of _two_site_update_backward_precorrect! (:729-759).
  void split_left(State& s, int i, double dts) {
    Ten Th = merge(s.t[i], s.t[i + 1]);
    Th.v = evolve(EL[i], ER[i + 2], P.W2[i], Th, dts);
    Ten U, V;
    split_theta(Th, 0, P.thr, P.max_bond, true, U, V, cnt);
    s.t[i + 1] = V;
    ER[i + 1] = update_right(s.t[i + 1], P.W[i + 1], ER[i + 2]);
    s.t[i] = U;
  }

  void backward(State& s, int i, double dts) {  // Algorithms.jl:713-760
    s.t[i + 1].v = evolve(EL[i + 1], ER[i + 2], P.W[i + 1], s.t[i + 1], -dts);
    split_left(s, i, dts);
  }

  void sweep(State& s) {
    if (P.tdvp_mode == YAQS_TDVP_1SITE)
      sweep_1site(s);
    else if (P.tdvp_mode == YAQS_TDVP_DYNAMIC)
      sweep_dynamic(s);
    else
      sweep_2site(s);
  }

  void sweep_2site(State& s) {  // _tdvp_sweep_hamiltonian_2site!, Algorithms.jl:580-603
    shift_oc(s, 0);
    const int L = s.L;
    const double dt = P.dt;
    init_envs(s);
    for (int i = 0; i <= L - 3; ++i) forward(s, i, dt / 2);
    if (L >= 2) split_left(s, L - 2, dt);
    for (int i = L - 3; i >= 0; --i) backward(s, i, dt / 2);
  }

  // exp(-i dt H_bond) C for the bond matrix C (k x r) between EL and ER
  // (project_bond, Algorithms.jl:222-226).
  vector<cd> evolve_bond(const Env& Le, const Env& Re, int k, int r, const vector<cd>& C, double dt) {
    auto op = [&](const vector<cd>& in, vector<cd>& out) {
      const int w = Le.w;
      // T1[a, m, kr] = sum_k L[a, m, k] C[k, kr];  out[a, b] = sum_{m, kr} T1[a, m, kr] R[b, m, kr]
      vector<cd> T1((size_t)Le.b * w * r);
      matmul(Le.b * w, r, k, Le.v.data(), in.data(), T1.data());
      out.assign((size_t)Le.b * Re.b, 0.0);
      for (int b = 0; b < Re.b; ++b)
        for (int kr = 0; kr < r; ++kr)
          for (int m = 0; m < w; ++m) {
            const cd rv = Re.at(b, m, kr);
            if (rv == cd(0)) continue;
            const cd* t = &T1[(size_t)Le.b * (m + (size_t)w * kr)];
            cd* o = &out[(size_t)Le.b * b];
            for (int a = 0; a < Le.b; ++a) o[a] += t[a] * rv;
          }
      cnt.flops += 8.0 * ((double)Le.b * w * k * r + (double)Le.b * w * r * Re.b);
    };
    return expm_krylov(op, C, dt, P.kp, cnt);
  }

  // site i = Q R (thin QR), Q -> site i, EL[i+1], R evolved by dtb and
  // absorbed into site i+1.
  void qr_bond_forward(State& s, int i, double dtb) {
    Ten& A = s.t[i];
    vector<cd> Q, R;
    house_qr(A.l * A.d, A.r, A.v.data(), Q, R);
    const int rn = std::min(A.l * A.d, A.r), r = A.r;
    Ten An(A.l, A.d, rn);
    An.v = Q;
    A = std::move(An);
    EL[i + 1] = update_left(s.t[i], P.W[i], EL[i]);
    R = evolve_bond(EL[i + 1], ER[i + 1], rn, r, R, dtb);
    Ten& N = s.t[i + 1];
    Ten Nn(rn, N.d, N.r);
    matmul(rn, N.d * N.r, r, R.data(), N.v.data(), Nn.v.data());
    N = std::move(Nn);
  }

  // site i = L Q (thin LQ), Q -> site i, ER[i], L evolved by dtb and
  // absorbed into site i-1.
  void lq_bond_backward(State& s, int i, double dtb) {
    Ten& A = s.t[i];
    vector<cd> Lm, Qm;
    house_lq(A.l, A.d * A.r, A.v.data(), Lm, Qm);
    const int rn = std::min(A.l, A.d * A.r), l = A.l;
    Ten An(rn, A.d, A.r);
    An.v = Qm;
    A = std::move(An);
    ER[i] = update_right(s.t[i], P.W[i], ER[i + 1]);
    Lm = evolve_bond(EL[i], ER[i], l, rn, Lm, dtb);
    Ten& Pv = s.t[i - 1];
    Ten Pn(Pv.l, Pv.d, rn);
    matmul(Pv.l * Pv.d, rn, l, Pv.v.data(), Lm.data(), Pn.v.data());
    Pv = std::move(Pn);
  }

  void evolve_site(State& s, int i, double dts) {
    s.t[i].v = evolve(EL[i], ER[i + 1], P.W[i], s.t[i], dts);
  }

  // _tdvp_sweep_hamiltonian_1site!, Algorithms.jl:472-533
  void sweep_1site(State& s) {
    shift_oc(s, 0);
    const int L = s.L;
    const double dt = P.dt;
    init_envs(s);
    for (int i = 0; i < L; ++i) {
      evolve_site(s, i, dt / 2);
      if (i < L - 1) qr_bond_forward(s, i, -dt / 2);
    }
    for (int i = L - 1; i >= 0; --i) {
      evolve_site(s, i, dt / 2);
      if (i > 0) lq_bond_backward(s, i, -dt / 2);
    }
    s.oc = 0;
  }

  // local_dynamic_tdvp (mqt-yaqs/src/mqt/yaqs/core/methods/tdvp.py:667-855),
  // in the Julia tensor layout: a 2-site update (split keeping
  // min(rank, max_bond) values) while the bond is below max_bond, else a
  // 1-site update with bond back-evolution; the last site (first site on
  // the way back) takes a 1-site update once a 1-site step reached it.
  void sweep_dynamic(State& s) {
    shift_oc(s, 0);
    const int L = s.L;
    const double dt = P.dt;
    init_envs(s);
    bool lock = false;
    for (int i = 0; i < L; ++i) {  // left to right (tdvp.py:706-781)
      const int bond = s.t[i].r;
      if (bond >= P.max_bond || lock) {
        evolve_site(s, i, dt / 2);
        if (i != L - 1) qr_bond_forward(s, i, -dt / 2);
        if (i == L - 2) lock = true;
      } else if (i == L - 1) {
        continue;
      } else {
        Ten Th = merge(s.t[i], s.t[i + 1]);
        Th.v = evolve(EL[i], ER[i + 2], P.W2[i], Th, dt / 2);
        Ten U, V;
        split_theta(Th, 3, P.thr, P.max_bond, false, U, V, cnt);
        s.t[i] = U;
        s.t[i + 1] = V;
        EL[i + 1] = update_left(s.t[i], P.W[i], EL[i]);
        if (i != L - 2) s.t[i + 1].v = evolve(EL[i + 1], ER[i + 2], P.W[i + 1], s.t[i + 1], -dt / 2);
      }
    }
    lock = false;
    for (int i = L - 1; i >= 0; --i) {  // right to left (tdvp.py:786-855)
      const int bond = s.t[i].l;
      if (bond >= P.max_bond || lock) {
        evolve_site(s, i, dt / 2);
        if (i != 0) {
          lq_bond_backward(s, i, -dt / 2);
          if (i == 1) lock = true;
        }
      } else if (i == 0) {
        continue;
      } else {
        Ten Th = merge(s.t[i - 1], s.t[i]);
        Th.v = evolve(EL[i - 1], ER[i + 1], P.W2[i - 1], Th, dt / 2);
        Ten U, V;
        split_theta(Th, 3, P.thr, P.max_bond, true, U, V, cnt);
        s.t[i - 1] = U;
        s.t[i] = V;
        ER[i] = update_right(s.t[i], P.W[i], ER[i + 1]);
        if (i != 1) s.t[i - 1].v = evolve(EL[i - 1], ER[i], P.W[i - 1], s.t[i - 1], -dt / 2);
      }
    }
    s.oc = 0;
  }
};

// ---------------------------------------------------------------------------
// Dissipation (Dissipation.jl:37-159), local processes
// ---------------------------------------------------------------------------
void apply_dissipation(const Problem& P, const NoiseSet& N, State& s, bool full_dt, double dt, Counters& cnt) {
  const int L = s.L;
  if (!N.present || N.all_zero) {  // :39-47
    for (int i = L - 1; i >= 1; --i) shift_oc(s, i - 1);
    return;
  }
  for (int i = L - 1; i >= 0; --i) {
    for (const auto& pr : N.procs) {
      if (pr.nsites == 1 && pr.s0 == i) {
        if (pr.pauli_name) {
          double f = std::exp(-0.5 * dt * pr.gamma);
          for (auto& x : s.t[i].v) x *= f;
        } else {
          apply_1site(s.t[i], full_dt ? pr.diss_full : pr.diss_half);
        }
      }
    }
    if (i > 0) {
      for (const auto& pr : N.procs) {
        if (pr.nsites == 2 && pr.s1 == i) {
          if (pr.lr) {  // handle_longrange_scalar! (Dissipation.jl:161-204)
            double f = std::exp(-0.5 * dt * pr.diss_rate);
            for (auto& x : s.t[i].v) x *= f;
          } else if (pr.pauli_name) {
            double f = std::exp(-0.5 * dt * pr.gamma);
            for (auto& x : s.t[i].v) x *= f;
          } else {
            Ten Th = merge(s.t[i - 1], s.t[i]);
            apply_2site(Th, full_dt ? pr.diss_full : pr.diss_half);
            Ten U, V;
            split_theta(Th, 1, P.thr, P.max_bond, false, U, V, cnt);
            s.t[i - 1] = U;
            s.t[i] = V;
          }
        }
      }
      shift_oc(s, i - 1);
    }
  }
}

// ---------------------------------------------------------------------------
// Stochastic process (StochasticProcess.jl:35-38, 89-212, 219-330)
// ---------------------------------------------------------------------------
// MPS.truncate! (MPS.jl:320-440): centre to site 1, one SVD sweep 1 -> L-1
// with the absolute min-2 rule (keep the crossing value, at most
// max_bond_dim), then normalize!.
void mps_truncate(const Problem& P, State& s, Counters& cnt) {
  shift_oc(s, 0);
  for (int i = 0; i + 1 < s.L; ++i) {
    Ten Th = merge(s.t[i], s.t[i + 1]);
    Ten U, V;
    split_theta(Th, 0, P.thr, P.max_bond, false, U, V, cnt);
    s.t[i] = std::move(U);
    s.t[i + 1] = std::move(V);
  }
  s.oc = s.L - 1;
  normalize_mps(s);
}

// MPO of a long-range process (build_mpo_phys, Noise.jl:71-131): identity
// outside [s0, s1]; row [1, sig] at s0; diag(1, 1) in between; column
// [alpha 1; beta tau] at s1.  Tensors (wl, out, in, wr).
Wt lr_mpo_site(const NoiseProc& pr, int k) {
  const int a = pr.s0, b = pr.s1;
  const int wl = (k > a && k <= b) ? 2 : 1, wr = (k >= a && k < b) ? 2 : 1;
  Wt W(wl, 2, wr);
  for (int po = 0; po < 2; ++po)
    for (int pi = 0; pi < 2; ++pi) {
      const cd id = po == pi ? 1.0 : 0.0;
      if (k < a || k > b) {
        W.at(0, po, pi, 0) = id;
      } else if (k == a) {
        W.at(0, po, pi, 0) = id;
        W.at(0, po, pi, 1) = pr.sig[po + 2 * pi];
      } else if (k < b) {
        W.at(0, po, pi, 0) = id;
        W.at(1, po, pi, 1) = id;
      } else {
        W.at(0, po, pi, 0) = pr.alpha * id;
        W.at(1, po, pi, 0) = pr.beta * pr.tau[po + 2 * pi];
      }
    }
  return W;
}

// apply_mpo_jump! (StochasticProcess.jl:46-82): contract the MPO into the
// MPS site by site, C[la,lw,po,ra,rw] = sum_pi A[la,pi,ra] W[lw,po,pi,rw]
// reshaped to (la*lw, po, ra*rw), then truncate!.
void apply_mpo_jump(const Problem& P, State& s, const NoiseProc& pr, Counters& cnt) {
  for (int k = 0; k < s.L; ++k) {
    const Ten& A = s.t[k];
    const Wt W = lr_mpo_site(pr, k);
    Ten C(A.l * W.wl, 2, A.r * W.wr);
    for (int rw = 0; rw < W.wr; ++rw)
      for (int ra = 0; ra < A.r; ++ra)
        for (int po = 0; po < 2; ++po)
          for (int lw = 0; lw < W.wl; ++lw)
            for (int la = 0; la < A.l; ++la) {
              cd acc = 0;
              for (int pi = 0; pi < 2; ++pi) acc += A.at(la, pi, ra) * W.at(lw, po, pi, rw);
              C.at(la + A.l * lw, po, ra + A.r * rw) = acc;
            }
    s.t[k] = std::move(C);
  }
  mps_truncate(P, s, cnt);
}

struct Cand {
  const NoiseProc* pr;
  double dp;
};

// create_probability_distribution (StochasticProcess.jl:89-212): the jump
// candidates in the reference's order with their unnormalised weights
// dt gamma ||L psi||^2 (1-site in site order, then 2-site adjacent, then the
// long-range processes).  Moves the orthogonality centre.
vector<Cand> jump_candidates(const Problem& P, const NoiseSet& N, State& s, double dt) {
  const int L = s.L;
  vector<Cand> cands;
  for (int site = 0; site < L; ++site) {
    shift_oc(s, site);
    for (const auto& pr : N.procs) {
      if (pr.nsites == 1 && pr.s0 == site) {
        double nr;
        if (pr.pauli_proc) {
          nr = tnorm2(s.t[site]);
        } else {
          Ten T = s.t[site];
          apply_1site(T, pr.mat);
          nr = tnorm2(T);
        }
        cands.push_back({&pr, dt * pr.gamma * nr});
      }
    }
    if (site < L - 1) {
      for (const auto& pr : N.procs) {
        if (pr.nsites == 2 && !pr.lr && pr.s0 == site) {
          double nr;
          if (pr.pauli_proc) {
            nr = tnorm2(s.t[site]);
          } else {
            Ten Th = merge(s.t[site], s.t[site + 1]);
            apply_2site(Th, pr.mat);
            nr = tnorm2(Th);
          }
          cands.push_back({&pr, dt * pr.gamma * nr});
        }
      }
    }
  }
  // long-range processes, after every local candidate (StochasticProcess.jl:169-202)
  for (const auto& pr : N.procs) {
    if (!pr.lr) continue;
    double nr;
    if (pr.pauli_proc) {
      nr = tnorm2(s.t[s.oc]);
    } else {  // applied to a copy, truncated and renormalised, then its norm
      State tmp = s;
      Counters scratch{};
      apply_mpo_jump(P, tmp, pr, scratch);
      nr = tnorm2(tmp.t[tmp.oc]);
    }
    cands.push_back({&pr, dt * pr.gamma * nr});
  }
  return cands;
}

bool stochastic_process(const Problem& P, const NoiseSet& N, State& s, double dt, Draws& rng, Counters& cnt) {
  double dp = 1.0 - scalar_product(s).real();
  if (N.procs.empty() || rng.next() >= dp) {
    shift_oc(s, 0);
    normalize_mps(s);
    return false;
  }
  vector<Cand> cands = jump_candidates(P, N, s, dt);
  double total = 0;
  for (auto& c : cands) total += c.dp;
  if (total == 0.0) {
    shift_oc(s, 0);
    normalize_mps(s);
    return false;
  }
  double r = rng.next();
  double acc = 0;
  size_t chosen = 0;
  for (size_t i = 0; i < cands.size(); ++i) {
    acc += cands[i].dp / total;
    if (r <= acc) {
      chosen = i;
      break;
    }
  }
  const NoiseProc& pr = *cands[chosen].pr;
  if (pr.lr) {
    // "pauli_long_range" has no branch of its own in the reference
    // (StochasticProcess.jl:311 tests "mpo_pauli"), so only the final
    // normalisation acts; "mpo_general" applies the operator.
    if (!pr.pauli_proc) apply_mpo_jump(P, s, pr, cnt);
  } else if (pr.nsites == 1) {
    shift_oc(s, pr.s0);
    apply_1site(s.t[pr.s0], pr.mat);
  } else {
    shift_oc(s, pr.s0);
    Ten Th = merge(s.t[pr.s0], s.t[pr.s0 + 1]);
    apply_2site(Th, pr.mat);
    Ten U, V;
    split_theta(Th, 1, P.thr, P.max_bond, false, U, V, cnt);
    s.t[pr.s0] = U;
    s.t[pr.s0 + 1] = V;
  }
  cnt.jumps++;
  normalize_mps(s);
  return true;
}

// ---------------------------------------------------------------------------
// Observables (SimulationConfigs.jl:42-56, MPS.jl:608-651)
// ---------------------------------------------------------------------------
double measure(const Obs& o, State& s) {
  if (o.kind == YAQS_OBS_LOCAL1) {
    shift_oc(s, o.s0);
    const Ten& A = s.t[o.s0];
    cd acc = 0;
    for (int r = 0; r < A.r; ++r)
      for (int l = 0; l < A.l; ++l)
        for (int p = 0; p < 2; ++p) {
          cd oa = 0;
          for (int k = 0; k < 2; ++k) oa += o.mat[p + 2 * k] * A.at(l, k, r);
          acc += std::conj(A.at(l, p, r)) * oa;
        }
    return acc.real();
  }
  if (o.kind == YAQS_OBS_LOCAL2) {
    shift_oc(s, o.s0);
    Ten Th = merge(s.t[o.s0], s.t[o.s0 + 1]);
    cd acc = 0;
    for (int r = 0; r < Th.r; ++r)
      for (int l = 0; l < Th.l; ++l)
        for (int p = 0; p < 4; ++p) {
          cd oa = 0;
          for (int k = 0; k < 4; ++k) oa += o.mat[p + 4 * k] * Th.at(l, k, r);
          acc += std::conj(Th.at(l, p, r)) * oa;
        }
    return acc.real();
  }
  // ENTROPY across the bond (s0, s0+1): Schmidt values of the center tensor.
  shift_oc(s, o.s0);
  const Ten& A = s.t[o.s0];
  const vector<double> S = svd_side(A.l * A.d, A.r, A.v.data(), SVD_LEFT).S;
  double nsq = 0;
  for (double x : S) nsq += x * x;
  double ent = 0;
  for (double x : S) {
    double p = x * x / nsq;
    if (p > 0) ent -= p * std::log(p);
  }
  return ent;
}

int max_bond(const State& s) {  // write_max_bond_dim, MPS.jl:168-174
  int m = 0;
  for (const auto& t : s.t) m = std::max(m, std::max(t.l, t.r));
  return m;
}

void evaluate(const Problem& P, State& s, double* out, int col, int ncols, int* chi_out) {
  for (size_t k = 0; k < P.obs.size(); ++k) out[k * ncols + col] = measure(P.obs[k], s);
  if (chi_out) chi_out[col] = max_bond(s);
}

// ---------------------------------------------------------------------------
// Trajectories (AnalogTJM.jl:21-176)
// ---------------------------------------------------------------------------
int run_trajectory(const Problem& P, long long traj, double* out, int* chi_out, Counters& cnt) {
  State s = P.psi0;  // deepcopy (AnalogTJM.jl:110)
  normalize_mps(s);  // Simulator.run normalises psi0 (Simulator.jl:128)
  Draws rng{&P, traj};
  const int nobs = (int)P.obs.size();
  const int ncols = P.sample_timesteps ? P.n_times : 1;
  const double dt = P.dt;
  Sweeper sw(P, cnt);
  if (P.order == 2) {
    if (P.sample_timesteps) evaluate(P, s, out, 0, ncols, chi_out);
    // initialize (AnalogTJM.jl:21-33)
    apply_dissipation(P, P.noise, s, false, dt / 2, cnt);
    if (P.noise.present) stochastic_process(P, P.noise, s, dt, rng, cnt);
    auto sample = [&](int j) {  // AnalogTJM.jl:62-81
      State psi = s;
      sw.sweep(psi);
      apply_dissipation(P, P.noise, psi, false, dt / 2, cnt);
      if (P.noise.present) stochastic_process(P, P.noise, psi, dt, rng, cnt);
      evaluate(P, psi, out, P.sample_timesteps ? j : 0, ncols, chi_out);
    };
    if (P.sample_timesteps && P.n_times > 1) sample(1);
    for (int j = 2; j < P.n_times; ++j) {
      sw.sweep(s);  // step_through (AnalogTJM.jl:40-55)
      apply_dissipation(P, P.noise, s, true, dt, cnt);
      if (P.noise.present) stochastic_process(P, P.noise, s, dt, rng, cnt);
      if (P.sample_timesteps || j == P.n_times - 1) sample(j);
    }
  } else {
    if (P.sample_timesteps) evaluate(P, s, out, 0, ncols, chi_out);
    for (int j = 1; j < P.n_times; ++j) {
      sw.sweep(s);
      if (P.noise.present) {
        apply_dissipation(P, P.noise, s, true, dt, cnt);
        stochastic_process(P, P.noise, s, dt, rng, cnt);
      }
      if (P.sample_timesteps)
        evaluate(P, s, out, j, ncols, chi_out);
      else if (j == P.n_times - 1)
        evaluate(P, s, out, 0, ncols, chi_out);
    }
  }
  (void)nobs;
  return rng.exhausted ? YAQS_E_RNG : YAQS_OK;
}

std::string g_err;
std::mutex g_err_mu;

int fail(int code, const std::string& msg) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_err = msg;
  return code;
}

void load_state(Problem& P, const yaqs_mps_desc* psi0) {
  const int L = psi0->L;
  P.L = L;
  P.psi0.L = L;
  P.psi0.oc = 0;
  P.psi0.t.resize(L);
  for (int i = 0; i < L; ++i) {
    int l = psi0->chi[i], r = psi0->chi[i + 1];
    Ten T(l, 2, r);
    const double* src = psi0->tensors[i];
    for (size_t k = 0; k < T.v.size(); ++k) T.v[k] = cd(src[2 * k], src[2 * k + 1]);
    P.psi0.t[i] = std::move(T);
  }
}

// Noise processes; the dissipators exp(-0.5 dt_eff gamma L^dag L) are
// precomputed for dt_eff = P.dt / 2 and P.dt (Dissipation.jl:62-69).
bool load_noise(Problem& P, const yaqs_noise_desc* noise, std::string& err) {
  P.noise.present = noise && noise->present;
  P.noise.all_zero = true;
  if (!P.noise.present) return true;
  for (int k = 0; k < noise->n; ++k) {
    const yaqs_noise_proc& q = noise->procs[k];
    NoiseProc pr{};
    pr.nsites = q.nsites;
    pr.s0 = q.site[0];
    pr.s1 = q.nsites == 2 ? q.site[1] : q.site[0];
    pr.gamma = q.strength;
    pr.pauli_name = q.pauli_name != 0;
    pr.pauli_proc = q.pauli_proc != 0;
    if (q.nsites < 1 || q.nsites > 2 || pr.s0 < 0 || pr.s1 >= P.L || pr.s1 < pr.s0) {
      err = "bad noise process sites";
      return false;
    }
    if (q.nsites == 2 && pr.s1 > pr.s0 + 1) {  // long-range: sig, tau, alpha, beta, dissipation rate
      if (!pr.pauli_name) {
        err = "Non-Pauli long-range processes not fully implemented";
        return false;
      }
      pr.lr = true;
      for (int e = 0; e < 4; ++e) {
        pr.sig[e] = cd(q.matrix[2 * e], q.matrix[2 * e + 1]);
        pr.tau[e] = cd(q.matrix[8 + 2 * e], q.matrix[9 + 2 * e]);
      }
      pr.alpha = cd(q.matrix[16], q.matrix[17]);
      pr.beta = cd(q.matrix[18], q.matrix[19]);
      pr.diss_rate = q.matrix[20];
      if (pr.gamma != 0.0) P.noise.all_zero = false;
      P.noise.procs.push_back(pr);
      continue;
    }
    int dd = q.nsites == 1 ? 2 : 4;
    for (int e = 0; e < dd * dd; ++e) pr.mat[e] = cd(q.matrix[2 * e], q.matrix[2 * e + 1]);
    cd LdL[16];
    for (int i = 0; i < dd; ++i)
      for (int j = 0; j < dd; ++j) {
        cd sacc = 0;
        for (int kk = 0; kk < dd; ++kk) sacc += std::conj(pr.mat[kk + dd * i]) * pr.mat[kk + dd * j];
        LdL[i + dd * j] = sacc;
      }
    herm_expm(dd, LdL, -0.5 * (P.dt / 2) * pr.gamma, pr.diss_half);
    herm_expm(dd, LdL, -0.5 * P.dt * pr.gamma, pr.diss_full);
    if (pr.gamma != 0.0) P.noise.all_zero = false;
    P.noise.procs.push_back(pr);
  }
  return true;
}

void load_obs_rng(Problem& P, const yaqs_obs_desc* obs, int n_obs, const yaqs_rng_desc* rng) {
  for (int k = 0; k < n_obs; ++k) {
    Obs o{};
    o.kind = obs[k].kind;
    o.s0 = obs[k].site[0];
    o.s1 = obs[k].site[1];
    int dd = o.kind == YAQS_OBS_LOCAL2 ? 4 : 2;
    for (int e = 0; e < dd * dd; ++e) o.mat[e] = cd(obs[k].matrix[2 * e], obs[k].matrix[2 * e + 1]);
    P.obs.push_back(o);
  }
  P.rng_mode = rng->mode;
  P.seed = rng->seed;
  P.uniforms = rng->uniforms;
  P.stride = rng->stride;
}

bool load_problem(Problem& P, const yaqs_mps_desc* psi0, const yaqs_mpo_desc* H, const yaqs_noise_desc* noise,
                  const yaqs_obs_desc* obs, int n_obs, const yaqs_tev_config* cfg, const yaqs_rng_desc* rng,
                  std::string& err) {
  if (!psi0 || !H || !cfg || !rng) {
    err = "null descriptor";
    return false;
  }
  const int L = psi0->L;
  if (L < 2 || H->L != L) {
    err = "need L >= 2 and matching MPO length";
    return false;
  }
  load_state(P, psi0);
  P.W.resize(L);
  for (int i = 0; i < L; ++i) {
    Wt W(H->w[i], 2, H->w[i + 1]);
    const double* src = H->tensors[i];
    for (size_t k = 0; k < W.v.size(); ++k) W.v[k] = cd(src[2 * k], src[2 * k + 1]);
    P.W[i] = std::move(W);
  }
  P.W2.resize(L - 1);
  for (int i = 0; i + 1 < L; ++i) P.W2[i] = merge_wt(P.W[i], P.W[i + 1]);
  P.dt = cfg->dt;
  P.n_times = cfg->n_times;
  P.num_traj = cfg->num_traj;
  P.max_bond = cfg->max_bond_dim;
  P.thr = cfg->truncation_threshold;
  P.order = cfg->order;
  P.sample_timesteps = cfg->sample_timesteps != 0;
  P.kp.kdim = cfg->krylov_dim;
  P.kp.tol = cfg->krylov_tol;
  P.kp.exit_tol = cfg->krylov_exit_tol;
  P.traj_offset = cfg->traj_offset;
  P.tdvp_mode = cfg->tdvp_mode;
  if (P.tdvp_mode < YAQS_TDVP_2SITE || P.tdvp_mode > YAQS_TDVP_DYNAMIC) {
    err = "bad tdvp_mode";
    return false;
  }
  if (P.n_times < 1 || P.num_traj < 1 || P.max_bond < 1 || P.kp.kdim < 1) {
    err = "bad config";
    return false;
  }
  if (!load_noise(P, noise, err)) return false;
  load_obs_rng(P, obs, n_obs, rng);
  return true;
}

// ---------------------------------------------------------------------------
// Digital TJM (DigitalTJM.jl:86-450), TEBD gate application
// ---------------------------------------------------------------------------
struct Gate {
  int kind;  // 0 barrier, 1 one-qubit, 2 two-qubit
  int a, b;  // sites as given
  cd mat[16];
  bool sample;
  bool has_gen;  // exp(-i coeff g1 (x) g2), g1 on a, g2 on b
  double coeff;
  cd g1[4], g2[4];
};

struct Circuit {
  vector<vector<int>> layers;  // indices into gates
  bool sample_at_start = false;
  vector<bool> sample_after;   // per layer
  int n_samples = 1;
};

// process_circuit (DigitalTJM.jl:86-145) and _sample_plan (:159-168).
Circuit process_circuit(const vector<Gate>& gates) {
  Circuit c;
  vector<int> cur;
  vector<char> busy;
  std::vector<std::pair<int, bool>> barriers;  // (index, is_sample)
  auto flush = [&]() {
    c.layers.push_back(cur);
    cur.clear();
    std::fill(busy.begin(), busy.end(), 0);
  };
  for (size_t g = 0; g < gates.size(); ++g) {
    const Gate& G = gates[g];
    int mx = std::max(G.a, G.b);
    if ((int)busy.size() <= mx) busy.resize(mx + 1, 0);
    if (G.kind == 0) {
      if (!cur.empty()) flush();
      barriers.push_back({(int)c.layers.size(), G.sample});
      continue;
    }
    bool overlap = busy[G.a] || (G.kind == 2 && busy[G.b]);
    if (overlap) flush();
    cur.push_back((int)g);
    busy[G.a] = 1;
    if (G.kind == 2) busy[G.b] = 1;
  }
  if (!cur.empty()) c.layers.push_back(cur);
  c.sample_after.assign(c.layers.size(), false);
  for (auto& bs : barriers) {
    if (!bs.second) continue;
    if (bs.first == 0) c.sample_at_start = true;
    else if (bs.first <= (int)c.layers.size()) c.sample_after[bs.first - 1] = true;
  }
  int n = c.sample_at_start ? 1 : 0;
  for (bool x : c.sample_after) n += x ? 1 : 0;
  c.n_samples = n == 0 ? 1 : n;
  return c;
}

const cd kSwap[16] = {1, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0, 0, 0, 0, 0, 1};

// apply_local_gate_exact! (DigitalTJM.jl:251-305)
void tebd_apply(const Problem& P, State& s, const cd* op, int s1, Counters& cnt) {
  shift_oc(s, s1);
  Ten Th = merge(s.t[s1], s.t[s1 + 1]);
  apply_2site(Th, op);
  Ten U, V;
  split_theta(Th, 2, P.thr, P.max_bond, false, U, V, cnt);
  s.t[s1] = U;
  s.t[s1 + 1] = V;
  s.oc = s1 + 1;
}

// apply_window! with method :TEBD (DigitalTJM.jl:307-334)
void apply_window_tebd(const Problem& P, State& s, const Gate& G, Counters& cnt) {
  const int s1 = std::min(G.a, G.b), s2 = std::max(G.a, G.b);
  if (s2 > s1 + 1) {
    for (int k = s2 - 1; k >= s1 + 1; --k) tebd_apply(P, s, kSwap, k, cnt);
    tebd_apply(P, s, G.mat, s1, cnt);
    for (int k = s1 + 1; k <= s2 - 1; ++k) tebd_apply(P, s, kSwap, k, cnt);
  } else {
    tebd_apply(P, s, G.mat, s1, cnt);
  }
}

// apply_window! with method :TDVP (DigitalTJM.jl:335-358): the window
// s1..s2 (padding 0) evolves under construct_window_mpo (DigitalTJM.jl:
// 192-236) by one _tdvp_sweep_circuit_2site! (Algorithms.jl:606-627):
// forward 2-site updates by +1 with back-evolution by -1 (:631-672), then the
// edge pair by +1 split to the right (:762-800); the centre ends on s2.
void apply_window_tdvp(const Problem& P, State& s, const Gate& G, Counters& cnt) {
  const int s1 = std::min(G.a, G.b), s2 = std::max(G.a, G.b), n = s2 - s1 + 1;
  shift_oc(s, s1);
  const cd* gs1 = G.a == s1 ? G.g1 : G.g2;  // the generator of the smaller site
  const cd* gs2 = G.a == s1 ? G.g2 : G.g1;
  vector<Wt> W(n, Wt(1, 2, 1));
  for (int j = 0; j < n; ++j)
    for (int po = 0; po < 2; ++po)
      for (int pi = 0; pi < 2; ++pi) {
        cd v = po == pi ? 1.0 : 0.0;
        if (j == 0) v = G.coeff * gs1[po + 2 * pi];
        else if (j == n - 1) v = gs2[po + 2 * pi];
        W[j].v[po + 2 * pi] = v;
      }
  vector<Wt> W2(n - 1);
  for (int j = 0; j + 1 < n; ++j) W2[j] = merge_wt(W[j], W[j + 1]);
  vector<Env> EL(n + 1), ER(n + 1);
  EL[0] = identity_env(s.t[s1].l, 1);
  ER[n] = identity_env(s.t[s2].r, 1);
  for (int j = n - 1; j >= 1; --j) ER[j] = update_right(s.t[s1 + j], W[j], ER[j + 1]);
  Sweeper sw(P, cnt);
  for (int j = 0; j + 2 < n; ++j) {  // forward (Algorithms.jl:617-620)
    Ten Th = merge(s.t[s1 + j], s.t[s1 + j + 1]);
    Th.v = sw.evolve(EL[j], ER[j + 2], W2[j], Th, 1.0);
    Ten U, V;
    split_theta(Th, 0, P.thr, P.max_bond, false, U, V, cnt);
    s.t[s1 + j] = U;
    EL[j + 1] = update_left(s.t[s1 + j], W[j], EL[j]);
    V.v = sw.evolve(EL[j + 1], ER[j + 2], W[j + 1], V, -1.0);
    s.t[s1 + j + 1] = V;
  }
  {  // edge (Algorithms.jl:762-800)
    const int j = n - 2;
    Ten Th = merge(s.t[s1 + j], s.t[s1 + j + 1]);
    Th.v = sw.evolve(EL[j], ER[j + 2], W2[j], Th, 1.0);
    Ten U, V;
    split_theta(Th, 0, P.thr, P.max_bond, false, U, V, cnt);
    s.t[s1 + j] = U;
    s.t[s1 + j + 1] = V;
  }
  s.oc = s2;
}

// create_local_noise_model (DigitalTJM.jl:172-188)
NoiseSet local_noise(const NoiseSet& N, int s1, int s2) {
  NoiseSet out;
  out.present = true;
  out.all_zero = true;
  for (const auto& pr : N.procs) {
    bool take = pr.nsites == 1 ? (pr.s0 == s1 || pr.s0 == s2)
                               : ((pr.s0 == s1 && pr.s1 == s2) || (pr.s0 == s2 && pr.s1 == s1));
    if (take) {
      out.procs.push_back(pr);
      if (pr.gamma != 0.0) out.all_zero = false;
    }
  }
  return out;
}

// run_digital_tjm (DigitalTJM.jl:363-450)
int run_digital(const Problem& P, const vector<Gate>& gates, const Circuit& C, long long traj, double* out,
                int* chi_out, Counters& cnt) {
  State s = P.psi0;
  normalize_mps(s);  // Simulator.jl:128
  Draws rng{&P, traj};
  const int ncols = C.n_samples;
  int col = 0;
  if (C.sample_at_start) evaluate(P, s, out, col++, ncols, chi_out);
  for (size_t l = 0; l < C.layers.size(); ++l) {
    for (int g : C.layers[l])
      if (gates[g].kind == 1) apply_1site(s.t[gates[g].a], gates[g].mat);  // apply_single_qubit_gate!
    for (int g : C.layers[l]) {
      const Gate& G = gates[g];
      if (G.kind != 2) continue;
      const bool lr = std::abs(G.a - G.b) > 1;
      if ((lr ? P.long_range_method : P.local_method) == YAQS_METHOD_TDVP)
        apply_window_tdvp(P, s, G, cnt);
      else
        apply_window_tebd(P, s, G, cnt);
      if (P.noise.present && !P.noise.procs.empty()) {
        NoiseSet loc = local_noise(P.noise, std::min(G.a, G.b), std::max(G.a, G.b));
        if (!loc.procs.empty()) {
          apply_dissipation(P, loc, s, true, 1.0, cnt);
          stochastic_process(P, loc, s, 1.0, rng, cnt);
        } else {
          normalize_mps(s);
        }
      } else {
        normalize_mps(s);
      }
    }
    if (C.sample_after[l]) evaluate(P, s, out, col++, ncols, chi_out);
  }
  if (!C.sample_at_start && col == 0 && !P.obs.empty()) evaluate(P, s, out, 0, ncols, chi_out);
  return rng.exhausted ? YAQS_E_RNG : YAQS_OK;
}

bool load_circuit(const yaqs_gate_desc* gates, int n, int L, vector<Gate>& out, std::string& err) {
  for (int g = 0; g < n; ++g) {
    const yaqs_gate_desc& q = gates[g];
    Gate G{};
    G.kind = q.kind;
    G.a = q.site[0];
    G.b = q.kind == 2 ? q.site[1] : q.site[0];
    G.sample = q.sample != 0;
    if (q.kind < 0 || q.kind > 2 || (q.kind != 0 && (G.a < 0 || G.a >= L || G.b < 0 || G.b >= L)) ||
        (q.kind == 2 && G.a == G.b)) {
      err = "bad gate descriptor";
      return false;
    }
    if (q.kind == 0) G.a = G.b = 0;
    int dd = q.kind == 2 ? 4 : 2;
    for (int e = 0; e < dd * dd && q.kind != 0; ++e) G.mat[e] = cd(q.matrix[2 * e], q.matrix[2 * e + 1]);
    G.has_gen = q.kind == 2 && q.has_generator;
    G.coeff = q.coeff;
    for (int e = 0; e < 4; ++e) {
      G.g1[e] = cd(q.gen1[2 * e], q.gen1[2 * e + 1]);
      G.g2[e] = cd(q.gen2[2 * e], q.gen2[2 * e + 1]);
    }
    out.push_back(G);
  }
  return true;
}

}  // namespace

// ===========================================================================
// extern "C" API of the oracle (ctypes, tests only)
// ===========================================================================
extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

// Installs (fn != null) or removes the CBLAS zgemm the contractions use and
// returns the previous one.  Not to be changed while a problem runs.
void* orc_set_zgemm(void* fn) {
  void* old = reinterpret_cast<void*>(g_zgemm);
  g_zgemm = reinterpret_cast<cblas_zgemm_t>(fn);
  return old;
}

// Runs trajectories [t_begin, t_end) of the problem on nthreads host threads.
// traj_out is [num_traj][n_obs][n_out] indexed by the absolute trajectory.
int orc_analog_run(const yaqs_mps_desc* psi0, const yaqs_mpo_desc* H, const yaqs_noise_desc* noise,
                   const yaqs_obs_desc* obs, int32_t n_obs, const yaqs_tev_config* cfg, const yaqs_rng_desc* rng,
                   int32_t t_begin, int32_t t_end, int32_t nthreads, double* traj_out, int32_t* maxchi_out,
                   yaqs_run_stats* stats) {
  Problem P;
  std::string err;
  if (!load_problem(P, psi0, H, noise, obs, n_obs, cfg, rng, err)) return fail(YAQS_E_ARG, err);
  const int ncols = P.sample_timesteps ? P.n_times : 1;
  if (t_begin < 0 || t_end > P.num_traj || t_begin > t_end) return fail(YAQS_E_ARG, "bad trajectory range");
  std::atomic<int> next(t_begin);
  std::atomic<int> status(YAQS_OK);
  std::mutex mu;
  Counters total;
  auto worker = [&]() {
    Counters c;
    for (;;) {
      int t = next.fetch_add(1);
      if (t >= t_end) break;
      vector<double> out((size_t)n_obs * ncols, 0.0);
      vector<int> chi(ncols, 0);
      int st = run_trajectory(P, t, out.data(), chi.data(), c);
      if (st != YAQS_OK) status.store(st);
      if (traj_out) std::copy(out.begin(), out.end(), traj_out + (size_t)t * n_obs * ncols);
      if (maxchi_out) std::copy(chi.begin(), chi.end(), maxchi_out + (size_t)t * ncols);
    }
    std::lock_guard<std::mutex> lk(mu);
    total.matvecs += c.matvecs;
    total.solves += c.solves;
    total.svds += c.svds;
    total.jumps += c.jumps;
    total.nonfinite += c.nonfinite;
    total.flops += c.flops;
  };
  int nt = std::max(1, (int)nthreads);
  vector<std::thread> th;
  for (int i = 0; i < nt; ++i) th.emplace_back(worker);
  for (auto& x : th) x.join();
  if (stats) {
    stats->matvecs = total.matvecs;
    stats->krylov_solves = total.solves;
    stats->svds = total.svds;
    stats->jumps = total.jumps;
    stats->nonfinite_fixes = total.nonfinite;
    stats->flops = total.flops;
    stats->device_ms = 0;
  }
  if (status.load() != YAQS_OK) return fail(status.load(), "injected uniform stream exhausted");
  return YAQS_OK;
}

int orc_digital_plan(const yaqs_gate_desc* gates, int32_t n_gates, int32_t* n_layers, int32_t* n_samples) {
  vector<Gate> G;
  std::string err;
  int L = 1;
  for (int g = 0; g < n_gates; ++g) L = std::max(L, std::max(gates[g].site[0], gates[g].site[1]) + 1);
  if (!load_circuit(gates, n_gates, L, G, err)) return fail(YAQS_E_ARG, err);
  Circuit C = process_circuit(G);
  *n_layers = (int32_t)C.layers.size();
  *n_samples = C.n_samples;
  return YAQS_OK;
}

// Digital TJM trajectories [t_begin, t_end) on nthreads host threads.
int orc_digital_run(const yaqs_mps_desc* psi0, const yaqs_gate_desc* gates, int32_t n_gates,
                    const yaqs_noise_desc* noise, const yaqs_obs_desc* obs, int32_t n_obs,
                    const yaqs_circuit_config* cfg, const yaqs_rng_desc* rng, int32_t t_begin, int32_t t_end,
                    int32_t nthreads, double* traj_out, int32_t* maxchi_out, yaqs_run_stats* stats) {
  if (!psi0 || !cfg || !rng || psi0->L < 2) return fail(YAQS_E_ARG, "bad descriptors");
  Problem P;
  std::string err;
  load_state(P, psi0);
  P.dt = 1.0;  // gate-level noise uses dt = 1 (DigitalTJM.jl:412-413)
  P.num_traj = cfg->num_traj;
  P.max_bond = cfg->max_bond_dim;
  P.thr = cfg->truncation_threshold;
  P.traj_offset = cfg->traj_offset;
  if (!load_noise(P, noise, err)) return fail(YAQS_E_ARG, err);
  load_obs_rng(P, obs, n_obs, rng);
  vector<Gate> G;
  if (!load_circuit(gates, n_gates, P.L, G, err)) return fail(YAQS_E_ARG, err);
  P.local_method = cfg->local_method;
  P.long_range_method = cfg->long_range_method;
  P.kp.kdim = 25;  // expm_krylov(..., 25) in the circuit sweeps (Algorithms.jl:185)
  P.kp.tol = 1e-10;
  P.kp.exit_tol = 1e-12;
  for (const Gate& g : G) {
    const bool lr = std::abs(g.a - g.b) > 1;
    if (g.kind == 2 && (lr ? P.long_range_method : P.local_method) == YAQS_METHOD_TDVP && !g.has_gen)
      return fail(YAQS_E_ARG, "a gate applied by TDVP needs its generator (GateLibrary.generator)");
  }
  Circuit C = process_circuit(G);
  const int ncols = C.n_samples;
  if (t_begin < 0 || t_end > P.num_traj || t_begin > t_end) return fail(YAQS_E_ARG, "bad trajectory range");
  std::atomic<int> next(t_begin);
  std::atomic<int> status(YAQS_OK);
  std::mutex mu;
  Counters total;
  auto worker = [&]() {
    Counters c;
    for (;;) {
      int t = next.fetch_add(1);
      if (t >= t_end) break;
      vector<double> out((size_t)n_obs * ncols, 0.0);
      vector<int> chi(ncols, 0);
      int st = run_digital(P, G, C, t, out.data(), chi.data(), c);
      if (st != YAQS_OK) status.store(st);
      if (traj_out) std::copy(out.begin(), out.end(), traj_out + (size_t)t * n_obs * ncols);
      if (maxchi_out) std::copy(chi.begin(), chi.end(), maxchi_out + (size_t)t * ncols);
    }
    std::lock_guard<std::mutex> lk(mu);
    total.svds += c.svds;
    total.jumps += c.jumps;
  };
  vector<std::thread> th;
  for (int i = 0; i < std::max(1, (int)nthreads); ++i) th.emplace_back(worker);
  for (auto& x : th) x.join();
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->svds = total.svds;
    stats->jumps = total.jumps;
  }
  if (status.load() != YAQS_OK) return fail(status.load(), "injected uniform stream exhausted");
  return YAQS_OK;
}

// Plain 2TDVP evolution without noise: n_steps sweeps of two_site_tdvp!, with
// local_expect of the given 1-site observables after every sweep (the loop
// of test/benchmark_tdvp.jl:195-212 and test/simulate_large_ising.jl:69-81).
// out is [n_steps+1][n_obs].
int orc_tdvp_evolve(const yaqs_mps_desc* psi0, const yaqs_mpo_desc* H, const yaqs_obs_desc* obs, int32_t n_obs,
                    const yaqs_tev_config* cfg, int32_t n_steps, double* out) {
  Problem P;
  std::string err;
  yaqs_rng_desc rng{YAQS_RNG_PHILOX, 0, nullptr, 0};
  if (!load_problem(P, psi0, H, nullptr, obs, n_obs, cfg, &rng, err)) return fail(YAQS_E_ARG, err);
  Counters c;
  State s = P.psi0;
  Sweeper sw(P, c);
  for (int k = 0; k < n_obs; ++k) out[k] = measure(P.obs[k], s);
  for (int t = 1; t <= n_steps; ++t) {
    sw.sweep(s);
    for (int k = 0; k < n_obs; ++k) out[(size_t)t * n_obs + k] = measure(P.obs[k], s);
  }
  return YAQS_OK;
}

// calculate_stochastic_factor (StochasticProcess.jl:35-38): dp = 1 - <psi|psi>
// of the state as given (no normalisation first).
int orc_stochastic_factor(const yaqs_mps_desc* psi, double* dp) {
  if (!psi || !dp || psi->L < 1) return fail(YAQS_E_ARG, "null argument");
  Problem P;
  load_state(P, psi);
  *dp = 1.0 - scalar_product(P.psi0).real();
  return YAQS_OK;
}

// create_probability_distribution (StochasticProcess.jl:89-212) on the
// initial state of a problem: the normalised weights in the reference's
// candidate order, each candidate's type (0 local_1, 1 local_2,
// 2 pauli_long_range, 3 mpo_general) and its two sites (0-based; the second
// repeats the first for 1-site candidates).  *n_out = 0 when every weight is
// zero, as the reference returns empty lists then.
int orc_probability_distribution(const yaqs_mps_desc* psi0, const yaqs_mpo_desc* H, const yaqs_noise_desc* noise,
                                 const yaqs_tev_config* cfg, double dt, int32_t cap, double* probs, int32_t* kinds,
                                 int32_t* sites, int32_t* n_out) {
  if (!probs || !kinds || !sites || !n_out) return fail(YAQS_E_ARG, "null argument");
  Problem P;
  std::string err;
  yaqs_rng_desc rng{YAQS_RNG_PHILOX, 0, nullptr, 0};
  if (!load_problem(P, psi0, H, noise, nullptr, 0, cfg, &rng, err)) return fail(YAQS_E_ARG, err);
  State s = P.psi0;
  vector<Cand> cands = jump_candidates(P, P.noise, s, dt);
  double total = 0;
  for (auto& c : cands) total += c.dp;
  *n_out = 0;
  if (total == 0.0) return YAQS_OK;
  if ((int)cands.size() > cap) return fail(YAQS_E_ARG, "candidate capacity too small");
  for (size_t i = 0; i < cands.size(); ++i) {
    const NoiseProc& pr = *cands[i].pr;
    probs[i] = cands[i].dp / total;
    kinds[i] = pr.lr ? (pr.pauli_proc ? 2 : 3) : (pr.nsites == 1 ? 0 : 1);
    sites[2 * i] = pr.s0;
    sites[2 * i + 1] = pr.nsites == 1 ? pr.s0 : pr.s1;
  }
  *n_out = (int32_t)cands.size();
  return YAQS_OK;
}

// Plain TDVP evolution without noise, returning <psi0|psi(t)> after n_steps
// sweeps of the configured mode (single_site_tdvp! / two_site_tdvp!, the
// eigenstate-phase checks of test/test_Algorithms.jl:37-95).
int orc_tdvp_overlap(const yaqs_mps_desc* psi0, const yaqs_mpo_desc* H, const yaqs_tev_config* cfg, int32_t n_steps,
                     double* overlap) {
  if (!overlap || n_steps < 0) return fail(YAQS_E_ARG, "bad argument");
  Problem P;
  std::string err;
  yaqs_rng_desc rng{YAQS_RNG_PHILOX, 0, nullptr, 0};
  if (!load_problem(P, psi0, H, nullptr, nullptr, 0, cfg, &rng, err)) return fail(YAQS_E_ARG, err);
  Counters c;
  State s = P.psi0;
  Sweeper sw(P, c);
  for (int t = 0; t < n_steps; ++t) sw.sweep(s);
  cd ov = scalar_product(s, P.psi0);  // scalar_product(mps, mps0) of the reference test
  overlap[0] = ov.real();
  overlap[1] = ov.imag();
  return YAQS_OK;
}

// apply_dissipation (Dissipation.jl:37-159) once on the initial state of a
// problem, with the process rates at cfg->dt (full_dt != 0) or cfg->dt / 2.
// The resulting tensors are written packed, site after site, in the
// (left, phys, right) column-major layout; chi_out gets the L+1 bond
// dimensions and *oc_out the 0-based orthogonality centre.
int orc_apply_dissipation(const yaqs_mps_desc* psi0, const yaqs_mpo_desc* H, const yaqs_noise_desc* noise,
                          const yaqs_tev_config* cfg, int32_t full_dt, int64_t capacity, double* tensors_out,
                          int32_t* chi_out, int32_t* oc_out) {
  if (!tensors_out || !chi_out || !oc_out) return fail(YAQS_E_ARG, "null argument");
  Problem P;
  std::string err;
  yaqs_rng_desc rng{YAQS_RNG_PHILOX, 0, nullptr, 0};
  if (!load_problem(P, psi0, H, noise, nullptr, 0, cfg, &rng, err)) return fail(YAQS_E_ARG, err);
  Counters c;
  State s = P.psi0;
  apply_dissipation(P, P.noise, s, full_dt != 0, full_dt ? P.dt : P.dt / 2, c);
  int64_t n = 0;
  for (int i = 0; i < s.L; ++i) n += (int64_t)s.t[i].v.size();
  if (n > capacity) return fail(YAQS_E_ARG, "tensor capacity too small");
  int64_t o = 0;
  for (int i = 0; i < s.L; ++i) {
    chi_out[i] = s.t[i].l;
    for (const cd& x : s.t[i].v) {
      tensors_out[2 * o] = x.real();
      tensors_out[2 * o + 1] = x.imag();
      ++o;
    }
  }
  chi_out[s.L] = s.t[s.L - 1].r;
  *oc_out = s.oc;
  return YAQS_OK;
}

// Component entry points used by the unit tests.
int orc_svd(int32_t m, int32_t n, const double* M, double* U, double* S, double* Vt) {
  vector<cd> A((size_t)m * n);
  for (size_t k = 0; k < A.size(); ++k) A[k] = cd(M[2 * k], M[2 * k + 1]);
  vector<cd> u, vt;
  vector<double> s;
  jacobi_svd(m, n, A.data(), u, s, vt);
  std::memcpy(U, u.data(), u.size() * sizeof(cd));
  std::memcpy(Vt, vt.data(), vt.size() * sizeof(cd));
  std::memcpy(S, s.data(), s.size() * sizeof(double));
  return YAQS_OK;
}

int orc_qr(int32_t m, int32_t n, const double* M, double* Q, double* R) {
  vector<cd> A((size_t)m * n);
  for (size_t k = 0; k < A.size(); ++k) A[k] = cd(M[2 * k], M[2 * k + 1]);
  vector<cd> q, r;
  house_qr(m, n, A.data(), q, r);
  std::memcpy(Q, q.data(), q.size() * sizeof(cd));
  std::memcpy(R, r.data(), r.size() * sizeof(cd));
  return YAQS_OK;
}

int orc_truncation_rank(int32_t n, const double* S, double thr, int32_t max_bond, int32_t rule) {
  vector<double> s(S, S + n);
  return rule == 0 ? keep_tdvp(s, thr, max_bond) : rule == 1 ? keep_relative(s, thr, max_bond) : keep_tebd(s, thr, max_bond);
}

// exp(-i dt H_eff) x for H_eff = project_site(L, R, W) with (chil, D, chir) x.
// L: (chil, wl, chil), R: (chir, wr, chir), W: (wl, D, D, wr).
int orc_expm_site(int32_t chil, int32_t D, int32_t chir, int32_t wl, int32_t wr, const double* Lp, const double* Rp,
                  const double* Wp, const double* x, double dt, int32_t kdim, double tol, double exit_tol, double* out,
                  int32_t* matvecs) {
  Env Le(chil, wl, chil), Re(chir, wr, chir);
  for (size_t k = 0; k < Le.v.size(); ++k) Le.v[k] = cd(Lp[2 * k], Lp[2 * k + 1]);
  for (size_t k = 0; k < Re.v.size(); ++k) Re.v[k] = cd(Rp[2 * k], Rp[2 * k + 1]);
  Wt W(wl, D, wr);
  for (size_t k = 0; k < W.v.size(); ++k) W.v[k] = cd(Wp[2 * k], Wp[2 * k + 1]);
  vector<cd> v((size_t)chil * D * chir);
  for (size_t k = 0; k < v.size(); ++k) v[k] = cd(x[2 * k], x[2 * k + 1]);
  KrylovParams kp;
  kp.kdim = kdim;
  kp.tol = tol;
  kp.exit_tol = exit_tol;
  Counters c;
  auto op = [&](const vector<cd>& in, vector<cd>& o) { project_site(Le, Re, W, chil, D, chir, in, o); };
  vector<cd> r = expm_krylov(op, v, dt, kp, c);
  std::memcpy(out, r.data(), r.size() * sizeof(cd));
  if (matvecs) *matvecs = (int32_t)c.matvecs;
  return YAQS_OK;
}

int orc_project_site(int32_t chil, int32_t D, int32_t chir, int32_t wl, int32_t wr, const double* Lp,
                     const double* Rp, const double* Wp, const double* x, double* out) {
  Env Le(chil, wl, chil), Re(chir, wr, chir);
  for (size_t k = 0; k < Le.v.size(); ++k) Le.v[k] = cd(Lp[2 * k], Lp[2 * k + 1]);
  for (size_t k = 0; k < Re.v.size(); ++k) Re.v[k] = cd(Rp[2 * k], Rp[2 * k + 1]);
  Wt W(wl, D, wr);
  for (size_t k = 0; k < W.v.size(); ++k) W.v[k] = cd(Wp[2 * k], Wp[2 * k + 1]);
  vector<cd> v((size_t)chil * D * chir), o;
  for (size_t k = 0; k < v.size(); ++k) v[k] = cd(x[2 * k], x[2 * k + 1]);
  project_site(Le, Re, W, chil, D, chir, v, o);
  std::memcpy(out, o.data(), o.size() * sizeof(cd));
  return YAQS_OK;
}

double orc_philox_uniform(uint64_t seed, uint64_t stream, uint64_t draw) { return philox_uniform(seed, stream, draw); }

}  // extern "C"

extern "C" {
// Raw Philox-4x32-10 block for known-answer tests.
void orc_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  uint32_t k[2] = {key[0], key[1]};
  for (int r = 0; r < 10; ++r) {
    philox_round(c, k);
    if (r < 9) {
      k[0] += 0x9E3779B9u;
      k[1] += 0xBB67AE85u;
    }
  }
  for (int i = 0; i < 4; ++i) out[i] = c[i];
}
}
