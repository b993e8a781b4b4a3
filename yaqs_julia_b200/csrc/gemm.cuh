// gemm.cuh — CTA-level complex FP64 GEMM with general strides.
//
// C(m,n) = op(A)(m,k) * op(B)(k,n)  [+ C if accumulate]
//   A element (m,k) at A[m*am + k*ak], conjugated if conjA
//   B element (k,n) at B[k*bk + n*bn], conjugated if conjB
//   C element (m,n) at C[m*cm + n*cn]
// Every tensor contraction of the TDVP path (Algorithms.jl:199-226) is
// written as one such GEMM over the reference's column-major layouts.
//
// Tiling: 64 x GBN_EFF output tiles (64 x 64 for a 256-thread program, 64 x
// 32 for a 128-thread one), 16-deep K slices staged in shared memory by
// cp.async (double buffered, zero-filled outside the matrix), each warp
// owning a 32 x 16 sub-tile.  Conjugation is applied when a slice is read
// from shared memory.
#pragma once
#include "common.cuh"

#define GBM 64
#define GBN 64
#define GBK 16
// Output columns of one CTA tile: the warps form a 2 x NW/2 grid of 32 x 16
// sub-tiles.
#define GBN_EFF (16 * (NW / 2))
static_assert(NW % 2 == 0 && GBN_EFF <= GBN, "the GEMM needs an even warp count of at most 8");

struct GemmSmem {
  cplx As[2][GBK][GBM + 1];
  cplx Bs[2][GBK][GBN + 1];
};

static __device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz) : "memory");
}
static __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
static __device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
static __device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

struct GemmArgs {
  int M, N, K;
  const cplx* A;
  long long am, ak;
  const cplx* B;
  long long bk, bn;
  cplx* C;
  long long cm, cn;
  bool conjA, conjB, accumulate;
};

static __device__ __forceinline__ GemmArgs gemm_args(int M, int N, int K, const cplx* A, long long am, long long ak,
                                              const cplx* B, long long bk, long long bn, cplx* C, long long cm,
                                              long long cn, bool conjA = false, bool conjB = false,
                                              bool accumulate = false) {
  GemmArgs g;
  g.M = M;
  g.N = N;
  g.K = K;
  g.A = A;
  g.am = am;
  g.ak = ak;
  g.B = B;
  g.bk = bk;
  g.bn = bn;
  g.C = C;
  g.cm = cm;
  g.cn = cn;
  g.conjA = conjA;
  g.conjB = conjB;
  g.accumulate = accumulate;
  return g;
}

// FP64 tensor-core product: D (8x8) += A (8x4, row) * B (4x8, col).
// Fragments (per lane, g = lane/4, t = lane%4): A[g][t], B[t][g],
// D[g][2t], D[g][2t+1].
static __device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// CTA-collective.  Ends with a cta_sync() so C is visible to all.
// Complex products run on the FP64 tensor cores (mma.sync m8n8k4): each
// warp owns a 32x16 complex sub-tile of the 64 x GBN_EFF CTA tile as 4x2
// blocks of 8x8, each block accumulating re and im with four real MMAs.
// Conjugation is a template parameter (a sign flip of the imaginary
// fragment).
template <bool CA, bool CB, int BK>
static __device__ __noinline__ void cta_gemm_t(const GemmArgs g, GemmSmem& sm) {
  ProfScope prof_scope_(PF_GEMM);
  const int tid = ltid();
  const int lane = tid & 31, wid = tid >> 5;
  const int wm = wid & 1, wn = wid >> 1;  // 2 x NW/2 warps
  const int gq = lane >> 2, tq = lane & 3;
  const bool a_m_fast = (g.am == 1) || (g.ak != 1);
  const bool b_n_fast = (g.bn == 1) || (g.bk != 1);
  const int nk = (g.K + BK - 1) / BK;
  for (int tm = 0; tm < g.M; tm += GBM) {
    for (int tn = 0; tn < g.N; tn += GBN_EFF) {
      double cr[4][2][2], ci[4][2][2];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          cr[i][j][0] = cr[i][j][1] = 0.0;
          ci[i][j][0] = ci[i][j][1] = 0.0;
        }
      auto issue = [&](int kc, int buf) {
        const int k0 = kc * BK;
        // A: GBM x BK values, B: BK x GBN_EFF values (equal counts with 8 warps)
#pragma unroll
        for (int e = 0; e < GBM * BK / NT; ++e) {
          const int idx = tid + NT * e;
          int mi, ki;
          if (a_m_fast) {
            mi = idx & (GBM - 1);
            ki = idx / GBM;
          } else {
            ki = idx & (BK - 1);
            mi = idx / BK;
          }
          const int mm = tm + mi, ka = k0 + ki;
          const bool va = mm < g.M && ka < g.K;
          cp_async16(&sm.As[buf][ki][mi], va ? g.A + (long long)mm * g.am + (long long)ka * g.ak : g.A, va);
          if (e < GBN_EFF * BK / NT) {
            int ni, kj;
            if (b_n_fast) {
              ni = idx & (GBN_EFF - 1);
              kj = idx / GBN_EFF;
            } else {
              kj = idx & (BK - 1);
              ni = idx / BK;
            }
            const int nn = tn + ni, kb = k0 + kj;
            const bool vb = nn < g.N && kb < g.K;
            cp_async16(&sm.Bs[buf][kj][ni], vb ? g.B + (long long)kb * g.bk + (long long)nn * g.bn : g.B, vb);
          }
        }
        cp_async_commit();
      };
      cta_sync();
      issue(0, 0);
      for (int kc = 0; kc < nk; ++kc) {
        const int buf = kc & 1;
        if (kc + 1 < nk) {
          issue(kc + 1, buf ^ 1);
          cp_async_wait_one();
        } else {
          cp_async_wait_all();
        }
        cta_sync();
#pragma unroll
        for (int k4 = 0; k4 < BK; k4 += 4) {
          double ar[4], ai[4], br[2], bi[2];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const cplx a = sm.As[buf][k4 + tq][wm * 32 + i * 8 + gq];
            ar[i] = a.x;
            ai[i] = CA ? -a.y : a.y;
          }
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const cplx b = sm.Bs[buf][k4 + tq][wn * 16 + j * 8 + gq];
            br[j] = b.x;
            bi[j] = CB ? -b.y : b.y;
          }
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              dmma884(cr[i][j][0], cr[i][j][1], ar[i], br[j]);
              dmma884(cr[i][j][0], cr[i][j][1], -ai[i], bi[j]);
              dmma884(ci[i][j][0], ci[i][j][1], ar[i], bi[j]);
              dmma884(ci[i][j][0], ci[i][j][1], ai[i], br[j]);
            }
        }
        cta_sync();
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int mm = tm + wm * 32 + i * 8 + gq;
        if (mm >= g.M) continue;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int nn = tn + wn * 16 + j * 8 + 2 * tq + h;
            if (nn >= g.N) continue;
            cplx* c = g.C + (long long)mm * g.cm + (long long)nn * g.cn;
            cplx v = make_double2(cr[i][j][h], ci[i][j][h]);
            if (g.accumulate) v = cadd(v, *c);
            *c = v;
          }
      }
    }
  }
  cta_sync();
}

// K slices 16 deep for long reductions, 8 deep for short ones (a short K
// would otherwise stage mostly zero padding).
template <int BK>
static __device__ __forceinline__ void cta_gemm_k(const GemmArgs g, GemmSmem& sm) {
  if (g.conjA) {
    if (g.conjB) cta_gemm_t<true, true, BK>(g, sm);
    else cta_gemm_t<true, false, BK>(g, sm);
  } else {
    if (g.conjB) cta_gemm_t<false, true, BK>(g, sm);
    else cta_gemm_t<false, false, BK>(g, sm);
  }
}

static __device__ __forceinline__ void cta_gemm(const GemmArgs g, GemmSmem& sm) {
  if (g.K >= 32)
    cta_gemm_k<GBK>(g, sm);
  else
    cta_gemm_k<8>(g, sm);
}
