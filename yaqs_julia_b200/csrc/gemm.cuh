// gemm.cuh — CTA-level complex FP64 GEMM with general strides.
//
// C(m,n) = op(A)(m,k) * op(B)(k,n)  [+ C if accumulate]
//   A element (m,k) at A[m*am + k*ak], conjugated if conjA
//   B element (k,n) at B[k*bk + n*bn], conjugated if conjB
//   C element (m,n) at C[m*cm + n*cn]
// Every tensor contraction of the TDVP path (Algorithms.jl:199-226) is
// written as one such GEMM over the reference's column-major layouts.
//
// Tiling: 64x64 output tiles, 8-deep K slices staged in shared memory by
// cp.async (double buffered, zero-filled outside the matrix), each of the
// 256 threads owning a 4x4 register tile with rows tx+16i and columns
// ty+16j (so stores along m are coalesced).  Conjugation is applied when a
// slice is read from shared memory.
#pragma once
#include "common.cuh"

#define GBM 64
#define GBN 64
#define GBK 8

struct GemmSmem {
  cplx As[2][GBK][GBM + 1];
  cplx Bs[2][GBK][GBN + 1];
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

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

__device__ __forceinline__ GemmArgs gemm_args(int M, int N, int K, const cplx* A, long long am, long long ak,
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

// CTA-collective.  Ends with a __syncthreads() so C is visible to all.
// Conjugation is a template parameter so the common unconjugated case has
// no extra arithmetic in the inner loop.
template <bool CA, bool CB>
__device__ __noinline__ void cta_gemm_t(const GemmArgs g, GemmSmem& sm) {
  ProfScope prof_scope_(PF_GEMM);
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const bool a_m_fast = (g.am == 1) || (g.ak != 1);
  const bool b_n_fast = (g.bn == 1) || (g.bk != 1);
  const int nk = (g.K + GBK - 1) / GBK;
  for (int tm = 0; tm < g.M; tm += GBM) {
    for (int tn = 0; tn < g.N; tn += GBN) {
      cplx acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
      auto issue = [&](int kc, int buf) {
        const int k0 = kc * GBK;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int idx = tid + NT * e;
          int mi, ki, ni, kj;
          if (a_m_fast) {
            mi = idx & 63;
            ki = idx >> 6;
          } else {
            ki = idx & 7;
            mi = idx >> 3;
          }
          if (b_n_fast) {
            ni = idx & 63;
            kj = idx >> 6;
          } else {
            kj = idx & 7;
            ni = idx >> 3;
          }
          const int mm = tm + mi, ka = k0 + ki, nn = tn + ni, kb = k0 + kj;
          const bool va = mm < g.M && ka < g.K, vb = nn < g.N && kb < g.K;
          cp_async16(&sm.As[buf][ki][mi], va ? g.A + (long long)mm * g.am + (long long)ka * g.ak : g.A, va);
          cp_async16(&sm.Bs[buf][kj][ni], vb ? g.B + (long long)kb * g.bk + (long long)nn * g.bn : g.B, vb);
        }
        cp_async_commit();
      };
      __syncthreads();
      issue(0, 0);
      for (int kc = 0; kc < nk; ++kc) {
        const int buf = kc & 1;
        if (kc + 1 < nk) {
          issue(kc + 1, buf ^ 1);
          cp_async_wait_one();
        } else {
          cp_async_wait_all();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GBK; ++kk) {
          cplx a[4], b[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) a[i] = sm.As[buf][kk][tx + 16 * i];
#pragma unroll
          for (int j = 0; j < 4; ++j) b[j] = sm.Bs[buf][kk][ty + 16 * j];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              // acc += op(a) * op(b) with op = conj where requested
              cplx& c = acc[i][j];
              const double ay = CA ? -a[i].y : a[i].y, by = CB ? -b[j].y : b[j].y;
              c.x = fma(a[i].x, b[j].x, c.x);
              c.x = fma(-ay, by, c.x);
              c.y = fma(a[i].x, by, c.y);
              c.y = fma(ay, b[j].x, c.y);
            }
        }
        __syncthreads();
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int nn = tn + ty + 16 * j;
        if (nn >= g.N) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          int mm = tm + tx + 16 * i;
          if (mm >= g.M) continue;
          cplx* c = g.C + (long long)mm * g.cm + (long long)nn * g.cn;
          cplx v = acc[i][j];
          if (g.accumulate) v = cadd(v, *c);
          *c = v;
        }
      }
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void cta_gemm(const GemmArgs g, GemmSmem& sm) {
  if (g.conjA) {
    if (g.conjB) cta_gemm_t<true, true>(g, sm);
    else cta_gemm_t<true, false>(g, sm);
  } else {
    if (g.conjB) cta_gemm_t<false, true>(g, sm);
    else cta_gemm_t<false, false>(g, sm);
  }
}
