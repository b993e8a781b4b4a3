// gemm_tf32.cuh — CTA-level complex FP32 GEMM on the tensor cores for the
// mixed-precision form.
//
// Same operand convention as gemm.cuh (C(m,n) = op(A)(m,k) op(B)(k,n) with
// general strides), operands complex FP32 (float2), C complex FP32 or FP64.
// Every real product X*Y runs as three TF32 products
//   X_hi Y_lo + X_lo Y_hi + X_hi Y_hi,   X_hi = tf32(X), X_lo = tf32(X - X_hi)
// (the 3xTF32 split), accumulated in FP32, which keeps FP32 accuracy; a
// complex product is four real ones (re = ar br - ai bi, im = ar bi + ai br).
// Tensor-core instruction: mma.sync m16n8k8 .tf32 with FP32 accumulators.
//
// Tiling: 64x64 output tiles, 8-deep K slices staged in shared memory by
// cp.async (8-byte copies, double buffered, zero-filled outside the matrix);
// 8 warps as 2 (m) x 4 (n), each owning a 32x16 complex sub-tile (2 x 2
// fragments of 16x8).
#pragma once
#include "gemm.cuh"

typedef float2 cflt;

#define TBM 64
#define TBN 64
#define TBK 8
#define TLD 72  // row stride of a K slice (floats2): 16 banks apart between k rows

struct GemmSmemF {
  cflt As[2][TBK][TLD];
  cflt Bs[2][TBK][TLD];
};

struct GemmArgsF {
  int M, N, K;
  const cflt* A;
  long long am, ak;
  const cflt* B;
  long long bk, bn;
  void* C;  // cflt* or cplx* (template parameter of the kernel routine)
  long long cm, cn;
  bool conjA, conjB, accumulate;
};

static __device__ __forceinline__ GemmArgsF gemm_args_f(int M, int N, int K, const cflt* A, long long am, long long ak,
                                                 const cflt* B, long long bk, long long bn, void* C, long long cm,
                                                 long long cn, bool conjA = false, bool conjB = false,
                                                 bool accumulate = false) {
  GemmArgsF g;
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

static __device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz) : "memory");
}

static __device__ __forceinline__ unsigned to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

static __device__ __forceinline__ void split_tf32(float x, unsigned& hi, unsigned& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

// D (16x8) += A (16x8, row) * B (8x8, col).  Fragments (g = lane/4,
// t = lane%4): a = {A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]},
// b = {B[t][g], B[t+4][g]}, d = {D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]}.
static __device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// d += x * y with the 3xTF32 split (small terms first).
static __device__ __forceinline__ void mma3(float (&d)[4], const unsigned (&xh)[4], const unsigned (&xl)[4],
                                     const unsigned (&yh)[2], const unsigned (&yl)[2]) {
  mma_tf32(d, xl, yh);
  mma_tf32(d, xh, yl);
  mma_tf32(d, xh, yh);
}

static __device__ __forceinline__ void store_c(cflt* c, float re, float im, bool acc) {
  if (acc) {
    cflt o = *c;
    re += o.x;
    im += o.y;
  }
  *c = make_float2(re, im);
}
static __device__ __forceinline__ void store_c(cplx* c, float re, float im, bool acc) {
  double r = re, i = im;
  if (acc) {
    cplx o = *c;
    r += o.x;
    i += o.y;
  }
  *c = make_double2(r, i);
}

// CTA-collective.  Ends with a cta_sync() so C is visible to all.
template <bool CA, bool CB, class TC>
static __device__ __noinline__ void cta_gemm_tf32_t(const GemmArgsF g, GemmSmemF& sm) {
  ProfScope prof_scope_(PF_GEMM);
  const int tid = ltid();
  const int lane = tid & 31, wid = tid >> 5;
  const int wm = wid & 1, wn = wid >> 1;  // 2 x 4 warps
  const int gq = lane >> 2, tq = lane & 3;
  const bool a_m_fast = (g.am == 1) || (g.ak != 1);
  const bool b_n_fast = (g.bn == 1) || (g.bk != 1);
  const int nk = (g.K + TBK - 1) / TBK;
  const unsigned SGN = 0x80000000u;
  TC* C = reinterpret_cast<TC*>(g.C);
  for (int tm = 0; tm < g.M; tm += TBM) {
    for (int tn = 0; tn < g.N; tn += TBN) {
      float cr[2][2][4], ci[2][2][4];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) cr[i][j][e] = ci[i][j][e] = 0.f;
      auto issue = [&](int kc, int buf) {
        const int k0 = kc * TBK;
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
          cp_async8(&sm.As[buf][ki][mi], va ? g.A + (long long)mm * g.am + (long long)ka * g.ak : g.A, va);
          cp_async8(&sm.Bs[buf][kj][ni], vb ? g.B + (long long)kb * g.bk + (long long)nn * g.bn : g.B, vb);
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
        unsigned arh[2][4], arl[2][4], aih[2][4], ail[2][4];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int m0 = wm * 32 + i * 16 + gq;
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const cflt a = sm.As[buf][tq + (e >> 1) * 4][m0 + (e & 1) * 8];
            split_tf32(a.x, arh[i][e], arl[i][e]);
            split_tf32(CA ? -a.y : a.y, aih[i][e], ail[i][e]);
          }
        }
        unsigned brh[2][2], brl[2][2], bih[2][2], bil[2][2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int n0 = wn * 16 + j * 8 + gq;
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const cflt b = sm.Bs[buf][tq + e * 4][n0];
            split_tf32(b.x, brh[j][e], brl[j][e]);
            split_tf32(CB ? -b.y : b.y, bih[j][e], bil[j][e]);
          }
        }
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          unsigned nih[4], nil[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            nih[e] = aih[i][e] ^ SGN;
            nil[e] = ail[i][e] ^ SGN;
          }
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            mma3(cr[i][j], arh[i], arl[i], brh[j], brl[j]);
            mma3(cr[i][j], nih, nil, bih[j], bil[j]);
            mma3(ci[i][j], arh[i], arl[i], bih[j], bil[j]);
            mma3(ci[i][j], aih[i], ail[i], brh[j], brl[j]);
          }
        }
        cta_sync();
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int mm = tm + wm * 32 + i * 16 + gq + (e >> 1) * 8;
            const int nn = tn + wn * 16 + j * 8 + 2 * tq + (e & 1);
            if (mm < g.M && nn < g.N)
              store_c(C + (long long)mm * g.cm + (long long)nn * g.cn, cr[i][j][e], ci[i][j][e], g.accumulate);
          }
    }
  }
  cta_sync();
}

template <class TC>
static __device__ __forceinline__ void cta_gemm_tf32(const GemmArgsF g, GemmSmemF& sm) {
  if (g.conjA) {
    if (g.conjB) cta_gemm_tf32_t<true, true, TC>(g, sm);
    else cta_gemm_tf32_t<true, false, TC>(g, sm);
  } else {
    if (g.conjB) cta_gemm_tf32_t<false, true, TC>(g, sm);
    else cta_gemm_tf32_t<false, false, TC>(g, sm);
  }
}

// FP64 -> FP32 conversion of n complex values.  CTA-collective.
static __device__ __forceinline__ void cta_to_f32(cflt* __restrict__ dst, const cplx* __restrict__ src, long long n) {
  for (long long i = ltid(); i < n; i += NT) {
    const cplx v = src[i];
    dst[i] = make_float2((float)v.x, (float)v.y);
  }
  cta_sync();
}
