// common.cuh — complex FP64 helpers and CTA-collective reductions.
//
// Every function marked "CTA-collective" must be called by all NT threads of
// the block with identical arguments; decisions derived from reductions are
// broadcast through shared memory so control flow stays uniform.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Threads of one trajectory program: 256, or 128 in the small-program
// digital kernel (engine_dg.cu defines NT before including this header).
#ifndef NT
#define NT 256
#endif
#define NW (NT / 32)

typedef double2 cplx;

// A trajectory program runs on NT threads: a whole 256-thread CTA, or, in
// the tensor-core kernel (YAQS_TC = 1, engine_tc.cu), one half of a
// 512-thread CTA whose two halves run independent programs (a kernel that
// holds tensor memory is given one CTA per SM, so it carries two slots per
// CTA).  Every CTA-collective routine synchronises its own NT threads and
// indexes threads and slots through these helpers; in the two-program
// kernel each half waits on its own named barrier (1 or 2).
#ifndef YAQS_TC
#define YAQS_TC 0
#endif
#if YAQS_TC
static __device__ __forceinline__ int ltid() { return (int)(threadIdx.x & (NT - 1)); }
static __device__ __forceinline__ int cta_half() { return (int)(threadIdx.x / NT); }
static __device__ __forceinline__ int cta_slot() { return (int)(blockIdx.x * 2 + threadIdx.x / NT); }
static __device__ __forceinline__ void cta_sync() {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + cta_half()), "n"(NT) : "memory");
}
#else
static __device__ __forceinline__ int ltid() { return (int)threadIdx.x; }
static __device__ __forceinline__ int cta_half() { return 0; }
static __device__ __forceinline__ int cta_slot() { return (int)blockIdx.x; }
static __device__ __forceinline__ void cta_sync() { __syncthreads(); }
#endif

// Optional per-slot phase timers (clock64 cycles), enabled when the host sets
// g_prof to a [slots][PROF_N] buffer.  Thread 0 of a program accumulates the
// elapsed time of each instrumented routine.
#define PROF_N 16
enum {
  PF_GEMM = 0, PF_WAPPLY = 1, PF_ORTH = 2, PF_TRIDIAG = 3, PF_SVD = 4, PF_SVDVEC = 5, PF_QR = 6, PF_QRQ = 7,
  PF_SCALAR = 8, PF_ENV = 9, PF_DISS = 10, PF_STOCH = 11, PF_EVAL = 12, PF_SWEEP = 13, PF_STEP = 14, PF_COPY = 15
};
static __device__ unsigned long long* g_prof = nullptr;  // one per translation unit
struct ProfScope {
  long long t0;
  int id;
  __device__ __forceinline__ ProfScope(int i) : id(i) { t0 = (g_prof && ltid() == 0) ? clock64() : 0; }
  __device__ __forceinline__ ~ProfScope() {
    if (g_prof && ltid() == 0) g_prof[(long long)cta_slot() * PROF_N + id] += (unsigned long long)(clock64() - t0);
  }
};

static __device__ __forceinline__ cplx cmk(double x, double y) { return make_double2(x, y); }
static __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return make_double2(a.x + b.x, a.y + b.y); }
static __device__ __forceinline__ cplx csub(cplx a, cplx b) { return make_double2(a.x - b.x, a.y - b.y); }
static __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
static __device__ __forceinline__ cplx cconj(cplx a) { return make_double2(a.x, -a.y); }
// conj(a) * b
static __device__ __forceinline__ cplx cmulc(cplx a, cplx b) {
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
static __device__ __forceinline__ cplx cscale(cplx a, double s) { return make_double2(a.x * s, a.y * s); }
static __device__ __forceinline__ double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }
// c += a * b
static __device__ __forceinline__ void cfma(cplx& c, cplx a, cplx b) {
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(a.y, b.x, c.y);
}
// c += conj(a) * b
static __device__ __forceinline__ void cfmac(cplx& c, cplx a, cplx b) {
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(-a.y, b.x, c.y);
}

static __device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
static __device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Shared scratch used by the reductions (NW*16+16 doubles).
struct RedScratch {
  double v[NW * 16 + 16];
};

// CTA-collective sum of NV values per thread; result broadcast to every thread.
// The warp partials are added in warp order w = 0 .. NW-1 either way.  For up
// to four values every thread adds them itself (two barriers: the partials
// are written, then read before anyone may write them again); for more, NV
// threads add one value each and publish it (three barriers, fewer shared
// loads).
template <int NV>
static __device__ __forceinline__ void block_sum_n(double (&x)[NV], RedScratch& rs) {
  const int lane = ltid() & 31, wid = ltid() >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) x[k] = warp_sum(x[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) rs.v[wid * NV + k] = x[k];
  }
  cta_sync();
  if (NV <= 4) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < NW; ++w) s += rs.v[w * NV + k];
      x[k] = s;
    }
    cta_sync();
    return;
  }
  if (ltid() < NV) {
    double s = 0.0;
    for (int w = 0; w < NW; ++w) s += rs.v[w * NV + ltid()];
    rs.v[NW * 16 + ltid()] = s;
  }
  cta_sync();
#pragma unroll
  for (int k = 0; k < NV; ++k) x[k] = rs.v[NW * 16 + k];
  cta_sync();
}

static __device__ __forceinline__ double block_sum(double v, RedScratch& rs) {
  double x[1] = {v};
  block_sum_n<1>(x, rs);
  return x[0];
}

static __device__ __forceinline__ double block_max(double v, RedScratch& rs) {
  const int lane = ltid() & 31, wid = ltid() >> 5;
  v = warp_max(v);
  if (lane == 0) rs.v[wid] = v;
  cta_sync();
  double s = rs.v[0];
#pragma unroll
  for (int w = 1; w < NW; ++w) s = fmax(s, rs.v[w]);
  cta_sync();
  return s;
}

// CTA-collective copy / fill helpers.
static __device__ __forceinline__ void cta_copy(cplx* __restrict__ dst, const cplx* __restrict__ src, long long n) {
  for (long long i = ltid(); i < n; i += NT) dst[i] = src[i];
}
static __device__ __forceinline__ void cta_zero(cplx* dst, long long n) {
  for (long long i = ltid(); i < n; i += NT) dst[i] = make_double2(0.0, 0.0);
}
static __device__ __forceinline__ void cta_scale(cplx* x, long long n, double s) {
  for (long long i = ltid(); i < n; i += NT) x[i] = cscale(x[i], s);
}
static __device__ __forceinline__ double cta_norm2(const cplx* x, long long n, RedScratch& rs) {
  double s = 0.0;
  for (long long i = ltid(); i < n; i += NT) s += cabs2(x[i]);
  return block_sum(s, rs);
}
