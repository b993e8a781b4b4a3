// tcgemm.cuh — CTA-level complex FP32 GEMM on the 5th-generation tensor
// cores (tcgen05), operands fed by TMA.
//
// C(m,n) = op(A)(m,k) op(B)(k,n) for complex FP32 operands held in staging
// buffers of global memory, each described by a 2D FP32 tensor map (inner
// dimension contiguous, a fixed row pitch).  A staged operand is either
// "MN-major" (each staged row is one k, the inner dimension runs over m or
// n) or "K-major" (each staged row is one m or n, the inner dimension runs
// over k).  The tensor map's box is fixed by that role:
//   A, MN-major: 128 complex (m) x 8 rows (k)      A, K-major: 8 complex (k) x 128 rows (m)
//   B, MN-major:  64 complex (n) x 8 rows (k)      B, K-major: 8 complex (k) x  64 rows (n)
//
// Arithmetic: the 3-product (Gauss) complex form
//   P1 = Ar Br,  P2 = Ai Bi,  P3 = (Ar + Ai)(Br + Bi)
//   re = P1 - P2,  im = P3 - P1 - P2,
// each real product X Y as three TF32 products X_hi Y_hi + X_hi Y_lo +
// X_lo Y_hi (X_hi = tf32(X), X_lo = tf32(X - X_hi)), accumulated in FP32 in
// tensor memory: nine tcgen05.mma.kind::tf32 (M = 128, N <= 64, K = 8) per
// K step into three accumulators of 64 columns each.
//
// Pipeline per 128 x 64 output tile, K in steps of 8: thread 0 issues the
// TMA loads of step k+1 (raw FP32 complex tiles into one of two raw
// buffers, completion on that buffer's mbarrier) while the 256 threads of
// the program wait for the MMAs of step k-1 to release the planes, then
// split the raw tile of step k into six TF32 planes (re, im, re+im; hi and
// lo) laid out in the canonical K-major no-swizzle layout the MMA reads
// (8-row x 16-byte core matrices; 128 bytes between the two K halves, 256
// bytes between 8-row groups); thread 0 then issues the nine MMAs and
// commits them to the plane mbarrier.  One plane buffer keeps the pipeline
// within the shared memory the FP64 GEMM staging already takes (60 KB).
// The epilogue reads the accumulators with tcgen05.ld (warp w owns TMEM
// lanes 32 (w % 4) .. +31, warps 0-3 the first 32 columns, warps 4-7 the
// rest) and writes C in FP32 or FP64 with general strides.
//
// Every wait is bounded; a wait that gives up sets TcState::fatal, after
// which every later call returns at once and the caller reports a timeout.
#pragma once
#include <cuda.h>
#include "common.cuh"

#define TC_BM 128
#define TC_BN 64
#define TC_BK 8
#define TC_TMEM_COLS 256  // three accumulators of 64 columns (power of two >= 192)
#define TMEM_PROGRAMS_PER_SM 2  // 512 TMEM columns per SM / TC_TMEM_COLS
#define TC_WAIT_SPINS (1LL << 24)

// Shared memory of the pipeline (never live together with the other GEMM or
// SVD staging; the engine keeps it in the same union).
// Pipeline depth: TC_RAW_STAGES raw TMA buffers (TMA runs that many K steps
// minus one ahead) and TC_PLANE_STAGES plane buffers (with two, the split of
// step k+1 overlaps the MMAs of step k).  The defaults fit the FP64 GEMM
// staging; the tensor-core kernel's translation unit may set deeper ones.
#ifndef TC_RAW_STAGES
#define TC_RAW_STAGES 2
#endif
#ifndef TC_PLANE_STAGES
#define TC_PLANE_STAGES 1
#endif
struct __align__(1024) TcSmem {
  float rawA[TC_RAW_STAGES][2048];             // 8 KB each: one A box (128 x 8 complex)
  float rawB[TC_RAW_STAGES][1024];             // 4 KB each: one B box (8 x 64 complex)
  unsigned planeA[TC_PLANE_STAGES][6][1024];   // 6 planes x (128 rows x 8 k) tf32
  unsigned planeB[TC_PLANE_STAGES][6][512];    // 6 planes x (64 rows x 8 k) tf32
};

// State that persists across calls (outside the union).
struct TcState {
  unsigned long long bar_raw[TC_RAW_STAGES];
  unsigned long long bar_mma[TC_PLANE_STAGES];
  unsigned tmem_base;
  unsigned ph_raw;  // bit s: parity of the next phase of bar_raw[s]
  unsigned ph_mma;  // bit s: parity of the next phase of bar_mma[s]
  int fatal;
};

// One staged operand.
struct TcOp {
  const CUtensorMap* map;  // tensor map in global memory (written before the launch)
  int mn;                  // 1: MN-major staging, 0: K-major staging
  int conj;                // use the complex conjugate
};

static __device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

static __device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
static __device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
static __device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of parity `parity`; false when it gave up.
static __device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  for (long long it = 0; it < TC_WAIT_SPINS; ++it) {
    if (mbar_test(bar, parity)) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

static __device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
static __device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

static __device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
static __device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
static __device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
static __device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Warp-collective TMEM allocation / release.
static __device__ __forceinline__ void tmem_alloc(unsigned* dst, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
static __device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
static __device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

static __device__ __forceinline__ void tc_mma_tf32(unsigned d_tmem, unsigned long long adesc, unsigned long long bdesc,
                                            unsigned idesc, unsigned accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
static __device__ __forceinline__ void tc_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
static __device__ __forceinline__ void tmem_ld16(unsigned taddr, float (&v)[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
static __device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor, canonical K-major layout without
// swizzle: LBO = bytes between the two 16-byte K halves of an 8-row core
// matrix group, SBO = bytes between consecutive 8-row groups.
static __device__ __forceinline__ unsigned long long tc_sdesc(const void* p, unsigned lbo, unsigned sbo) {
  unsigned long long d = (unsigned long long)((smem_u32(p) >> 4) & 0x3FFFu);
  d |= (unsigned long long)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (unsigned long long)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;  // descriptor version of sm_100
  return d;         // base offset 0, absolute LBO mode, no swizzle
}

// Instruction descriptor: TF32 x TF32 -> FP32, A and B K-major, M = 128, N.
static __device__ __forceinline__ unsigned tc_idesc(int n) {
  return (1u << 4)            // D format FP32
         | (2u << 7)          // A format TF32
         | (2u << 10)         // B format TF32
         | ((unsigned)(n >> 3) << 17) | ((unsigned)(TC_BM >> 4) << 24);
}

static __device__ __forceinline__ unsigned tf32_rna(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

// Byte offset of (row r, k quad q) inside a K-major plane.
static __device__ __forceinline__ int tc_plane_off(int r, int q) { return (r >> 3) * 256 + q * 128 + (r & 7) * 16; }

// Splits four complex values (one row, one k quad) into the six planes.
static __device__ __forceinline__ void tc_split_store(unsigned* planes, int plane_words, int r, int q, const float2 (&v)[4]) {
  unsigned hr[4], lr[4], hi_[4], li[4], hs[4], ls[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float re = v[j].x, im = v[j].y, su = re + im;
    hr[j] = tf32_rna(re);
    lr[j] = tf32_rna(re - __uint_as_float(hr[j]));
    hi_[j] = tf32_rna(im);
    li[j] = tf32_rna(im - __uint_as_float(hi_[j]));
    hs[j] = tf32_rna(su);
    ls[j] = tf32_rna(su - __uint_as_float(hs[j]));
  }
  const int w = tc_plane_off(r, q) >> 2;
  *reinterpret_cast<uint4*>(planes + 0 * plane_words + w) = make_uint4(hr[0], hr[1], hr[2], hr[3]);
  *reinterpret_cast<uint4*>(planes + 1 * plane_words + w) = make_uint4(lr[0], lr[1], lr[2], lr[3]);
  *reinterpret_cast<uint4*>(planes + 2 * plane_words + w) = make_uint4(hi_[0], hi_[1], hi_[2], hi_[3]);
  *reinterpret_cast<uint4*>(planes + 3 * plane_words + w) = make_uint4(li[0], li[1], li[2], li[3]);
  *reinterpret_cast<uint4*>(planes + 4 * plane_words + w) = make_uint4(hs[0], hs[1], hs[2], hs[3]);
  *reinterpret_cast<uint4*>(planes + 5 * plane_words + w) = make_uint4(ls[0], ls[1], ls[2], ls[3]);
}

// Reads the four complex values of row r (global r0 + r), k quad q of a raw
// box; zero outside the matrix.  rows_box: 128 (A) or 64 (B).
static __device__ __forceinline__ void tc_raw_quad(const float* raw, int mn, int rows_box, int r, int q, bool row_ok, int k0,
                                            int K, bool conj, float2 (&v)[4]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = 4 * q + j;
    float2 x = make_float2(0.f, 0.f);
    if (row_ok && k0 + k < K) {
      const int e = mn ? (k * rows_box + r) : (r * TC_BK + k);
      x = *reinterpret_cast<const float2*>(raw + 2 * e);
      if (conj) x.y = -x.y;
    }
    v[j] = x;
  }
}

static __device__ __forceinline__ void tc_store_c(float2* c, float re, float im, bool acc) {
  if (acc) {
    const float2 o = *c;
    re += o.x;
    im += o.y;
  }
  *c = make_float2(re, im);
}
static __device__ __forceinline__ void tc_store_c(double2* c, float re, float im, bool acc) {
  double r = re, i = im;
  if (acc) {
    const double2 o = *c;
    r += o.x;
    i += o.y;
  }
  *c = make_double2(r, i);
}

// Called once per program before the first tc_gemm: thread-0 barrier
// set-up and a warp-0 allocation of TC_TMEM_COLS columns.  Collective over
// the program's NT threads.  The kernel relinquishes the CTA's allocation
// permit once every program of the CTA has allocated.
static __device__ __forceinline__ void tc_setup(TcState& st) {
  if (ltid() == 0) {
    for (int r = 0; r < TC_RAW_STAGES; ++r) mbar_init(&st.bar_raw[r], 1);
    for (int r = 0; r < TC_PLANE_STAGES; ++r) mbar_init(&st.bar_mma[r], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    st.ph_raw = 0;
    st.ph_mma = 0;
    st.fatal = 0;
  }
  if (ltid() < 32) tmem_alloc(&st.tmem_base, TC_TMEM_COLS);
  tc_fence_before();
  cta_sync();
  tc_fence_after();
}

// Releases the program's TMEM columns.  Collective over the program's
// threads; its last call.
static __device__ __forceinline__ void tc_teardown(TcState& st) {
  tc_fence_before();
  cta_sync();
  tc_fence_after();
  if (ltid() < 32) tmem_dealloc(st.tmem_base, TC_TMEM_COLS);
}

// C = op(A) op(B) (+ C when accumulate), M x N x K, C element (m, n) at
// C[m cm + n cn], TC = float2 or double2.  Returns false after a wait gave
// up (the CTA's tensor-core state is then unusable).  CTA-collective; ends
// with C visible to the whole CTA.
template <class TC>
static __device__ __noinline__ bool tc_gemm(int M, int N, int K, const TcOp A, const TcOp B, TC* C, long long cm, long long cn,
                                     bool accumulate, TcSmem& s, TcState& st) {
  ProfScope prof_scope_(PF_GEMM);
  const int tid = ltid(), lane = tid & 31, wid = tid >> 5;
  cta_sync();
  if (st.fatal) return false;
  // producers of the staged operands wrote them through the generic proxy
  fence_async_global();
  if (tid == 0) {  // the tensor maps live in global memory: start their descriptor fetch
    tma_prefetch_map(A.map);
    tma_prefetch_map(B.map);
  }
  cta_sync();
  unsigned ph_raw = st.ph_raw, ph_mma = st.ph_mma;
  bool ok = true;
  const int nM = (M + TC_BM - 1) / TC_BM, nN = (N + TC_BN - 1) / TC_BN, nK = (K + TC_BK - 1) / TC_BK;
  const unsigned BYTES = (TC_BM + TC_BN) * TC_BK * 8;
  const int G = nM * nN * nK;  // K steps of all tiles, one stream
  // TMA of step g into raw stage g % TC_RAW_STAGES
  auto issue = [&](int g) {
    const int t = g / nK, kc = g - t * nK, stg = g % TC_RAW_STAGES;
    const int m0 = (t / nN) * TC_BM, n0 = (t % nN) * TC_BN, k0 = kc * TC_BK;
    mbar_arrive_expect_tx(&st.bar_raw[stg], BYTES);
    if (A.mn)
      tma_load_2d(s.rawA[stg], A.map, 2 * m0, k0, &st.bar_raw[stg]);
    else
      tma_load_2d(s.rawA[stg], A.map, 2 * k0, m0, &st.bar_raw[stg]);
    if (B.mn)
      tma_load_2d(s.rawB[stg], B.map, 2 * n0, k0, &st.bar_raw[stg]);
    else
      tma_load_2d(s.rawB[stg], B.map, 2 * k0, n0, &st.bar_raw[stg]);
  };
  unsigned pend = 0;  // bit p: a commit on bar_mma[p] not yet waited for
  auto wait_mma = [&](int p) {
    if (pend & (1u << p)) {
      ok &= mbar_wait(&st.bar_mma[p], (ph_mma >> p) & 1);
      ph_mma ^= 1u << p;
      pend &= ~(1u << p);
    }
  };
  if (tid == 0)
    for (int g = 0; g < TC_RAW_STAGES - 1 && g < G; ++g) issue(g);
  for (int t = 0; t < nM * nN; ++t) {
    const int m0 = (t / nN) * TC_BM, n0 = (t % nN) * TC_BN;
    const int nrem = min(TC_BN, N - n0);
    const int nmma = (nrem + 15) & ~15;
    const unsigned idesc = tc_idesc(nmma);
    for (int kc = 0; kc < nK; ++kc) {
      const int g = t * nK + kc;
      const int sg = g % TC_RAW_STAGES, pl = g % TC_PLANE_STAGES;
      // raw stage (g - 1) % R was split at step g - 1, before its barrier
      if (tid == 0 && g + TC_RAW_STAGES - 1 < G) issue(g + TC_RAW_STAGES - 1);
      ok &= mbar_wait(&st.bar_raw[sg], (ph_raw >> sg) & 1);
      ph_raw ^= 1u << sg;
      wait_mma(pl);  // the MMAs that last read these planes are done
      const int k0 = kc * TC_BK;
      {  // A: 128 rows x 2 k quads, one item per thread
        const int r = tid & 127, q = tid >> 7;
        float2 v[4];
        tc_raw_quad(s.rawA[sg], A.mn, TC_BM, r, q, m0 + r < M, k0, K, A.conj != 0, v);
        tc_split_store(&s.planeA[pl][0][0], 1024, r, q, v);
      }
      if (tid < 128) {  // B: 64 rows x 2 k quads
        const int r = tid & 63, q = tid >> 6;
        float2 v[4];
        tc_raw_quad(s.rawB[sg], B.mn, TC_BN, r, q, n0 + r < N, k0, K, B.conj != 0, v);
        tc_split_store(&s.planeB[pl][0][0], 512, r, q, v);
      }
      fence_async_smem();
      cta_sync();
      if (tid == 0) {
        tc_fence_after();
        const unsigned* pa = &s.planeA[pl][0][0];
        const unsigned* pb = &s.planeB[pl][0][0];
#pragma unroll
        for (int acc = 0; acc < 3; ++acc) {
          const unsigned long long ah = tc_sdesc(pa + (2 * acc) * 1024, 128, 256);
          const unsigned long long al = tc_sdesc(pa + (2 * acc + 1) * 1024, 128, 256);
          const unsigned long long bh = tc_sdesc(pb + (2 * acc) * 512, 128, 256);
          const unsigned long long bl = tc_sdesc(pb + (2 * acc + 1) * 512, 128, 256);
          const unsigned d = st.tmem_base + acc * TC_BN;
          tc_mma_tf32(d, ah, bl, idesc, kc > 0 ? 1u : 0u);
          tc_mma_tf32(d, al, bh, idesc, 1u);
          tc_mma_tf32(d, ah, bh, idesc, 1u);
        }
        tc_commit(&st.bar_mma[pl]);
      }
      pend |= 1u << pl;
    }
    // all MMAs of the tile done (commits complete in issue order)
    for (int p = 0; p < TC_PLANE_STAGES; ++p) wait_mma((t * nK + nK + p) % TC_PLANE_STAGES);
    tc_fence_after();
    // epilogue
    const int quarter = wid & 3, half = wid >> 2;
    const int m = m0 + quarter * 32 + lane;
    const unsigned lane_addr = st.tmem_base + ((unsigned)(quarter * 32) << 16);
#pragma unroll 1
    for (int c16 = 0; c16 < 2; ++c16) {
      const int col = half * 32 + c16 * 16;
      if (col >= nrem) break;  // uniform per warp
      float p1[16], p2[16], p3[16];
      tmem_ld16(lane_addr + 0 * TC_BN + col, p1);
      tmem_ld16(lane_addr + 1 * TC_BN + col, p2);
      tmem_ld16(lane_addr + 2 * TC_BN + col, p3);
      tmem_wait_ld();
      if (m < M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = n0 + col + j;
          if (n < N) tc_store_c(C + (long long)m * cm + (long long)n * cn, p1[j] - p2[j], p3[j] - p1[j] - p2[j], accumulate);
        }
      }
    }
    tc_fence_before();
    cta_sync();
  }
  if (!ok) st.fatal = 1;  // benign race: every writer stores 1
  cta_sync();
  if (tid == 0) {
    st.ph_raw = ph_raw;
    st.ph_mma = ph_mma;
  }
  const bool good = !st.fatal;
  cta_sync();
  return good;
}
