// engine_tc.cu — the tensor-core trajectory kernel: the mixed-precision
// analog program whose H_eff products run on tcgen05 (dev_heff_tc).
//
// It lives in its own translation unit because a kernel that holds tensor
// memory is given one CTA per SM: this kernel therefore runs two
// independent 256-thread trajectory programs per 512-thread CTA (each with
// its own shared memory, named barrier and 256 TMEM columns), while the
// kernels of engine.cu, compiled without any tcgen05 code, keep two CTAs
// per SM.
#define YAQS_TC 1
// Pipeline depth of this unit (tcgemm.cuh defaults: 2 raw, 1 plane buffer).
// Measured on the L=30 chi=64 products: 3 or 4 raw buffers and 2 plane
// buffers gave no faster GEMM (79 us for M=320 N=128 K=64 in every case)
// and the larger shared memory cost the whole kernel 7 % through L1.
#include "program.cuh"
#include "serve.cuh"
#include "engine_tc.h"

__global__ void __launch_bounds__(2 * NT, 1) tjm_step_kernel_tc(const DevParams P, int first, int count) {
  extern __shared__ __align__(16) unsigned char smraw[];
  CtaSmem* both = reinterpret_cast<CtaSmem*>(align_smem_1024(smraw));
  CtaSmem& sm = both[cta_half()];
  tc_setup(sm.e.tc);
  __syncthreads();  // both programs hold their columns: the CTA allocates no more
  if (threadIdx.x < 32) tmem_relinquish();
  run_units(P, sm, first, count, [](Ctx& c, int j) { run_step(c, j); });
  tc_teardown(sm.e.tc);
}

cudaError_t tc_kernel_prepare(int* programs_per_sm, size_t* smem_per_cta) {
  // sized here: this unit's CtaSmem holds its own (deeper) pipeline buffers
  const size_t smem = 2 * sizeof(CtaSmem) + 1024;  // one alignment slack per CTA
  cudaError_t e = cudaFuncSetAttribute(tjm_step_kernel_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tjm_step_kernel_tc, 2 * NT, smem);
  if (e != cudaSuccess) return e;
  *programs_per_sm = 2 * per_sm;
  *smem_per_cta = smem;
  return cudaSuccess;
}

cudaError_t tc_kernel_launch(int slots, size_t smem_per_cta, cudaStream_t stream, const DevParams& P, int first,
                             int count) {
  tjm_step_kernel_tc<<<slots / 2, 2 * NT, smem_per_cta, stream>>>(P, first, count);
  return cudaGetLastError();
}

// The server's kernel when it admits mixed-precision runs: the serve loop
// (serve.cuh) in two programs per CTA; FP64 and digital units run in it too.
__global__ void __launch_bounds__(2 * NT, 1) serve_kernel_tc(const BatchRun* runs, int nruns, int total_units,
                                                             int* counter) {
  extern __shared__ __align__(16) unsigned char smraw[];
  CtaSmem* both = reinterpret_cast<CtaSmem*>(align_smem_1024(smraw));
  CtaSmem& sm = both[cta_half()];
  __shared__ __align__(16) BatchRun br[2];
  tc_setup(sm.e.tc);
  __syncthreads();
  if (threadIdx.x < 32) tmem_relinquish();
  serve_units(runs, nruns, total_units, counter, sm, br[cta_half()]);
  tc_teardown(sm.e.tc);
}

cudaError_t tc_serve_prepare(int* programs_per_sm, size_t* smem_per_cta) {
  const size_t smem = 2 * sizeof(CtaSmem) + 1024;
  cudaError_t e = cudaFuncSetAttribute(serve_kernel_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_kernel_tc, 2 * NT, smem);
  if (e != cudaSuccess) return e;
  *programs_per_sm = 2 * per_sm;
  *smem_per_cta = smem;
  return cudaSuccess;
}

cudaError_t tc_serve_launch(int slots, size_t smem_per_cta, cudaStream_t stream, const BatchRun* runs, int nruns,
                            int total_units, int* counter) {
  serve_kernel_tc<<<slots / 2, 2 * NT, smem_per_cta, stream>>>(runs, nruns, total_units, counter);
  return cudaGetLastError();
}

// The autotuner's measurement: every program of the launch stages synthetic
// operands of one bucket's shape in its own slot (the environments of bonds
// bl and br, sizes l x D x r) and applies H_eff `reps` times in the product
// form the table `form` selects.  Values are deterministic and of unit size.
__global__ void __launch_bounds__(2 * NT, 1) tune_heff_kernel_tc(const DevParams P, const unsigned char* form, int bl,
                                                                 int br, int l, int D, int r, int site, int reps) {
  extern __shared__ __align__(16) unsigned char smraw[];
  CtaSmem* both = reinterpret_cast<CtaSmem*>(align_smem_1024(smraw));
  CtaSmem& sm = both[cta_half()];
  tc_setup(sm.e.tc);
  __syncthreads();
  if (threadIdx.x < 32) tmem_relinquish();
  DevParams Q = P;
  Q.tune = form;
  const int slot = cta_slot();
  Ctx c{Q, sm, Q.ws + (long long)slot * Q.lay.total, Q.wsi + (long long)slot * Q.lay.itotal, slot, 0, nullptr, nullptr};
  cplx* L = envL(c, bl);
  cplx* R = envR(c, br);
  cplx* x = c.ws + Q.lay.Q;
  cplx* y = x + Q.kry_n;
  const long long nl = (long long)l * Q.w[bl] * l, nr = (long long)r * Q.w[br] * r, nx = (long long)l * D * r;
  for (long long e = ltid(); e < nl; e += NT) L[e] = make_double2(1.0 / (1 + e % 7), 0.5 / (1 + e % 5));
  for (long long e = ltid(); e < nr; e += NT) R[e] = make_double2(0.5 / (1 + e % 3), 1.0 / (1 + e % 11));
  for (long long e = ltid(); e < nx; e += NT) x[e] = make_double2(1.0 / (1 + e % 13), 0.25);
  cta_sync();
  const WMat& W = D == 1 ? Q.wm_bond[bl] : D == 2 ? Q.wm_heff1[site] : Q.wm_heff2[site];
  const HeffOp h = make_heff(c, l, D, r, bl, br, W);
  for (int k = 0; k < reps; ++k) dev_heff(h, x, y, sm.e);
  tc_teardown(sm.e.tc);
}

cudaError_t tc_tune_time(const DevParams& P, int slots, const unsigned char* form, int bl, int br, int l, int D, int r,
                         int site, int reps, float* ms) {
  const size_t smem = 2 * sizeof(CtaSmem) + 1024;
  cudaError_t e = cudaFuncSetAttribute(tune_heff_kernel_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  cudaEvent_t e0, e1;
  if ((e = cudaEventCreate(&e0)) != cudaSuccess) return e;
  if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
    cudaEventDestroy(e0);
    return e;
  }
  tune_heff_kernel_tc<<<slots / 2, 2 * NT, smem>>>(P, form, bl, br, l, D, r, site, 1);  // warm-up
  cudaEventRecord(e0);
  tune_heff_kernel_tc<<<slots / 2, 2 * NT, smem>>>(P, form, bl, br, l, D, r, site, reps);
  cudaEventRecord(e1);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return e;
}

cudaError_t tc_set_prof(unsigned long long* buf) { return cudaMemcpyToSymbol(g_prof, &buf, sizeof(buf)); }

// One complex FP32 product per CTA on the tensor cores (tcgen05 + TMA): the
// yaqs_batched_cgemm_tf32 component, with the pipeline of the engine.
struct CgemmSmem {
  TcSmem t;
  TcState st;
};
__global__ void __launch_bounds__(NT, 1) cgemm_tc_kernel(int M, int N, int K, const CUtensorMap* maps, int a_mn,
                                                         int conj_a, int b_mn, int conj_b, float2* C, int* status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  CgemmSmem& sm = *reinterpret_cast<CgemmSmem*>(align_smem_1024(smraw));
  tc_setup(sm.st);
  const TcOp A{maps + 2 * blockIdx.x, a_mn, conj_a};
  const TcOp B{maps + 2 * blockIdx.x + 1, b_mn, conj_b};
  const bool ok = tc_gemm<float2>(M, N, K, A, B, C + (long long)M * N * blockIdx.x, 1, M, false, sm.t, sm.st);
  if (ltid() == 0) status[blockIdx.x] = ok ? 0 : 1;
  tc_teardown(sm.st);
}

cudaError_t tc_cgemm_launch(int batch, int M, int N, int K, const CUtensorMap* maps, int a_mn, int conj_a, int b_mn,
                            int conj_b, float2* C, int* status) {
  const size_t smem = sizeof(CgemmSmem) + 1024;
  cudaError_t e = cudaFuncSetAttribute(cgemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  cgemm_tc_kernel<<<batch, NT, smem>>>(M, N, K, maps, a_mn, conj_a, b_mn, conj_b, C, status);
  return cudaGetLastError();
}
