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
