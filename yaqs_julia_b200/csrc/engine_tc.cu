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
#include "program.cuh"
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

cudaError_t tc_kernel_prepare(size_t smem_per_program, int* programs_per_sm, size_t* smem_per_cta) {
  const size_t smem = 2 * (smem_per_program - 1024) + 1024;  // one alignment slack per CTA
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

cudaError_t tc_set_prof(unsigned long long* buf) { return cudaMemcpyToSymbol(g_prof, &buf, sizeof(buf)); }
