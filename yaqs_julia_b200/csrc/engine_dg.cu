// engine_dg.cu — the digital trajectory kernel in 128-thread programs.
//
// A digital trajectory at the bond dimensions of Trotter circuits (2 x 2 up
// to a few dozen square) leaves most of a 256-thread program idle between
// its barriers: its merges, 4 x 4 gates, QR and Jacobi SVD steps are small
// and latency bound.  This unit compiles the same program (digital.cuh and
// everything under it) for 128 threads, so three CTAs fit on an SM (shared
// memory bounds it: one CtaSmem each) and half again as many trajectories
// advance at once with fewer threads waiting at each barrier.  The GEMM
// accumulates each output over K in the same order as the 256-thread kernel
// (its tile is 64 x 32 instead of 64 x 64); reductions add the same terms
// in another order, so the two kernels agree to rounding.
#define NT 128
#include "digital.cuh"
#include "program.cuh"
#include "engine_dg.h"

__global__ void __launch_bounds__(NT, 3) digital_step_kernel_dg(const DevParams P, const DigParams D, int first,
                                                                int count) {
  extern __shared__ __align__(16) unsigned char smraw[];
  CtaSmem& sm = *reinterpret_cast<CtaSmem*>(align_smem_1024(smraw));
  run_units(P, sm, first, count, [&D](Ctx& c, int j) { run_digital_step(c, D, j); });
}

cudaError_t dg_kernel_prepare(int* programs_per_sm, size_t* smem_per_cta) {
  const size_t smem = cta_smem_bytes();
  cudaError_t e =
      cudaFuncSetAttribute(digital_step_kernel_dg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, digital_step_kernel_dg, NT, smem);
  if (e != cudaSuccess) return e;
  *programs_per_sm = per_sm;
  *smem_per_cta = smem;
  return cudaSuccess;
}

cudaError_t dg_kernel_launch(int slots, size_t smem_per_cta, cudaStream_t stream, const DevParams& P,
                             const DigParams& D, int first, int count) {
  digital_step_kernel_dg<<<slots, NT, smem_per_cta, stream>>>(P, D, first, count);
  return cudaGetLastError();
}

cudaError_t dg_set_prof(unsigned long long* buf) { return cudaMemcpyToSymbol(g_prof, &buf, sizeof(buf)); }
