// engine_tc.h — host interface of the tensor-core trajectory kernel
// (engine_tc.cu), the mixed form whose H_eff products run on tcgen05.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>

struct DevParams;
struct BatchRun;

// Sets the kernel's attributes and returns in *programs_per_sm how many
// programs (two per CTA) fit on one SM and in *smem_per_cta the dynamic
// shared memory to launch a CTA with (this unit's pipeline is deeper than the
// other kernels', so only it knows the size).
cudaError_t tc_kernel_prepare(int* programs_per_sm, size_t* smem_per_cta);
// One launch over `slots` programs (an even count) of the launch-list
// positions first .. first+count-1.
cudaError_t tc_kernel_launch(int slots, size_t smem_per_cta, cudaStream_t stream, const DevParams& P, int first,
                             int count);
// Points this translation unit's phase timers at [slots][PROF_N] (or null).
cudaError_t tc_set_prof(unsigned long long* buf);
// yaqs_batched_cgemm_tf32's kernel: one product per CTA, maps[2b], maps[2b+1]
// the staged A and B of problem b, status[b] = 1 when a pipeline wait gave up.
cudaError_t tc_cgemm_launch(int batch, int M, int N, int K, const CUtensorMap* maps, int a_mn, int conj_a,
                            int b_mn, int conj_b, float2* C, int* status);
// The server's two-program kernel (serve.cuh's loop), for servers that admit
// mixed-precision runs: attributes and occupancy, then one launch per batch.
cudaError_t tc_serve_prepare(int* programs_per_sm, size_t* smem_per_cta);
cudaError_t tc_serve_launch(int slots, size_t smem_per_cta, cudaStream_t stream, const BatchRun* runs, int nruns,
                            int total_units, int* counter);
// The autotuner's timing of one product form on one bucket shape: a launch
// over every slot of the run applying H_eff `reps` times to synthetic
// operands (environments of bonds bl, br; l x D x r; the MPO map of `site`);
// form: the per-bucket table (entries 0 = tcgen05, 1 = mma.sync).
cudaError_t tc_tune_time(const DevParams& P, int slots, const unsigned char* form, int bl, int br, int l, int D, int r,
                         int site, int reps, float* ms);
