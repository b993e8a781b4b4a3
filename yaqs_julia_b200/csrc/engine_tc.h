// engine_tc.h — host interface of the tensor-core trajectory kernel
// (engine_tc.cu), the mixed form whose H_eff products run on tcgen05.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

struct DevParams;

// Sets the kernel's attributes for `smem_per_program` bytes of dynamic shared
// memory per trajectory program (alignment slack included) and returns in
// *programs_per_sm how many programs (two per CTA) fit on one SM and in
// *smem_per_cta the bytes to launch a CTA with.
cudaError_t tc_kernel_prepare(size_t smem_per_program, int* programs_per_sm, size_t* smem_per_cta);
// One launch over `slots` programs (an even count) of the launch-list
// positions first .. first+count-1.
cudaError_t tc_kernel_launch(int slots, size_t smem_per_cta, cudaStream_t stream, const DevParams& P, int first,
                             int count);
// Points this translation unit's phase timers at [slots][PROF_N] (or null).
cudaError_t tc_set_prof(unsigned long long* buf);
