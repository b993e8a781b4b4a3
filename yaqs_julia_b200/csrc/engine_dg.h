// engine_dg.h — host interface of the small-program digital kernel
// (engine_dg.cu): the digital TJM program on 128-thread CTAs, three per SM.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

struct DevParams;
struct DigParams;

// Sets the kernel's attributes and returns in *programs_per_sm how many
// 128-thread programs fit on one SM and in *smem_per_cta the dynamic shared
// memory of one (this unit's CtaSmem; only it knows the size).
cudaError_t dg_kernel_prepare(int* programs_per_sm, size_t* smem_per_cta);
// One launch over `slots` programs of the launch-list positions
// first .. first+count-1.
cudaError_t dg_kernel_launch(int slots, size_t smem_per_cta, cudaStream_t stream, const DevParams& P,
                             const DigParams& D, int first, int count);
// Points this translation unit's phase timers at [slots][PROF_N] (or null).
cudaError_t dg_set_prof(unsigned long long* buf);
