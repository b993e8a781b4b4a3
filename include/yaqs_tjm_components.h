/*
 * yaqs_tjm_components.h — batched device kernels of the TJM engine exposed
 * one at a time.  Each runs one CTA per problem of the batch, on host
 * buffers (copied in and out), with the same device code the trajectory
 * engine uses.  Layouts are column-major interleaved complex, as in
 * yaqs_tjm.h.  They replace, one for one, the reference's per-call numerics:
 *
 *   yaqs_batched_svd          svd(Mat) in split_mps_tensor_svd
 *                             (src/Algorithms.jl:409-445) in the split form
 *                             the forward sweep uses: orthonormal U, the
 *                             singular values descending and S*Vt = U^H M.
 *   yaqs_batched_qr           qr(Mat) of right_qr / shift_orthogonality_center!
 *                             (src/Decompositions.jl:18-36, src/MPS.jl:197-202).
 *   yaqs_batched_project_site project_site / _project_site_ws!
 *                             (src/Algorithms.jl:215-220, :330-361).
 *   yaqs_batched_expm_site    expm_krylov(project_site, x, dt, 25)
 *                             (src/Algorithms.jl:144-187).
 */
#ifndef YAQS_TJM_COMPONENTS_H
#define YAQS_TJM_COMPONENTS_H

#include <stdint.h>

#include "yaqs_tjm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* M: batch x (m x n); U: batch x (m x k); S: batch x k; SVt: batch x (k x n);
 * k = min(m, n) <= 256, m + n <= 2048. */
int yaqs_batched_svd(yaqs_ctx* ctx, int32_t batch, int32_t m, int32_t n, const double* M, double* U,
                     double* S, double* SVt);

/* M: batch x (m x n); Q: batch x (m x k); R: batch x (k x n). */
int yaqs_batched_qr(yaqs_ctx* ctx, int32_t batch, int32_t m, int32_t n, const double* M, double* Q,
                    double* R);

/* L: batch x (chil, wl, chil); R: batch x (chir, wr, chir); W: (wl, D, D, wr) shared;
 * x, out: batch x (chil, D, chir).  D is 2 (one site) or 4 (two merged sites). */
int yaqs_batched_project_site(yaqs_ctx* ctx, int32_t batch, int32_t chil, int32_t D, int32_t chir,
                              int32_t wl, int32_t wr, const double* L, const double* R, const double* W,
                              const double* x, double* out);

/* out = exp(-i dt H_eff) x; matvecs (optional) receives the Lanczos length per problem. */
int yaqs_batched_expm_site(yaqs_ctx* ctx, int32_t batch, int32_t chil, int32_t D, int32_t chir,
                           int32_t wl, int32_t wr, const double* L, const double* R, const double* W,
                           const double* x, double dt, int32_t krylov_dim, double krylov_tol,
                           double krylov_exit_tol, double* out, int32_t* matvecs);

/* Complex FP32 product C = op(A) op(B) on the tensor cores, the building
 * block of the mixed-precision form's H_eff and environment contractions
 * (the @tensor products of src/Algorithms.jl:199-226, :330-361, in complex
 * FP32): tcgen05 MMAs in the 3-product complex form with the 3xTF32 split,
 * operand tiles loaded by TMA.  A: batch x (M x K), column-major
 * (a_kmajor = 0) or row-major (a_kmajor = 1); B: batch x (K x N), row-major
 * (b_kmajor = 0) or column-major (b_kmajor = 1); C: batch x (M x N)
 * column-major; interleaved complex64.  conj_a / conj_b conjugate the
 * operand. */
int yaqs_batched_cgemm_tf32(yaqs_ctx* ctx, int32_t batch, int32_t M, int32_t N, int32_t K, const float* A,
                            int32_t a_kmajor, int32_t conj_a, const float* B, int32_t b_kmajor, int32_t conj_b,
                            float* C);

/*
 * yaqs_batched_svd without any device allocation (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc: a host whose device
 * memory is owned by its own pool allocator (Julia's CUDA.jl, PyTorch), or
 * a code path where an allocation would synchronise the device or could fail
 * mid-run.  M, U, S and SVt are DEVICE pointers with the layouts of
 * yaqs_batched_svd; the call enqueues one kernel on `stream` (a
 * cudaStream_t, NULL for the default stream) and returns without waiting.
 * Scratch comes from a fixed 8 MiB array compiled into the library (held by
 * every GPU that loads it until exit): batch * (4 max(m,n)^2 + max(m,n) +
 * 256) complex values plus 256 ints per problem must fit, otherwise the call
 * returns YAQS_E_ARG before launching anything.  yaqs_ctx_create looks up
 * the array's device address for its device and sets the kernel's
 * shared-memory limit (this loads the library onto that GPU), so a call does
 * no set-up of its own; create the context before any stream capture, and
 * create a new one after a cudaDeviceReset.  All calls share
 * the one array and every call rewrites the scratch words it reads, so a
 * call never depends on an earlier one; calls that overlap on the GPU (two
 * streams, two threads) race on the array and must be serialised by the
 * caller.
 */
int yaqs_batched_svd_noalloc(yaqs_ctx* ctx, int32_t batch, int32_t m, int32_t n, const double* M,
                             double* U, double* S, double* SVt, void* stream);

/* The autotuner's decisions on this context's device: one row of 8 doubles
 * per measured shape (chi_l, D, chi_r, w_l, w_r, form, us per product in the
 * tcgen05 form, us per product in the mma.sync form), form 0 = tcgen05,
 * 1 = mma.sync.  The mixed form's H_eff products (project_site,
 * src/Algorithms.jl:215-220) take the chosen form per shape bucket; shapes
 * are measured once per process when a run first needs them.  Writes at
 * most `capacity` rows and the total number into *count. */
int yaqs_autotune_results(yaqs_ctx* ctx, double* rows, int32_t capacity, int32_t* count);

/* Measured FP64 FMA throughput of the device (TFLOP/s, best of 5 runs of a
 * DFMA loop over every SM): the denominator of the FP64 form's roofline. */
int yaqs_fp64_peak(yaqs_ctx* ctx, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* YAQS_TJM_COMPONENTS_H */
