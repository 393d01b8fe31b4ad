// FP64 BLAS-1 helpers used by the Lanczos driver (device scalars, stream-ordered).
#pragma once
#include "ctn_common.h"

namespace ctn {
// bytes of the reduction workspace (partials + ticket); must be zeroed once before first use
size_t reduce_ws_bytes();
// the same for dot2s_f64 (two reductions in one pass)
size_t reduce2_ws_bytes();
ctn_status dot_f64(const double *x, const double *y, int64_t n, double *out, double *ws, cudaStream_t st);
// FP32 x (the split-precision matvec's result) against an FP64 y
ctn_status dot_f64(const float *x, const double *y, int64_t n, double *out, double *ws, cudaStream_t st);
// dst = w - alpha p1 - beta p0 with an FP32 w, ||dst|| -> *nrm (dst: the next Krylov slot)
ctn_status lanczos_update_to_f64(const float *w, const double *p1, const double *p0, double *dst, int64_t n,
                                 const double *alpha, const double *beta, double *nrm, double *ws, cudaStream_t st);
ctn_status nrm2_f64(const double *x, int64_t n, double *out, double *ws, cudaStream_t st);
ctn_status axpy_f64(const double *x, double *y, int64_t n, const double *a, double a_scale, cudaStream_t st);
ctn_status scal_f64(double *x, int64_t n, const double *a, int invert, cudaStream_t st);
ctn_status lanczos_update_f64(double *w, const double *p1, const double *p0, int64_t n, const double *alpha,
                              const double *beta, double *nrm, double *ws, cudaStream_t st);
// Krylov steps on unnormalised storage u_j = s_j q_j (s on device):
//   out_a = <w, a> / s^2, out_b = <w, b> / s  (s null: no scaling)
ctn_status dot2s_f64(const double *w, const double *a, const double *b, int64_t n, const double *s, double *out_a,
                     double *out_b, double *ws2, cudaStream_t st);
// the same with an FP32 w (the split-precision matvec output)
ctn_status dot2s_f64(const float *w, const double *a, const double *b, int64_t n, const double *s, double *out_a,
                     double *out_b, double *ws2, cudaStream_t st);
//   dst = (w - alpha u) / s - (s / sp) up - gamma q and ||dst|| -> nrm  (up, q may be null)
ctn_status lanczos_step_f64(const double *w, const double *u, const double *up, const double *q, double *dst,
                            int64_t n, const double *alpha, const double *gamma, const double *s, const double *sp,
                            double *nrm, double *ws, cudaStream_t st);
ctn_status lanczos_step_f64(const float *w, const double *u, const double *up, const double *q, double *dst,
                            int64_t n, const double *alpha, const double *gamma, const double *s, const double *sp,
                            double *nrm, double *ws, cudaStream_t st);
// dot2s_f64 then lanczos_step_f64 (out_a -> alpha, out_b -> gamma, q required) in one
// cooperative launch with a bounded grid barrier; ws and ws2 as for the two; a barrier wait
// that runs out sets *err (device word, zeroed by the caller) and alpha to NaN.  Returns
// CTN_ERR_UNSUPPORTED without launching when the device has no cooperative launch.
ctn_status krylov_step_f64(const double *w, const double *u, const double *up, const double *q, double *dst,
                           int64_t n, const double *s, const double *sp, double *out_alpha, double *out_gamma,
                           double *nrm, double *ws, double *ws2, unsigned *err, cudaStream_t st);
ctn_status krylov_step_f64(const float *w, const double *u, const double *up, const double *q, double *dst,
                           int64_t n, const double *s, const double *sp, double *out_alpha, double *out_gamma,
                           double *nrm, double *ws, double *ws2, unsigned *err, cudaStream_t st);
ctn_status div_copy_f64(const double *x, double *y, int64_t n, const double *a, cudaStream_t st);
ctn_status combine_f64(const double *K, int64_t n, int m, const double *c, double *out, cudaStream_t st);
// block Krylov helpers (basis V: m vectors of n doubles back to back)
size_t multidot_ws_doubles(int m);  // zeroed before first use (its first word is the ticket)
//   h[j] (+)= <V[j], w>, j < m
ctn_status multidot_f64(const double *V, const double *w, int64_t n, int m, double *h, int accumulate, double *ws,
                        cudaStream_t st);
//   w -= sum_j h[j] V[j]
ctn_status multiaxpy_f64(const double *V, const double *h, int64_t n, int m, double *w, cudaStream_t st);
//   out[c] = sum_j Y[j * ldy + c] V[j], c < nc
ctn_status basis_combine_f64(const double *V, int64_t n, int m, const double *Y, int ldy, int nc, double *out,
                             cudaStream_t st);
}  // namespace ctn
