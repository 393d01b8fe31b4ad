// FP64 BLAS-1 helpers used by the Lanczos driver (device scalars, stream-ordered).
#pragma once
#include "ctn_common.h"

namespace ctn {
// bytes of the reduction workspace (partials + ticket); must be zeroed once before first use
size_t reduce_ws_bytes();
// the same for dot2_f64 (two reductions in one pass)
size_t reduce2_ws_bytes();
ctn_status dot2_f64(const double *w, const double *a, const double *b, int64_t n, double *out_a, double *out_b,
                    double *ws2, cudaStream_t st);
ctn_status dot_f64(const double *x, const double *y, int64_t n, double *out, double *ws, cudaStream_t st);
ctn_status nrm2_f64(const double *x, int64_t n, double *out, double *ws, cudaStream_t st);
ctn_status axpy_f64(const double *x, double *y, int64_t n, const double *a, double a_scale, cudaStream_t st);
ctn_status scal_f64(double *x, int64_t n, const double *a, int invert, cudaStream_t st);
ctn_status lanczos_update_f64(double *w, const double *p1, const double *p0, int64_t n, const double *alpha,
                              const double *beta, double *nrm, double *ws, cudaStream_t st);
ctn_status lanczos_update3_f64(double *w, const double *p1, const double *p0, const double *q, int64_t n,
                               const double *alpha, const double *beta, const double *gamma, double *nrm, double *ws,
                               cudaStream_t st);
ctn_status div_copy_f64(const double *x, double *y, int64_t n, const double *a, cudaStream_t st);
ctn_status combine_f64(const double *K, int64_t n, int m, const double *c, double *out, cudaStream_t st);
}  // namespace ctn
