// Shared helpers for the cytnx_b200 C ABI: thread-local error text, CUDA checks.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/cytnx_b200.h"

namespace ctn {

void set_error(const char *fmt, ...);

inline ctn_status cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
  set_error("%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  return CTN_ERR_CUDA;
}

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// ground-state Lanczos (capi.cpp); speculate queues each next iteration before the host
// solve of the current one (matvecs without side effects only: one extra call at the end);
// w_f32: mv writes its result as n floats
ctn_status lanczos_gnd(int (*mv)(void *, const double *, double *, void *), void *user, const double *psi0,
                       int64_t n, int maxiter, double cvgcrit, double *krylov, double *work, double *eigvec,
                       double *energy, int *iters, cudaStream_t st, bool speculate, bool w_f32);
// restarted split-precision ground state (capi.cpp); w_f32: mv_lo writes its result as n floats
ctn_status lanczos_refined(int (*mv_lo)(void *, const double *, double *, void *), void *u_lo,
                           int (*mv_hi)(void *, const double *, double *, void *), void *u_hi, const double *psi0,
                           int64_t n, int krydim, int max_restarts, double tol, double *krylov, double *work,
                           double *eigvec, double *energy, double *residual, int *restarts, int64_t *counts,
                           cudaStream_t st, bool w_f32);

}  // namespace ctn

#define CTN_CUDA(call)                                                 \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) return ctn::cuda_fail(e_, #call, __FILE__, __LINE__); \
  } while (0)

#define CTN_CHECK_LAUNCH()                                             \
  do {                                                                 \
    cudaError_t e_ = cudaGetLastError();                               \
    if (e_ != cudaSuccess) return ctn::cuda_fail(e_, "kernel launch", __FILE__, __LINE__); \
  } while (0)

#define CTN_REQUIRE(cond, ...)                                         \
  do {                                                                 \
    if (!(cond)) {                                                     \
      ctn::set_error(__VA_ARGS__);                                     \
      return CTN_ERR_INVALID;                                          \
    }                                                                  \
  } while (0)

#define CTN_TRY(call)                                                  \
  do {                                                                 \
    ctn_status s_ = (call);                                            \
    if (s_ != CTN_OK) return s_;                                       \
  } while (0)
