// FP64 BLAS-1 for the Lanczos recurrence: warp-shuffle reductions and fused updates.
//
// Replaces the per-block cublasDdot / cublasDnrm2 / elementwise kernels the reference
// drives from Lanczos_Gnd_Ut (src/linalg/Lanczos_Gnd_Ut.cpp:95-140, BlockUniTensor
// Norm :1356-1375 and Add_/Sub_/Mul_ :1703-1815).  All blocks of a block-sparse
// tensor live in one flat buffer here, so each BLAS-1 step is ONE kernel over the
// whole vector instead of one library call per block.  Reductions: grid-stride
// loads in 16-byte vectors, warp __shfl_down_sync trees, one partial per CTA in
// shared memory, and a last-CTA-done finish (threadfence + atomic ticket) so the
// result is complete in device memory when the kernel ends -- deterministic
// summation order for a fixed grid.
#include <algorithm>

#include "ctn_common.h"
#include "blas1.cuh"

namespace ctn {

namespace {
constexpr int RT = 256;       // threads per CTA
constexpr int MAXCTA = 1024;  // partials buffer size

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[RT / 32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = lane < RT / 32 ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

// finish: last CTA sums the partials in a fixed order; op 0 = plain, 1 = sqrt
__device__ void finish(double part, double *partials, unsigned *ticket, double *out, int op) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = part;
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  double v = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += RT) v += ((volatile double *)partials)[i];
  v = block_sum(v);
  if (threadIdx.x == 0) {
    *out = op == 1 ? sqrt(v) : v;
    *ticket = 0u;  // re-arm for the next launch
  }
}

__global__ void __launch_bounds__(RT) k_dot(const double *__restrict__ x, const double *__restrict__ y,
                                           int64_t n, double *partials, unsigned *ticket,
                                           double *out, int op) {
  double s = 0.0;
  const int64_t tid = (int64_t)blockIdx.x * RT + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * RT;
  const bool vec = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
  if (vec) {
    const int64_t n2 = n / 2;
    const double2 *x2 = reinterpret_cast<const double2 *>(x);
    const double2 *y2 = reinterpret_cast<const double2 *>(y);
    for (int64_t i = tid; i < n2; i += step) {
      double2 a = x2[i], b = y2[i];
      s = fma(a.x, b.x, s);
      s = fma(a.y, b.y, s);
    }
    if (tid == 0 && (n & 1)) s = fma(x[n - 1], y[n - 1], s);
  } else {
    for (int64_t i = tid; i < n; i += step) s = fma(x[i], y[i], s);
  }
  s = block_sum(s);
  finish(s, partials, ticket, out, op);
}

// y += (a_scale * *a) * x
__global__ void __launch_bounds__(RT) k_axpy(const double *__restrict__ x, double *__restrict__ y,
                                            int64_t n, const double *a, double a_scale) {
  const double al = a_scale * (*a);
  const int64_t step = (int64_t)gridDim.x * RT;
  for (int64_t i = (int64_t)blockIdx.x * RT + threadIdx.x; i < n; i += step) y[i] = fma(al, x[i], y[i]);
}

// x *= a (or x /= a when invert)
__global__ void __launch_bounds__(RT) k_scal(double *__restrict__ x, int64_t n, const double *a, int invert) {
  const double al = *a;
  const int64_t step = (int64_t)gridDim.x * RT;
  for (int64_t i = (int64_t)blockIdx.x * RT + threadIdx.x; i < n; i += step) x[i] = invert ? x[i] / al : x[i] * al;
}

// w = w - alpha*p1 - beta*p0 ; and ||w||^2 reduction in the same pass.  alpha from
// device memory (just computed by k_dot), beta from device memory.
__global__ void __launch_bounds__(RT) k_lanczos_update(double *__restrict__ w, const double *__restrict__ p1,
                                                      const double *__restrict__ p0, int64_t n,
                                                      const double *alpha, const double *beta,
                                                      double *partials, unsigned *ticket, double *nrm) {
  const double a = *alpha;
  const double b = p0 ? *beta : 0.0;
  double s = 0.0;
  const int64_t step = (int64_t)gridDim.x * RT;
  for (int64_t i = (int64_t)blockIdx.x * RT + threadIdx.x; i < n; i += step) {
    double v = w[i] - a * p1[i];
    if (p0) v -= b * p0[i];
    w[i] = v;
    s = fma(v, v, s);
  }
  s = block_sum(s);
  finish(s, partials, ticket, nrm, 1);
}

// w -= alpha*p1 + beta*p0 + gamma*q, ||w|| to *nrm (p0 / q may be null)
__global__ void __launch_bounds__(RT) k_lanczos_update3(double *__restrict__ w, const double *__restrict__ p1,
                                                       const double *__restrict__ p0, const double *__restrict__ q,
                                                       int64_t n, const double *alpha, const double *beta,
                                                       const double *gamma, double *partials, unsigned *ticket,
                                                       double *nrm) {
  const double a = *alpha;
  const double b = p0 ? *beta : 0.0;
  const double c = q ? *gamma : 0.0;
  double s = 0.0;
  const int64_t step = (int64_t)gridDim.x * RT;
  for (int64_t i = (int64_t)blockIdx.x * RT + threadIdx.x; i < n; i += step) {
    double v = w[i] - a * p1[i];
    if (p0) v -= b * p0[i];
    if (q) v -= c * q[i];
    w[i] = v;
    s = fma(v, v, s);
  }
  s = block_sum(s);
  finish(s, partials, ticket, nrm, 1);
}

// y = x / *a (y = 0 when *a is zero: a Lanczos breakdown leaves the next vector empty)
__global__ void __launch_bounds__(RT) k_div_copy(const double *__restrict__ x, double *__restrict__ y,
                                                int64_t n, const double *a) {
  const double al = *a;
  const bool zero = al == 0.0;
  const int64_t step = (int64_t)gridDim.x * RT;
  for (int64_t i = (int64_t)blockIdx.x * RT + threadIdx.x; i < n; i += step) y[i] = zero ? 0.0 : x[i] / al;
}

// <w, a> and <w, b> in one pass over w (two reductions, partials side by side)
__global__ void __launch_bounds__(RT) k_dot2(const double *__restrict__ w, const double *__restrict__ a,
                                            const double *__restrict__ b, int64_t n, double *partials,
                                            unsigned *ticket, double *out_a, double *out_b) {
  double sa = 0.0, sb = 0.0;
  const int64_t step = (int64_t)gridDim.x * RT;
  for (int64_t i = (int64_t)blockIdx.x * RT + threadIdx.x; i < n; i += step) {
    const double x = w[i];
    sa = fma(x, a[i], sa);
    sb = fma(x, b[i], sb);
  }
  sa = block_sum(sa);
  sb = block_sum(sb);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = sa;
    partials[2 * blockIdx.x + 1] = sb;
    __threadfence();
    const unsigned t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  double va = 0.0, vb = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += RT) {
    va += ((volatile double *)partials)[2 * i];
    vb += ((volatile double *)partials)[2 * i + 1];
  }
  va = block_sum(va);
  vb = block_sum(vb);
  if (threadIdx.x == 0) {
    *out_a = va;
    *out_b = vb;
    *ticket = 0u;
  }
}

// out = sum_j c[j] * K[j]  (Krylov combination), c on device
__global__ void __launch_bounds__(RT) k_combine(const double *__restrict__ K, int64_t n, int m,
                                               const double *__restrict__ c, double *__restrict__ out) {
  const int64_t step = (int64_t)gridDim.x * RT;
  for (int64_t i = (int64_t)blockIdx.x * RT + threadIdx.x; i < n; i += step) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) s = fma(c[j], K[(int64_t)j * n + i], s);
    out[i] = s;
  }
}

int grid_for(int64_t n) {
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 148;
  }
  int64_t g = (n + RT * 4 - 1) / (RT * 4);
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, std::min<int64_t>((int64_t)nsm * 4, MAXCTA)));
}
}  // namespace

size_t reduce_ws_bytes() { return (MAXCTA + 8) * sizeof(double); }
size_t reduce2_ws_bytes() { return (2 * MAXCTA + 8) * sizeof(double); }

// ws2 layout: [2 * MAXCTA partials][ticket]
ctn_status dot2_f64(const double *w, const double *a, const double *b, int64_t n, double *out_a, double *out_b,
                    double *ws2, cudaStream_t st) {
  const int g = grid_for(n);
  k_dot2<<<g, RT, 0, st>>>(w, a, b, n, ws2, reinterpret_cast<unsigned *>(ws2 + 2 * MAXCTA), out_a, out_b);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}

// ws layout: [partials MAXCTA doubles][ticket (8 bytes)]
ctn_status dot_f64(const double *x, const double *y, int64_t n, double *out, double *ws, cudaStream_t st) {
  int g = grid_for(n);
  k_dot<<<g, RT, 0, st>>>(x, y, n, ws, reinterpret_cast<unsigned *>(ws + MAXCTA), out, 0);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status nrm2_f64(const double *x, int64_t n, double *out, double *ws, cudaStream_t st) {
  int g = grid_for(n);
  k_dot<<<g, RT, 0, st>>>(x, x, n, ws, reinterpret_cast<unsigned *>(ws + MAXCTA), out, 1);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status axpy_f64(const double *x, double *y, int64_t n, const double *a, double a_scale, cudaStream_t st) {
  k_axpy<<<grid_for(n), RT, 0, st>>>(x, y, n, a, a_scale);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status scal_f64(double *x, int64_t n, const double *a, int invert, cudaStream_t st) {
  k_scal<<<grid_for(n), RT, 0, st>>>(x, n, a, invert);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status lanczos_update_f64(double *w, const double *p1, const double *p0, int64_t n, const double *alpha,
                              const double *beta, double *nrm, double *ws, cudaStream_t st) {
  int g = grid_for(n);
  k_lanczos_update<<<g, RT, 0, st>>>(w, p1, p0, n, alpha, beta, ws, reinterpret_cast<unsigned *>(ws + MAXCTA), nrm);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status lanczos_update3_f64(double *w, const double *p1, const double *p0, const double *q, int64_t n,
                               const double *alpha, const double *beta, const double *gamma, double *nrm, double *ws,
                               cudaStream_t st) {
  const int g = std::min(grid_for(n), MAXCTA);
  k_lanczos_update3<<<g, RT, 0, st>>>(w, p1, p0, q, n, alpha, beta, gamma, ws,
                                      reinterpret_cast<unsigned *>(ws + MAXCTA), nrm);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status div_copy_f64(const double *x, double *y, int64_t n, const double *a, cudaStream_t st) {
  k_div_copy<<<grid_for(n), RT, 0, st>>>(x, y, n, a);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status combine_f64(const double *K, int64_t n, int m, const double *c, double *out, cudaStream_t st) {
  k_combine<<<grid_for(n), RT, 0, st>>>(K, n, m, c, out);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}

}  // namespace ctn
