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

// two consecutive elements (pair index i) of w as doubles: one 16-byte load for FP64, one
// 8-byte load for FP32
__device__ __forceinline__ double2 ld_pair(const double *w, int64_t i) {
  return reinterpret_cast<const double2 *>(w)[i];
}
__device__ __forceinline__ double2 ld_pair(const float *w, int64_t i) {
  const float2 v = reinterpret_cast<const float2 *>(w)[i];
  return make_double2((double)v.x, (double)v.y);
}

template <typename XT>
__global__ void __launch_bounds__(RT) k_dot(const XT *__restrict__ x, const double *__restrict__ y,
                                           int64_t n, double *partials, unsigned *ticket,
                                           double *out, int op) {
  double s = 0.0;
  const int64_t tid = (int64_t)blockIdx.x * RT + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * RT;
  const bool vec = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
  if (vec) {
    const int64_t n2 = n / 2;
    const double2 *y2 = reinterpret_cast<const double2 *>(y);
    for (int64_t i = tid; i < n2; i += step) {
      const double2 a = ld_pair(x, i), b = y2[i];
      s = fma(a.x, b.x, s);
      s = fma(a.y, b.y, s);
    }
    if (tid == 0 && (n & 1)) s = fma((double)x[n - 1], y[n - 1], s);
  } else {
    for (int64_t i = tid; i < n; i += step) s = fma((double)x[i], y[i], s);
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
  const int64_t tid = (int64_t)blockIdx.x * RT + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * RT;
  auto one = [&](double wv, double pv1, double pv0) -> double {
    double v = wv - a * pv1;
    if (p0) v -= b * pv0;
    s = fma(v, v, s);
    return v;
  };
  const bool vec = ((reinterpret_cast<uintptr_t>(w) | reinterpret_cast<uintptr_t>(p1) |
                     reinterpret_cast<uintptr_t>(p0)) & 15) == 0;
  if (vec) {
    const int64_t n2 = n / 2;
    double2 *w2 = reinterpret_cast<double2 *>(w);
    const double2 *a2 = reinterpret_cast<const double2 *>(p1), *b2 = reinterpret_cast<const double2 *>(p0);
    const double2 z = make_double2(0.0, 0.0);
    for (int64_t i = tid; i < n2; i += step) {
      const double2 x = w2[i], y = a2[i], q = p0 ? b2[i] : z;
      w2[i] = make_double2(one(x.x, y.x, q.x), one(x.y, y.y, q.y));
    }
    if (tid == 0 && (n & 1)) w[n - 1] = one(w[n - 1], p1[n - 1], p0 ? p0[n - 1] : 0.0);
  } else {
    for (int64_t i = tid; i < n; i += step) w[i] = one(w[i], p1[i], p0 ? p0[i] : 0.0);
  }
  s = block_sum(s);
  finish(s, partials, ticket, nrm, 1);
}

// dst = w - alpha*p1 - beta*p0 (w FP32: the split-precision matvec's result) and ||dst||
// in the same pass; dst is the next (unnormalised) Krylov slot
__global__ void __launch_bounds__(RT) k_lanczos_update_to(const float *__restrict__ w, const double *__restrict__ p1,
                                                         const double *__restrict__ p0, double *__restrict__ dst,
                                                         int64_t n, const double *alpha, const double *beta,
                                                         double *partials, unsigned *ticket, double *nrm) {
  const double a = *alpha;
  const double b = p0 ? *beta : 0.0;
  double s = 0.0;
  const int64_t tid = (int64_t)blockIdx.x * RT + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * RT;
  auto one = [&](double wv, double pv1, double pv0) -> double {
    double v = wv - a * pv1;
    if (p0) v -= b * pv0;
    s = fma(v, v, s);
    return v;
  };
  const bool vec = ((reinterpret_cast<uintptr_t>(w) | reinterpret_cast<uintptr_t>(p1) |
                     reinterpret_cast<uintptr_t>(p0) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0;
  if (vec) {
    const int64_t n2 = n / 2;
    double2 *d2 = reinterpret_cast<double2 *>(dst);
    const double2 *a2 = reinterpret_cast<const double2 *>(p1), *b2 = reinterpret_cast<const double2 *>(p0);
    const double2 z = make_double2(0.0, 0.0);
    for (int64_t i = tid; i < n2; i += step) {
      const double2 x = ld_pair(w, i), y = a2[i], q = p0 ? b2[i] : z;
      d2[i] = make_double2(one(x.x, y.x, q.x), one(x.y, y.y, q.y));
    }
    if (tid == 0 && (n & 1)) dst[n - 1] = one((double)w[n - 1], p1[n - 1], p0 ? p0[n - 1] : 0.0);
  } else {
    for (int64_t i = tid; i < n; i += step) dst[i] = one((double)w[i], p1[i], p0 ? p0[i] : 0.0);
  }
  s = block_sum(s);
  finish(s, partials, ticket, nrm, 1);
}

// y = x / *a (y = 0 when *a is zero: a Lanczos breakdown leaves the next vector empty)
// (x == y allowed: each element is read, then written, by the same thread)
__global__ void __launch_bounds__(RT) k_div_copy(const double *x, double *y, int64_t n, const double *a) {
  const double al = *a;
  const bool zero = al == 0.0;
  const int64_t tid = (int64_t)blockIdx.x * RT + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * RT;
  if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0) {
    const int64_t n2 = n / 2;
    const double2 *x2 = reinterpret_cast<const double2 *>(x);
    double2 *y2 = reinterpret_cast<double2 *>(y);
    for (int64_t i = tid; i < n2; i += step) {
      const double2 v = x2[i];
      y2[i] = zero ? make_double2(0.0, 0.0) : make_double2(v.x / al, v.y / al);
    }
    if (tid == 0 && (n & 1)) y[n - 1] = zero ? 0.0 : x[n - 1] / al;
  } else {
    for (int64_t i = tid; i < n; i += step) y[i] = zero ? 0.0 : x[i] / al;
  }
}

// ---- Krylov steps on unnormalised storage.  The restarted Lanczos keeps u_j = s_j q_j
// (s_j = |u_j|, a device scalar) instead of normalising every new vector in a separate
// pass: the matvec is linear, so w = H u_j serves for H q_j = w / s_j, and the scale
// goes into the coefficients.  Both kernels read 16-byte vectors, two per array per
// thread and iteration, when every pointer is 16-byte aligned.

__device__ __forceinline__ double safe_inv(double s) { return s != 0.0 ? 1.0 / s : 0.0; }


// <w, a> / s^2 and <w, b> / s in one pass (s = *s_ptr, 1 when s_ptr is null; a zero s
// gives zeros: the vector behind it is empty after a breakdown)
template <bool VEC, typename WT>
__global__ void __launch_bounds__(RT) k_dot2s(const WT *__restrict__ w, const double *__restrict__ a,
                                             const double *__restrict__ b, int64_t n, const double *s_ptr,
                                             double *partials, unsigned *ticket, double *out_a, double *out_b) {
  double sa = 0.0, sb = 0.0;
  const int64_t tid = (int64_t)blockIdx.x * RT + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * RT;
  if (VEC) {
    const int64_t n2 = n / 2;
    const double2 *a2 = reinterpret_cast<const double2 *>(a), *b2 = reinterpret_cast<const double2 *>(b);
    for (int64_t i = tid; i < n2; i += 2 * step) {
      const bool two = i + step < n2;
      const double2 x0 = ld_pair(w, i), y0 = a2[i], z0 = b2[i];
      double2 x1 = make_double2(0.0, 0.0), y1 = x1, z1 = x1;
      if (two) {
        x1 = ld_pair(w, i + step);
        y1 = a2[i + step];
        z1 = b2[i + step];
      }
      sa = fma(x0.x, y0.x, sa);
      sa = fma(x0.y, y0.y, sa);
      sb = fma(x0.x, z0.x, sb);
      sb = fma(x0.y, z0.y, sb);
      sa = fma(x1.x, y1.x, sa);
      sa = fma(x1.y, y1.y, sa);
      sb = fma(x1.x, z1.x, sb);
      sb = fma(x1.y, z1.y, sb);
    }
    if (tid == 0 && (n & 1)) {
      sa = fma((double)w[n - 1], a[n - 1], sa);
      sb = fma((double)w[n - 1], b[n - 1], sb);
    }
  } else {
    for (int64_t i = tid; i < n; i += step) {
      const double x = (double)w[i];
      sa = fma(x, a[i], sa);
      sb = fma(x, b[i], sb);
    }
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
    const double inv = s_ptr ? safe_inv(*s_ptr) : 1.0;
    *out_a = va * inv * inv;
    *out_b = vb * inv;
    *ticket = 0u;
  }
}

// dst = (w - alpha u) / s - (s / sp) up - gamma q,  ||dst|| -> *nrm.  alpha and gamma are
// the coefficients of q_j = u / s (from k_dot2s with the same s); up = u_{j-1} with its
// own scale sp, so (s / sp) up = beta_{j-1} q_{j-1}.  up and q may be null.
template <bool VEC, typename WT>
__global__ void __launch_bounds__(RT) k_lanczos_step(const WT *__restrict__ w, const double *__restrict__ u,
                                                    const double *__restrict__ up, const double *__restrict__ q,
                                                    double *__restrict__ dst, int64_t n, const double *alpha,
                                                    const double *gamma, const double *s_ptr, const double *sp_ptr,
                                                    double *partials, unsigned *ticket, double *nrm) {
  const double s = *s_ptr;
  const double inv = safe_inv(s);
  const double ca = *alpha * inv;
  const double cp = up ? s * safe_inv(*sp_ptr) : 0.0;
  const double cg = q ? *gamma : 0.0;
  double acc = 0.0;
  const int64_t tid = (int64_t)blockIdx.x * RT + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * RT;
  auto one = [&](double wv, double uv, double pv, double qv) -> double {
    double v = fma(-ca, uv, wv * inv);
    v = fma(-cp, pv, v);
    v = fma(-cg, qv, v);
    acc = fma(v, v, acc);
    return v;
  };
  if (VEC) {
    const int64_t n2 = n / 2;
    const double2 *u2 = reinterpret_cast<const double2 *>(u), *p2 = reinterpret_cast<const double2 *>(up),
                  *q2 = reinterpret_cast<const double2 *>(q);
    double2 *d2 = reinterpret_cast<double2 *>(dst);
    const double2 z = make_double2(0.0, 0.0);
    for (int64_t i = tid; i < n2; i += 2 * step) {
      const bool two = i + step < n2;
      const double2 w0 = ld_pair(w, i), u0 = u2[i], p0 = up ? p2[i] : z, q0 = q ? q2[i] : z;
      double2 w1 = z, u1 = z, p1 = z, q1 = z;
      if (two) {
        w1 = ld_pair(w, i + step);
        u1 = u2[i + step];
        if (up) p1 = p2[i + step];
        if (q) q1 = q2[i + step];
      }
      d2[i] = make_double2(one(w0.x, u0.x, p0.x, q0.x), one(w0.y, u0.y, p0.y, q0.y));
      if (two) d2[i + step] = make_double2(one(w1.x, u1.x, p1.x, q1.x), one(w1.y, u1.y, p1.y, q1.y));
    }
    if (tid == 0 && (n & 1)) {
      const int64_t k = n - 1;
      dst[k] = one((double)w[k], u[k], up ? up[k] : 0.0, q ? q[k] : 0.0);
    }
  } else {
    for (int64_t i = tid; i < n; i += step) dst[i] = one((double)w[i], u[i], up ? up[i] : 0.0, q ? q[i] : 0.0);
  }
  acc = block_sum(acc);
  finish(acc, partials, ticket, nrm, 1);
}

// The two kernels above in one cooperative launch: pass 1 (alpha and gamma as in k_dot2s,
// the partials summed by every CTA in the order k_dot2s's last CTA uses), a grid-wide barrier, pass 2 (the update and the norm as in k_lanczos_step)
// over the same elements, whose w, u and q are then read again from L2.  One launch and one
// ramp instead of two.  The barrier is a counter and a generation word in the two-sum
// workspace; every wait on it is bounded (about a second), after which the CTA raises *err,
// writes NaN to alpha and leaves.  A cooperative launch makes all CTAs resident at once, so
// the barrier completes unless the launch itself went wrong.
constexpr long long BARRIER_SPINS = 1ll << 24;  // x ~64 ns of sleep: about a second

// `extra` > 0 (the self-test only) waits for arrivals that never come
__device__ __forceinline__ bool grid_barrier(unsigned *count, unsigned *gen, unsigned extra, long long spins) {
  __shared__ int passed;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g0 = *(volatile unsigned *)gen;
    __threadfence();
    const unsigned a = atomicAdd(count, 1u);
    if (a == gridDim.x - 1 + extra) {
      *(volatile unsigned *)count = 0u;  // re-arm for the next launch
      __threadfence();
      atomicAdd(gen, 1u);
      passed = 1;
    } else {
      passed = 0;
      for (long long it = 0; it < spins; ++it) {
        if (*(volatile unsigned *)gen != g0) {
          passed = 1;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return passed != 0;
}

template <bool VEC, typename WT>
__global__ void __launch_bounds__(RT, 4) k_krylov_step(const WT *__restrict__ w, const double *__restrict__ u,
                                                   const double *__restrict__ up, const double *__restrict__ q,
                                                   double *__restrict__ dst, int64_t n, const double *s_ptr,
                                                   const double *sp_ptr, double *out_alpha, double *out_gamma,
                                                   double *nrm, double *ws, double *ws2, unsigned *err,
                                                   unsigned extra, long long spins) {
  const int64_t tid = (int64_t)blockIdx.x * RT + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * RT;
  // ---- pass 1: <w, u> and <w, q>
  double sa = 0.0, sb = 0.0;
  if (VEC) {
    const int64_t n2 = n / 2;
    const double2 *a2 = reinterpret_cast<const double2 *>(u), *b2 = reinterpret_cast<const double2 *>(q);
    for (int64_t i = tid; i < n2; i += 2 * step) {
      const bool two = i + step < n2;
      const double2 x0 = ld_pair(w, i), y0 = a2[i], z0 = b2[i];
      double2 x1 = make_double2(0.0, 0.0), y1 = x1, z1 = x1;
      if (two) {
        x1 = ld_pair(w, i + step);
        y1 = a2[i + step];
        z1 = b2[i + step];
      }
      sa = fma(x0.x, y0.x, sa);
      sa = fma(x0.y, y0.y, sa);
      sb = fma(x0.x, z0.x, sb);
      sb = fma(x0.y, z0.y, sb);
      sa = fma(x1.x, y1.x, sa);
      sa = fma(x1.y, y1.y, sa);
      sb = fma(x1.x, z1.x, sb);
      sb = fma(x1.y, z1.y, sb);
    }
    if (tid == 0 && (n & 1)) {
      sa = fma((double)w[n - 1], u[n - 1], sa);
      sb = fma((double)w[n - 1], q[n - 1], sb);
    }
  } else {
    for (int64_t i = tid; i < n; i += step) {
      const double x = (double)w[i];
      sa = fma(x, u[i], sa);
      sb = fma(x, q[i], sb);
    }
  }
  sa = block_sum(sa);
  sb = block_sum(sb);
  if (threadIdx.x == 0) {
    ws2[2 * blockIdx.x] = sa;
    ws2[2 * blockIdx.x + 1] = sb;
  }
  unsigned *bar = reinterpret_cast<unsigned *>(ws2 + 2 * MAXCTA + 2);  // [count, generation]
  if (!grid_barrier(bar, bar + 1, extra, spins)) {
    if (threadIdx.x == 0) {
      atomicExch(err, 1u);
      *out_alpha = __longlong_as_double(0x7ff8000000000000ll);
    }
    return;
  }
  // ---- every CTA: alpha, gamma from all partials (k_dot2s's order)
  double va = 0.0, vb = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += RT) {
    va += ((volatile double *)ws2)[2 * i];
    vb += ((volatile double *)ws2)[2 * i + 1];
  }
  va = block_sum(va);
  vb = block_sum(vb);
  __shared__ double coef[2];
  const double s = *s_ptr;
  const double inv = safe_inv(s);
  if (threadIdx.x == 0) {
    coef[0] = va * inv * inv;  // alpha
    coef[1] = vb * inv;        // gamma
    if (blockIdx.x == 0) {
      *out_alpha = coef[0];
      *out_gamma = coef[1];
    }
  }
  __syncthreads();
  // ---- pass 2: the update of k_lanczos_step
  const double ca = coef[0] * inv;
  const double cp = up ? s * safe_inv(*sp_ptr) : 0.0;
  const double cg = coef[1];
  double acc = 0.0;
  auto one = [&](double wv, double uv, double pv, double qv) -> double {
    double v = fma(-ca, uv, wv * inv);
    v = fma(-cp, pv, v);
    v = fma(-cg, qv, v);
    acc = fma(v, v, acc);
    return v;
  };
  if (VEC) {
    const int64_t n2 = n / 2;
    const double2 *u2 = reinterpret_cast<const double2 *>(u), *p2 = reinterpret_cast<const double2 *>(up),
                  *q2 = reinterpret_cast<const double2 *>(q);
    double2 *d2 = reinterpret_cast<double2 *>(dst);
    const double2 z = make_double2(0.0, 0.0);
    for (int64_t i = tid; i < n2; i += 2 * step) {
      const bool two = i + step < n2;
      const double2 w0 = ld_pair(w, i), u0 = u2[i], p0 = up ? p2[i] : z, q0 = q2[i];
      double2 w1 = z, u1 = z, p1 = z, q1 = z;
      if (two) {
        w1 = ld_pair(w, i + step);
        u1 = u2[i + step];
        if (up) p1 = p2[i + step];
        q1 = q2[i + step];
      }
      d2[i] = make_double2(one(w0.x, u0.x, p0.x, q0.x), one(w0.y, u0.y, p0.y, q0.y));
      if (two) d2[i + step] = make_double2(one(w1.x, u1.x, p1.x, q1.x), one(w1.y, u1.y, p1.y, q1.y));
    }
    if (tid == 0 && (n & 1)) {
      const int64_t k = n - 1;
      dst[k] = one((double)w[k], u[k], up ? up[k] : 0.0, q[k]);
    }
  } else {
    for (int64_t i = tid; i < n; i += step) dst[i] = one((double)w[i], u[i], up ? up[i] : 0.0, q[i]);
  }
  acc = block_sum(acc);
  finish(acc, ws, reinterpret_cast<unsigned *>(ws + MAXCTA), nrm, 1);
}

// out = sum_j c[j] * K[j]  (Krylov combination), c on device
// (16-byte loads of four Krylov vectors at a time when every row is 16-byte aligned)
template <bool VEC>
__global__ void __launch_bounds__(RT) k_combine(const double *__restrict__ K, int64_t n, int m,
                                               const double *__restrict__ c, double *__restrict__ out) {
  const int64_t tid = (int64_t)blockIdx.x * RT + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * RT;
  if (VEC) {
    const int64_t n2 = n / 2;
    const double2 *K2 = reinterpret_cast<const double2 *>(K);
    double2 *o2 = reinterpret_cast<double2 *>(out);
    for (int64_t i = tid; i < n2; i += step) {
      double sx = 0.0, sy = 0.0;
      int j = 0;
      for (; j + 4 <= m; j += 4) {
        const double2 a0 = K2[(int64_t)j * n2 + i], a1 = K2[(int64_t)(j + 1) * n2 + i];
        const double2 a2 = K2[(int64_t)(j + 2) * n2 + i], a3 = K2[(int64_t)(j + 3) * n2 + i];
        sx = fma(c[j], a0.x, sx);
        sy = fma(c[j], a0.y, sy);
        sx = fma(c[j + 1], a1.x, sx);
        sy = fma(c[j + 1], a1.y, sy);
        sx = fma(c[j + 2], a2.x, sx);
        sy = fma(c[j + 2], a2.y, sy);
        sx = fma(c[j + 3], a3.x, sx);
        sy = fma(c[j + 3], a3.y, sy);
      }
      for (; j < m; ++j) {
        const double2 a = K2[(int64_t)j * n2 + i];
        sx = fma(c[j], a.x, sx);
        sy = fma(c[j], a.y, sy);
      }
      o2[i] = make_double2(sx, sy);
    }
  } else {
    for (int64_t i = tid; i < n; i += step) {
      double s = 0.0;
      for (int j = 0; j < m; ++j) s = fma(c[j], K[(int64_t)j * n + i], s);
      out[i] = s;
    }
  }
}

// ---- block Krylov kernels for the thick-restart Lanczos (k extreme eigenpairs).
// The basis V holds m vectors of n doubles back to back (V[j] = V + j * n).

// h[j] = <V[j], w> for j < m (accumulate: h[j] += ...).  Each CTA reduces its slice of
// every dot and writes m partials; the last CTA sums them in a fixed order.
__global__ void __launch_bounds__(RT) k_multidot(const double *__restrict__ V, const double *__restrict__ w,
                                                int64_t n, int m, double *partials, unsigned *ticket, double *h,
                                                int accumulate) {
  const int64_t step = (int64_t)gridDim.x * RT;
  for (int j = 0; j < m; ++j) {
    const double *v = V + (int64_t)j * n;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * RT + threadIdx.x; i < n; i += step) s = fma(v[i], w[i], s);
    s = block_sum(s);
    if (threadIdx.x == 0) partials[(int64_t)blockIdx.x * m + j] = s;
  }
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  for (int j = threadIdx.x; j < m; j += RT) {
    double v = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) v += ((volatile double *)partials)[(int64_t)b * m + j];
    h[j] = accumulate ? h[j] + v : v;
  }
  __syncthreads();
  if (threadIdx.x == 0) *ticket = 0u;
}

// w -= sum_j V[j] h[j]  (j < m)
__global__ void __launch_bounds__(RT) k_multiaxpy(const double *__restrict__ V, const double *__restrict__ h,
                                                 int64_t n, int m, double *__restrict__ w) {
  const int64_t step = (int64_t)gridDim.x * RT;
  for (int64_t i = (int64_t)blockIdx.x * RT + threadIdx.x; i < n; i += step) {
    double s = w[i];
    for (int j = 0; j < m; ++j) s = fma(-h[j], V[(int64_t)j * n + i], s);
    w[i] = s;
  }
}

// out[c] = sum_j V[j] Y[j * ldy + c]  (c < nc, j < m): Ritz vectors from the basis
__global__ void __launch_bounds__(RT) k_basis_combine(const double *__restrict__ V, int64_t n, int m,
                                                     const double *__restrict__ Y, int ldy, int nc,
                                                     double *__restrict__ out) {
  const int64_t step = (int64_t)gridDim.x * RT;
  for (int64_t i = (int64_t)blockIdx.x * RT + threadIdx.x; i < n; i += step) {
    for (int c = 0; c < nc; ++c) {
      double s = 0.0;
      for (int j = 0; j < m; ++j) s = fma(Y[j * ldy + c], V[(int64_t)j * n + i], s);
      out[(int64_t)c * n + i] = s;
    }
  }
}

// streaming kernels of the refined Lanczos step: up to MAXCTA CTAs (about seven per SM) for
// more loads in flight
int grid_stream(int64_t n) {
  const int64_t g = (n + RT * 4 - 1) / (RT * 4);
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, MAXCTA));
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

// ws2 layout (dot2s_f64, krylov_step_f64): [2 * MAXCTA partials][ticket][spare][barrier count][barrier generation]
// ws layout: [partials MAXCTA doubles][ticket (8 bytes)]
ctn_status dot_f64(const float *x, const double *y, int64_t n, double *out, double *ws, cudaStream_t st) {
  int g = grid_for(n);
  k_dot<float><<<g, RT, 0, st>>>(x, y, n, ws, reinterpret_cast<unsigned *>(ws + MAXCTA), out, 0);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status lanczos_update_to_f64(const float *w, const double *p1, const double *p0, double *dst, int64_t n,
                                 const double *alpha, const double *beta, double *nrm, double *ws, cudaStream_t st) {
  int g = grid_for(n);
  k_lanczos_update_to<<<g, RT, 0, st>>>(w, p1, p0, dst, n, alpha, beta, ws, reinterpret_cast<unsigned *>(ws + MAXCTA),
                                        nrm);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status dot_f64(const double *x, const double *y, int64_t n, double *out, double *ws, cudaStream_t st) {
  int g = grid_for(n);
  k_dot<double><<<g, RT, 0, st>>>(x, y, n, ws, reinterpret_cast<unsigned *>(ws + MAXCTA), out, 0);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status nrm2_f64(const double *x, int64_t n, double *out, double *ws, cudaStream_t st) {
  int g = grid_for(n);
  k_dot<double><<<g, RT, 0, st>>>(x, x, n, ws, reinterpret_cast<unsigned *>(ws + MAXCTA), out, 1);
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
static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <typename WT>
static ctn_status dot2s_any(const WT *w, const double *a, const double *b, int64_t n, const double *s, double *out_a,
                            double *out_b, double *ws2, cudaStream_t st) {
  const int g = grid_stream(n);
  unsigned *ticket = reinterpret_cast<unsigned *>(ws2 + 2 * MAXCTA);
  if (aligned16(w) && aligned16(a) && aligned16(b))
    k_dot2s<true, WT><<<g, RT, 0, st>>>(w, a, b, n, s, ws2, ticket, out_a, out_b);
  else
    k_dot2s<false, WT><<<g, RT, 0, st>>>(w, a, b, n, s, ws2, ticket, out_a, out_b);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status dot2s_f64(const double *w, const double *a, const double *b, int64_t n, const double *s, double *out_a,
                     double *out_b, double *ws2, cudaStream_t st) {
  return dot2s_any(w, a, b, n, s, out_a, out_b, ws2, st);
}
ctn_status dot2s_f64(const float *w, const double *a, const double *b, int64_t n, const double *s, double *out_a,
                     double *out_b, double *ws2, cudaStream_t st) {
  return dot2s_any(w, a, b, n, s, out_a, out_b, ws2, st);
}

template <typename WT>
static ctn_status lanczos_step_any(const WT *w, const double *u, const double *up, const double *q, double *dst,
                                   int64_t n, const double *alpha, const double *gamma, const double *s,
                                   const double *sp, double *nrm, double *ws, cudaStream_t st) {
  const int g = grid_stream(n);
  unsigned *ticket = reinterpret_cast<unsigned *>(ws + MAXCTA);
  const bool vec = aligned16(w) && aligned16(u) && aligned16(dst) && (!up || aligned16(up)) && (!q || aligned16(q));
  if (vec)
    k_lanczos_step<true, WT><<<g, RT, 0, st>>>(w, u, up, q, dst, n, alpha, gamma, s, sp, ws, ticket, nrm);
  else
    k_lanczos_step<false, WT><<<g, RT, 0, st>>>(w, u, up, q, dst, n, alpha, gamma, s, sp, ws, ticket, nrm);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status lanczos_step_f64(const double *w, const double *u, const double *up, const double *q, double *dst,
                            int64_t n, const double *alpha, const double *gamma, const double *s, const double *sp,
                            double *nrm, double *ws, cudaStream_t st) {
  return lanczos_step_any(w, u, up, q, dst, n, alpha, gamma, s, sp, nrm, ws, st);
}
ctn_status lanczos_step_f64(const float *w, const double *u, const double *up, const double *q, double *dst,
                            int64_t n, const double *alpha, const double *gamma, const double *s, const double *sp,
                            double *nrm, double *ws, cudaStream_t st) {
  return lanczos_step_any(w, u, up, q, dst, n, alpha, gamma, s, sp, nrm, ws, st);
}

// the fused step: one cooperative launch of k_krylov_step with k_dot2s's grid (capped at the
// CTAs that fit on the device at once); CTN_ERR_UNSUPPORTED when the device has no
// cooperative launch (the caller then runs the two kernels)
template <typename WT>
static ctn_status krylov_step_any(const WT *w, const double *u, const double *up, const double *q, double *dst,
                                  int64_t n, const double *s, const double *sp, double *out_alpha,
                                  double *out_gamma, double *nrm, double *ws, double *ws2, unsigned *err,
                                  cudaStream_t st, unsigned extra = 0, long long spins = BARRIER_SPINS) {
  const bool vec = aligned16(w) && aligned16(u) && aligned16(dst) && (!up || aligned16(up)) && aligned16(q);
  void (*kern)(const WT *, const double *, const double *, const double *, double *, int64_t, const double *,
               const double *, double *, double *, double *, double *, double *, unsigned *, unsigned, long long) =
      vec ? k_krylov_step<true, WT> : k_krylov_step<false, WT>;
  // resident CTAs of this kernel on the device (queried once per device: the step runs hundreds
  // of times per solve); 0 = the device has no cooperative launch
  static int resident[64][2];
  static bool known[64][2];
  int dev = 0;
  CTN_CUDA(cudaGetDevice(&dev));
  const int di = dev & 63;
  if (!known[di][vec]) {
    int coop = 0, nsm = 0, occ = 0;
    CTN_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    CTN_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CTN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, RT, 0));
    resident[di][vec] = coop ? std::max(1, nsm * occ) : 0;
    known[di][vec] = true;
  }
  if (resident[di][vec] == 0) return CTN_ERR_UNSUPPORTED;
  const int g = std::min(grid_stream(n), resident[di][vec]);
  void *args[] = {(void *)&w,   (void *)&u,         (void *)&up,        (void *)&q,   (void *)&dst,
                  (void *)&n,   (void *)&s,         (void *)&sp,        (void *)&out_alpha,
                  (void *)&out_gamma, (void *)&nrm, (void *)&ws,        (void *)&ws2, (void *)&err,
                  (void *)&extra, (void *)&spins};
  CTN_CUDA(cudaLaunchCooperativeKernel((const void *)kern, dim3(g), dim3(RT), args, 0, st));
  return CTN_OK;
}
ctn_status krylov_step_f64(const double *w, const double *u, const double *up, const double *q, double *dst,
                           int64_t n, const double *s, const double *sp, double *out_alpha, double *out_gamma,
                           double *nrm, double *ws, double *ws2, unsigned *err, cudaStream_t st) {
  return krylov_step_any(w, u, up, q, dst, n, s, sp, out_alpha, out_gamma, nrm, ws, ws2, err, st);
}
ctn_status krylov_step_f64(const float *w, const double *u, const double *up, const double *q, double *dst,
                           int64_t n, const double *s, const double *sp, double *out_alpha, double *out_gamma,
                           double *nrm, double *ws, double *ws2, unsigned *err, cudaStream_t st) {
  return krylov_step_any(w, u, up, q, dst, n, s, sp, out_alpha, out_gamma, nrm, ws, ws2, err, st);
}

ctn_status div_copy_f64(const double *x, double *y, int64_t n, const double *a, cudaStream_t st) {
  k_div_copy<<<grid_for(n), RT, 0, st>>>(x, y, n, a);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status combine_f64(const double *K, int64_t n, int m, const double *c, double *out, cudaStream_t st) {
  if ((n & 1) == 0 && aligned16(K) && aligned16(out))
    k_combine<true><<<grid_stream(n), RT, 0, st>>>(K, n, m, c, out);
  else
    k_combine<false><<<grid_for(n), RT, 0, st>>>(K, n, m, c, out);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}

// ws layout: [ticket (8 bytes, fixed place for every m)][grid * m partials]; ws must hold
// multidot_ws_doubles(m_max) doubles
size_t multidot_ws_doubles(int m) { return (size_t)MAXCTA * (size_t)m + 8; }
ctn_status multidot_f64(const double *V, const double *w, int64_t n, int m, double *h, int accumulate, double *ws,
                        cudaStream_t st) {
  const int g = grid_for(n);
  k_multidot<<<g, RT, 0, st>>>(V, w, n, m, ws + 8, reinterpret_cast<unsigned *>(ws), h, accumulate);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status multiaxpy_f64(const double *V, const double *h, int64_t n, int m, double *w, cudaStream_t st) {
  k_multiaxpy<<<grid_for(n), RT, 0, st>>>(V, h, n, m, w);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}
ctn_status basis_combine_f64(const double *V, int64_t n, int m, const double *Y, int ldy, int nc, double *out,
                             cudaStream_t st) {
  k_basis_combine<<<grid_for(n), RT, 0, st>>>(V, n, m, Y, ldy, nc, out);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}

}  // namespace ctn

// Self-test of the fused Krylov step's bounded grid barrier: one launch on a small vector whose
// barrier waits for one arrival more than the grid has, so every CTA's wait runs out after
// `spin_limit` probes, raises the error word and leaves.
namespace ctn {
ctn_status selftest_barrier_timeout(long long spin_limit, cudaStream_t st) {
  const int64_t n = 1 << 14;
  const size_t wsb = reduce_ws_bytes(), ws2b = reduce2_ws_bytes();
  const size_t bytes = 4 * n * sizeof(double) + wsb + ws2b + 8 * sizeof(double);
  double *buf = nullptr;
  CTN_CUDA(cudaMalloc(&buf, bytes));
  ctn_status rc = cudaMemsetAsync(buf, 0, bytes, st) == cudaSuccess ? CTN_OK : CTN_ERR_CUDA;
  double *w = buf, *u = buf + n, *q = buf + 2 * n, *dst = buf + 3 * n;
  double *ws = buf + 4 * n, *ws2 = ws + wsb / sizeof(double), *scal = ws2 + ws2b / sizeof(double);
  unsigned *err = reinterpret_cast<unsigned *>(scal + 7);
  const double one = 1.0;
  if (rc == CTN_OK && cudaMemcpyAsync(scal, &one, sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
    rc = CTN_ERR_CUDA;
  if (rc == CTN_OK)
    rc = krylov_step_any<double>(w, u, nullptr, q, dst, n, scal, nullptr, scal + 1, scal + 2, scal + 3, ws, ws2, err,
                                 st, 1u, spin_limit);
  unsigned herr = 0;
  if (rc == CTN_OK && (cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                       cudaStreamSynchronize(st) != cudaSuccess))
    rc = CTN_ERR_CUDA;
  cudaFree(buf);
  if (rc != CTN_OK) return rc;
  if (herr) {
    set_error("fused Krylov step: the grid barrier's bounded wait expired");
    return CTN_ERR_TIMEOUT;
  }
  set_error("ctn_selftest_barrier_timeout: the kernel passed its barrier");
  return CTN_ERR_INVALID;
}
}  // namespace ctn

extern "C" ctn_status ctn_selftest_barrier_timeout(long long spin_limit, void *stream) {
  CTN_REQUIRE(spin_limit > 0, "ctn_selftest_barrier_timeout: spin_limit must be positive");
  return ctn::selftest_barrier_timeout(spin_limit, ctn::as_stream(stream));
}
