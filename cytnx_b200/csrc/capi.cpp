// C ABI plumbing: error text, dtype table, BLAS-1 entry points, the symmetric
// tridiagonal eigensolver and the Lanczos ground-state driver.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <numeric>
#include <vector>

#include "blas1.cuh"
#include "ctn_common.h"

namespace ctn {
static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

// one zeroed reduction workspace per device for the stand-alone BLAS-1 entry points
static std::mutex g_ws_mu;
static double *g_ws[64] = {nullptr};
static ctn_status device_ws(double **ws) {
  int dev = 0;
  CTN_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_ws_mu);
  if (!g_ws[dev]) {
    CTN_CUDA(cudaMalloc(&g_ws[dev], reduce_ws_bytes()));
    CTN_CUDA(cudaMemset(g_ws[dev], 0, reduce_ws_bytes()));
  }
  *ws = g_ws[dev];
  return CTN_OK;
}

// Symmetric tridiagonal eigenproblem by the implicit symmetric QR algorithm with
// Wilkinson shifts (Golub & Van Loan, Matrix Computations, 4th ed., Algorithms 8.3.2
// "implicit symmetric QR step" and 8.3.3 "symmetric QR"): the trailing unreduced window
// [lo, hi] of T is swept by Givens rotations that chase the shift's bulge down the band,
// and off-diagonals below eps * (|d_i| + |d_i+1|) split the problem.  d: diagonal (n),
// e: off-diagonal (n-1).  Eigenvalues ascending; z (n x n, row-major) receives the
// eigenvectors as ROWS, the is_row=true layout linalg::Tridiag returns
// (src/linalg/Tridiag.cpp:83-95).  With zrows == nullptr no rotation is accumulated
// (O(n^2) instead of O(n^3)); the eigenvalues do not depend on it and are bit-identical.
// The sweeps run on the reversed matrix J T J (J the exchange matrix), i.e. the bulge moves
// from the last row towards the first and rows deflate from the top: on Lanczos
// tridiagonals this keeps the leading eigenvector components, which the Lanczos drivers
// combine (exp(tau T) e_1, the Ritz vectors), accurate to rounding; the top-down order
// lost up to two digits there (the stopping value |exp(tau T)[i][0]| of Lanczos_Exp then
// stalled above 1e-14).
static ctn_status tql(int n, const double *din, const double *ein, double *w, double *zrows) {
  std::vector<double> d(n), e(n > 1 ? n - 1 : 1, 0.0);
  for (int i = 0; i < n; ++i) d[i] = din[n - 1 - i];
  for (int i = 0; i + 1 < n; ++i) e[i] = ein[n - 2 - i];
  // vec[j * n + k]: component k of the j-th column of the accumulated rotation product V
  // (T_input = V T_current V^T), so the two columns a rotation touches are contiguous
  std::vector<double> vec(zrows ? (size_t)n * n : 0, 0.0);
  if (zrows)
    for (int j = 0; j < n; ++j) vec[(size_t)j * n + j] = 1.0;
  const double eps = std::numeric_limits<double>::epsilon();
  auto negligible = [&](int i) {
    return std::fabs(e[i]) <= eps * (std::fabs(d[i]) + std::fabs(d[i + 1])) || std::fabs(e[i]) < 1e-300;
  };
  // rotation R = [[c, s], [-s, c]] on coordinates (k, k+1): T <- R T R^T, V <- V R^T
  auto rotate_vectors = [&](int k, double c, double s) {
    if (!zrows) return;
    double *u = &vec[(size_t)k * n], *v = &vec[(size_t)(k + 1) * n];
    for (int i = 0; i < n; ++i) {
      const double a = u[i], b = v[i];
      u[i] = c * a + s * b;
      v[i] = c * b - s * a;
    }
  };
  long long budget = 60ll * std::max(n, 1);
  int hi = n - 1;
  while (hi > 0) {
    if (negligible(hi - 1)) {
      e[hi - 1] = 0.0;
      --hi;
      continue;
    }
    int lo = hi - 1;
    while (lo > 0 && !negligible(lo - 1)) --lo;
    if (--budget < 0) {
      set_error("ctn_tridiag_eigh: QR iteration did not converge");
      return CTN_ERR_NUMERIC;
    }
    // Wilkinson shift: the eigenvalue of the trailing 2 x 2 block closer to d[hi]
    const double half = 0.5 * (d[hi - 1] - d[hi]);
    const double off = e[hi - 1];
    const double den = half + (half >= 0.0 ? 1.0 : -1.0) * std::hypot(half, off);
    const double mu = d[hi] - (den != 0.0 ? off * off / den : 0.0);
    // implicit QR step: the first rotation comes from the shifted first column, each
    // later one removes the bulge the previous one created below the band
    double x = d[lo] - mu, z = e[lo];
    for (int k = lo; k < hi; ++k) {
      const double r = std::hypot(x, z);
      const double c = r != 0.0 ? x / r : 1.0, s = r != 0.0 ? z / r : 0.0;
      if (k > lo) e[k - 1] = r;
      const double p = d[k], q = e[k], t = d[k + 1];
      const double cc = c * c, ss = s * s, cs = c * s;
      d[k] = cc * p + 2.0 * cs * q + ss * t;
      d[k + 1] = ss * p - 2.0 * cs * q + cc * t;
      e[k] = cs * (t - p) + (cc - ss) * q;
      rotate_vectors(k, c, s);
      if (k + 1 < hi) {
        z = s * e[k + 1];  // the new bulge at (k + 2, k)
        e[k + 1] *= c;
        x = e[k];
      }
    }
  }
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return d[a] < d[b]; });
  for (int j = 0; j < n; ++j) {
    w[j] = d[idx[j]];
    if (zrows) {
      const double *src = &vec[(size_t)idx[j] * n];
      for (int k = 0; k < n; ++k) zrows[(size_t)j * n + k] = src[n - 1 - k];  // undo the reversal
    }
  }
  return CTN_OK;
}
}  // namespace ctn

extern "C" const char *ctn_last_error(void) { return ctn::g_err; }
extern "C" int ctn_version(void) { return 100; }
extern "C" size_t ctn_dtype_size(int dtype) {
  switch (dtype) {
    case CTN_COMPLEX128: return 16;
    case CTN_COMPLEX64: return 8;
    case CTN_FLOAT64: return 8;
    case CTN_FLOAT32: return 4;
    case CTN_INT64: return 8;
    case CTN_UINT64: return 8;
    case CTN_INT32: return 4;
    case CTN_UINT32: return 4;
    case CTN_INT16: return 2;
    case CTN_UINT16: return 2;
    case CTN_BOOL: return 1;
  }
  return 0;
}

extern "C" ctn_status ctn_dot_f64(const double *x, const double *y, int64_t n, double *out, void *stream) {
  double *ws;
  CTN_TRY(ctn::device_ws(&ws));
  return ctn::dot_f64(x, y, n, out, ws, ctn::as_stream(stream));
}
extern "C" ctn_status ctn_nrm2_f64(const double *x, int64_t n, double *out, void *stream) {
  double *ws;
  CTN_TRY(ctn::device_ws(&ws));
  return ctn::nrm2_f64(x, n, out, ws, ctn::as_stream(stream));
}
extern "C" ctn_status ctn_axpy_f64(const double *x, double *y, int64_t n, const double *a_dev, double a_scale,
                                   void *stream) {
  return ctn::axpy_f64(x, y, n, a_dev, a_scale, ctn::as_stream(stream));
}
extern "C" ctn_status ctn_scal_f64(double *x, int64_t n, const double *a_dev, int invert, void *stream) {
  return ctn::scal_f64(x, n, a_dev, invert, ctn::as_stream(stream));
}

extern "C" ctn_status ctn_tridiag_eigh(int n, const double *d, const double *e, double *w, double *z) {
  CTN_REQUIRE(n >= 0 && d && w, "ctn_tridiag_eigh: bad argument");
  if (n == 0) return CTN_OK;
  return ctn::tql(n, d, e, w, z);
}

namespace ctn {
// per-thread pinned landing slots for the per-iteration scalars: a device-to-host copy into
// pageable memory returns only when it has completed, which would hold the host at every
// queued read; into pinned memory it is queued like a kernel.  128 bytes per calling thread,
// allocated on first use and left to the process exit (no CUDA call from thread teardown)
static ctn_status pinned_scalars(double **out) {
  static thread_local double *buf = nullptr;
  if (!buf) CTN_CUDA(cudaHostAlloc((void **)&buf, 16 * sizeof(double), cudaHostAllocPortable));
  *out = buf;
  return CTN_OK;
}

// Lanczos_Gnd_Ut (src/linalg/Lanczos_Gnd_Ut.cpp:29-162): 3-term recurrence, Tridiag
// re-solved each iteration, stop on |dE| < cvgcrit or beta == 0; the Ritz vector is
// the combination of the stored Krylov vectors.  The vectors stay on the device; the
// two scalars per iteration come to the host as the reference's .item() calls do.
// speculate: queue iteration i+1 on the device before the host solves iteration i's
// tridiagonal, so the host solve runs under the next matvec; the iteration queued after the
// last one runs and is discarded (one extra matvec, results unchanged).  Only for matvecs
// without side effects.
ctn_status lanczos_gnd(int (*mv)(void *, const double *, double *, void *), void *user, const double *psi0,
                       int64_t n, int maxiter, double cvgcrit, double *krylov, double *work, double *eigvec,
                       double *energy, int *iters, cudaStream_t st, bool speculate, bool w_f32) {
  CTN_REQUIRE(maxiter >= 2, "[Lanczos] Maxiter must >1");
  CTN_REQUIRE(cvgcrit > 0, "[Lanczos] converge criteria must >0");
  CTN_REQUIRE(n > 0, "[Lanczos] empty vector");
  double *w = work;                      // new_psi
  // device scalars: [0] |psi0|, [1] alpha, [2] / [3] the norms of w, alternately written by one
  // update and read as beta (the coefficient of psi_{i-1}) by the next, so no value travels
  // back to the device; one host read of [1..3] per iteration (the reference's .item() calls)
  double *scal = work + n;
  double *ws = work + n + 8;             // reduction workspace (zeroed below)
  double *cdev = ws + reduce_ws_bytes() / sizeof(double);
  double *pin;
  CTN_TRY(pinned_scalars(&pin));
  cudaEvent_t ev[2] = {nullptr, nullptr};
  struct EvGuard {
    cudaEvent_t *e;
    ~EvGuard() {
      for (int k = 0; k < 2; ++k)
        if (e[k]) cudaEventDestroy(e[k]);
    }
  } guard{ev};
  for (int k = 0; k < 2; ++k) CTN_CUDA(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
  CTN_CUDA(cudaMemsetAsync(ws, 0, reduce_ws_bytes(), st));
  // psi_1 = Tin / |Tin|
  CTN_TRY(nrm2_f64(psi0, n, scal + 0, ws, st));
  CTN_CUDA(cudaMemcpyAsync(pin + 8, scal + 0, sizeof(double), cudaMemcpyDeviceToHost, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  CTN_REQUIRE(pin[8] > 0 && std::isfinite(pin[8]), "[Lanczos] initial vector has zero or non-finite norm");
  CTN_TRY(div_copy_f64(psi0, krylov, n, scal + 0, st));
  // iteration i on the device: (i >= 1) psi_i = w / beta_{i-1}; w = H psi_i; alpha_i = <w, psi_i>;
  // w -= alpha_i psi_i + beta_{i-1} psi_{i-1}; beta_i = |w|; alpha_i, beta_i -> pinned slot i & 1
  // w_f32 (split-precision matvecs): mv writes w as n floats, the update writes its FP64 result
  // straight into the next Krylov slot, which the next iteration scales in place
  auto queue = [&](int i) -> ctn_status {
    double *pi = krylov + (int64_t)i * n;
    double *b_new = scal + 2 + (i & 1);
    const double *b_old = i ? scal + 2 + ((i - 1) & 1) : nullptr;
    if (i) CTN_TRY(div_copy_f64(w_f32 ? pi : w, pi, n, b_old, st));
    if (mv(user, pi, w, st) != 0) return CTN_ERR_CUDA;
    if (w_f32) {
      const float *wf = reinterpret_cast<const float *>(w);
      CTN_TRY(dot_f64(wf, pi, n, scal + 1, ws, st));
      CTN_TRY(lanczos_update_to_f64(wf, pi, i ? pi - n : nullptr, pi + n, n, scal + 1, b_old, b_new, ws, st));
    } else {
      CTN_TRY(dot_f64(w, pi, n, scal + 1, ws, st));
      CTN_TRY(lanczos_update_f64(w, pi, i ? pi - n : nullptr, n, scal + 1, b_old, b_new, ws, st));
    }
    CTN_CUDA(cudaMemcpyAsync(pin + 4 * (i & 1), scal + 1, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaEventRecord(ev[i & 1], st));
    return CTN_OK;
  };
  std::vector<double> As, Bs, evals, evecs;
  double E = 0.0;
  int it = 0;
  CTN_TRY(queue(0));
  for (int i = 0; i < maxiter; ++i) {
    it = i + 1;
    CTN_CUDA(cudaEventSynchronize(ev[i & 1]));
    const double alpha = pin[4 * (i & 1)], beta = pin[4 * (i & 1) + 1 + (i & 1)];
    As.push_back(alpha);
    const bool more = beta != 0.0 && i + 1 < maxiter;
    if (speculate && more) CTN_TRY(queue(i + 1));
    const int m = (int)As.size();
    evals.assign(m, 0.0);
    // eigenvalues only inside the loop: the Ritz vector is needed once, after it
    if (m == 1)
      evals[0] = alpha;
    else
      CTN_TRY(tql(m, As.data(), Bs.data(), evals.data(), nullptr));
    Bs.push_back(beta);
    if (beta == 0.0) break;
    if (i >= 1) {
      if (std::fabs(E - evals[0]) < cvgcrit) break;
    }
    E = evals[0];
    if (!speculate && more) CTN_TRY(queue(i + 1));
  }
  // eigenvector = sum_n kry[n] psi_s[n] over the tridiagonal size
  const int m = (int)evals.size();
  evecs.assign((size_t)m * m, 0.0);
  if (m == 1)
    evecs[0] = 1.0;
  else
    CTN_TRY(tql(m, As.data(), Bs.data(), evals.data(), evecs.data()));
  CTN_CUDA(cudaMemcpyAsync(cdev, evecs.data(), sizeof(double) * m, cudaMemcpyHostToDevice, st));
  CTN_TRY(combine_f64(krylov, n, m, cdev, eigvec, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  *energy = evals[0];
  *iters = it;
  return CTN_OK;
}
}  // namespace ctn

namespace ctn {
// Restarted ground-state Lanczos with a low-precision matvec and one FP64 refinement
// matvec per restart.  Each cycle starts from the current unit vector q0 = v:
//   w = H_hi q0 (FP64): theta = <q0, w>, r = w - theta q0, rho = |r|  -- the FP64
//   Rayleigh quotient and eigen-residual of v; stop when rho <= tol * |theta|;
//   q1 = r / rho, then q_{j+1} from w = H_lo q_j with the three-term recurrence and an
//   FP64 re-orthogonalisation of w against q0 at every step;
//   the (krydim x krydim) tridiagonal T is solved in FP64 and v <- normalised sum y_j q_j.
// The low-precision products only ever act on the correction directions q_j (j >= 1),
// whose weight in v shrinks with rho, so the FP64 residual keeps falling below the
// matvec error.  Returned energy and residual are the FP64 Rayleigh quotient and |r| of
// the returned vector (measured by the last FP64 matvec).
ctn_status lanczos_refined(int (*mv_lo)(void *, const double *, double *, void *), void *u_lo,
                           int (*mv_hi)(void *, const double *, double *, void *), void *u_hi, const double *psi0,
                           int64_t n, int krydim, int max_restarts, double tol, double *krylov, double *work,
                           double *eigvec, double *energy, double *residual, int *restarts, int64_t *counts,
                           cudaStream_t st, bool w_f32) {
  CTN_REQUIRE(krydim >= 2 && max_restarts >= 1 && n > 0 && tol >= 0, "[Lanczos refined] bad argument");
  // work: [w n][scalars 8][reduction ws][two-sum ws][Ritz coefficients m][alpha m][beta m]
  double *w = work;
  double *scal = work + n;  // [0] norm [1] theta [3] rho [4] gamma (overlap with q0) [6] error word
  double *ws = work + n + 8;
  double *ws2 = ws + reduce_ws_bytes() / sizeof(double);
  double *cdev = ws2 + reduce2_ws_bytes() / sizeof(double);
  double *alpha = cdev + krydim;
  double *beta = alpha + krydim;
  CTN_CUDA(cudaMemsetAsync(ws, 0, reduce_ws_bytes() + reduce2_ws_bytes(), st));
  unsigned *err = reinterpret_cast<unsigned *>(scal + 6);
  CTN_CUDA(cudaMemsetAsync(err, 0, sizeof(double), st));
  bool fused = true;  // one cooperative launch per Krylov step while the device supports it
  double host = 0.0;
  int64_t n_lo = 0, n_hi = 0;
  CTN_TRY(nrm2_f64(psi0, n, scal + 0, ws, st));
  CTN_CUDA(cudaMemcpyAsync(&host, scal + 0, sizeof(double), cudaMemcpyDeviceToHost, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  CTN_REQUIRE(host > 0 && std::isfinite(host), "[Lanczos refined] initial vector has zero or non-finite norm");
  CTN_TRY(div_copy_f64(psi0, krylov, n, scal + 0, st));
  double theta = 0.0, rho = 0.0;
  int c = 0;
  std::vector<double> As(krydim), Bs(krydim), coef(krydim), evals, evecs;
  // Krylov storage: slot 0 holds the unit vector q0; slot j >= 1 holds u_j = s_j q_j with
  // s_j = beta[j-1] = |u_j| (never normalised in a separate pass: H u_j = s_j H q_j, and
  // the scales enter the recurrence coefficients and the final combination)
  for (c = 0; c < max_restarts; ++c) {
    double *q0 = krylov;
    double *u1 = krylov + n;
    // FP64 refinement: theta = <q0, H q0>, u1 = r = H q0 - theta q0, rho = |r|  (alpha[0], beta[0])
    if (mv_hi(u_hi, q0, u1, st) != 0) return CTN_ERR_CUDA;
    ++n_hi;
    CTN_TRY(dot_f64(u1, q0, n, alpha + 0, ws, st));
    CTN_TRY(lanczos_update_f64(u1, q0, nullptr, n, alpha + 0, nullptr, beta + 0, ws, st));
    double tr[2];
    CTN_CUDA(cudaMemcpyAsync(&tr[0], alpha + 0, sizeof(double), cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaMemcpyAsync(&tr[1], beta + 0, sizeof(double), cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaStreamSynchronize(st));  // the one host synchronisation of a cycle
    theta = tr[0];
    rho = tr[1];
    CTN_REQUIRE(std::isfinite(theta) && std::isfinite(rho), "[Lanczos refined] non-finite Rayleigh quotient");
    if (rho <= tol * std::fabs(theta) || rho == 0.0 || c == max_restarts - 1) break;
    // low-precision Krylov steps, all scalars kept on the device (no host round trip):
    //   w = H u_j;  alpha_j = <w, u_j> / s_j^2, gamma = <w, q0> / s_j;
    //   u_{j+1} = (w - alpha_j u_j) / s_j - beta_{j-1} q_{j-1} - gamma q0, beta_j = |u_{j+1}|
    // (for j = 1, q_{j-1} is q0 and its measured overlap gamma replaces beta_0).  The last
    // step needs alpha only: beta_{m-1} is not an entry of the m x m tridiagonal.
    for (int j = 1; j < krydim; ++j) {
      const double *uj = krylov + (int64_t)j * n;
      const double *up = j >= 2 ? krylov + (int64_t)(j - 1) * n : nullptr;
      if (mv_lo(u_lo, uj, w, st) != 0) return CTN_ERR_CUDA;
      ++n_lo;
      auto step = [&](const auto *wv) -> ctn_status {
        if (fused && j + 1 < krydim) {
          const ctn_status r = krylov_step_f64(wv, uj, up, q0, krylov + (int64_t)(j + 1) * n, n, beta + j - 1,
                                               j >= 2 ? beta + j - 2 : nullptr, alpha + j, scal + 4, beta + j, ws,
                                               ws2, err, st);
          if (r != CTN_ERR_UNSUPPORTED) return r;
          fused = false;
        }
        CTN_TRY(dot2s_f64(wv, uj, q0, n, beta + j - 1, alpha + j, scal + 4, ws2, st));
        if (j + 1 < krydim)
          CTN_TRY(lanczos_step_f64(wv, uj, up, q0, krylov + (int64_t)(j + 1) * n, n, alpha + j, scal + 4,
                                   beta + j - 1, j >= 2 ? beta + j - 2 : nullptr, beta + j, ws, st));
        return CTN_OK;
      };
      // w_f32: the low-precision matvec wrote w as n floats (its own error is far above FP32 rounding)
      if (w_f32) CTN_TRY(step(reinterpret_cast<const float *>(w)));
      else CTN_TRY(step(static_cast<const double *>(w)));
    }
    CTN_CUDA(cudaMemcpyAsync(As.data(), alpha, sizeof(double) * krydim, cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaMemcpyAsync(Bs.data(), beta, sizeof(double) * krydim, cudaMemcpyDeviceToHost, st));
    unsigned err_host = 0;
    CTN_CUDA(cudaMemcpyAsync(&err_host, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaStreamSynchronize(st));
    if (err_host) {
      set_error("[Lanczos refined] the grid barrier of a fused Krylov step gave up waiting");
      return CTN_ERR_TIMEOUT;
    }
    // a zero beta (breakdown) ends the Krylov space there
    int m = krydim;
    for (int j = 0; j + 1 < krydim; ++j)
      if (!(Bs[j] > 0.0) || !std::isfinite(Bs[j])) {
        m = j + 1;
        break;
      }
    for (int j = 0; j < m; ++j)
      CTN_REQUIRE(std::isfinite(As[j]), "[Lanczos refined] non-finite recurrence coefficient");
    evals.assign(m, 0.0);
    evecs.assign((size_t)m * m, 0.0);
    CTN_TRY(tql(m, As.data(), Bs.data(), evals.data(), evecs.data()));
    // v = y_0 q0 + sum_{j>=1} y_j u_j / s_j  (s_j = beta_{j-1} > 0 for j < m)
    coef[0] = evecs[0];
    for (int j = 1; j < m; ++j) coef[j] = evecs[j] / Bs[j - 1];
    CTN_CUDA(cudaMemcpyAsync(cdev, coef.data(), sizeof(double) * m, cudaMemcpyHostToDevice, st));
    CTN_TRY(combine_f64(krylov, n, m, cdev, w, st));
    CTN_TRY(nrm2_f64(w, n, scal + 0, ws, st));
    CTN_TRY(div_copy_f64(w, krylov, n, scal + 0, st));
  }
  CTN_CUDA(cudaMemcpyAsync(eigvec, krylov, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  *energy = theta;
  if (residual) *residual = rho;
  if (restarts) *restarts = c;
  if (counts) {
    counts[0] = n_lo;
    counts[1] = n_hi;
  }
  return CTN_OK;
}
}  // namespace ctn

extern "C" ctn_status ctn_lanczos_refined(ctn_matvec_fn matvec_lo, void *user_lo, ctn_matvec_fn matvec_hi,
                                          void *user_hi, const double *psi0, int64_t n, int krydim, int max_restarts,
                                          double tol, double *krylov, double *work, double *eigvec, double *energy,
                                          double *residual, int *restarts, int64_t *matvecs, void *stream) {
  CTN_REQUIRE(matvec_lo && matvec_hi && psi0 && krylov && work && eigvec && energy,
              "ctn_lanczos_refined: null argument");
  return ctn::lanczos_refined(matvec_lo, user_lo, matvec_hi, user_hi, psi0, n, krydim, max_restarts, tol, krylov,
                              work, eigvec, energy, residual, restarts, matvecs, ctn::as_stream(stream),
                              /*w_f32=*/false);
}

extern "C" ctn_status ctn_lanczos_gnd(ctn_matvec_fn matvec, void *user, const double *psi0, int64_t n, int maxiter,
                                      double cvgcrit, double *krylov, double *work, double *eigvec, double *energy,
                                      int *iters, void *stream) {
  return ctn::lanczos_gnd(matvec, user, psi0, n, maxiter, cvgcrit, krylov, work, eigvec, energy, iters,
                          ctn::as_stream(stream), /*speculate=*/false, /*w_f32=*/false);
}

namespace ctn {
// Dense symmetric eigenproblem by the cyclic Jacobi method (Golub & Van Loan, Matrix
// Computations, sec. 8.5: two-sided rotations that zero one off-diagonal pair at a time,
// swept until the off-diagonal mass is negligible).  a: n x n row-major (copied);
// w: eigenvalues (diagonal order); z: n x n row-major, eigenvectors as COLUMNS.
static ctn_status jacobi_eigh(int n, const double *ain, double *w, double *z) {
  std::vector<double> a(ain, ain + (size_t)n * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) z[(size_t)i * n + j] = i == j ? 1.0 : 0.0;
  double fro = 0.0;
  for (double x : a) fro += x * x;
  fro = std::sqrt(fro);
  bool done = n <= 1 || fro == 0.0;
  for (int sweep = 0; sweep < 100 && !done; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) off += a[(size_t)i * n + j] * a[(size_t)i * n + j];
    if (std::sqrt(off) <= 1e-18 * fro) {
      done = true;
      break;
    }
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double tau = (a[(size_t)q * n + q] - a[(size_t)p * n + p]) / (2.0 * apq);
        const double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < n; ++k) {  // A <- A J (columns p, q)
          const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
          a[(size_t)k * n + p] = c * akp - s * akq;
          a[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // A <- J^T A (rows p, q)
          const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
          a[(size_t)p * n + k] = c * apk - s * aqk;
          a[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {  // Z <- Z J
          const double zkp = z[(size_t)k * n + p], zkq = z[(size_t)k * n + q];
          z[(size_t)k * n + p] = c * zkp - s * zkq;
          z[(size_t)k * n + q] = s * zkp + c * zkq;
        }
      }
    if (sweep == 99) {
      set_error("ctn_sym_eigh: Jacobi sweeps did not converge");
      return CTN_ERR_NUMERIC;
    }
  }
  for (int i = 0; i < n; ++i) w[i] = a[(size_t)i * n + i];
  return CTN_OK;
}

// work layout: [w n][H (ncv + 1) x ncv][Y ncv x ncv][scalars 8][h ncv + 9][multidot ws]
// [reduction ws][restart combination n x ncv]
size_t lanczos_which_work_doubles(int64_t n, int ncv) {
  const size_t ld = (size_t)ncv + 1;
  return (size_t)n + ld * ncv + (size_t)ncv * ncv + 8 + ld + 8 + multidot_ws_doubles((int)ld) +
         reduce_ws_bytes() / sizeof(double) + (size_t)n * (size_t)ncv;
}

// Thick-restart Lanczos for the k extreme eigenpairs of a symmetric operator (Wu & Simon,
// SIAM J. Matrix Anal. Appl. 22 (2000) 602; the symmetric Krylov-Schur restart of Stewart,
// SIAM J. Matrix Anal. Appl. 23 (2001) 601).  It computes what the reference obtains from
// ARPACK's implicitly restarted Lanczos (src/linalg/Lanczos.cpp:250-402: dsaupd/dseupd,
// which = SA / LA / LM, ncv = min(n, 2k + 10) by default, convergence of a Ritz pair when
// its estimate |beta_m y_m| <= tol * max(eps^(2/3), |theta|), tol <= 0 meaning machine
// precision).  Each cycle extends the basis to ncv vectors with full (twice-applied
// classical Gram-Schmidt) re-orthogonalisation on the device, solves the projected
// matrix on the host, and keeps k + (m - k) / 2 wanted Ritz vectors plus the residual
// direction for the next cycle.
ctn_status lanczos_which(int (*mv)(void *, const double *, double *, void *), void *user, const double *v0,
                         int64_t n, int which, int k, int ncv, int maxiter, double tol, double *V, double *work,
                         double *evals, double *evecs, int *iters, int *nconv_out, cudaStream_t st) {
  CTN_REQUIRE(which >= 0 && which <= 2, "[ERROR][Lanczos] 'which' should be 'LM', 'LA', 'SA'");
  CTN_REQUIRE(n > 0 && k >= 1 && k <= n, "[ERROR][Lanczos] k should be in 1..n");
  CTN_REQUIRE(maxiter >= 1, "[ERROR][Lanczos] Maxiter must be >= 1");
  CTN_REQUIRE(tol >= 0, "[ERROR][Lanczos] cvg_crit should be >= 0");
  if (ncv == 0) ncv = (int)std::min<int64_t>(n, 2 * (int64_t)k + 10);
  CTN_REQUIRE(ncv <= n && (ncv > k || ncv == n), "[ERROR][Lanczos] ncv should be 2+k<=ncv<=nx");
  const int ld = ncv + 1;  // device H: column j at H + j * ld (rows 0..j+1)
  double *w = work;
  double *Hd = w + n;
  double *Yd = Hd + (size_t)ld * ncv;
  double *scal = Yd + (size_t)ncv * ncv;  // [0] norm [1] one [2..] spare
  double *tmp_h = scal + 8;                // ld doubles
  double *mws = tmp_h + ld + 8;            // multidot workspace
  double *rws = mws + multidot_ws_doubles(ld);
  double *Vtmp = rws + reduce_ws_bytes() / sizeof(double);  // n x ncv: restart combination
  CTN_CUDA(cudaMemsetAsync(mws, 0, multidot_ws_doubles(ld) * sizeof(double), st));
  CTN_CUDA(cudaMemsetAsync(rws, 0, reduce_ws_bytes(), st));
  CTN_CUDA(cudaMemsetAsync(Hd, 0, sizeof(double) * (size_t)ld * ncv, st));
  const double one = 1.0;
  CTN_CUDA(cudaMemcpyAsync(scal + 1, &one, sizeof(double), cudaMemcpyHostToDevice, st));
  CTN_TRY(nrm2_f64(v0, n, scal + 0, rws, st));
  double nrm0 = 0.0;
  CTN_CUDA(cudaMemcpyAsync(&nrm0, scal + 0, sizeof(double), cudaMemcpyDeviceToHost, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  CTN_REQUIRE(nrm0 > 0 && std::isfinite(nrm0), "[ERROR][Lanczos] initial vector has zero or non-finite norm");
  CTN_TRY(div_copy_f64(v0, V, n, scal + 0, st));

  const double eps = std::numeric_limits<double>::epsilon() * 0.5;  // unit roundoff (dlamch 'E')
  const double eps23 = std::pow(eps, 2.0 / 3.0);
  const double tol_eff = tol > 0 ? tol : eps;
  std::vector<double> Hh((size_t)ld * ncv), T, th, Y, theta_kept;
  std::vector<int> order;
  int p = 0, it = 0, nconv = 0, m = 0;
  bool finished = false;
  std::vector<double> Ysel;
  for (it = 0; it < maxiter && !finished; ++it) {
    for (int j = p; j < ncv; ++j) {
      if (mv(user, V + (int64_t)j * n, w, st) != 0) return CTN_ERR_CUDA;
      double *hj = Hd + (size_t)j * ld;
      CTN_TRY(multidot_f64(V, w, n, j + 1, hj, 0, mws, st));
      CTN_TRY(multiaxpy_f64(V, hj, n, j + 1, w, st));
      CTN_TRY(multidot_f64(V, w, n, j + 1, tmp_h, 0, mws, st));  // second Gram-Schmidt pass
      CTN_TRY(multiaxpy_f64(V, tmp_h, n, j + 1, w, st));
      CTN_TRY(axpy_f64(tmp_h, hj, j + 1, scal + 1, 1.0, st));
      CTN_TRY(nrm2_f64(w, n, hj + j + 1, rws, st));
      CTN_TRY(div_copy_f64(w, V + (int64_t)(j + 1) * n, n, hj + j + 1, st));
    }
    CTN_CUDA(cudaMemcpyAsync(Hh.data(), Hd, sizeof(double) * Hh.size(), cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaStreamSynchronize(st));
    double anorm = 0.0;
    for (int i = 0; i < p; ++i) anorm = std::max(anorm, std::fabs(theta_kept[i]));
    for (int j = p; j < ncv; ++j)
      for (int i = 0; i <= j + 1; ++i) {
        CTN_REQUIRE(std::isfinite(Hh[(size_t)j * ld + i]), "[ERROR][Lanczos] non-finite projection");
        anorm = std::max(anorm, std::fabs(Hh[(size_t)j * ld + i]));
      }
    m = ncv;
    bool breakdown = false;
    for (int j = p; j < ncv; ++j)
      if (Hh[(size_t)j * ld + j + 1] <= 64.0 * eps * anorm) {  // invariant subspace reached
        m = j + 1;
        breakdown = true;
        break;
      }
    // projected matrix: the kept Ritz values on the diagonal of the first p rows, the
    // Gram-Schmidt coefficients of the extension columns (couplings included) above it
    T.assign((size_t)m * m, 0.0);
    for (int i = 0; i < p; ++i) T[(size_t)i * m + i] = theta_kept[i];
    for (int j = p; j < m; ++j)
      for (int i = 0; i <= j; ++i) T[(size_t)i * m + j] = T[(size_t)j * m + i] = Hh[(size_t)j * ld + i];
    th.assign(m, 0.0);
    Y.assign((size_t)m * m, 0.0);
    CTN_TRY(jacobi_eigh(m, T.data(), th.data(), Y.data()));
    order.resize(m);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      if (which == 0) return th[a] < th[b];               // SA
      if (which == 1) return th[a] > th[b];               // LA
      return std::fabs(th[a]) > std::fabs(th[b]);         // LM
    });
    const double beta_last = breakdown ? 0.0 : Hh[(size_t)(m - 1) * ld + m];
    const int kk_want = std::min(k, m);
    nconv = 0;
    for (int c = 0; c < kk_want; ++c) {
      const double est = std::fabs(beta_last * Y[(size_t)(m - 1) * m + order[c]]);
      if (est <= tol_eff * std::max(eps23, std::fabs(th[order[c]]))) ++nconv;
    }
    if (nconv >= k || breakdown || it == maxiter - 1) {
      finished = true;
      break;
    }
    // thick restart: keep kk wanted Ritz vectors, then the residual direction v_m
    const int kk = std::max(k, std::min(m - 1, k + (m - k) / 2));
    Ysel.assign((size_t)m * kk, 0.0);
    for (int j = 0; j < m; ++j)
      for (int c = 0; c < kk; ++c) Ysel[(size_t)j * kk + c] = Y[(size_t)j * m + order[c]];
    CTN_CUDA(cudaMemcpyAsync(Yd, Ysel.data(), sizeof(double) * Ysel.size(), cudaMemcpyHostToDevice, st));
    double *comb = Vtmp;
    CTN_TRY(basis_combine_f64(V, n, m, Yd, kk, kk, comb, st));
    CTN_CUDA(cudaMemcpyAsync(V, comb, sizeof(double) * (size_t)n * kk, cudaMemcpyDeviceToDevice, st));
    CTN_CUDA(cudaMemcpyAsync(V + (int64_t)kk * n, V + (int64_t)m * n, sizeof(double) * (size_t)n,
                             cudaMemcpyDeviceToDevice, st));
    theta_kept.assign(kk, 0.0);
    for (int c = 0; c < kk; ++c) theta_kept[c] = th[order[c]];
    CTN_CUDA(cudaStreamSynchronize(st));  // Ysel is reused by the next cycle
    p = kk;
  }
  // eigenpairs in the reference's order (sort_indices of Lanczos.cpp: by value or |value|)
  for (int c = 0; c < k; ++c) evals[c] = c < m ? th[order[c]] : 0.0;
  if (evecs) {
    const int kc = std::min(k, m);
    Ysel.assign((size_t)m * kc, 0.0);
    for (int j = 0; j < m; ++j)
      for (int c = 0; c < kc; ++c) Ysel[(size_t)j * kc + c] = Y[(size_t)j * m + order[c]];
    CTN_CUDA(cudaMemcpyAsync(Yd, Ysel.data(), sizeof(double) * Ysel.size(), cudaMemcpyHostToDevice, st));
    CTN_TRY(basis_combine_f64(V, n, m, Yd, kc, kc, evecs, st));
  }
  CTN_CUDA(cudaStreamSynchronize(st));
  if (iters) *iters = it + (finished ? 1 : 0);
  if (nconv_out) *nconv_out = nconv;
  return CTN_OK;
}
}  // namespace ctn

extern "C" size_t ctn_lanczos_which_work_doubles(int64_t n, int ncv) {
  return ctn::lanczos_which_work_doubles(n, ncv);
}

extern "C" ctn_status ctn_lanczos_which(ctn_matvec_fn matvec, void *user, const double *v0, int64_t n, int which,
                                        int k, int ncv, int maxiter, double tol, double *basis, double *work,
                                        double *evals, double *evecs, int *iters, int *nconv, void *stream) {
  CTN_REQUIRE(matvec && v0 && basis && work && evals, "ctn_lanczos_which: null argument");
  return ctn::lanczos_which(matvec, user, v0, n, which, k, ncv, maxiter, tol, basis, work, evals, evecs, iters, nconv,
                            ctn::as_stream(stream));
}

extern "C" ctn_status ctn_sym_eigh(int n, const double *a, double *w, double *z) {
  CTN_REQUIRE(n >= 0 && a && w && z, "ctn_sym_eigh: bad argument");
  return ctn::jacobi_eigh(n, a, w, z);
}

namespace ctn {
// exp(tau H) v by the Lanczos projection of Lanczos_Exp (src/linalg/Lanczos_Exp.cpp:264-369):
// plain three-term recurrence from v / |v|, breakdown when beta <= 100 eps scale sqrt(i)
// (scale = running max of |alpha| + |beta| + |beta_prev| and 1), stop when the bottom-left
// element of exp(tau T_i) falls below cvgcrit, result V exp(tau T) V^T v with the
// un-normalised input.  T is symmetric tridiagonal, so exp(tau T) is formed from its
// eigenpairs (the reference calls a general ExpM; the matrices agree to rounding).  Real
// and imaginary parts of tau; out_im may be null when tau is real.
ctn_status lanczos_exp(int (*mv)(void *, const double *, double *, void *), void *user, const double *vin,
                       int64_t n, double tau_re, double tau_im, double cvgcrit, int maxiter, double *V, double *work,
                       double *out_re, double *out_im, int *iters, cudaStream_t st) {
  CTN_REQUIRE(cvgcrit > 0, "[ERROR][Lanczos_Exp] converge criteria must >0");
  CTN_REQUIRE(maxiter >= 2, "[ERROR][Lanczos_Exp] Maxiter must >1");
  CTN_REQUIRE(n > 0, "[ERROR][Lanczos_Exp] empty vector");
  CTN_REQUIRE(tau_im == 0.0 || out_im, "[ERROR][Lanczos_Exp] complex tau needs the imaginary output");
  const int mmax = (int)std::min<int64_t>(maxiter, n);
  double *w = work;                  // matvec output / recurrence vector
  double *scal = work + n;           // [0] |v| [1] alpha [2] beta (coefficient of v_old) [3] |w|
  double *cdev = scal + 8;           // V^T v (mmax) then the output coefficients
  double *mws = cdev + 2 * mmax + 8;
  double *rws = mws + multidot_ws_doubles(mmax);
  CTN_CUDA(cudaMemsetAsync(mws, 0, multidot_ws_doubles(mmax) * sizeof(double), st));
  CTN_CUDA(cudaMemsetAsync(rws, 0, reduce_ws_bytes(), st));
  double h[4];
  auto fetch2 = [&](int a, int b) -> ctn_status {
    CTN_CUDA(cudaMemcpyAsync(&h[a], scal + a, sizeof(double), cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaMemcpyAsync(&h[b], scal + b, sizeof(double), cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaStreamSynchronize(st));
    return CTN_OK;
  };
  CTN_TRY(nrm2_f64(vin, n, scal + 0, rws, st));
  CTN_TRY(div_copy_f64(vin, V, n, scal + 0, st));
  if (mv(user, V, w, st) != 0) return CTN_ERR_CUDA;
  CTN_TRY(dot_f64(w, V, n, scal + 1, rws, st));
  CTN_TRY(lanczos_update_f64(w, V, nullptr, n, scal + 1, nullptr, scal + 3, rws, st));
  CTN_TRY(fetch2(1, 3));
  CTN_REQUIRE(std::isfinite(h[1]) && std::isfinite(h[3]), "[ERROR][Lanczos_Exp] non-finite recurrence");
  const double eps = std::numeric_limits<double>::epsilon();
  std::vector<double> al{h[1]}, be;  // diagonal, off-diagonal
  double beta_prev = 0.0, scale = std::max(std::fabs(h[1]), 1.0), wnorm = h[3];
  double alpha = h[1];
  std::vector<double> ev, z, Bre, Bim;
  // B = exp(tau T) for the current T (m x m, row-major), real and imaginary parts
  auto expm = [&](int m) -> ctn_status {
    ev.assign(m, 0.0);
    z.assign((size_t)m * m, 0.0);
    CTN_TRY(tql(m, al.data(), be.data(), ev.data(), z.data()));
    Bre.assign((size_t)m * m, 0.0);
    Bim.assign((size_t)m * m, 0.0);
    for (int j = 0; j < m; ++j) {
      const double mag = std::exp(tau_re * ev[j]);
      const double er = mag * std::cos(tau_im * ev[j]), ei = mag * std::sin(tau_im * ev[j]);
      const double *zj = &z[(size_t)j * m];
      for (int a = 0; a < m; ++a)
        for (int b = 0; b < m; ++b) {
          Bre[(size_t)a * m + b] += er * zj[a] * zj[b];
          Bim[(size_t)a * m + b] += ei * zj[a] * zj[b];
        }
    }
    return CTN_OK;
  };
  int m = 1;
  bool have_B = false;
  for (int i = 1; i < mmax; ++i) {
    const double beta = wnorm;
    scale = std::max(scale, std::max(std::fabs(alpha) + std::fabs(beta) + std::fabs(beta_prev), 1.0));
    if (!(beta > 100.0 * eps * scale * std::sqrt((double)i))) break;  // no new direction
    CTN_TRY(div_copy_f64(w, V + (int64_t)i * n, n, scal + 3, st));
    m = i + 1;
    be.push_back(beta);
    CTN_CUDA(cudaMemcpyAsync(scal + 2, &be.back(), sizeof(double), cudaMemcpyHostToDevice, st));
    if (mv(user, V + (int64_t)i * n, w, st) != 0) return CTN_ERR_CUDA;
    CTN_TRY(dot_f64(w, V + (int64_t)i * n, n, scal + 1, rws, st));
    CTN_TRY(lanczos_update_f64(w, V + (int64_t)i * n, V + (int64_t)(i - 1) * n, n, scal + 1, scal + 2, scal + 3,
                               rws, st));
    CTN_TRY(fetch2(1, 3));
    CTN_REQUIRE(std::isfinite(h[1]) && std::isfinite(h[3]), "[ERROR][Lanczos_Exp] non-finite recurrence");
    alpha = h[1];
    wnorm = h[3];
    al.push_back(alpha);
    beta_prev = beta;
    CTN_TRY(expm(m));
    have_B = true;
    const double err = std::hypot(Bre[(size_t)i * m], Bim[(size_t)i * m]);
    if (err < cvgcrit) break;
  }
  if (!have_B) CTN_TRY(expm(m));
  // out = V B (V^T v): c = V^T v on the device, the coefficients on the host
  CTN_TRY(multidot_f64(V, vin, n, m, cdev, 0, mws, st));
  std::vector<double> c(m), dre(m, 0.0), dim(m, 0.0);
  CTN_CUDA(cudaMemcpyAsync(c.data(), cdev, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  for (int a = 0; a < m; ++a)
    for (int b = 0; b < m; ++b) {
      dre[a] += Bre[(size_t)a * m + b] * c[b];
      dim[a] += Bim[(size_t)a * m + b] * c[b];
    }
  CTN_CUDA(cudaMemcpyAsync(cdev, dre.data(), sizeof(double) * m, cudaMemcpyHostToDevice, st));
  CTN_TRY(basis_combine_f64(V, n, m, cdev, 1, 1, out_re, st));
  if (out_im) {
    CTN_CUDA(cudaMemcpyAsync(cdev + mmax, dim.data(), sizeof(double) * m, cudaMemcpyHostToDevice, st));
    CTN_TRY(basis_combine_f64(V, n, m, cdev + mmax, 1, 1, out_im, st));
  }
  CTN_CUDA(cudaStreamSynchronize(st));
  if (iters) *iters = m;
  return CTN_OK;
}
}  // namespace ctn

extern "C" size_t ctn_lanczos_exp_work_doubles(int64_t n, int maxiter) {
  const int mmax = (int)std::min<int64_t>(maxiter, n);
  return (size_t)n + 8 + 2 * (size_t)mmax + 8 + ctn::multidot_ws_doubles(mmax) + ctn::reduce_ws_bytes() / sizeof(double);
}

extern "C" ctn_status ctn_lanczos_exp(ctn_matvec_fn matvec, void *user, const double *v, int64_t n, double tau_re,
                                      double tau_im, double cvgcrit, int maxiter, double *basis, double *work,
                                      double *out_re, double *out_im, int *iters, void *stream) {
  CTN_REQUIRE(matvec && v && basis && work && out_re, "ctn_lanczos_exp: null argument");
  return ctn::lanczos_exp(matvec, user, v, n, tau_re, tau_im, cvgcrit, maxiter, basis, work, out_re, out_im, iters,
                          ctn::as_stream(stream));
}
