// C ABI plumbing: error text, dtype table, BLAS-1 entry points, the symmetric
// tridiagonal eigensolver and the Lanczos ground-state driver.
#include <algorithm>
#include <cmath>
#include <cstring>
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

// Symmetric tridiagonal eigenproblem by the implicit QL algorithm with Wilkinson-type
// shifts (the EISPACK tql2 / "tqli" scheme: Bowdler, Martin, Reinsch & Wilkinson,
// Numer. Math. 11 (1968) 293-306).  d: diagonal (n), e: sub-diagonal (n-1).
// Eigenvalues ascending; z (n x n, row-major) receives eigenvectors as ROWS, which is
// the is_row=true layout linalg::Tridiag returns (src/linalg/Tridiag.cpp:83-95).
static ctn_status tql(int n, const double *din, const double *ein, double *w, double *zrows) {
  std::vector<double> d(din, din + n), e(n, 0.0);
  for (int i = 0; i + 1 < n; ++i) e[i] = ein[i];
  std::vector<double> z((size_t)n * n, 0.0);  // column-major accumulation: z[k + n*i] = comp k of vec i
  for (int i = 0; i < n; ++i) z[(size_t)i * n + i] = 1.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    int m;
    do {
      for (m = l; m < n - 1; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= 1e-300 || std::fabs(e[m]) + dd == dd) break;
      }
      if (m != l) {
        if (++iter > 200) {
          set_error("ctn_tridiag_eigh: QL iteration did not converge");
          return CTN_ERR_NUMERIC;
        }
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = std::hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
        double s = 1.0, c = 1.0, p = 0.0;
        int i;
        bool early = false;
        for (i = m - 1; i >= l; --i) {
          double f = s * e[i];
          const double b = c * e[i];
          r = std::hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            d[i + 1] -= p;
            e[m] = 0.0;
            early = true;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - b;
          double *zi = &z[(size_t)i * n], *zi1 = &z[(size_t)(i + 1) * n];
          for (int k = 0; k < n; ++k) {
            f = zi1[k];
            zi1[k] = s * zi[k] + c * f;
            zi[k] = c * zi[k] - s * f;
          }
        }
        if (early) continue;
        d[l] -= p;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return d[a] < d[b]; });
  for (int j = 0; j < n; ++j) {
    w[j] = d[idx[j]];
    if (zrows) std::memcpy(zrows + (size_t)j * n, &z[(size_t)idx[j] * n], sizeof(double) * n);
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
// Lanczos_Gnd_Ut (src/linalg/Lanczos_Gnd_Ut.cpp:29-162): 3-term recurrence, Tridiag
// re-solved each iteration, stop on |dE| < cvgcrit or beta == 0; the Ritz vector is
// the combination of the stored Krylov vectors.  The vectors stay on the device; the
// two scalars per iteration come to the host as the reference's .item() calls do.
ctn_status lanczos_gnd(int (*mv)(void *, const double *, double *, void *), void *user, const double *psi0,
                       int64_t n, int maxiter, double cvgcrit, double *krylov, double *work, double *eigvec,
                       double *energy, int *iters, cudaStream_t st) {
  CTN_REQUIRE(maxiter >= 2, "[Lanczos] Maxiter must >1");
  CTN_REQUIRE(cvgcrit > 0, "[Lanczos] converge criteria must >0");
  CTN_REQUIRE(n > 0, "[Lanczos] empty vector");
  double *w = work;                      // new_psi
  double *scal = work + n;               // device scalars [0]=norm [1]=alpha [2]=beta [3]=nrm
  double *ws = work + n + 8;             // reduction workspace (zeroed below)
  CTN_CUDA(cudaMemsetAsync(ws, 0, reduce_ws_bytes(), st));
  double host[4];
  auto fetch = [&](int idx, double *dst) -> ctn_status {
    CTN_CUDA(cudaMemcpyAsync(dst, scal + idx, sizeof(double), cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaStreamSynchronize(st));
    return CTN_OK;
  };
  // psi_1 = Tin / |Tin|
  CTN_TRY(nrm2_f64(psi0, n, scal + 0, ws, st));
  CTN_TRY(fetch(0, &host[0]));
  CTN_REQUIRE(host[0] > 0 && std::isfinite(host[0]), "[Lanczos] initial vector has zero or non-finite norm");
  CTN_TRY(div_copy_f64(psi0, krylov, n, scal + 0, st));
  std::vector<double> As, Bs, evals, evecs;
  int nk = 1;  // Krylov vectors stored
  // i = 0
  if (mv(user, krylov, w, st) != 0) return CTN_ERR_CUDA;
  CTN_TRY(dot_f64(w, krylov, n, scal + 1, ws, st));
  CTN_TRY(lanczos_update_f64(w, krylov, nullptr, n, scal + 1, scal + 2, scal + 3, ws, st));
  CTN_TRY(fetch(1, &host[1]));
  CTN_TRY(fetch(3, &host[3]));
  double alpha = host[1], beta = host[3];
  As.push_back(alpha);
  Bs.push_back(beta);
  if (beta == 0.0) {
    *energy = alpha;
    *iters = 1;
    CTN_CUDA(cudaMemcpyAsync(eigvec, krylov, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    return CTN_OK;
  }
  CTN_CUDA(cudaMemcpyAsync(scal + 2, &beta, sizeof(double), cudaMemcpyHostToDevice, st));
  CTN_TRY(div_copy_f64(w, krylov + n, n, scal + 3, st));
  nk = 2;
  double E = alpha;
  evals.assign(1, alpha);
  evecs.assign(1, 1.0);
  int it = 1;
  for (int i = 1; i < maxiter; ++i) {
    it = i + 1;
    const double *p1 = krylov + (int64_t)i * n;
    const double *p0 = krylov + (int64_t)(i - 1) * n;
    if (mv(user, p1, w, st) != 0) return CTN_ERR_CUDA;
    CTN_TRY(dot_f64(w, p1, n, scal + 1, ws, st));
    // beta (old) is at scal[2]
    CTN_TRY(lanczos_update_f64(w, p1, p0, n, scal + 1, scal + 2, scal + 3, ws, st));
    CTN_TRY(fetch(1, &host[1]));
    CTN_TRY(fetch(3, &host[3]));
    alpha = host[1];
    As.push_back(alpha);
    const int m = (int)As.size();
    evals.assign(m, 0.0);
    evecs.assign((size_t)m * m, 0.0);
    CTN_TRY(tql(m, As.data(), Bs.data(), evals.data(), evecs.data()));
    beta = host[3];
    Bs.push_back(beta);
    if (beta == 0.0) break;
    CTN_CUDA(cudaMemcpyAsync(scal + 2, &beta, sizeof(double), cudaMemcpyHostToDevice, st));
    CTN_TRY(div_copy_f64(w, krylov + (int64_t)(i + 1) * n, n, scal + 3, st));
    nk = i + 2;
    const double ediff = std::fabs(E - evals[0]);
    if (ediff < cvgcrit) break;
    E = evals[0];
  }
  (void)nk;
  // eigenvector = sum_n kry[n] psi_s[n] over the tridiagonal size
  const int m = (int)evals.size();
  double *coef = scal + 4;  // need m doubles: place after ws instead if m > 4
  double *cdev = ws + reduce_ws_bytes() / sizeof(double);
  (void)coef;
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
                           cudaStream_t st) {
  CTN_REQUIRE(krydim >= 2 && max_restarts >= 1 && n > 0 && tol >= 0, "[Lanczos refined] bad argument");
  // work: [w n][scalars 8][reduction ws][two-sum ws][Ritz coefficients m][alpha m][beta m]
  double *w = work;
  double *scal = work + n;  // [0] norm [1] theta [3] rho [4] gamma (overlap with q0)
  double *ws = work + n + 8;
  double *ws2 = ws + reduce_ws_bytes() / sizeof(double);
  double *cdev = ws2 + reduce2_ws_bytes() / sizeof(double);
  double *alpha = cdev + krydim;
  double *beta = alpha + krydim;
  CTN_CUDA(cudaMemsetAsync(ws, 0, reduce_ws_bytes() + reduce2_ws_bytes(), st));
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
      CTN_TRY(dot2s_f64(w, uj, q0, n, beta + j - 1, alpha + j, scal + 4, ws2, st));
      if (j + 1 < krydim)
        CTN_TRY(lanczos_step_f64(w, uj, up, q0, krylov + (int64_t)(j + 1) * n, n, alpha + j, scal + 4, beta + j - 1,
                                 j >= 2 ? beta + j - 2 : nullptr, beta + j, ws, st));
    }
    CTN_CUDA(cudaMemcpyAsync(As.data(), alpha, sizeof(double) * krydim, cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaMemcpyAsync(Bs.data(), beta, sizeof(double) * krydim, cudaMemcpyDeviceToHost, st));
    CTN_CUDA(cudaStreamSynchronize(st));
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
                              work, eigvec, energy, residual, restarts, matvecs, ctn::as_stream(stream));
}

extern "C" ctn_status ctn_lanczos_gnd(ctn_matvec_fn matvec, void *user, const double *psi0, int64_t n, int maxiter,
                                      double cvgcrit, double *krylov, double *work, double *eigvec, double *energy,
                                      int *iters, void *stream) {
  return ctn::lanczos_gnd(matvec, user, psi0, n, maxiter, cvgcrit, krylov, work, eigvec, energy, iters,
                          ctn::as_stream(stream));
}
