// Grouped FP64 GEMM on the B200 FP64 tensor pipe (DMMA, mma.sync m16n8k16 .f64).
//
// One launch computes every output block of a block-sparse contraction:
//   C_t = sum_{p in pairs(t)} op(A_p) * op(B_p)     (row-major C_t, m_t x n_t)
// which is what BlockUniTensor::contract issues as one Matmul (non-MKL build,
// src/BlockUniTensor.cpp:1180-1223) or one Gemm_Batch group entry (MKL build,
// :1114-1177) per block pair; the reference's GPU Gemm_Batch is a serial loop of
// cublasDgemm calls (src/backend/linalg_internal_gpu/cuGemm_Batch_internal.cu:23-64).
// Here a CTA owns one 64x64 tile of one output block and walks the whole K range of
// all its pairs, so every output element is written exactly once (no atomics, no
// zero-fill pass; tasks with no pair write zeros, matching Init's zeros blocks).
// Operands are read in place from the block storage with per-pair leading
// dimensions and an optional transpose, staged through shared memory by a
// 2-stage cp.async pipeline.  FP64 has no tcgen05 kind, so the legacy-warp DMMA
// instruction is the FP64 tensor path on sm_100a.
#include <algorithm>
#include <vector>

#include "ctn_common.h"
#include "gemm_f64.cuh"

namespace ctn {

namespace {
constexpr int BK = 16;  // k depth of a stage; tiles are BM x BN = 64 x 64, 64 x 32 or 32 x 32
constexpr int PAD = 4;
constexpr int NTHREADS = 128;

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D(16x8) += A(16x16) B(16x8), FP64, one warp.  Fragments (groupID g = lane/4,
// t = lane%4): a[i] = A[g + 8*(i&1)][t + 4*(i>>1)], b[i] = B[t + 4*i][g],
// c[0..1] = C[g][2t..2t+1], c[2..3] = C[g+8][2t..2t+1].
__device__ __forceinline__ void dmma_16x8x16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// Shared-memory tiles keep the operand's contiguous global axis contiguous, so the
// cp.async writes are conflict-free; the +4 double padding makes every fragment read
// pattern below conflict-free as well (bank = 8*x + 2*y for the 4x4 lanes of a phase).
template <bool TA, bool TB, int BM, int BN>
struct SmemT {
  double A[2][TA ? BK : BM][(TA ? BM : BK) + PAD];
  double B[2][TB ? BN : BK][(TB ? BK : BN) + PAD];
};

template <bool TA, bool TB, int BM, int BN>
__device__ __forceinline__ void load_stage(SmemT<TA, TB, BM, BN> &sm, int buf, const double *__restrict__ A,
                                           const double *__restrict__ B, const GemmPairD &p, int m, int n,
                                           int m0, int n0, int k0) {
  const int tid = threadIdx.x;
  const double *Ap = A + p.a_off;
  const double *Bp = B + p.b_off;
#pragma unroll
  for (int i = 0; i < (BM * BK) / NTHREADS; ++i) {
    const int idx = tid + i * NTHREADS;
    if (!TA) {  // A[m][k]: k contiguous
      const int mm = idx / BK, kk = idx % BK;
      const int gm = m0 + mm, gk = k0 + kk;
      const bool ok = gm < m && gk < p.k;
      cp_async8(&sm.A[buf][mm][kk], ok ? Ap + (int64_t)gm * p.lda + gk : Ap, ok);
    } else {  // A stored [k][m]: m contiguous
      const int kk = idx / BM, mm = idx % BM;
      const int gm = m0 + mm, gk = k0 + kk;
      const bool ok = gm < m && gk < p.k;
      cp_async8(&sm.A[buf][kk][mm], ok ? Ap + (int64_t)gk * p.lda + gm : Ap, ok);
    }
  }
#pragma unroll
  for (int i = 0; i < (BN * BK) / NTHREADS; ++i) {
    const int idx = tid + i * NTHREADS;
    if (!TB) {  // B[k][n]: n contiguous
      const int kk = idx / BN, nn = idx % BN;
      const int gn = n0 + nn, gk = k0 + kk;
      const bool ok = gn < n && gk < p.k;
      cp_async8(&sm.B[buf][kk][nn], ok ? Bp + (int64_t)gk * p.ldb + gn : Bp, ok);
    } else {  // B stored [n][k]: k contiguous
      const int nn = idx / BK, kk = idx % BK;
      const int gn = n0 + nn, gk = k0 + kk;
      const bool ok = gn < n && gk < p.k;
      cp_async8(&sm.B[buf][nn][kk], ok ? Bp + (int64_t)gn * p.ldb + gk : Bp, ok);
    }
  }
}

// Each of the 4 warps computes a (BM / 2) x (BN / 2) quarter of the tile: 64 x 64 tiles 2 x 4
// m16n8 products per k step, 64 x 32 tiles 2 x 2 (plans with too few 64 x 64 tiles to fill the
// SMs), 32 x 32 tiles 1 x 2 (plans of small blocks, where 64-row tiles are mostly padding).
template <bool TA, bool TB, int BM, int BN>
__global__ void __launch_bounds__(NTHREADS) k_gemm_grouped_f64(
    const double *__restrict__ A, const double *__restrict__ B, double *__restrict__ C,
    const GemmTaskD *__restrict__ tasks, const GemmPairD *__restrict__ pairs,
    const GemmTileD *__restrict__ tiles, int64_t ntiles) {
  constexpr int MI = BM / 32;  // m16 products per warp
  constexpr int NJ = BN / 16;  // n8 products per warp
  __shared__ __align__(16) SmemT<TA, TB, BM, BN> sm;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp >> 1) * (BM / 2), wn = (warp & 1) * (BN / 2);
  const int g = lane >> 2, t4 = lane & 3;
  for (int64_t ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
    const GemmTileD tile = tiles[ti];
    const GemmTaskD task = tasks[tile.task];
    const int m0 = tile.m0, n0 = tile.n0;
    double acc[MI][NJ][4];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

    // flattened (pair, k-tile) iteration with a 2-deep cp.async pipeline
    int pi = 0, kt = 0;
    const int npairs = task.pair_count;
    while (pi < npairs && pairs[task.pair_begin + pi].k <= 0) ++pi;
    int buf = 0;
    bool have = pi < npairs;
    GemmPairD cur;
    if (have) {
      cur = pairs[task.pair_begin + pi];
      load_stage<TA, TB, BM, BN>(sm, 0, A, B, cur, task.m, task.n, m0, n0, 0);
    }
    cp_async_commit();
    while (have) {
      int npi = pi, nkt = kt + 1;
      GemmPairD nxt = cur;
      if (nkt * BK >= cur.k) {
        nkt = 0;
        ++npi;
        while (npi < npairs && pairs[task.pair_begin + npi].k <= 0) ++npi;
        if (npi < npairs) nxt = pairs[task.pair_begin + npi];
      }
      const bool have_next = npi < npairs;
      if (have_next) load_stage<TA, TB, BM, BN>(sm, buf ^ 1, A, B, nxt, task.m, task.n, m0, n0, nkt * BK);
      cp_async_commit();
      cp_async_wait<1>();
      __syncthreads();
      double a[MI][8], b[NJ][4];
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int r = wm + i * 16 + g + 8 * (e & 1), k = t4 + 4 * (e >> 1);
          a[i][e] = TA ? sm.A[buf][k][r] : sm.A[buf][r][k];
        }
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = t4 + 4 * e, cidx = wn + j * 8 + g;
          b[j][e] = TB ? sm.B[buf][cidx][k] : sm.B[buf][k][cidx];
        }
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) dmma_16x8x16(acc[i][j], a[i], b[j]);
      __syncthreads();
      buf ^= 1;
      pi = npi;
      kt = nkt;
      cur = nxt;
      have = have_next;
    }
    cp_async_wait<0>();
    double *Cp = C + task.c_off;
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int r0 = m0 + wm + i * 16 + g;
        const int c0 = n0 + wn + j * 8 + 2 * t4;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = r0 + h * 8;
          if (r < task.m) {
            if (c0 < task.n) Cp[(int64_t)r * task.ldc + c0] = acc[i][j][2 * h];
            if (c0 + 1 < task.n) Cp[(int64_t)r * task.ldc + c0 + 1] = acc[i][j][2 * h + 1];
          }
        }
      }
    __syncthreads();
  }
}
}  // namespace

void build_tiles_f64(const std::vector<GemmTaskD> &tasks, const std::vector<GemmPairD> &pairs,
                     std::vector<GemmTileD> &tiles, int bm, int bn) {
  tiles.clear();
  std::vector<std::pair<double, GemmTileD>> tmp;
  for (size_t t = 0; t < tasks.size(); ++t) {
    const GemmTaskD &tk = tasks[t];
    double kt = 0;
    for (int p = 0; p < tk.pair_count; ++p) kt += std::max(0, pairs[tk.pair_begin + p].k);
    for (int m0 = 0; m0 < tk.m; m0 += bm)
      for (int n0 = 0; n0 < tk.n; n0 += bn) {
        GemmTileD g;
        g.task = (int32_t)t;
        g.m0 = m0;
        g.n0 = n0;
        tmp.push_back({kt + 1.0, g});
      }
  }
  // longest-first so the tail of the grid is made of cheap tiles
  std::stable_sort(tmp.begin(), tmp.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
  tiles.reserve(tmp.size());
  for (auto &x : tmp) tiles.push_back(x.second);
}

ctn_status launch_gemm_f64(const double *A, const double *B, double *C, const GemmTaskD *d_tasks,
                           const GemmPairD *d_pairs, const GemmTileD *d_tiles, int64_t ntiles, int flags,
                           int bm, int bn, cudaStream_t st) {
  if (ntiles == 0) return CTN_OK;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // 128 threads, ~17 KB smem: up to 8+ CTAs per SM resident
  const int64_t grid = std::min<int64_t>(ntiles, (int64_t)nsm * 12);
  auto go = [&](auto kern) { kern<<<(unsigned)grid, NTHREADS, 0, st>>>(A, B, C, d_tasks, d_pairs, d_tiles, ntiles); };
  if (bm == 32) {
    switch (flags & 3) {
      case 0: go(k_gemm_grouped_f64<false, false, 32, 32>); break;
      case 1: go(k_gemm_grouped_f64<true, false, 32, 32>); break;
      case 2: go(k_gemm_grouped_f64<false, true, 32, 32>); break;
      default: go(k_gemm_grouped_f64<true, true, 32, 32>); break;
    }
  } else if (bn == 32) {
    switch (flags & 3) {
      case 0: go(k_gemm_grouped_f64<false, false, 64, 32>); break;
      case 1: go(k_gemm_grouped_f64<true, false, 64, 32>); break;
      case 2: go(k_gemm_grouped_f64<false, true, 64, 32>); break;
      default: go(k_gemm_grouped_f64<true, true, 64, 32>); break;
    }
  } else {
    switch (flags & 3) {
      case 0: go(k_gemm_grouped_f64<false, false, 64, 64>); break;
      case 1: go(k_gemm_grouped_f64<true, false, 64, 64>); break;
      case 2: go(k_gemm_grouped_f64<false, true, 64, 64>); break;
      default: go(k_gemm_grouped_f64<true, true, 64, 64>); break;
    }
  }
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}

}  // namespace ctn

extern "C" size_t ctn_gemm_grouped_scratch_bytes(int64_t ntasks, int64_t npairs) {
  // tasks + pairs + tiles (upper bound: tiles counted at execution; reserve generously)
  (void)ntasks;
  (void)npairs;
  return 0;
}
