// Device-side task tables of the grouped FP64 GEMM and the owning host object.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

#include "ctn_common.h"

namespace ctn {

#ifndef F64_NARROW_BELOW
#define F64_NARROW_BELOW 6  // 64 x 32 tiles when a plan has fewer 64 x 64 tiles than this many per SM
#endif
#ifndef F64_SMALL_PADDING
#define F64_SMALL_PADDING 1.25  // 32 x 32 tiles when the wider tiles execute this many times the products of 32 x 32 tiles
#endif

struct GemmTaskD {
  int64_t c_off;
  int32_t m, n, ldc;
  int32_t pair_begin, pair_count;
  int32_t pad_;
};
struct GemmPairD {
  int64_t a_off, b_off;
  int32_t k, lda, ldb, flags;  // flags bit0: A stored [k][m]; bit1: B stored [n][k]
};
struct GemmTileD {
  int32_t task;
  int32_t m0, n0;
};

void build_tiles_f64(const std::vector<GemmTaskD> &tasks, const std::vector<GemmPairD> &pairs,
                     std::vector<GemmTileD> &tiles, int bm, int bn);
ctn_status launch_gemm_f64(const double *A, const double *B, double *C, const GemmTaskD *d_tasks,
                           const GemmPairD *d_pairs, const GemmTileD *d_tiles, int64_t ntiles, int flags,
                           int bm, int bn, cudaStream_t st);

// Host tables + their device copy (uploaded once, on the first launch on a device).
struct GroupedGemmF64 {
  std::vector<GemmTaskD> tasks;
  std::vector<GemmPairD> pairs;
  std::vector<GemmTileD> tiles;
  void *d_mem = nullptr;
  int d_dev = -1;
  double flops = 0.0;
  int flags = 0;          // operand orientation shared by every pair of the plan
  int bm = 64, bn = 64;   // tile: 64 x 64; 64 x 32 when 64 x 64 would not fill the SMs; 32 x 32 for small blocks
  bool mixed = false;     // pairs disagree on the orientation (rejected at run time)

  // products the tiles execute, with K padded to the 16-deep stages
  double executed(int tm, int tn) const {
    double w = 0.0;
    for (const auto &t : tasks) {
      double kp = 0.0;
      for (int p = 0; p < t.pair_count; ++p) kp += (double)((std::max(0, pairs[t.pair_begin + p].k) + 15) / 16 * 16);
      w += (double)((t.m + tm - 1) / tm) * tm * (double)((t.n + tn - 1) / tn) * tn * kp;
    }
    return w;
  }
  void finalize() {
    // fewer than six 64 x 64 tiles per SM (148 SMs; about 1.5 waves of four resident CTAs):
    // 64 x 32 tiles, twice as many CTAs, less padding on narrow groups and a fuller last wave;
    // blocks so small that these tiles execute F64_SMALL_PADDING times the products of 32 x 32
    // tiles (D ~ 1000 two-site problems: sectors of 2-68 states): 32 x 32 tiles
    bm = 64;
    bn = 64;
    build_tiles_f64(tasks, pairs, tiles, bm, bn);
    if (tiles.size() < F64_NARROW_BELOW * 148) bn = 32;
    if (executed(bm, bn) > F64_SMALL_PADDING * executed(32, 32)) bm = bn = 32;
    if (bm != 64 || bn != 64) build_tiles_f64(tasks, pairs, tiles, bm, bn);
    flags = pairs.empty() ? 0 : (pairs[0].flags & 3);
    mixed = false;
    for (const auto &p : pairs) mixed |= ((p.flags & 3) != flags);
    flops = 0.0;
    for (const auto &t : tasks)
      for (int p = 0; p < t.pair_count; ++p)
        flops += 2.0 * t.m * (double)t.n * (double)pairs[t.pair_begin + p].k;
  }
  size_t table_bytes() const {
    return tasks.size() * sizeof(GemmTaskD) + pairs.size() * sizeof(GemmPairD) +
           tiles.size() * sizeof(GemmTileD) + 64;
  }
  ctn_status upload(cudaStream_t st) {
    int dev = 0;
    CTN_CUDA(cudaGetDevice(&dev));
    if (d_mem && d_dev == dev) return CTN_OK;
    if (d_mem) {
      cudaFree(d_mem);
      d_mem = nullptr;
    }
    CTN_CUDA(cudaMalloc(&d_mem, table_bytes()));
    d_dev = dev;
    char *p = (char *)d_mem;
    if (!tasks.empty()) CTN_CUDA(cudaMemcpyAsync(p, tasks.data(), tasks.size() * sizeof(GemmTaskD), cudaMemcpyHostToDevice, st));
    p += tasks.size() * sizeof(GemmTaskD);
    if (!pairs.empty()) CTN_CUDA(cudaMemcpyAsync(p, pairs.data(), pairs.size() * sizeof(GemmPairD), cudaMemcpyHostToDevice, st));
    p += pairs.size() * sizeof(GemmPairD);
    if (!tiles.empty()) CTN_CUDA(cudaMemcpyAsync(p, tiles.data(), tiles.size() * sizeof(GemmTileD), cudaMemcpyHostToDevice, st));
    // pageable host memory: make sure the copies finished before the vectors can change
    CTN_CUDA(cudaStreamSynchronize(st));
    return CTN_OK;
  }
  ctn_status run(const double *A, const double *B, double *C, cudaStream_t st) {
    if (mixed) {
      set_error("grouped GEMM: all pairs of one plan must share the operand orientation flags");
      return CTN_ERR_UNSUPPORTED;
    }
    CTN_TRY(upload(st));
    const char *p = (const char *)d_mem;
    const GemmTaskD *dt = (const GemmTaskD *)p;
    const GemmPairD *dp = (const GemmPairD *)(p + tasks.size() * sizeof(GemmTaskD));
    const GemmTileD *dl = (const GemmTileD *)(p + tasks.size() * sizeof(GemmTaskD) + pairs.size() * sizeof(GemmPairD));
    return launch_gemm_f64(A, B, C, dt, dp, dl, (int64_t)tiles.size(), flags, bm, bn, st);
  }
  ~GroupedGemmF64() {
    if (d_mem) cudaFree(d_mem);
  }
};

}  // namespace ctn
