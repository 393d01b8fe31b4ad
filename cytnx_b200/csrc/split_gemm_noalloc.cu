// Allocation-free form of the dense split-precision GEMM (ctn_split_gemm_f64).
//
// Some programs that call this library cannot let it allocate device memory: hosts
// that hand the whole GPU to their own pool allocator at start-up and forbid side
// allocations by plugins, codes that run under a fixed device-memory budget where a
// hidden cudaMalloc could fail mid-run, and foreign-language callers (Fortran/C DMRG
// drivers binding the C ABI) that have no device allocator to offer for a workspace.
// For them this entry point keeps all of its scratch -- the hi/lo operand panels, the
// task tables and the kernel's error word -- in one file-scope __device__ array of a
// fixed size, and calls no cudaMalloc, cudaFree or other allocating routine.
//
// Properties callers must know:
//  * the array holds kNoAllocScratchBytes (32 MiB) on every GPU that loads the
//    library, from module load until process exit;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current); make that first
//    call before any stream capture on that device.  The address is kept for the
//    process: a device reset (cudaDeviceReset) or a new primary context on that device
//    is not supported afterwards;
//  * every call on a device uses the same array and leaves its contents behind; the call
//    clears the regions that must start at zero itself.  Calls whose work overlaps on
//    the GPU (different streams, or host threads without ordering) race on the array:
//    serialise them;
//  * problems whose scratch exceeds the array are rejected with CTN_ERR_INVALID before
//    any GPU work is issued.
#include <cstring>
#include <mutex>
#include <vector>

#include "ctn_common.h"
#include "tc_gemm.cuh"

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_split_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_scratch_mu;
void *g_scratch_addr[64] = {nullptr};

// device address of g_split_scratch on the current device (looked up once per device)
ctn_status scratch_address(uint8_t **out) {
  int dev = 0;
  CTN_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    ctn::set_error("ctn_split_gemm_f64_noalloc: device ordinal %d out of range", dev);
    return CTN_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_split_scratch);
    if (e != cudaSuccess || p == nullptr)
      return ctn::cuda_fail(e == cudaSuccess ? cudaErrorInvalidSymbol : e, "cudaGetSymbolAddress(g_split_scratch)",
                            __FILE__, __LINE__);
    g_scratch_addr[dev] = p;
  }
  *out = (uint8_t *)g_scratch_addr[dev];
  return CTN_OK;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

extern "C" ctn_status ctn_split_gemm_f64_noalloc(int64_t M, int64_t N, int64_t K, const double *A, const double *B,
                                                 double *C, int precision, void *stream) {
  CTN_REQUIRE(M > 0 && N > 0 && K > 0 && A && B && C, "ctn_split_gemm_f64_noalloc: bad argument");
  CTN_REQUIRE(precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3,
              "ctn_split_gemm_f64_noalloc: precision must be CTN_PREC_3XTF32 or CTN_PREC_BF16X3");
  CTN_REQUIRE(M < (1 << 30) && N < (1 << 30) && K < (1 << 30), "ctn_split_gemm_f64_noalloc: dimension too large");
  const int kind = precision == CTN_PREC_BF16X3 ? ctn::TC_BF16 : ctn::TC_TF32;
  const int bn = 128;
  const int64_t ks = ctn::tc_k_per_slice(kind);
  const int64_t kb = (K + ks - 1) / ks, mt = (M + ctn::TC_BM - 1) / ctn::TC_BM, nt = (N + bn - 1) / bn;
  const size_t a_bytes = (size_t)(mt * kb) * 2 * ctn::TC_A_TILE;         // hi and lo tiles interleaved
  const size_t b_bytes = (size_t)(nt * kb) * 2 * bn * ctn::TC_ROW_BYTES;
  // scratch layout: [A panel][B panel][err][group][tiles][rowmap][pack segs][pack prefixes]
  size_t o = 0;
  const size_t o_a = o;
  o += a_bytes;
  const size_t o_b = o;
  o += b_bytes;
  const size_t o_err = o;
  o = align_up(o + 256, 256);
  const size_t o_grp = o;
  o = align_up(o + sizeof(ctn::TcGroup), 256);
  const size_t o_tiles = o;
  o = align_up(o + (size_t)(mt * nt) * sizeof(ctn::TcTile), 256);
  const size_t o_rows = o;
  o = align_up(o + (size_t)M * sizeof(int64_t), 256);
  const size_t o_segs = o;
  o = align_up(o + 2 * sizeof(ctn::PackSeg), 256);
  const size_t o_begin = o;
  o = align_up(o + 4 * sizeof(int64_t), 256);
  if (o > kNoAllocScratchBytes) {
    ctn::set_error(
        "ctn_split_gemm_f64_noalloc: M=%lld N=%lld K=%lld needs %zu scratch bytes, more than the %zu-byte static "
        "device array; use ctn_split_gemm_f64 with a caller-provided workspace",
        (long long)M, (long long)N, (long long)K, o, kNoAllocScratchBytes);
    return CTN_ERR_INVALID;
  }
  uint8_t *S = nullptr;
  CTN_TRY(scratch_address(&S));
  cudaStream_t st = ctn::as_stream(stream);

  // host copies of the tables (same layout ctn_split_gemm_f64 builds)
  ctn::TcGroup g{};
  g.a_off = 0;
  g.b_off = 0;
  g.M = (int32_t)M;
  g.N = (int32_t)N;
  g.K = (int32_t)K;
  g.mt = (int32_t)mt;
  g.nt = (int32_t)nt;
  g.kb = (int32_t)kb;
  g.mode = 1;
  g.ldc = (int32_t)N;
  g.c_off = 0;
  g.rm_off = 0;
  std::vector<ctn::TcTile> tiles;
  tiles.reserve(mt * nt);
  for (int32_t m = 0; m < mt; ++m)
    for (int32_t n = 0; n < nt; ++n) tiles.push_back(ctn::TcTile{0, m, n, 0});
  std::vector<int64_t> rowmap(M);
  for (int64_t r = 0; r < M; ++r) rowmap[r] = r * N;
  const ctn::PackSeg segs[2] = {
      {0, K, 1, (int32_t)M, (int32_t)K, 0, 0, 0, ctn::TC_BM, (int32_t)kb},  // A[M][K]
      {0, 1, N, (int32_t)N, (int32_t)K, 0, 0, 0, bn, (int32_t)kb}};         // B^T rows = n, k stride N
  const int64_t E = kind == ctn::TC_TF32 ? 4 : 8;
  const int64_t ca = ((K + E - 1) / E) * M, cb = ((K + E - 1) / E) * N;
  const int64_t begin[4] = {0, ca, 0, cb};

  // what must start at zero: operand panels (padding) and the error word
  CTN_CUDA(cudaMemsetAsync(S, 0, o_err + 256, st));
  CTN_CUDA(cudaMemcpyAsync(S + o_grp, &g, sizeof(g), cudaMemcpyHostToDevice, st));
  CTN_CUDA(cudaMemcpyAsync(S + o_tiles, tiles.data(), tiles.size() * sizeof(ctn::TcTile), cudaMemcpyHostToDevice, st));
  CTN_CUDA(cudaMemcpyAsync(S + o_rows, rowmap.data(), rowmap.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  CTN_CUDA(cudaMemcpyAsync(S + o_segs, segs, sizeof(segs), cudaMemcpyHostToDevice, st));
  CTN_CUDA(cudaMemcpyAsync(S + o_begin, begin, sizeof(begin), cudaMemcpyHostToDevice, st));
  const ctn::PackSeg *dsegs = (const ctn::PackSeg *)(S + o_segs);
  const int64_t *dbeg = (const int64_t *)(S + o_begin);
  CTN_TRY(ctn::pack_launch_tables(kind, dsegs, dbeg, 1, ca, A, 0, S + o_a, ctn::TC_BM, st));
  CTN_TRY(ctn::pack_launch_tables(kind, dsegs + 1, dbeg + 2, 1, cb, B, 0, S + o_b, bn, st));
  int *err = (int *)(S + o_err);
  CTN_TRY(ctn::tc_launch_tables(kind, bn, (const ctn::TcGroup *)(S + o_grp), (const ctn::TcTile *)(S + o_tiles),
                                (int64_t)tiles.size(), (const int64_t *)(S + o_rows), S + o_a, S + o_b, nullptr, C,
                                err, st));
  int herr = 0;
  CTN_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  if (herr) {
    ctn::set_error("ctn_split_gemm_f64_noalloc: a bounded wait in the tcgen05 kernel expired (code %d)", herr);
    return CTN_ERR_TIMEOUT;
  }
  return CTN_OK;
}
