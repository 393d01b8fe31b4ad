// Tensor permute (materialisation of a lazy permutation) for sm_100a.
//
// Semantics of the reference (src/backend/utils_internal_cpu/Movemem_cpu.cpp:152-191,
// src/backend/utils_internal_gpu/cuMovemem_gpu.cu:60-94): for a row-major tensor of
// old_shape, out has new_shape[i] = old_shape[mapper[i]] and
// out[sum_i new_stride[i] * idx_old[mapper[i]]] = in[idx_old].  Pure data movement,
// bit-exact for every dtype.
//
// B200 design: the permutation is first reduced (size-1 axes dropped, axes that stay
// adjacent merged), then one of two kernels runs:
//  * the innermost axis is preserved -> a row-gather copy in 16-byte vectors where the
//    row length and pointers allow (every warp reads and writes whole contiguous runs);
//  * otherwise a 32x32-element shared-memory tiled transpose between the input's
//    fastest axis and the output's fastest axis, so both the HBM reads and the HBM
//    writes are coalesced; all remaining axes are batch axes decomposed per tile.
// No per-call allocation or host<->device copy of stride vectors: the reduced
// geometry travels as kernel parameters (the reference mallocs and copies two
// stride arrays per call, cuMovemem_gpu.cu:139-152).
#include <algorithm>
#include <cstring>
#include <vector>

#include "ctn_common.h"

namespace ctn {

constexpr int kMaxRank = 16;

struct PermGeom {
  int rank;                   // reduced rank (>= 2 here)
  int64_t n;                  // total elements
  int64_t out_shape[kMaxRank];    // new shape (reduced)
  int64_t in_stride_of_out[kMaxRank];  // input stride of the old axis at new position i
};

struct alignas(16) U128 {
  uint64_t a, b;
};

template <int N>
struct VecT;
template <>
struct VecT<1> { using T = uint8_t; };
template <>
struct VecT<2> { using T = uint16_t; };
template <>
struct VecT<4> { using T = uint32_t; };
template <>
struct VecT<8> { using T = uint64_t; };
template <>
struct VecT<16> { using T = U128; };

// ---------------------------------------------------------------- row gather
// The last new axis equals the last old axis.  Each "unit" is V bytes; the row of
// the innermost axis holds row_units units.  For out unit u: row = u / row_units,
// col = u % row_units; the row's input offset comes from decomposing `row` over
// the new axes 0..rank-2.
template <typename U>
__global__ void __launch_bounds__(256) k_row_gather(const U *__restrict__ src, U *__restrict__ dst,
                                                    PermGeom g, int64_t row_units,
                                                    int64_t total_units, int64_t in_row_stride_units_scale) {
  int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * blockDim.x;
  for (; u < total_units; u += step) {
    int64_t row = u / row_units;
    int64_t col = u - row * row_units;
    int64_t off = 0;  // input element offset of the row start
    int64_t r = row;
    for (int i = g.rank - 2; i >= 0; --i) {
      int64_t d = g.out_shape[i];
      int64_t q = r / d;
      off += (r - q * d) * g.in_stride_of_out[i];
      r = q;
    }
    dst[u] = src[off / in_row_stride_units_scale + col];
  }
}

// ---------------------------------------------------------------- tiled transpose
// Input fastest axis "a" (new position pa), output fastest axis "b" (old axis with
// input stride sb).  Tile: 32 (b) x 32 (a) elements; block 32 x 8 threads.
struct TransGeom {
  int nbatch_dims;
  int64_t na, nb;           // sizes of axes a and b
  int64_t out_stride_a;     // output stride of axis a
  int64_t in_stride_b;      // input stride of axis b
  int64_t tiles_a, tiles_b; // tile counts
  int64_t batch;            // number of batch points
  int64_t bshape[kMaxRank]; // batch axes (new order, row-major over them)
  int64_t bin[kMaxRank];    // their input strides
  int64_t bout[kMaxRank];   // their output strides
};

template <typename T>
__global__ void __launch_bounds__(256) k_transpose(const T *__restrict__ src, T *__restrict__ dst,
                                                   TransGeom g) {
  __shared__ T tile[32][33];
  const int64_t ntile = g.tiles_a * g.tiles_b;
  const int64_t total = ntile * g.batch;
  for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
    int64_t bidx = t / ntile;
    int64_t tt = t - bidx * ntile;
    int64_t tb = tt / g.tiles_a;
    int64_t ta = tt - tb * g.tiles_a;
    int64_t in_off = 0, out_off = 0;
    int64_t r = bidx;
    for (int i = g.nbatch_dims - 1; i >= 0; --i) {
      int64_t d = g.bshape[i];
      int64_t q = r / d;
      int64_t c = r - q * d;
      in_off += c * g.bin[i];
      out_off += c * g.bout[i];
      r = q;
    }
    const int64_t a0 = ta * 32, b0 = tb * 32;
    // read: rows of b, contiguous along a
    const int64_t ia = a0 + threadIdx.x;
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
      int64_t ib = b0 + threadIdx.y + j;
      if (ia < g.na && ib < g.nb) tile[threadIdx.y + j][threadIdx.x] = src[in_off + ib * g.in_stride_b + ia];
    }
    __syncthreads();
    // write: rows of a, contiguous along b
    const int64_t ob = b0 + threadIdx.x;
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
      int64_t oa = a0 + threadIdx.y + j;
      if (oa < g.na && ob < g.nb) dst[out_off + oa * g.out_stride_a + ob] = tile[threadIdx.x][threadIdx.y + j];
    }
    __syncthreads();
  }
}

static int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Reduce (drop size-1 axes, merge axes that stay adjacent).  Returns reduced rank.
static int reduce_perm(int rank, const uint64_t *old_shape, const uint64_t *mapper, int64_t *rshape,
                       int *rmap) {
  // keep old axes with extent > 1
  int keep_idx[kMaxRank];
  int nk = 0;
  int old_to_k[kMaxRank];
  for (int j = 0; j < rank; ++j) {
    old_to_k[j] = -1;
    if (old_shape[j] != 1) {
      old_to_k[j] = nk;
      keep_idx[nk++] = j;
    }
  }
  int64_t kshape[kMaxRank];
  for (int k = 0; k < nk; ++k) kshape[k] = (int64_t)old_shape[keep_idx[k]];
  int kmap[kMaxRank];
  int nm = 0;
  for (int i = 0; i < rank; ++i)
    if (old_to_k[mapper[i]] >= 0) kmap[nm++] = old_to_k[mapper[i]];
  // merge: old axes k and k+1 merge if k+1 immediately follows k in the new order
  int group_of[kMaxRank];
  int ng = 0;
  int64_t gshape[kMaxRank];
  for (int k = 0; k < nk; ++k) {
    bool merge = false;
    if (k > 0) {
      for (int i = 0; i + 1 < nm; ++i)
        if (kmap[i] == k - 1 && kmap[i + 1] == k) merge = true;
    }
    if (merge) {
      group_of[k] = ng - 1;
      gshape[ng - 1] *= kshape[k];
    } else {
      group_of[k] = ng;
      gshape[ng++] = kshape[k];
    }
  }
  int r = 0;
  for (int i = 0; i < nm; ++i) {
    int g = group_of[kmap[i]];
    if (r == 0 || rmap[r - 1] != g) rmap[r++] = g;
  }
  for (int g = 0; g < ng; ++g) rshape[g] = gshape[g];
  return ng;
}

template <int ES>
static ctn_status launch_perm(const void *src, void *dst, int rank, const uint64_t *old_shape,
                              const uint64_t *mapper, cudaStream_t st) {
  using T = typename VecT<ES>::T;
  int64_t n = 1;
  for (int i = 0; i < rank; ++i) n *= (int64_t)old_shape[i];
  if (n == 0) return CTN_OK;
  int64_t rshape[kMaxRank];
  int rmap[kMaxRank];
  int r = reduce_perm(rank, old_shape, mapper, rshape, rmap);
  bool ident = true;
  for (int i = 0; i < r; ++i) ident &= (rmap[i] == i);
  if (r <= 1 || ident) {
    CTN_CUDA(cudaMemcpyAsync(dst, src, (size_t)n * ES, cudaMemcpyDeviceToDevice, st));
    return CTN_OK;
  }
  int64_t in_stride[kMaxRank];
  int64_t acc = 1;
  for (int j = r - 1; j >= 0; --j) {
    in_stride[j] = acc;
    acc *= rshape[j];
  }
  int64_t out_shape[kMaxRank], out_stride[kMaxRank];
  for (int i = 0; i < r; ++i) out_shape[i] = rshape[rmap[i]];
  acc = 1;
  for (int i = r - 1; i >= 0; --i) {
    out_stride[i] = acc;
    acc *= out_shape[i];
  }
  const int nsm = sm_count();
  if (rmap[r - 1] == r - 1) {
    PermGeom g;
    g.rank = r;
    g.n = n;
    for (int i = 0; i < r; ++i) {
      g.out_shape[i] = out_shape[i];
      g.in_stride_of_out[i] = in_stride[rmap[i]];
    }
    const int64_t L = rshape[r - 1];
    const int64_t bytes_row = L * ES;
    const uintptr_t al = reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst);
    int vb = ES;  // unit bytes
    for (int cand = 16; cand > ES; cand /= 2)
      if (bytes_row % cand == 0 && al % cand == 0) {
        vb = cand;
        break;
      }
    const int64_t scale = vb / ES;  // elements per unit
    const int64_t row_units = L / scale;
    const int64_t total_units = n / scale;
    const int64_t blocks = std::min<int64_t>((total_units + 255) / 256, (int64_t)nsm * 16);
    switch (vb) {
      case 16:
        k_row_gather<U128><<<(unsigned)blocks, 256, 0, st>>>((const U128 *)src, (U128 *)dst, g, row_units, total_units, scale);
        break;
      case 8:
        k_row_gather<uint64_t><<<(unsigned)blocks, 256, 0, st>>>((const uint64_t *)src, (uint64_t *)dst, g, row_units, total_units, scale);
        break;
      case 4:
        k_row_gather<uint32_t><<<(unsigned)blocks, 256, 0, st>>>((const uint32_t *)src, (uint32_t *)dst, g, row_units, total_units, scale);
        break;
      case 2:
        k_row_gather<uint16_t><<<(unsigned)blocks, 256, 0, st>>>((const uint16_t *)src, (uint16_t *)dst, g, row_units, total_units, scale);
        break;
      default:
        k_row_gather<uint8_t><<<(unsigned)blocks, 256, 0, st>>>((const uint8_t *)src, (uint8_t *)dst, g, row_units, total_units, scale);
    }
    CTN_CHECK_LAUNCH();
    return CTN_OK;
  }
  TransGeom g;
  const int a = r - 1;        // input fastest (old axis)
  const int b = rmap[r - 1];  // old axis that is output fastest
  int pa = 0;
  for (int i = 0; i < r; ++i)
    if (rmap[i] == a) pa = i;
  g.na = rshape[a];
  g.nb = rshape[b];
  g.out_stride_a = out_stride[pa];
  g.in_stride_b = in_stride[b];
  g.tiles_a = (g.na + 31) / 32;
  g.tiles_b = (g.nb + 31) / 32;
  g.nbatch_dims = 0;
  g.batch = 1;
  for (int i = 0; i < r; ++i) {
    const int j = rmap[i];
    if (j == a || j == b) continue;
    g.bshape[g.nbatch_dims] = rshape[j];
    g.bin[g.nbatch_dims] = in_stride[j];
    g.bout[g.nbatch_dims] = out_stride[i];
    g.nbatch_dims++;
    g.batch *= rshape[j];
  }
  const int64_t total = g.tiles_a * g.tiles_b * g.batch;
  const int64_t blocks = std::min<int64_t>(total, (int64_t)nsm * 32);
  k_transpose<T><<<(unsigned)blocks, dim3(32, 8), 0, st>>>((const T *)src, (T *)dst, g);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}

static ctn_status permute_impl(const void *src, void *dst, int dtype, int rank,
                               const uint64_t *old_shape, const uint64_t *mapper, cudaStream_t st) {
  const size_t es = ctn_dtype_size(dtype);
  CTN_REQUIRE(es != 0, "ctn_permute: unknown dtype %d", dtype);
  CTN_REQUIRE(rank >= 0 && rank <= kMaxRank, "ctn_permute: rank %d out of range", rank);
  bool seen[kMaxRank] = {false};
  for (int i = 0; i < rank; ++i) {
    CTN_REQUIRE(mapper[i] < (uint64_t)rank && !seen[mapper[i]], "ctn_permute: invalid mapper");
    seen[mapper[i]] = true;
  }
  if (rank == 0) {
    CTN_CUDA(cudaMemcpyAsync(dst, src, es, cudaMemcpyDeviceToDevice, st));
    return CTN_OK;
  }
  switch (es) {
    case 1: return launch_perm<1>(src, dst, rank, old_shape, mapper, st);
    case 2: return launch_perm<2>(src, dst, rank, old_shape, mapper, st);
    case 4: return launch_perm<4>(src, dst, rank, old_shape, mapper, st);
    case 8: return launch_perm<8>(src, dst, rank, old_shape, mapper, st);
    case 16: return launch_perm<16>(src, dst, rank, old_shape, mapper, st);
  }
  set_error("ctn_permute: unsupported element size");
  return CTN_ERR_UNSUPPORTED;
}

}  // namespace ctn

extern "C" ctn_status ctn_permute(const void *src, void *dst, int dtype, int rank,
                                  const uint64_t *old_shape, const uint64_t *mapper, void *stream) {
  return ctn::permute_impl(src, dst, dtype, rank, old_shape, mapper, ctn::as_stream(stream));
}

extern "C" ctn_status ctn_permute_blocks(const void *src, void *dst, int dtype, int rank,
                                         int64_t nblocks, const uint64_t *old_shapes,
                                         const int64_t *src_offs, const int64_t *dst_offs,
                                         const uint64_t *mapper, void *stream) {
  const size_t es = ctn_dtype_size(dtype);
  CTN_REQUIRE(es != 0, "ctn_permute_blocks: unknown dtype %d", dtype);
  for (int64_t b = 0; b < nblocks; ++b) {
    CTN_TRY(ctn::permute_impl((const char *)src + src_offs[b] * es, (char *)dst + dst_offs[b] * es,
                              dtype, rank, old_shapes + b * rank, mapper, ctn::as_stream(stream)));
  }
  return CTN_OK;
}
