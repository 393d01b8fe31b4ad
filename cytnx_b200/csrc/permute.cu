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
//  * otherwise a tiled transpose between the input's fastest axis and the output's
//    fastest axis, so both the HBM reads and the HBM writes are coalesced; all remaining
//    axes are batch axes decomposed per tile.  For 1-, 2- and 4-byte elements, when the
//    input strides allow a tensor map (16-byte multiples, at most 3 batch axes), the
//    tiles are staged by TMA: a persistent CTA double-buffers (128 bytes of the input's
//    fastest axis) x 64 tiles into shared memory with cp.async.bulk.tensor
//    (SWIZZLE_128B, so the column reads of the transpose spread over the banks) and
//    writes 16-byte vectors along the output's fastest axis.  Otherwise (8-byte
//    elements, short output axes, other strides) a 32x32-element shared-memory tile
//    kernel runs.
// No per-call allocation or host<->device copy of stride vectors: the reduced
// geometry travels as kernel parameters (the reference mallocs and copies two
// stride arrays per call, cuMovemem_gpu.cu:139-152).

#include <algorithm>
#include <cstring>
#include <vector>

#include "ctn_common.h"
#include "tmap.h"

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
// IT: index type of the decomposition (32-bit when every index fits: integer division
// is several times cheaper than in 64 bits, and it runs once per copied unit).  The input
// strides in g are in units (the host divides them exactly: every stride of an outer axis is
// a multiple of the row, which is a whole number of units).
template <typename U, typename IT>
__global__ void __launch_bounds__(256) k_row_gather(const U *__restrict__ src, U *__restrict__ dst,
                                                    PermGeom g, int64_t row_units, int64_t total_units) {
  int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t step = (int64_t)gridDim.x * blockDim.x;
  const IT ru = (IT)row_units;
  for (; u < total_units; u += step) {
    const IT uu = (IT)u;
    IT row = uu / ru;
    const IT col = uu - row * ru;
    int64_t off = 0;  // input unit offset of the row start
    for (int i = g.rank - 2; i >= 0; --i) {
      const IT d = (IT)g.out_shape[i];
      const IT q = row / d;
      off += (int64_t)(row - q * d) * g.in_stride_of_out[i];
      row = q;
    }
    dst[u] = src[off + col];
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

// IT: the integer type of the tile and batch index arithmetic (32-bit when the tile count
// and every batch axis fit, which turns the per-tile divisions from 64-bit software routines
// into 32-bit ones); element offsets stay 64-bit.
template <typename T, typename IT>
__global__ void __launch_bounds__(256) k_transpose(const T *__restrict__ src, T *__restrict__ dst,
                                                   TransGeom g) {
  __shared__ T tile[32][33];
  const IT tiles_a = (IT)g.tiles_a;
  const IT ntile = (IT)(g.tiles_a * g.tiles_b);
  const IT total = (IT)(g.tiles_a * g.tiles_b * g.batch);
  for (IT t = blockIdx.x; t < total; t += gridDim.x) {
    const IT bidx = t / ntile;
    const IT tt = t - bidx * ntile;
    const IT tb = tt / tiles_a;
    const IT ta = tt - tb * tiles_a;
    int64_t in_off = 0, out_off = 0;
    IT r = bidx;
    for (int i = g.nbatch_dims - 1; i >= 0; --i) {
      const IT d = (IT)g.bshape[i];
      const IT q = r / d;
      const IT c = r - q * d;
      in_off += (int64_t)c * g.bin[i];
      out_off += (int64_t)c * g.bout[i];
      r = q;
    }
    const int64_t a0 = (int64_t)ta * 32, b0 = (int64_t)tb * 32;
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

// Short output axis (nb < 16): one thread per (batch point, a) writes the nb consecutive
// output elements of its row, reading them at input stride in_stride_b; the reads of a
// warp are coalesced along a and the writes are contiguous runs.
template <typename T>
__global__ void __launch_bounds__(256) k_transpose_short(const T *__restrict__ src, T *__restrict__ dst, TransGeom g) {
  const int64_t rows = g.na * g.batch;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < rows; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t bidx = t / g.na;
    const int64_t ia = t - bidx * g.na;
    int64_t in_off = 0, out_off = 0;
    for (int i = g.nbatch_dims - 1; i >= 0; --i) {
      const int64_t d = g.bshape[i];
      const int64_t q = bidx / d;
      const int64_t c = bidx - q * d;
      in_off += c * g.bin[i];
      out_off += c * g.bout[i];
      bidx = q;
    }
    const T *s = src + in_off + ia;
    T *o = dst + out_off + ia * g.out_stride_a;
    T v[16];
#pragma unroll
    for (int b = 0; b < 16; ++b)
      if (b < g.nb) v[b] = s[b * g.in_stride_b];
#pragma unroll
    for (int b = 0; b < 16; ++b)
      if (b < g.nb) o[b] = v[b];
  }
}

// Short output axis (nb < 16) under a long input axis (na >= 256): a CTA stages a tile of
// TA = 256 x APT consecutive a by all nb b of one batch point in shared memory.  Reads:
// nb coalesced input rows, all APT x nb loads of a thread issued together.  Writes: when
// the output stride of a equals nb the tile is ONE contiguous output run of cnt_a x nb
// elements, written in 16-byte vectors when the run starts on a 16-byte boundary;
// otherwise the tile's runs of nb elements go out in warp-wide sweeps.  NB bounds nb at
// compile time so the staging registers stay few (occupancy carries the bytes in flight).
constexpr int STAGED_THREADS = 256;

template <typename T, int NB, int APT, typename IT>
__global__ void __launch_bounds__(STAGED_THREADS) k_transpose_staged(const T *__restrict__ src, T *__restrict__ dst,
                                                                     TransGeom g) {
  extern __shared__ __align__(16) unsigned char staged_smem[];
  T *tile = reinterpret_cast<T *>(staged_smem);
  constexpr int TA = STAGED_THREADS * APT;
  const int nb = (int)g.nb;
  const int tid = threadIdx.x;
  const IT tiles_a = (IT)((g.na + TA - 1) / TA);
  const IT total = (IT)((g.na + TA - 1) / TA * g.batch);
  for (IT t = blockIdx.x; t < total; t += gridDim.x) {
    IT bidx = t / tiles_a;
    const int64_t a0 = (int64_t)(t - bidx * tiles_a) * TA;
    int64_t in_off = 0, out_off = 0;
    for (int i = g.nbatch_dims - 1; i >= 0; --i) {
      const IT d = (IT)g.bshape[i];
      const IT q = bidx / d;
      const IT c = bidx - q * d;
      in_off += (int64_t)c * g.bin[i];
      out_off += (int64_t)c * g.bout[i];
      bidx = q;
    }
    const int cnt_a = (int)(g.na - a0 < TA ? g.na - a0 : TA);
    const T *s = src + in_off + a0;
    T v[APT][NB];
#pragma unroll
    for (int p = 0; p < APT; ++p)
#pragma unroll
      for (int b = 0; b < NB; ++b)
        if (b < nb && p * STAGED_THREADS + tid < cnt_a) v[p][b] = s[(int64_t)b * g.in_stride_b + p * STAGED_THREADS + tid];
    __syncthreads();  // the previous tile's writers are done reading the stage
#pragma unroll
    for (int p = 0; p < APT; ++p)
#pragma unroll
      for (int b = 0; b < NB; ++b)
        if (b < nb && p * STAGED_THREADS + tid < cnt_a) tile[(p * STAGED_THREADS + tid) * nb + b] = v[p][b];
    __syncthreads();
    const int cnt = cnt_a * nb;  // elements staged
    if (g.out_stride_a == nb) {
      T *o = dst + out_off + a0 * nb;
      if (sizeof(T) < 16 && (reinterpret_cast<uintptr_t>(o) & 15) == 0) {
        constexpr int V = 16 / sizeof(T);
        const int nv = cnt / V;
        const uint4 *s4 = reinterpret_cast<const uint4 *>(tile);
        uint4 *o4 = reinterpret_cast<uint4 *>(o);
        for (int i = tid; i < nv; i += STAGED_THREADS) o4[i] = s4[i];
        for (int i = nv * V + tid; i < cnt; i += STAGED_THREADS) o[i] = tile[i];
      } else {
        for (int i = tid; i < cnt; i += STAGED_THREADS) o[i] = tile[i];
      }
    } else {
      for (int i = tid; i < cnt; i += STAGED_THREADS) {
        const int a = i / nb, b = i - a * nb;
        dst[out_off + (a0 + a) * g.out_stride_a + b] = tile[i];
      }
    }
  }
}

// Launches k_transpose_staged when the geometry suits it (na >= 256, nb < 16, the stage
// within 48 KB); returns false otherwise.
template <typename T, int NB>
static bool launch_staged_nb(const void *src, void *dst, const TransGeom &g, int nsm, cudaStream_t st) {
  int apt = NB <= 8 ? 2 : 1;
  if ((size_t)STAGED_THREADS * apt * g.nb * sizeof(T) > 48 * 1024) apt = 1;
  const size_t smem = (size_t)STAGED_THREADS * apt * g.nb * sizeof(T);
  if (smem > 48 * 1024) return false;
  const int64_t ta = (int64_t)STAGED_THREADS * apt;
  const int64_t total = (g.na + ta - 1) / ta * g.batch;
  const int64_t blocks = std::min<int64_t>(total, (int64_t)nsm * 64);
  const bool narrow = total + blocks < ((int64_t)1 << 32);  // 32-bit tile arithmetic
  if (apt == 2 && narrow)
    k_transpose_staged<T, NB, 2, uint32_t><<<(unsigned)blocks, STAGED_THREADS, smem, st>>>((const T *)src, (T *)dst, g);
  else if (apt == 2)
    k_transpose_staged<T, NB, 2, int64_t><<<(unsigned)blocks, STAGED_THREADS, smem, st>>>((const T *)src, (T *)dst, g);
  else if (narrow)
    k_transpose_staged<T, NB, 1, uint32_t><<<(unsigned)blocks, STAGED_THREADS, smem, st>>>((const T *)src, (T *)dst, g);
  else
    k_transpose_staged<T, NB, 1, int64_t><<<(unsigned)blocks, STAGED_THREADS, smem, st>>>((const T *)src, (T *)dst, g);
  return true;
}

template <typename T>
static bool launch_staged(const void *src, void *dst, const TransGeom &g, int nsm, cudaStream_t st) {
  if (g.na < STAGED_THREADS || g.nb >= 16 || g.nb < 2) return false;
  if (g.nb <= 2) return launch_staged_nb<T, 2>(src, dst, g, nsm, st);
  if (g.nb <= 4) return launch_staged_nb<T, 4>(src, dst, g, nsm, st);
  if (g.nb <= 8) return launch_staged_nb<T, 8>(src, dst, g, nsm, st);
  return launch_staged_nb<T, 16>(src, dst, g, nsm, st);
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

// ---------------------------------------------------------------- TMA-staged transpose
// Tile: TA = 128 / ES elements of axis a (one 128-byte swizzle row) x TB = tma_tb(ES) of axis b.
// The tensor map views the input as [batch2][batch1][batch0][b][a] (a fastest); the
// shared-memory image of a box row b is 128 bytes whose 16-byte chunks are XOR-swizzled
// with (b & 7).  The 256 threads write the tile as 16-byte output vectors (16 / ES
// consecutive b of one a), TA * TB * ES / 4096 of them each.
// b rows per staged tile: 128 for 1- and 2-byte elements (16 KB tiles; int16 4.37 -> 4.83 TB/s
// against 64 rows), 64 for 4-byte ones (128 rows: f32 4.56 -> 4.30 TB/s)
constexpr int tma_tb(int es) { return es <= 2 ? 128 : 64; }
constexpr int TMA_THREADS = 256;
constexpr long long TMA_SPIN = 1ll << 26;  // mbarrier probes before giving up

struct TmaGeom {
  int64_t na, nb;
  int64_t tiles_a, tiles_b, batch;
  int nbatch;
  int64_t bshape[3];  // batch extents (tensor-map order: innermost first)
  int64_t bout[3];    // their output strides (elements)
  int64_t out_stride_a;
  int *err;
};

__device__ __forceinline__ uint32_t smem32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// rotate a 128-bit value (little-endian words) left by `bits` (0..127)
__device__ __forceinline__ uint4 rotl128(uint4 x, int bits) {
  const int w = bits >> 5, s = bits & 31;
  if (w & 2) {
    uint32_t t = x.x; x.x = x.z; x.z = t;
    t = x.y; x.y = x.w; x.w = t;
  }
  if (w & 1) {
    const uint32_t t = x.w;
    x.w = x.z; x.z = x.y; x.y = x.x; x.x = t;
  }
  uint4 y;
  y.x = __funnelshift_l(x.w, x.x, s);
  y.y = __funnelshift_l(x.x, x.y, s);
  y.z = __funnelshift_l(x.y, x.z, s);
  y.w = __funnelshift_l(x.z, x.w, s);
  return y;
}

// IT: integer type of the tile and batch index arithmetic (32-bit when it fits)
template <int ES, typename IT>
__global__ void __launch_bounds__(TMA_THREADS) k_transpose_tma(const __grid_constant__ CUtensorMap in_map,
                                                              uint8_t *__restrict__ dst, TmaGeom g) {
  constexpr int TA = 128 / ES;
  constexpr int TMA_TB = tma_tb(ES);
  constexpr int TILE = TMA_TB * 128;                   // bytes per staged tile
  constexpr int VEC = 16 / ES;                         // elements per output vector
  constexpr int CHUNKS = TMA_TB / VEC;                 // output vectors per a (along b)
  constexpr int AROWS = TMA_THREADS / CHUNKS;          // a rows written per pass
  __shared__ __align__(1024) uint8_t buf[2][TILE];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int stop;
  const IT tiles_a = (IT)g.tiles_a;
  const IT ntile = (IT)(g.tiles_a * g.tiles_b);
  const IT total = (IT)(g.tiles_a * g.tiles_b * g.batch);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem32(&bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem32(&bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    stop = 0;
  }
  __syncthreads();
  struct C5 {
    int x0, x1, x2, x3, x4;
  };
  auto coords = [&](IT t) -> C5 {
    IT bidx = t / ntile;
    const IT tt = t - bidx * ntile;
    const IT tb = tt / tiles_a, ta = tt - tb * tiles_a;
    C5 c{(int)(ta * TA), (int)(tb * TMA_TB), 0, 0, 0};
    if (g.nbatch > 0) {
      const IT d = (IT)g.bshape[0];
      const IT q = bidx / d;
      c.x2 = (int)(bidx - q * d);
      bidx = q;
    }
    if (g.nbatch > 1) {
      const IT d = (IT)g.bshape[1];
      const IT q = bidx / d;
      c.x3 = (int)(bidx - q * d);
      bidx = q;
    }
    if (g.nbatch > 2) c.x4 = (int)bidx;
    return c;
  };
  auto issue = [&](IT t, int slot) {
    const C5 c = coords(t);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem32(&bar[slot])), "r"(TILE)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];" ::"r"(smem32(buf[slot])),
        "l"(reinterpret_cast<uint64_t>(&in_map)), "r"(c.x0), "r"(c.x1), "r"(c.x2), "r"(c.x3), "r"(c.x4),
        "r"(smem32(&bar[slot]))
        : "memory");
  };
  IT t = blockIdx.x;
  if (threadIdx.x == 0 && t < total) issue(t, 0);
  uint32_t phase[2] = {0, 0};
  for (int i = 0; t < total; ++i, t += gridDim.x) {
    const int slot = i & 1;
    const IT tn = t + gridDim.x;
    if (threadIdx.x == 0) {
      if (tn < total) issue(tn, slot ^ 1);  // that buffer was released by the last __syncthreads
      bool ok = false;
      for (long long k = 0; k < TMA_SPIN && !ok; ++k) {
        uint32_t r;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(r)
            : "r"(smem32(&bar[slot])), "r"(phase[slot])
            : "memory");
        ok = r != 0;
      }
      if (!ok) {
        atomicCAS(g.err, 0, 1);
        stop = 1;
      }
    }
    __syncthreads();
    if (stop) break;
    phase[slot] ^= 1;
    const C5 c = coords(t);
    int64_t out_base = 0;
    if (g.nbatch > 0) out_base += (int64_t)c.x2 * g.bout[0];
    if (g.nbatch > 1) out_base += (int64_t)c.x3 * g.bout[1];
    if (g.nbatch > 2) out_base += (int64_t)c.x4 * g.bout[2];
    const uint8_t *tile = buf[slot];
    // A warp covers CW output vectors (along b) of 32 / CW a rows.  Staged row bl sits at
    // bl * 128 bytes with its 16-byte chunks XOR-swizzled by (bl & 7), so the rows that the
    // CW lanes of one a row read at step e must differ in (bl & 7) to reach different
    // banks: lane ch reads its VEC rows in an order rotated by `rot` and the assembled
    // vector is rotated back in registers.  Every staged load of the warp is then one
    // shared-memory wavefront (8 distinct chunks, or lanes sharing a 32-bit word).
    constexpr int CW = CHUNKS < 8 ? CHUNKS : 8;   // output vectors per a row within a warp
    constexpr int WG = CHUNKS / CW;               // warps per a row
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ch_lo = lane % CW;
    const int ch = (warp % WG) * CW + ch_lo, ar = (warp / WG) * (32 / CW) + lane / CW;
    const int rot = VEC >= 8 ? (ch_lo * (8 / CW)) & (VEC - 1) : (ch_lo >> 1) & (VEC - 1);
#pragma unroll
    for (int a_off = 0; a_off < TA; a_off += AROWS) {
      const int al = a_off + ar;  // local a
      const int64_t ag = c.x0 + al, bg0 = c.x1 + ch * VEC;
      if (al >= TA || ag >= g.na || bg0 >= g.nb) continue;
      using T = typename VecT<ES>::T;
      union {
        T e[VEC];
        uint4 q;
      } v;
      const int byte = al * ES;
#pragma unroll
      for (int e = 0; e < VEC; ++e) {
        const int bl = ch * VEC + ((e + rot) & (VEC - 1));  // local b = staged row
        const int sw = (((byte >> 4) ^ (bl & 7)) << 4) | (byte & 15);
        v.e[e] = *reinterpret_cast<const T *>(tile + bl * 128 + sw);
      }
      v.q = rotl128(v.q, rot * ES * 8);  // element j of the vector is staged row ch * VEC + j
      T *o = reinterpret_cast<T *>(dst) + (out_base + ag * g.out_stride_a + bg0);
      const int nvalid = g.nb - bg0 < VEC ? (int)(g.nb - bg0) : VEC;
      if (nvalid == VEC && ((reinterpret_cast<uintptr_t>(o) & 15) == 0)) {
        *reinterpret_cast<uint4 *>(o) = v.q;
      } else {
        for (int e = 0; e < nvalid; ++e) o[e] = v.e[e];
      }
    }
    __syncthreads();  // this buffer may be refilled
  }
  // an early stop may leave the prefetched tile in flight: wait for it (bounded)
  if (threadIdx.x == 0 && stop) {
    for (int s2 = 0; s2 < 2; ++s2)
      for (long long k = 0; k < TMA_SPIN; ++k) {
        uint32_t r;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(r)
            : "r"(smem32(&bar[s2])), "r"(phase[s2])
            : "memory");
        if (r) break;
      }
  }
}

static int *tma_err_word() {
  static int *w = nullptr;
  static int dev_of = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (!w || dev_of != dev) {
    if (cudaMalloc(&w, sizeof(int)) != cudaSuccess) return nullptr;
    cudaMemset(w, 0, sizeof(int));
    dev_of = dev;
  }
  return w;
}

// TMA path for the transpose case; returns false (nothing launched) when the geometry
// does not fit a tensor map
template <int ES>
static bool try_transpose_tma(const void *src, void *dst, int r, const int64_t *rshape, const int *rmap,
                              const int64_t *in_stride, const int64_t *out_stride, cudaStream_t st, ctn_status *res) {
  constexpr int TA = 128 / ES;
  constexpr int TMA_TB = tma_tb(ES);
  const int a = r - 1, b = rmap[r - 1];
  if (r - 2 > 3) return false;
  int64_t nel = 1;
  for (int i = 0; i < r; ++i) nel *= rshape[i];
  if (nel * ES < (1 << 20)) return false;  // small tensors: the plain tile kernel (no tensor map to encode)
  if ((reinterpret_cast<uintptr_t>(src) & 15) != 0) return false;
  int pa = 0;
  for (int i = 0; i < r; ++i)
    if (rmap[i] == a) pa = i;
  TmaGeom g;
  g.na = rshape[a];
  g.nb = rshape[b];
  g.out_stride_a = out_stride[pa];
  g.tiles_a = (g.na + TA - 1) / TA;
  g.tiles_b = (g.nb + TMA_TB - 1) / TMA_TB;
  g.nbatch = 0;
  g.batch = 1;
  cuuint64_t dims[5] = {1, 1, 1, 1, 1}, strides[4] = {0, 0, 0, 0};
  dims[0] = (cuuint64_t)g.na;
  dims[1] = (cuuint64_t)g.nb;
  strides[0] = (cuuint64_t)(in_stride[b] * ES);
  for (int i = r - 1; i >= 0; --i) {  // batch axes, innermost output axis first
    const int j = rmap[i];
    if (j == a || j == b) continue;
    dims[2 + g.nbatch] = (cuuint64_t)rshape[j];
    strides[1 + g.nbatch] = (cuuint64_t)(in_stride[j] * ES);
    g.bshape[g.nbatch] = rshape[j];
    g.bout[g.nbatch] = out_stride[i];
    g.nbatch++;
    g.batch *= rshape[j];
  }
  for (int i = 0; i < 1 + g.nbatch; ++i)
    if (strides[i] % 16 != 0 || strides[i] >= (1ull << 40)) return false;
  for (int i = 1 + g.nbatch; i < 4; ++i) strides[i] = strides[g.nbatch] * (cuuint64_t)dims[1 + g.nbatch];
  for (int i = 0; i < 5; ++i)
    if (dims[i] > (1ull << 31)) return false;
  if (g.tiles_a * g.tiles_b * g.batch > (1ll << 40)) return false;
  g.err = tma_err_word();
  if (!g.err) return false;
  CUtensorMap map;
  const cuuint32_t box[5] = {(cuuint32_t)TA, (cuuint32_t)TMA_TB, 1, 1, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUtensorMapDataType dt = ES == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                 : ES == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                                 : ES == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32
                                           : CU_TENSOR_MAP_DATA_TYPE_UINT64;
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) return false;
  if (enc(&map, dt, 5, const_cast<void *>(src), dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  const int64_t total = g.tiles_a * g.tiles_b * g.batch;
  const int64_t blocks = std::min<int64_t>(total, (int64_t)sm_count() * 8);
  if (total + 2 * blocks < ((int64_t)1 << 32))  // t and t + grid stay below 2^32
    k_transpose_tma<ES, uint32_t><<<(unsigned)blocks, TMA_THREADS, 0, st>>>(map, (uint8_t *)dst, g);
  else
    k_transpose_tma<ES, int64_t><<<(unsigned)blocks, TMA_THREADS, 0, st>>>(map, (uint8_t *)dst, g);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("CUDA error %s in k_transpose_tma", cudaGetErrorString(e));
    *res = CTN_ERR_CUDA;
  } else {
    *res = CTN_OK;
  }
  return true;
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
    for (int i = 0; i + 1 < r; ++i) g.in_stride_of_out[i] /= scale;  // exact: multiples of L
    const int64_t row_units = L / scale;
    const int64_t total_units = n / scale;
    const int64_t blocks = std::min<int64_t>((total_units + 255) / 256, (int64_t)nsm * 16);
    const bool small = total_units < (1ll << 31);
#define CTN_ROW_GATHER(UT)                                                                                        \
  if (small)                                                                                                     \
    k_row_gather<UT, uint32_t><<<(unsigned)blocks, 256, 0, st>>>((const UT *)src, (UT *)dst, g, row_units,     \
                                                                 total_units);                                \
  else                                                                                                           \
    k_row_gather<UT, int64_t><<<(unsigned)blocks, 256, 0, st>>>((const UT *)src, (UT *)dst, g, row_units,      \
                                                                total_units);
    switch (vb) {
      case 16:
        CTN_ROW_GATHER(U128);
        break;
      case 8:
        CTN_ROW_GATHER(uint64_t);
        break;
      case 4:
        CTN_ROW_GATHER(uint32_t);
        break;
      case 2:
        CTN_ROW_GATHER(uint16_t);
        break;
      default:
        CTN_ROW_GATHER(uint8_t);
    }
#undef CTN_ROW_GATHER
    CTN_CHECK_LAUNCH();
    return CTN_OK;
  }
  // TMA staging pays for 1-, 2- and 4-byte elements (f32 4.3 vs 2.9 TB/s, 16-bit 3.0 vs 1.5 TB/s
  // on a 512 MB transpose); for 8-byte elements the 32x32 register tile is faster (4.9 vs 4.3
  // TB/s), and a short output axis (< 16) wastes most of a staged tile
  if (ES <= 4 && rshape[rmap[r - 1]] >= 16) {
    ctn_status res = CTN_OK;
    if (try_transpose_tma<(ES <= 4 ? ES : 4)>(src, dst, r, rshape, rmap, in_stride, out_stride, st, &res)) return res;
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
  if (g.nb < 16) {
    if (launch_staged<T>(src, dst, g, nsm, st)) {
      CTN_CHECK_LAUNCH();
      return CTN_OK;
    }
    const int64_t rows = g.na * g.batch;
    const int64_t blocks = std::min<int64_t>((rows + 255) / 256, (int64_t)nsm * 16);
    k_transpose_short<T><<<(unsigned)blocks, 256, 0, st>>>((const T *)src, (T *)dst, g);
    CTN_CHECK_LAUNCH();
    return CTN_OK;
  }
  const int64_t total = g.tiles_a * g.tiles_b * g.batch;
  const int64_t blocks = std::min<int64_t>(total, (int64_t)nsm * 32);
  // 32-bit tile arithmetic when the loop variable cannot pass 2^32 (t < total + grid)
  if (total + blocks < ((int64_t)1 << 32))
    k_transpose<T, uint32_t><<<(unsigned)blocks, dim3(32, 8), 0, st>>>((const T *)src, (T *)dst, g);
  else
    k_transpose<T, int64_t><<<(unsigned)blocks, dim3(32, 8), 0, st>>>((const T *)src, (T *)dst, g);
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
