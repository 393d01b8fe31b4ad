// tcgen05 split-precision grouped GEMM (see tc_gemm.cuh for the operand format).
//
// Persistent, warp-specialised CTA of 192 threads, one CTA per SM:
//   warp 0  (1 thread)  producer: per K slice, 4 bulk copies (A_hi, A_lo, B_hi, B_lo)
//                        into an S-stage shared-memory ring, completion on mbarriers;
//   warp 1  (1 thread)  MMA issuer: tcgen05.mma kind::tf32 / kind::f16 (BF16), M=128,
//                        N=BN, accumulating lo*hi + hi*lo + hi*hi into a TMEM buffer;
//                        tcgen05.commit releases a ring slot / publishes a finished tile;
//   warps 2-5           epilogue: tcgen05.ld (32x32b) of the accumulator, FP32 or FP64
//                        stores; two TMEM accumulator buffers let the epilogue of tile i
//                        overlap the main loop of tile i+1.
// Every wait is bounded: on expiry the kernel records an error code in p.err, drains
// its own bulk copies and MMAs (again bounded), frees its TMEM and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <numeric>
#include <queue>
#include <cstring>

#include "tc_gemm.cuh"
#include "tmap.h"

namespace ctn {

int nsm_count() {
  int dev = 0, n = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();  // no device here: clear the error, use the B200 count
    n = 148;
  }
  return n > 0 ? n : 148;
}

namespace {

constexpr int NTHREADS_TC = 192;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait; returns false (and records `code`) when `limit` probes found the phase
// incomplete, or early once another role has recorded an error
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int code, long long limit) {
  for (long long i = 0; i < limit; ++i) {
    if (mbar_try(bar, parity)) return true;
    if ((i & 1023) == 1023 && *(volatile int *)err != 0) return false;  // another role gave up
  }
  atomicCAS(err, 0, code);
  return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}


// UMMA shared-memory descriptor of a K-major SWIZZLE_64B operand tile: start address, stride
// byte offset = one 8-row atom (512 B), descriptor version 1, layout type 4 (64-byte swizzle);
// the leading byte offset is unused for K-major swizzled operands
__device__ __forceinline__ uint64_t smem_desc(const void *p) {
  const uint64_t a = smem_u32(p);
  return ((a & 0x3FFFFull) >> 4) | (1ull << 16) | ((uint64_t)(TC_ATOM_BYTES >> 4) << 32) | (1ull << 46) |
         (4ull << 61);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accum, int kind) {
  if (kind == TC_TF32) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
  }
}
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// 16 TMEM lanes x 32 columns (four 256-bit groups): lane t of the warp receives, for group j,
// r[4j], r[4j+1] = row (t / 4), columns 8j + 2 (t % 4) + {0, 1} and r[4j+2], r[4j+3] = the same
// columns of row (t / 4) + 8 (rows relative to the lane in `addr`)
__device__ __forceinline__ void tmem_ld_frag16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.16x256b.x4.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}
// two adjacent output columns (col, col + 1) of one row from registers: FP32 row-strided or
// row-mapped output (8-byte store when aligned) or FP64 row-mapped output (16-byte store)
__device__ __forceinline__ void epi_store_pair(int mode, int64_t dst, int col, int ncols, uint32_t a, uint32_t b,
                                               float *c32, double *c64) {
  if (dst < 0 || col >= ncols) return;
  const int64_t o = dst + col;
  const bool two = col + 1 < ncols;
  if (mode != 1) {
    float *q = c32 + o;
    if (two && (o & 1) == 0) {
      *reinterpret_cast<float2 *>(q) = make_float2(__uint_as_float(a), __uint_as_float(b));
    } else {
      q[0] = __uint_as_float(a);
      if (two) q[1] = __uint_as_float(b);
    }
  } else {
    double *q = c64 + o;
    if (two && (o & 1) == 0) {
      *reinterpret_cast<double2 *>(q) = make_double2((double)__uint_as_float(a), (double)__uint_as_float(b));
    } else {
      q[0] = (double)__uint_as_float(a);
      if (two) q[1] = (double)__uint_as_float(b);
    }
  }
}

// Epilogue store of one 32-column piece of a warp's 32 accumulator rows.  Each lane holds
// its row's 32 FP32 values (TMEM lane = row); they are staged in the warp's padded
// shared-memory slab (row stride 36 floats: 16-byte aligned, 4-way bank spread) and
// written back 8 lanes per row, so every store instruction covers 4 whole 128-byte
// FP32 row segments (or 4 x 256-byte FP64 segments) instead of 32 scattered 16-byte
// pieces of 32 different rows.
constexpr int EPI_LD = 36;                        // floats per staged row
constexpr int EPI_WARP_FLOATS = 32 * EPI_LD;      // one warp's slab
constexpr int EPI_BYTES = 4 * EPI_WARP_FLOATS * 4;  // four epilogue warps

__device__ __forceinline__ void epi_store_piece(const uint32_t (&v)[32], float *slab, int lane, int64_t dst,
                                                int cg0, int ncol_tile, int mode, float *c32, double *c64) {
  // stage: lane = row
#pragma unroll
  for (int j = 0; j < 8; ++j)
    *reinterpret_cast<float4 *>(slab + lane * EPI_LD + 4 * j) =
        make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]), __uint_as_float(v[4 * j + 2]),
                    __uint_as_float(v[4 * j + 3]));
  __syncwarp();
  const int sub = lane >> 3, ch = lane & 7;  // 4 rows per round, 8 chunks of 4 columns per row
  const int c = ch * 4;                      // first column of this lane's chunk inside the piece
  int64_t rdst[8];
  float4 x[8];
#pragma unroll
  for (int it = 0; it < 8; ++it) rdst[it] = __shfl_sync(0xffffffffu, dst, it * 4 + sub);
#pragma unroll
  for (int it = 0; it < 8; ++it) x[it] = *reinterpret_cast<const float4 *>(slab + (it * 4 + sub) * EPI_LD + c);
  const int nv = min(4, ncol_tile - c);
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    if (rdst[it] < 0 || nv <= 0) continue;
    if (mode != 1) {
      float *o = c32 + rdst[it] + cg0 + c;
      if (nv == 4 && ((reinterpret_cast<uintptr_t>(o) & 15) == 0)) {
        *reinterpret_cast<float4 *>(o) = x[it];
      } else {
        const float xs[4] = {x[it].x, x[it].y, x[it].z, x[it].w};
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (e < nv) o[e] = xs[e];
      }
    } else {
      double *o = c64 + rdst[it] + cg0 + c;
      if (nv == 4 && ((reinterpret_cast<uintptr_t>(o) & 15) == 0)) {
        reinterpret_cast<double2 *>(o)[0] = make_double2((double)x[it].x, (double)x[it].y);
        reinterpret_cast<double2 *>(o)[1] = make_double2((double)x[it].z, (double)x[it].w);
      } else {
        const float xs[4] = {x[it].x, x[it].y, x[it].z, x[it].w};
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (e < nv) o[e] = (double)xs[e];
      }
    }
  }
  __syncwarp();  // the slab is reused by the next piece
}

// Direct form: each lane stores its own row's piece (16-byte vector stores when aligned).
// Cheaper than staging when the tiles are mostly empty (small blocks) or the rows are
// scattered FP64 rows.
__device__ __forceinline__ void epi_store_direct(const uint32_t (&v)[32], int64_t dst, int cg0, int ncol, int mode,
                                                 float *c32, double *c64) {
  if (mode != 1) {
    float *o = c32 + dst + cg0;
    if (ncol == 32 && ((reinterpret_cast<uintptr_t>(o) & 15) == 0)) {
#pragma unroll
      for (int j = 0; j < 8; ++j)
        *reinterpret_cast<float4 *>(o + 4 * j) = make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]),
                                                             __uint_as_float(v[4 * j + 2]), __uint_as_float(v[4 * j + 3]));
    } else {
#pragma unroll
      for (int e = 0; e < 32; ++e)
        if (e < ncol) o[e] = __uint_as_float(v[e]);
    }
  } else {
    double *o = c64 + dst + cg0;
    if (ncol == 32 && ((reinterpret_cast<uintptr_t>(o) & 15) == 0)) {
#pragma unroll
      for (int j = 0; j < 16; ++j)
        *reinterpret_cast<double2 *>(o + 2 * j) =
            make_double2((double)__uint_as_float(v[2 * j]), (double)__uint_as_float(v[2 * j + 1]));
    } else {
#pragma unroll
      for (int e = 0; e < 32; ++e)
        if (e < ncol) o[e] = (double)__uint_as_float(v[e]);
    }
  }
}

// A stage holds SPS consecutive K slices: [SPS A tile pairs (hi, lo)][SPS B tile pairs].  The
// K slices of one row tile are consecutive tiles in the panels, so each operand of a stage is
// one bulk copy of SPS tile pairs; two slices per stage (long-K groups) keep the copies large,
// one slice per stage (short-K groups) keeps the ring deep.
template <int KIND, int BN, int STAGES, int SPS>
struct TcSmem {
  static constexpr int A_BYTES = TC_A_TILE;
  static constexpr int B_BYTES = BN * TC_ROW_BYTES;
  static constexpr int B_OFF = SPS * 2 * A_BYTES;  // the B tile pairs of a stage
  static constexpr int STAGE_BYTES = SPS * (2 * A_BYTES + 2 * B_BYTES);
  static constexpr int RING = STAGES * STAGE_BYTES;
  static constexpr int BAR_OFF = RING;                 // full[S], empty[S], tfull[2], tempty[2], drain
  static constexpr int EPI_OFF = RING + 1024;  // four warps' epilogue slabs (1024-aligned: TMA store boxes)
  // two 4 KB TMA store boxes per epilogue warp when they fit beside the ring (a piece is
  // written into one box while the previous piece's store still reads the other)
  static constexpr int EPI_DB_BYTES = 4 * 2 * 4096;
  static constexpr bool EPI_DB = EPI_OFF + EPI_DB_BYTES + 1024 <= 227 * 1024;
  static constexpr int TOTAL = EPI_OFF + (EPI_DB ? EPI_DB_BYTES : EPI_BYTES);
};

template <int KIND, int BN, int STAGES, int SPS>
__global__ void __launch_bounds__(NTHREADS_TC, 1) k_tc_gemm(TcParams p) {
  using SM = TcSmem<KIND, BN, STAGES, SPS>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + SM::BAR_OFF);
  uint64_t *empty = full + STAGES;
  uint64_t *tfull = empty + STAGES;
  uint64_t *tempty = tfull + 2;
  uint64_t *drain = tempty + 2;
  uint32_t *tmem_holder = (uint32_t *)(drain + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // two accumulator buffers; the allocation is a power of two >= 32 columns
  constexpr uint32_t TMEM_COLS = 2 * BN <= 64 ? 64 : 2 * BN <= 128 ? 128 : 2 * BN <= 256 ? 256 : 512;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], 4);
    }
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;

  constexpr uint32_t FMT = KIND == TC_TF32 ? 2u : 1u;
  // instruction descriptor without its N field: each tile sets N to the columns it has
  // (the last tile of a group is narrower than BN; N is rounded up to a multiple of 16,
  // the padded panel rows are zero), so no MMA work and no B bytes go to padding
  constexpr uint32_t IDESC0 = (1u << 4) | (FMT << 7) | (FMT << 10) | ((uint32_t)(TC_BM >> 4) << 24);
  auto tile_n = [](const TcGroup &g, const TcTile &tl) -> int {
    const int rem = g.N - tl.nt * BN;
    return rem >= BN ? BN : ((rem + 15) & ~15);
  };
  constexpr int KSTEPS = TC_ROW_BYTES / 32;  // MMA K per instruction = 32 bytes of the 64-byte slice

  if (warp == 0 && lane == 0) {
    // ---------------------------------------------------------------- producer
    int stage = 0;
    uint32_t phase = 0;
    uint32_t filled[STAGES];
    for (int s = 0; s < STAGES; ++s) filled[s] = 0;
    bool ok = true;
    for (int64_t t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
      const TcTile tl = p.tiles[t];
      const TcGroup g = p.groups[tl.group];
      const uint32_t b_bytes = (uint32_t)tile_n(g, tl) * TC_ROW_BYTES;  // the tile's B rows only
      for (int kb = 0; kb < g.kb; kb += SPS) {
        const int n = min(SPS, g.kb - kb);  // K slices in this stage
        if (!mbar_wait(&empty[stage], phase ^ 1, p.err, 1, p.spin_limit)) {
          ok = false;
          break;
        }
        if (p.skip_copies) {  // self-test of the error path: nothing arrives on this stage
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1;
          }
          continue;
        }
        uint8_t *st = smem + stage * SM::STAGE_BYTES;
        mbar_expect_tx(&full[stage], (uint32_t)n * (2 * SM::A_BYTES + 2 * b_bytes));
        // tiles are stored hi then lo and the K slices of a row tile back to back: A's n pairs are
        // one copy, B's too when the tile is full width
        const int64_t ao = g.a_off + ((int64_t)tl.mt * g.kb + kb) * (2 * SM::A_BYTES);
        const int64_t bo = g.b_off + ((int64_t)tl.nt * g.kb + kb) * (2 * SM::B_BYTES);
        bulk_g2s(st, p.a + ao, (uint32_t)n * 2 * SM::A_BYTES, &full[stage]);
        if (b_bytes == (uint32_t)SM::B_BYTES) {
          bulk_g2s(st + SM::B_OFF, p.b + bo, (uint32_t)n * 2 * SM::B_BYTES, &full[stage]);
        } else {
          for (int q = 0; q < n; ++q) {
            uint8_t *sb = st + SM::B_OFF + q * 2 * SM::B_BYTES;
            const int64_t bq = bo + (int64_t)q * 2 * SM::B_BYTES;
            bulk_g2s(sb, p.b + bq, b_bytes, &full[stage]);
            bulk_g2s(sb + SM::B_BYTES, p.b + bq + SM::B_BYTES, b_bytes, &full[stage]);
          }
        }
        filled[stage]++;
        if (++stage == STAGES) {
          stage = 0;
          phase ^= 1;
        }
      }
    }
    // drain: every issued fill must have landed before the CTA may exit
    for (int s = 0; s < STAGES; ++s)
      if (filled[s]) mbar_wait(&full[s], (filled[s] - 1) & 1, p.err, 5, p.spin_limit);
  } else if (warp == 1 && lane == 0) {
    // ---------------------------------------------------------------- MMA issuer
    int stage = 0;
    uint32_t phase = 0;
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    bool issued = false;
    for (int64_t t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
      const TcTile tl = p.tiles[t];
      const TcGroup g = p.groups[tl.group];
      const uint32_t idesc = IDESC0 | ((uint32_t)(tile_n(g, tl) >> 3) << 17);
      if (!mbar_wait(&tempty[acc], acc_phase ^ 1, p.err, 2, p.spin_limit)) break;
      tc_fence_after();
      const uint32_t d = tmem_base + (uint32_t)(acc * BN);
      for (int kb = 0; kb < g.kb; kb += SPS) {
        const int n = min(SPS, g.kb - kb);
        if (!mbar_wait(&full[stage], phase, p.err, 3, p.spin_limit)) {
          ok = false;
          break;
        }
        tc_fence_after();
        uint8_t *st = smem + stage * SM::STAGE_BYTES;
#pragma unroll
        for (int q = 0; q < SPS; ++q) {
          if (q >= n) break;
          const uint64_t ahi = smem_desc(st + q * 2 * SM::A_BYTES), alo = smem_desc(st + q * 2 * SM::A_BYTES + SM::A_BYTES);
          const uint64_t bhi = smem_desc(st + SM::B_OFF + q * 2 * SM::B_BYTES);
          const uint64_t blo = smem_desc(st + SM::B_OFF + q * 2 * SM::B_BYTES + SM::B_BYTES);
#pragma unroll
          for (int j = 0; j < KSTEPS; ++j) {
            const uint64_t adv = (uint64_t)(j * 32) >> 4;  // +32 bytes along K inside the swizzle row
            tc_mma(d, alo + adv, bhi + adv, idesc, ((kb + q) | j) != 0, KIND);
            tc_mma(d, ahi + adv, blo + adv, idesc, 1u, KIND);
            tc_mma(d, ahi + adv, bhi + adv, idesc, 1u, KIND);
          }
        }
        issued = true;
        tc_commit(&empty[stage]);
        if (++stage == STAGES) {
          stage = 0;
          phase ^= 1;
        }
      }
      if (!ok) break;
      tc_commit(&tfull[acc]);
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1;
      }
    }
    // all MMAs of this CTA complete before TMEM is released
    if (issued) {
      tc_commit(drain);
      mbar_wait(drain, 0, p.err, 6, p.spin_limit);
    }
  } else if (warp >= 2) {
    // ---------------------------------------------------------------- epilogue
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    float *slab = reinterpret_cast<float *>(smem + SM::EPI_OFF) + (warp - 2) * EPI_WARP_FLOATS;
    int acc = 0;
    uint32_t acc_phase = 0;
    uint32_t pieces = 0;  // TMA-stored pieces of this warp (alternates the store boxes)
    for (int64_t t = blockIdx.x; t < p.ntiles; t += gridDim.x) {
      const TcTile tl = p.tiles[t];
      const TcGroup g = p.groups[tl.group];
      // warp-uniform bounded wait (the TMEM loads below are .sync.aligned)
      int okw = 0;
      if (lane == 0) okw = mbar_wait(&tfull[acc], acc_phase, p.err, 4, p.spin_limit) ? 1 : 0;
      okw = __shfl_sync(0xffffffffu, okw, 0);
      __syncwarp();
      if (!okw) break;
      tc_fence_after();
      const int r = tl.mt * TC_BM + q * 32 + lane;
      const uint32_t base = tmem_base + (uint32_t)(acc * BN) + ((uint32_t)(q * 32) << 16);
      int64_t dst = -1;  // this lane's row start in the output (-1: row beyond M)
      if (r < g.M) dst = g.mode == 0 ? g.c_off + (int64_t)r * g.ldc : p.rowmap[g.rm_off + r];
      // Each lane owns one accumulator row (TMEM lane = row); every 32-column piece goes
      // through the warp's shared-memory slab so that the global stores cover whole row
      // segments (epi_store_piece).  Storing straight from registers (one row per lane)
      // made every store instruction touch 32 rows and kept the epilogue of a 128 x 192
      // FP32 tile at ~4 us, longer than the next tile's MMAs.
      const bool any_row = __any_sync(0xffffffffu, dst >= 0);  // warp-uniform: rows of this quarter inside M
      // Row-strided FP32 output with a tensor map: each 32 x 32 piece goes into this warp's
      // 4 KB box (SWIZZLE_128B layout, conflict-free) and one lane stores it with a 2-D TMA
      // store; rows past M and columns past N are clipped by the tensor map.  The box is
      // reused once the previous store has read it (bulk-group wait on the read).
      const bool tma_out = p.cmaps != nullptr && g.mode == 0 && p.epi_staged == 1;
      // row-mapped FP64 groups launched with only an FP32 output go out as FP32 (mode 2)
      const int mode = (g.mode == 1 && p.c64 == nullptr) ? 2 : g.mode;
      // Fragment form (epi_staged == 2): no shared memory at all.  16-lane x 32-column TMEM
      // fragments put 4 lanes on 8 consecutive columns of one row, so each store instruction
      // writes 8 rows x 32 bytes (FP32) or 8 x 64 bytes (FP64) of whole sectors straight from
      // registers; the main loop of the next tile keeps the shared-memory bandwidth, which the
      // operand copies and the three products' operand reads already fill.
      if (p.epi_staged == 2) {
#pragma unroll 1
        for (int h = 0; h < 2 && any_row; ++h) {
          const int ra = tl.mt * TC_BM + q * 32 + 16 * h + (lane >> 2), rb = ra + 8;
          int64_t da = -1, db = -1;
          if (ra < g.M) da = g.mode == 0 ? g.c_off + (int64_t)ra * g.ldc : p.rowmap[g.rm_off + ra];
          if (rb < g.M) db = g.mode == 0 ? g.c_off + (int64_t)rb * g.ldc : p.rowmap[g.rm_off + rb];
          if (!__any_sync(0xffffffffu, da >= 0 || db >= 0)) continue;  // warp-uniform
          const uint32_t hb = base + ((uint32_t)(16 * h) << 16);
          // columns of this tile only: a 32-column fragment may reach past BN (into the other
          // accumulator's columns), which belong to the next tile
          const int cend = min(g.N, (tl.nt + 1) * BN);
#pragma unroll 1
          for (int c0 = 0; c0 < BN; c0 += 32) {
            if (tl.nt * BN + c0 >= g.N) break;  // warp-uniform: past the group's last column
            uint32_t v[16];
            tmem_ld_frag16(hb + c0, v);
            tmem_wait_ld();
            const int cb = tl.nt * BN + c0 + 2 * (lane & 3);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              epi_store_pair(mode, da, cb + 8 * j, cend, v[4 * j], v[4 * j + 1], p.c32, p.c64);
              epi_store_pair(mode, db, cb + 8 * j, cend, v[4 * j + 2], v[4 * j + 3], p.c32, p.c64);
            }
          }
        }
      }
#pragma unroll 1
      for (int c0 = 0; c0 < BN && any_row && p.epi_staged != 2; c0 += 32) {
        uint32_t v[32];
        tmem_ld16(base + c0, *reinterpret_cast<uint32_t(*)[16]>(&v[0]));
        tmem_ld16(base + c0 + 16, *reinterpret_cast<uint32_t(*)[16]>(&v[16]));
        tmem_wait_ld();
        const int cg0 = tl.nt * BN + c0;
        if (cg0 >= g.N) continue;  // warp-uniform: the whole piece is past the tile edge
        const int ncol = min(min(32, BN - c0), g.N - cg0);  // a 32-column piece may pass the tile edge
        // a 32 x 32 TMA box is clipped at the group's last column only: a piece that passes the
        // tile edge while the group goes on (BN not a multiple of 32) is stored directly
        if (tma_out && c0 + 32 > BN && (tl.nt + 1) * BN < g.N) {
          if (dst >= 0) epi_store_direct(v, dst, cg0, ncol, mode, p.c32, p.c64);
        } else if (tma_out) {
          uint8_t *box = reinterpret_cast<uint8_t *>(smem + SM::EPI_OFF) +
                         (SM::EPI_DB ? (warp - 2) * 8192 + (pieces & 1) * 4096 : (warp - 2) * 4096);
          if (lane == 0) {
            if (SM::EPI_DB)
              asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");  // the other box may still be read
            else
              asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          }
          ++pieces;
          __syncwarp();
#pragma unroll
          for (int j = 0; j < 8; ++j)
            *reinterpret_cast<float4 *>(box + lane * 128 + ((j ^ (lane & 7)) << 4)) =
                make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]), __uint_as_float(v[4 * j + 2]),
                            __uint_as_float(v[4 * j + 3]));
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) {
            const CUtensorMap *map = reinterpret_cast<const CUtensorMap *>(p.cmaps) + tl.group;
            const int row0 = tl.mt * TC_BM + q * 32;
            asm volatile(
                "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                    reinterpret_cast<uint64_t>(map)),
                "r"(cg0), "r"(row0), "r"(smem_u32(box))
                : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          }
        } else if (p.epi_staged == 1) {
          epi_store_piece(v, slab, lane, dst, cg0, ncol, mode, p.c32, p.c64);
        } else if (dst >= 0) {
          epi_store_direct(v, dst, cg0, ncol, mode, p.c32, p.c64);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[acc]);
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1;
      }
    }
    if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // this warp's TMA stores done
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
  }
}

// ------------------------------------------------------------------ 2-CTA (cta_group::2) form
// A pair of CTAs (a cluster of 2) computes one 256 x BN tile: each CTA stages its own
// 128 rows of A and half (BN/2 rows) of B per K slice, the leader (cluster rank 0) issues
// tcgen05.mma.cta_group::2 with M = 256, which reads A from both CTAs and B from both
// halves, and each CTA's TMEM receives the accumulator rows of its own 128 rows.  Per SM
// this moves half of B per tile, so the operand ingest per flop drops by a third (BN=128)
// to a half (BN=256) against the 1-CTA form.
// Synchronisation: both CTAs load their operand slices with 2-D TMA copies of the
// (pre-swizzled) panels in the cta_group::2 form, which completes the bytes on the
// leader's full barrier; the leader's producer expects the bytes of both CTAs.  The
// leader's MMA commits are multicast to both CTAs' empty / tfull barriers; the
// follower's epilogue warps arrive on the leader's tempty barriers.  Every wait is
// bounded; both CTAs meet at a cluster barrier before TMEM is released.  No load is a
// multicast: each CTA reads its own slices of this GPU's memory.
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// shared::cluster address of the same shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t peer_addr(const void *p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
// 2-D TMA load of `rows` rows x 64 bytes at row y of a panel viewed as [rows][64 B]
// (no swizzle: the panel bytes are copied as they are); completes on the leader's
// barrier `bar_cluster` (cta_group::2)
__device__ __forceinline__ void tma_rows_pair(void *dst, const CUtensorMap *map, int y, uint32_t bar_cluster) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(y), "r"(bar_cluster)
      : "memory");
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
__device__ __forceinline__ void tc_mma2(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accum, int kind) {
  if (kind == TC_TF32) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
  }
}
// arrive on the barrier at this offset in both CTAs of the pair once the MMAs complete
__device__ __forceinline__ void tc_commit2_both(uint64_t *bar) {
  asm volatile(
      "{\n\t.reg .b16 m;\n\tmov.b16 m, 3;\n\t"
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], m;\n\t}" ::"r"(
          smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tc_commit2_local(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

template <int KIND, int BN, int STAGES>
struct TcSmem2 {
  static constexpr int A_BYTES = TC_A_TILE;              // this CTA's 128 rows
  static constexpr int B_BYTES = (BN / 2) * TC_ROW_BYTES;  // this CTA's half of B
  static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int RING = STAGES * STAGE_BYTES;
  static constexpr int BAR_OFF = RING;  // full[S], empty[S], tfull[2], tempty[2], drain
  static constexpr int EPI_OFF = RING + 1024;  // 1024-aligned: TMA store boxes
  static constexpr int TOTAL = EPI_OFF + EPI_BYTES;
};

template <int KIND, int BN, int STAGES>
__global__ void __launch_bounds__(NTHREADS_TC, 1) k_tc_gemm_pair(TcParams p, const __grid_constant__ CUtensorMap ta,
                                                                  const __grid_constant__ CUtensorMap tb) {
  using SM = TcSmem2<KIND, BN, STAGES>;
  static_assert(BN % 16 == 0 && BN >= 32 && BN <= 256, "2-CTA tile width");
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + SM::BAR_OFF);
  uint64_t *empty = full + STAGES;
  uint64_t *tfull = empty + STAGES;
  uint64_t *tempty = tfull + 2;
  uint64_t *drain = tempty + 2;
  uint32_t *tmem_holder = (uint32_t *)(drain + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();  // 0: leader (issues the MMAs), 1: follower
  const int64_t pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  constexpr uint32_t TMEM_COLS = 2 * BN <= 64 ? 64 : 2 * BN <= 128 ? 128 : 2 * BN <= 256 ? 256 : 512;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);  // leader: its producer's expect_tx (bytes of both CTAs)
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], 8);  // leader: 4 own + 4 follower epilogue warps
    }
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  cluster_sync_all();  // both CTAs' barriers initialised and TMEM allocated
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;

  constexpr uint32_t FMT = KIND == TC_TF32 ? 2u : 1u;
  constexpr uint32_t IDESC =
      (1u << 4) | (FMT << 7) | (FMT << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(256 >> 4) << 24);
  constexpr int KSTEPS = TC_ROW_BYTES / 32;

  if (warp == 0 && lane == 0) {
    // ---------------------------------------------------------------- producer (both CTAs)
    int stage = 0;
    uint32_t phase = 0;
    uint32_t filled[STAGES];
    for (int s = 0; s < STAGES; ++s) filled[s] = 0;
    bool ok = true;
    for (int64_t t = pair; t < p.ntiles && ok; t += npairs) {
      const TcTile tl = p.tiles[t];
      const TcGroup g = p.groups[tl.group];
      const int mt128 = 2 * tl.mt + (int)rank;  // this CTA's 128-row A tile (panels hold an even count)
      for (int kb = 0; kb < g.kb; ++kb) {
        if (!mbar_wait(&empty[stage], phase ^ 1, p.err, 1, p.spin_limit)) {
          ok = false;
          break;
        }
        uint8_t *st = smem + stage * SM::STAGE_BYTES;
        if (rank == 0) mbar_expect_tx(&full[stage], 2 * SM::STAGE_BYTES);
        const uint32_t fb = peer_addr(&full[stage], 0);
        // panel rows of 64 bytes: A tile (mt128, kb) hi + lo (256 rows, one box) and this
        // CTA's half of the B tile (nt, kb): the B panels of the 2-CTA form hold BN/2-row tiles
        // (hi then lo), half 2 nt + rank, so it is one box of BN rows as well
        const int ya = (int)((g.a_off + ((int64_t)mt128 * g.kb + kb) * (2 * SM::A_BYTES)) / TC_ROW_BYTES);
        const int yb =
            (int)((g.b_off + ((int64_t)(2 * tl.nt + (int)rank) * g.kb + kb) * (2 * SM::B_BYTES)) / TC_ROW_BYTES);
        tma_rows_pair(st, &ta, ya, fb);
        tma_rows_pair(st + 2 * SM::A_BYTES, &tb, yb, fb);
        filled[stage]++;
        if (++stage == STAGES) {
          stage = 0;
          phase ^= 1;
        }
      }
    }
    // drain: the leader's full barriers count the bytes of both CTAs, so the leader waits
    // for every issued fill; the follower is held at the final cluster barrier meanwhile
    if (rank == 0)
      for (int s = 0; s < STAGES; ++s)
        if (filled[s]) mbar_wait(&full[s], (filled[s] - 1) & 1, p.err, 5, p.spin_limit);
  } else if (warp == 1 && lane == 0 && rank == 0) {
    // ---------------------------------------------------------------- MMA issuer (leader)
    int stage = 0;
    uint32_t phase = 0;
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    bool issued = false;
    for (int64_t t = pair; t < p.ntiles && ok; t += npairs) {
      const TcGroup g = p.groups[p.tiles[t].group];
      if (!mbar_wait(&tempty[acc], acc_phase ^ 1, p.err, 2, p.spin_limit)) break;
      tc_fence_after();
      const uint32_t d = tmem_base + (uint32_t)(acc * BN);
      for (int kb = 0; kb < g.kb; ++kb) {
        if (!mbar_wait(&full[stage], phase, p.err, 3, p.spin_limit)) {
          ok = false;
          break;
        }
        tc_fence_after();
        uint8_t *st = smem + stage * SM::STAGE_BYTES;
        const uint64_t ahi = smem_desc(st), alo = smem_desc(st + SM::A_BYTES);
        const uint64_t bhi = smem_desc(st + 2 * SM::A_BYTES), blo = smem_desc(st + 2 * SM::A_BYTES + SM::B_BYTES);
#pragma unroll
        for (int j = 0; j < KSTEPS; ++j) {
          const uint64_t adv = (uint64_t)(j * 32) >> 4;
          tc_mma2(d, alo + adv, bhi + adv, IDESC, (kb | j) != 0, KIND);
          tc_mma2(d, ahi + adv, blo + adv, IDESC, 1u, KIND);
          tc_mma2(d, ahi + adv, bhi + adv, IDESC, 1u, KIND);
        }
        issued = true;
        tc_commit2_both(&empty[stage]);
        if (++stage == STAGES) {
          stage = 0;
          phase ^= 1;
        }
      }
      if (!ok) break;
      tc_commit2_both(&tfull[acc]);
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1;
      }
    }
    if (issued) {
      tc_commit2_local(drain);
      mbar_wait(drain, 0, p.err, 6, p.spin_limit);
    }
  } else if (warp >= 2) {
    // ---------------------------------------------------------------- epilogue (both CTAs)
    const int q = warp & 3;
    float *slab = reinterpret_cast<float *>(smem + SM::EPI_OFF) + (warp - 2) * EPI_WARP_FLOATS;
    int acc = 0;
    uint32_t acc_phase = 0;
    const uint32_t leader_tempty0 = peer_addr(&tempty[0], 0), leader_tempty1 = peer_addr(&tempty[1], 0);
    for (int64_t t = pair; t < p.ntiles; t += npairs) {
      const TcTile tl = p.tiles[t];
      const TcGroup g = p.groups[tl.group];
      int okw = 0;
      if (lane == 0) okw = mbar_wait(&tfull[acc], acc_phase, p.err, 4, p.spin_limit) ? 1 : 0;
      okw = __shfl_sync(0xffffffffu, okw, 0);
      __syncwarp();
      if (!okw) break;
      tc_fence_after();
      const int r = (2 * tl.mt + (int)rank) * TC_BM + q * 32 + lane;
      const uint32_t base = tmem_base + (uint32_t)(acc * BN) + ((uint32_t)(q * 32) << 16);
      int64_t dst = -1;
      if (r < g.M) dst = g.mode == 0 ? g.c_off + (int64_t)r * g.ldc : p.rowmap[g.rm_off + r];
      const bool any_row = __any_sync(0xffffffffu, dst >= 0);  // warp-uniform: rows of this quarter inside M
      // row-strided FP32 output with a tensor map: TMA stores of 32 x 32 pieces (as in k_tc_gemm)
      const bool tma_out = p.cmaps != nullptr && g.mode == 0 && p.epi_staged != 0;
      // row-mapped FP64 groups launched with only an FP32 output go out as FP32 (mode 2)
      const int mode = (g.mode == 1 && p.c64 == nullptr) ? 2 : g.mode;
      uint8_t *box = reinterpret_cast<uint8_t *>(smem + SM::EPI_OFF) + (warp - 2) * 4096;
#pragma unroll 1
      for (int c0 = 0; c0 < BN && any_row; c0 += 32) {
        uint32_t v[32];
        tmem_ld16(base + c0, *reinterpret_cast<uint32_t(*)[16]>(&v[0]));
        tmem_ld16(base + c0 + 16, *reinterpret_cast<uint32_t(*)[16]>(&v[16]));
        tmem_wait_ld();
        const int cg0 = tl.nt * BN + c0;
        if (cg0 >= g.N) continue;  // warp-uniform: the whole piece is past the tile edge
        const int ncol = min(min(32, BN - c0), g.N - cg0);  // a 32-column piece may pass the tile edge
        // a 32 x 32 TMA box is clipped at the group's last column only: a piece that passes the
        // tile edge while the group goes on (BN not a multiple of 32) is stored directly
        if (tma_out && c0 + 32 > BN && (tl.nt + 1) * BN < g.N) {
          if (dst >= 0) epi_store_direct(v, dst, cg0, ncol, mode, p.c32, p.c64);
        } else if (tma_out) {
          if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          __syncwarp();
#pragma unroll
          for (int j = 0; j < 8; ++j)
            *reinterpret_cast<float4 *>(box + lane * 128 + ((j ^ (lane & 7)) << 4)) =
                make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]), __uint_as_float(v[4 * j + 2]),
                            __uint_as_float(v[4 * j + 3]));
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) {
            const CUtensorMap *map = reinterpret_cast<const CUtensorMap *>(p.cmaps) + tl.group;
            const int row0 = (2 * tl.mt + (int)rank) * TC_BM + q * 32;
            asm volatile(
                "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                    reinterpret_cast<uint64_t>(map)),
                "r"(cg0), "r"(row0), "r"(smem_u32(box))
                : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          }
        } else if (p.epi_staged) {  // the 2-CTA form has no fragment form: staged for 1 and 2
          epi_store_piece(v, slab, lane, dst, cg0, ncol, mode, p.c32, p.c64);
        } else if (dst >= 0) {
          epi_store_direct(v, dst, cg0, ncol, mode, p.c32, p.c64);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        if (rank == 0) mbar_arrive(&tempty[acc]);
        else mbar_arrive_remote(acc == 0 ? leader_tempty0 : leader_tempty1);
      }
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1;
      }
    }
    if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // this warp's TMA stores done
  }
  tc_fence_before();
  cluster_sync_all();  // no CTA leaves while its peer may still touch its shared memory or TMEM
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
  }
}

// ------------------------------------------------------------------ packing
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

struct PackParams {
  const PackSeg *segs;
  const int64_t *begin;  // chunk prefix per segment (nseg + 1)
  int nseg;
  int64_t nchunks;
  int kind;
  int src_f32;
  const void *src;
  uint8_t *hi, *lo;
};

__global__ void __launch_bounds__(256) k_pack(PackParams p) {
  const int64_t step = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < p.nchunks; c += step) {
    int lo_s = 0, hi_s = p.nseg - 1;
    while (lo_s < hi_s) {  // last segment with begin <= c
      const int mid = (lo_s + hi_s + 1) >> 1;
      if (p.begin[mid] <= c) lo_s = mid;
      else hi_s = mid - 1;
    }
    const PackSeg s = p.segs[lo_s];
    const int64_t cl = c - p.begin[lo_s];
    const int r = (int)(cl % s.rows);
    const int kc = (int)(cl / s.rows);
    const int E = p.kind == TC_TF32 ? 4 : 8;  // elements per 16-byte chunk
    const int kloc = kc * E;
    double x[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      x[e] = 0.0;
      if (e < E && kloc + e < s.cols) {
        const int64_t idx = s.src_off + (int64_t)r * s.sr + (int64_t)(kloc + e) * s.sk;
        x[e] = p.src_f32 ? (double)((const float *)p.src)[idx] : ((const double *)p.src)[idx];
      }
    }
    const int64_t off = s.panel_off + tc_panel_offset(s.row0 + r, s.k0 + kloc, s.tile_rows, s.kb, p.kind);
    if (p.kind == TC_TF32) {
      float h[4], l[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        h[e] = to_tf32((float)x[e]);
        l[e] = to_tf32((float)(x[e] - (double)h[e]));
      }
      *(float4 *)(p.hi + off) = make_float4(h[0], h[1], h[2], h[3]);
      *(float4 *)(p.lo + off) = make_float4(l[0], l[1], l[2], l[3]);
    } else {
      __nv_bfloat16 h[8], l[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        h[e] = __double2bfloat16(x[e]);
        l[e] = __double2bfloat16(x[e] - (double)__bfloat162float(h[e]));
      }
      *(uint4 *)(p.hi + off) = *(uint4 *)h;
      *(uint4 *)(p.lo + off) = *(uint4 *)l;
    }
  }
}

constexpr int PACK_THREADS = 256;
#ifndef PACK_TILE_WAVES_X2
#define PACK_TILE_WAVES_X2 2
#endif
constexpr int PACK_UNROLL = 4;
constexpr int PACK_ITEM = PACK_THREADS * PACK_UNROLL;

struct PackItemParams {
  const PackSeg *segs;
  const PackItem *items;
  const int64_t *begin;  // chunk prefix sums per segment (nseg + 1)
  int64_t nitems, nchunks;
  int kind;
  int src_f32;
  const void *src;
  uint8_t *hi, *lo;
};

// hi/lo split of one chunk (E elements) and its two 16-byte stores
template <int KIND>
__device__ __forceinline__ void store_split(const double (&x)[8], uint8_t *hi, uint8_t *lo, int64_t off) {
  if (KIND == TC_TF32) {
    float h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      h[e] = to_tf32((float)x[e]);
      l[e] = to_tf32((float)(x[e] - (double)h[e]));
    }
    *(float4 *)(hi + off) = make_float4(h[0], h[1], h[2], h[3]);
    *(float4 *)(lo + off) = make_float4(l[0], l[1], l[2], l[3]);
  } else {
    __nv_bfloat16 h[8], l[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      h[e] = __double2bfloat16(x[e]);
      l[e] = __double2bfloat16(x[e] - (double)__bfloat162float(h[e]));
    }
    *(uint4 *)(hi + off) = *(uint4 *)h;
    *(uint4 *)(lo + off) = *(uint4 *)l;
  }
}

template <bool F32>
__device__ __forceinline__ double load_src(const void *src, int64_t idx) {
  return F32 ? (double)__ldg((const float *)src + idx) : __ldg((const double *)src + idx);
}

// One CTA per work item of PACK_ITEM consecutive chunks; an item may span many small
// segments (each thread finds its own segment by a binary search over the few the item
// overlaps), so tiny blocks do not waste CTAs.  Rows fastest inside a segment, so the
// source reads (rows are the contiguous axis of every operand packed here) coalesce.
template <int KIND, bool F32>
__global__ void __launch_bounds__(PACK_THREADS) k_pack_items(PackItemParams p) {
  constexpr int E = KIND == TC_TF32 ? 4 : 8;
  for (int64_t it = blockIdx.x; it < p.nitems; it += gridDim.x) {
    const PackItem wi = p.items[it];
#pragma unroll
    for (int j = 0; j < PACK_UNROLL; ++j) {
      const int64_t g = wi.chunk0 + threadIdx.x + j * PACK_THREADS;
      if (g >= p.nchunks) break;
      int lo_s = wi.seg0, hi_s = wi.seg1;  // last segment with begin <= g
      while (lo_s < hi_s) {
        const int mid = (lo_s + hi_s + 1) >> 1;
        if (__ldg(p.begin + mid) <= g) lo_s = mid;
        else hi_s = mid - 1;
      }
      const PackSeg s = p.segs[lo_s];
      const int64_t cl = g - __ldg(p.begin + lo_s);
      const int r = (int)(cl % s.rows);
      const int kloc = (int)(cl / s.rows) * E;
      double x[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        x[e] = 0.0;
        if (e < E && kloc + e < s.cols)
          x[e] = load_src<F32>(p.src, s.src_off + (int64_t)r * s.sr + (int64_t)(kloc + e) * s.sk);
      }
      const int64_t off = s.panel_off + tc_panel_offset(s.row0 + r, s.k0 + kloc, s.tile_rows, s.kb, KIND);
      store_split<KIND>(x, p.hi, p.lo, off);
    }
  }
}

// Transposing pack for segments whose rows are the contiguous source axis (sr == 1):
// a CTA loads a 32-row x 32-k (TF32) or 32 x 64 (BF16) tile with coalesced reads along
// the rows (all of a thread's loads issued together), stages it in shared memory, then
// each thread writes one 16-byte chunk with the 8 chunks of a panel row on 8 consecutive
// threads (a panel row of two 64-byte K slices per 8 threads).
using PackTileItem = PackTileItemH;  // rows r0..r0+31, local k chunks kc0..kc0+7
struct PackTileParams {
  const PackSeg *segs;
  const PackTileItem *items;
  int64_t nitems;
  int kind;
  int src_f32;
  const void *src;
  uint8_t *hi, *lo;
};

template <int KIND, bool F32>
__device__ __forceinline__ void pack_tile_load(const PackTileParams &p, const PackTileItem &wi,
                                               double (&v)[32 * 8 * (KIND == TC_TF32 ? 4 : 8) / 256]) {
  constexpr int PER = 32 * 8 * (KIND == TC_TF32 ? 4 : 8) / 256;
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int idx = threadIdx.x + u * 256;
    const int r = idx & 31, k = idx >> 5;
    v[u] = 0.0;
    if (r < wi.nrows && k < wi.ncols) v[u] = load_src<F32>(p.src, wi.src + r + (int64_t)k * wi.sk);
  }
}

// Persistent: each CTA walks items it, it + grid, ...; two items' descriptors and source
// loads are in registers at any time (the one being split and stored and the next), and the
// item after next is loaded as soon as the staging tile has taken the current one, so the
// reads of the whole pack are in flight from the start when it spans about one wave.
template <int KIND, bool F32>
__device__ __forceinline__ void pack_tile_step(const PackTileParams &p, double (*T)[33], PackTileItem &w,
                                               double (&v)[32 * 8 * (KIND == TC_TF32 ? 4 : 8) / 256], int64_t next) {
  constexpr int E = KIND == TC_TF32 ? 4 : 8;
  constexpr int PER = 32 * 8 * E / 256;
  const PackTileItem cur = w;
  __syncthreads();  // the previous item's readers are done with T
  // column r of staged row k sits at r ^ (k / E % 8): the 8-byte reads below (thread (r, c)
  // reads rows c * E + e) then spread over all 16 double-width banks (two threads each, the
  // minimum); without it the BF16 reads were 4-way conflicts
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int idx = threadIdx.x + u * 256;
    const int k = idx >> 5;
    T[k][(idx & 31) ^ ((k / E) & 7)] = v[u];
  }
  __syncthreads();
  if (next < p.nitems) {
    w = p.items[next];
    pack_tile_load<KIND, F32>(p, w, v);
  }
  const int r = threadIdx.x >> 3, c = threadIdx.x & 7;
  if (r >= cur.nrows || c * E >= cur.ncols) return;
  const int64_t off = cur.panel_off + tc_panel_offset(cur.row0 + r, cur.k0 + c * E, cur.tile_rows, cur.kb, KIND);
  double x[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) x[e] = e < E ? T[c * E + e][r ^ c] : 0.0;
  store_split<KIND>(x, p.hi, p.lo, off);
}

template <int KIND, bool F32>
__global__ void __launch_bounds__(256, 4) k_pack_tile(PackTileParams p) {
  constexpr int E = KIND == TC_TF32 ? 4 : 8;
  constexpr int PER = 32 * 8 * E / 256;  // source elements per thread per item
  __shared__ double T[8 * E][33];
  const int64_t g = gridDim.x;
  int64_t it = blockIdx.x;
  if (it >= p.nitems) return;
  PackTileItem wa = p.items[it], wb = wa;
  double va[PER], vb[PER];
  pack_tile_load<KIND, F32>(p, wa, va);
  if (it + g < p.nitems) {
    wb = p.items[it + g];
    pack_tile_load<KIND, F32>(p, wb, vb);
  }
  for (;;) {
    pack_tile_step<KIND, F32>(p, T, wa, va, it + 2 * g);
    it += g;
    if (it >= p.nitems) break;
    pack_tile_step<KIND, F32>(p, T, wb, vb, it + 2 * g);
    it += g;
    if (it >= p.nitems) break;
  }
}



template <int KIND, int BN, int STAGES, int SPS>
ctn_status launch_tc(const TcParams &prm, int64_t ntiles, cudaStream_t st) {
  using SM = TcSmem<KIND, BN, STAGES, SPS>;
  const int smem = SM::TOTAL + 1024;
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    CTN_CUDA(cudaFuncSetAttribute(k_tc_gemm<KIND, BN, STAGES, SPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_set[dev & 63] = true;
  }
  const int grid = (int)std::min<int64_t>(ntiles, nsm_count());
  k_tc_gemm<KIND, BN, STAGES, SPS><<<grid, NTHREADS_TC, smem, st>>>(prm);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}

// 2-D view [bytes / 64][64] (uint8, no swizzle) of a panel buffer, boxes of `box_rows` rows
static ctn_status encode_rows_map(CUtensorMap *m, const void *base, int64_t bytes, int box_rows) {
  const cuuint64_t dims[2] = {(cuuint64_t)TC_ROW_BYTES, (cuuint64_t)(bytes / TC_ROW_BYTES)};
  const cuuint64_t strides[1] = {(cuuint64_t)TC_ROW_BYTES};
  const cuuint32_t box[2] = {(cuuint32_t)TC_ROW_BYTES, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) {
    set_error("tcgen05 2-CTA GEMM: the driver provides no cuTensorMapEncodeTiled");
    return CTN_ERR_UNSUPPORTED;
  }
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides,
                                            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("tcgen05 2-CTA GEMM: cuTensorMapEncodeTiled failed (%d)", (int)r);
    return CTN_ERR_CUDA;
  }
  return CTN_OK;
}

template <int KIND, int BN, int STAGES>
ctn_status launch_tc_pair(const TcParams &prm, int64_t ntiles, cudaStream_t st) {
  using SM = TcSmem2<KIND, BN, STAGES>;
  const int smem = SM::TOTAL + 1024;
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    CTN_CUDA(cudaFuncSetAttribute(k_tc_gemm_pair<KIND, BN, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem));
    attr_set[dev & 63] = true;
  }
  const int pairs = (int)std::min<int64_t>(ntiles, nsm_count() / 2);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * pairs, 1, 1);
  cfg.blockDim = dim3(NTHREADS_TC, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CUtensorMap ma, mb;
  CTN_REQUIRE(prm.a_bytes > 0 && prm.b_bytes > 0 && prm.a_bytes % TC_ROW_BYTES == 0 &&
                  prm.b_bytes % TC_ROW_BYTES == 0,
              "tcgen05 2-CTA GEMM: panel sizes unknown");
  CTN_TRY(encode_rows_map(&ma, prm.a, prm.a_bytes, 2 * TC_BM));  // hi + lo of one A tile per box
  CTN_TRY(encode_rows_map(&mb, prm.b, prm.b_bytes, BN));  // hi + lo of one BN/2-row half tile per box
  CTN_CUDA(cudaLaunchKernelEx(&cfg, k_tc_gemm_pair<KIND, BN, STAGES>, prm, ma, mb));
  return CTN_OK;
}

// ring depth: the most stages (at most 8) that fit in 227 KiB next to the barriers, the
// alignment slack and the epilogue buffers (double TMA boxes for the 1-CTA form)
constexpr int TC_SMEM_MAX = 227 * 1024;
constexpr int tc_stages_1cta(int bn, int sps) {
  return (TC_SMEM_MAX - 2048 - 4 * 2 * 4096) / (sps * (2 * TC_A_TILE + 2 * bn * TC_ROW_BYTES)) < 8
             ? (TC_SMEM_MAX - 2048 - 4 * 2 * 4096) / (sps * (2 * TC_A_TILE + 2 * bn * TC_ROW_BYTES))
             : 8;
}
constexpr int tc_stages_pair(int bn) {
  return (TC_SMEM_MAX - 2048 - EPI_BYTES) / (2 * TC_A_TILE + bn * TC_ROW_BYTES) < 8
             ? (TC_SMEM_MAX - 2048 - EPI_BYTES) / (2 * TC_A_TILE + bn * TC_ROW_BYTES)
             : 8;
}

template <int KIND>
ctn_status launch_tc_pair_kind(int bn, const TcParams &prm, cudaStream_t st) {
  switch (bn) {
    case 128: return launch_tc_pair<KIND, 128, tc_stages_pair(128)>(prm, prm.ntiles, st);
    case 192: return launch_tc_pair<KIND, 192, tc_stages_pair(192)>(prm, prm.ntiles, st);
    case 256: return launch_tc_pair<KIND, 256, tc_stages_pair(256)>(prm, prm.ntiles, st);
  }
  set_error("tcgen05 2-CTA GEMM: unsupported tile width %d (128, 192, 256)", bn);
  return CTN_ERR_UNSUPPORTED;
}

// tile widths compiled (UMMA M=128 allows N = 16..256 in steps of 16); the ring depth is
// the largest that fits next to the epilogue boxes (SPS x (2 x 8 KiB A + 2 x BN x 64 B B) per stage)
template <int KIND, int BN>
ctn_status launch_tc_sps(int sps, const TcParams &prm, cudaStream_t st) {
  if (sps == 2) return launch_tc<KIND, BN, tc_stages_1cta(BN, 2), 2>(prm, prm.ntiles, st);
  return launch_tc<KIND, BN, tc_stages_1cta(BN, 1), 1>(prm, prm.ntiles, st);
}
template <int KIND>
ctn_status launch_tc_kind(int bn, int sps, const TcParams &prm, cudaStream_t st) {
  switch (bn) {
    case 32: return launch_tc_sps<KIND, 32>(sps, prm, st);
    case 48: return launch_tc_sps<KIND, 48>(sps, prm, st);
    case 64: return launch_tc_sps<KIND, 64>(sps, prm, st);
    case 96: return launch_tc_sps<KIND, 96>(sps, prm, st);
    case 128: return launch_tc_sps<KIND, 128>(sps, prm, st);
    case 144: return launch_tc_sps<KIND, 144>(sps, prm, st);
    case 160: return launch_tc_sps<KIND, 160>(sps, prm, st);
    case 192: return launch_tc_sps<KIND, 192>(sps, prm, st);
    case 256: return launch_tc_sps<KIND, 256>(sps, prm, st);
  }
  set_error("tcgen05 GEMM: unsupported tile width %d (32, 48, 64, 96, 128, 144, 160, 192, 256)", bn);
  return CTN_ERR_UNSUPPORTED;
}
ctn_status launch_tc_any(int kind, int bn, bool pair, int sps, const TcParams &prm, cudaStream_t st) {
  if (pair)
    return kind == TC_TF32 ? launch_tc_pair_kind<TC_TF32>(bn, prm, st) : launch_tc_pair_kind<TC_BF16>(bn, prm, st);
  return kind == TC_TF32 ? launch_tc_kind<TC_TF32>(bn, sps, prm, st) : launch_tc_kind<TC_BF16>(bn, sps, prm, st);
}

}  // namespace

bool tc_tile_width_supported(int w) {
  if (w < 0) return w == -128 || w == -192 || w == -256;  // 2-CTA (256-row) tiles
  const int bn = w;
  return bn == 32 || bn == 48 || bn == 64 || bn == 96 || bn == 128 || bn == 144 || bn == 160 || bn == 192 ||
         bn == 256;
}

int TcGemm::add_group(int M, int N, int K, int mode, int64_t c_off, int ldc, int64_t rm_off) {
  TcGroup g;
  const int ks = tc_k_per_slice(kind);
  g.M = M;
  g.N = N;
  g.K = K;
  g.mt = (M + TC_BM - 1) / TC_BM;
  g.nt = (N + bn - 1) / bn;
  g.kb = (K + ks - 1) / ks;
  const int mt_alloc = pair ? (g.mt + 1) / 2 * 2 : g.mt;  // 2-CTA tiles read 128-row A tiles in pairs
  g.mode = mode;
  g.c_off = c_off;
  g.ldc = ldc;
  g.rm_off = rm_off;
  g.a_off = a_bytes;
  g.b_off = b_bytes;
  a_bytes += (int64_t)mt_alloc * g.kb * 2 * TC_A_TILE;     // hi + lo tiles
  b_bytes += (int64_t)g.nt * g.kb * 2 * bn * TC_ROW_BYTES;
  groups.push_back(g);
  flops += 2.0 * M * (double)N * K;
  return (int)groups.size() - 1;
}

void TcGemm::stats(double *out) const {
  const int ks = tc_k_per_slice(kind);
  const int rows = pair ? 2 * TC_BM : TC_BM;
  double exec = 0.0, bytes = 0.0, own = 0.0;
  for (const TcGroup &g : groups) {
    if (g.kb == 0) continue;
    own += 2.0 * tc_elem_bytes(kind) * ((double)g.M * g.K + (double)g.N * g.K);
    const int mtiles = pair ? (g.mt + 1) / 2 : g.mt;
    for (int n = 0; n < g.nt; ++n) {
      const int rem = g.N - n * bn;
      const int neff = rem >= bn ? bn : (rem + 15) / 16 * 16;
      exec += 2.0 * mtiles * rows * (double)neff * g.kb * ks;
      bytes += (double)mtiles * g.kb * 2.0 * ((double)rows * TC_ROW_BYTES + (double)neff * TC_ROW_BYTES);
    }
  }
  out[0] = flops;
  out[1] = exec;
  out[2] = bytes;
  out[3] = own;
}

void TcGemm::finalize() {
  // staged epilogue when the tiles are mostly filled (whole row segments pay off); direct
  // when most of every tile lies outside its group (small blocks)
  double used = 0.0, cover = 0.0;
  for (const TcGroup &g : groups) {
    used += (double)g.M * g.N;
    cover += (double)(pair ? (g.mt + 1) / 2 * 2 : g.mt) * TC_BM * (double)g.nt * bn;
  }
  epi_staged = epi_auto = (cover > 0.0 && used >= 0.5 * cover) ? 1 : 0;
  std::vector<std::pair<int, TcTile>> tmp;
  for (size_t i = 0; i < groups.size(); ++i) {
    const TcGroup &g = groups[i];
    if (g.kb == 0) continue;
    const int mtiles = pair ? (g.mt + 1) / 2 : g.mt;  // 2-CTA: m counts 256-row tiles
    for (int m = 0; m < mtiles; ++m)
      for (int n = 0; n < g.nt; ++n) tmp.push_back({g.kb, TcTile{(int32_t)i, m, n, 0}});
  }
  std::stable_sort(tmp.begin(), tmp.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
  tiles.clear();
  double ksum = 0.0;
  for (auto &x : tmp) {
    tiles.push_back(x.second);
    ksum += x.first;
  }
  // two K slices per stage when the tiles' K is long (fewer, larger copies per stage), one when
  // it is short (a deeper ring over the few slices a tile has)
  sps = (!tiles.empty() && ksum >= TC_SPS2_MEAN_SLICES * (double)tiles.size()) ? 2 : 1;
}

// Order of the uploaded tile table.  The kernels hand tiles to their W persistent workers
// round-robin (worker w takes positions w, w + W, ...), so worker w gets R + 1 tiles when
// w < n mod W and R = n / W otherwise.  Within those counts the tiles are assigned largest
// first to the least-loaded worker (work = tile width x K slices), then laid out so that the
// round-robin walk visits that assignment.  The first round is the largest-first order itself.
static std::vector<TcTile> balance_tiles(const std::vector<TcTile> &tiles, const std::vector<TcGroup> &groups,
                                         int bn, int64_t W) {
  const int64_t n = (int64_t)tiles.size();
  if (W <= 0 || n <= W) return tiles;
  const int64_t R = n / W, rem = n % W;
  std::vector<double> work(n);
  for (int64_t i = 0; i < n; ++i) {
    const TcTile &t = tiles[i];
    const TcGroup &g = groups[t.group];
    const int neff = t.nt == g.nt - 1 ? (g.N - t.nt * bn + 15) / 16 * 16 : bn;
    work[i] = (double)neff * g.kb;
  }
  std::vector<int64_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return work[a] > work[b]; });
  using Slot = std::pair<double, int64_t>;
  std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>> heap;
  for (int64_t w = 0; w < W; ++w) heap.push({0.0, w});
  std::vector<std::vector<int64_t>> lists(W);
  for (int64_t i : idx) {
    const Slot sl = heap.top();
    heap.pop();
    lists[sl.second].push_back(i);
    const int64_t cap = R + (sl.second < rem ? 1 : 0);
    if ((int64_t)lists[sl.second].size() < cap) heap.push({sl.first + work[i], sl.second});
  }
  std::vector<TcTile> out(n);
  for (int64_t w = 0; w < W; ++w)
    for (size_t k = 0; k < lists[w].size(); ++k) out[(int64_t)k * W + w] = tiles[lists[w][k]];
  return out;
}

ctn_status TcGemm::upload(cudaStream_t st) {
  int dev = 0;
  CTN_CUDA(cudaGetDevice(&dev));
  if (d_mem && d_dev == dev) return CTN_OK;
  if (d_mem) cudaFree(d_mem);
  d_mem = nullptr;
  const size_t bytes = groups.size() * sizeof(TcGroup) + tiles.size() * sizeof(TcTile) +
                       rowmap.size() * sizeof(int64_t) + 256;
  CTN_CUDA(cudaMalloc(&d_mem, bytes));
  d_dev = dev;
  char *q = (char *)d_mem;
  if (!groups.empty()) CTN_CUDA(cudaMemcpyAsync(q, groups.data(), groups.size() * sizeof(TcGroup), cudaMemcpyHostToDevice, st));
  q += groups.size() * sizeof(TcGroup);
  // the workers of the launch: CTAs (1-CTA form) or CTA pairs (2-CTA form)
  const int64_t workers = std::min<int64_t>((int64_t)tiles.size(), pair ? nsm_count() / 2 : nsm_count());
  const std::vector<TcTile> order = balance ? balance_tiles(tiles, groups, bn, workers) : tiles;
  if (!order.empty()) CTN_CUDA(cudaMemcpyAsync(q, order.data(), order.size() * sizeof(TcTile), cudaMemcpyHostToDevice, st));
  q += tiles.size() * sizeof(TcTile);
  if (!rowmap.empty()) CTN_CUDA(cudaMemcpyAsync(q, rowmap.data(), rowmap.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  CTN_CUDA(cudaStreamSynchronize(st));  // the host vectors (order among them) must outlive the copies
  return CTN_OK;
}

ctn_status TcGemm::bind_c32(float *c32, cudaStream_t st) {
  if (!c32) return CTN_OK;
  bool any = false;
  for (const auto &g : groups) any |= g.mode == 0;
  if (!any) return CTN_OK;
  int dev = 0;
  CTN_CUDA(cudaGetDevice(&dev));
  if (d_cmaps && cmaps_for == c32 && cmaps_dev == dev) return CTN_OK;
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) return CTN_OK;  // no driver entry point: the plain staged stores stay in use
  std::vector<CUtensorMap> maps(groups.size());
  std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
  for (size_t i = 0; i < groups.size(); ++i) {
    const TcGroup &g = groups[i];
    if (g.mode != 0) continue;
    void *base = c32 + g.c_off;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || ((int64_t)g.ldc * 4) % 16 != 0) return CTN_OK;
    const cuuint64_t dims[2] = {(cuuint64_t)g.N, (cuuint64_t)g.M};
    const cuuint64_t strides[1] = {(cuuint64_t)g.ldc * 4};
    const cuuint32_t box[2] = {32, 32};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(&maps[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return CTN_OK;  // keep the plain stores
  }
  if (d_cmaps && cmaps_dev != dev) {
    cudaFree(d_cmaps);
    d_cmaps = nullptr;
  }
  if (!d_cmaps) CTN_CUDA(cudaMalloc(&d_cmaps, maps.size() * sizeof(CUtensorMap)));
  CTN_CUDA(cudaMemcpyAsync(d_cmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  cmaps_for = c32;
  cmaps_dev = dev;
  return CTN_OK;
}

ctn_status TcGemm::run(const uint8_t *a, const uint8_t *b, float *c32, double *c64, int *err, cudaStream_t st) {
  if (tiles.empty()) return CTN_OK;
  CTN_TRY(upload(st));
  TcParams prm;
  int dev = 0;
  CTN_CUDA(cudaGetDevice(&dev));
  prm.cmaps = (d_cmaps && c32 && cmaps_for == c32 && cmaps_dev == dev) ? d_cmaps : nullptr;
  const char *q = (const char *)d_mem;
  prm.groups = (const TcGroup *)q;
  prm.tiles = (const TcTile *)(q + groups.size() * sizeof(TcGroup));
  prm.rowmap = (const int64_t *)(q + groups.size() * sizeof(TcGroup) + tiles.size() * sizeof(TcTile));
  prm.ntiles = (int64_t)tiles.size();
  prm.epi_staged = epi_staged;
  prm.a_bytes = a_bytes;
  prm.b_bytes = b_bytes;
  prm.a = a;
  prm.b = b;
  prm.spin_limit = spin_limit;
  prm.skip_copies = skip_copies;
  prm.c32 = c32;
  prm.c64 = c64;
  prm.err = err;
  return launch_tc_any(kind, bn, pair, sps, prm, st);
}

ctn_status tc_launch_tables(int kind, int bn, const TcGroup *d_groups, const TcTile *d_tiles, int64_t ntiles,
                            const int64_t *d_rowmap, const uint8_t *a, const uint8_t *b, float *c32, double *c64,
                            int *err, cudaStream_t st) {
  if (ntiles == 0) return CTN_OK;
  TcParams prm;
  prm.cmaps = nullptr;
  prm.groups = d_groups;
  prm.tiles = d_tiles;
  prm.rowmap = d_rowmap;
  prm.ntiles = ntiles;
  prm.epi_staged = 0;
  prm.a_bytes = 0;
  prm.b_bytes = 0;
  prm.a = a;
  prm.b = b;
  prm.spin_limit = TC_SPIN_LIMIT;
  prm.skip_copies = 0;
  prm.c32 = c32;
  prm.c64 = c64;
  prm.err = err;
  return launch_tc_any(kind, bn, false, 1, prm, st);
}

ctn_status pack_launch_tables(int kind, const PackSeg *d_segs, const int64_t *d_begin, int nseg, int64_t nchunks,
                              const void *src, int src_is_f32, uint8_t *panel, int tile_rows, cudaStream_t st) {
  if (nchunks == 0) return CTN_OK;
  uint8_t *hi = panel, *lo = panel + tc_lo_delta(tile_rows);
  PackParams prm;
  prm.segs = d_segs;
  prm.begin = d_begin;
  prm.nseg = nseg;
  prm.nchunks = nchunks;
  prm.kind = kind;
  prm.src_f32 = src_is_f32;
  prm.src = src;
  prm.hi = hi;
  prm.lo = lo;
  const int64_t grid = std::min<int64_t>((nchunks + 255) / 256, (int64_t)nsm_count() * 16);
  k_pack<<<(unsigned)grid, 256, 0, st>>>(prm);
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}

TcGemm::~TcGemm() {
  if (d_mem) cudaFree(d_mem);
  if (d_cmaps) cudaFree(d_cmaps);
}

void Packer::finalize() {
  seg_chunk_begin.assign(segs.size() + 1, 0);
  const int E = kind == TC_TF32 ? 4 : 8;
  for (size_t i = 0; i < segs.size(); ++i) {
    const int64_t kc = (segs[i].cols + E - 1) / E;
    seg_chunk_begin[i + 1] = seg_chunk_begin[i] + kc * segs[i].rows;
  }
  nchunks = seg_chunk_begin.back();
  chunk_items(seg_chunk_begin, PACK_ITEM, items);
  tile_items.clear();
  bool all_rows = !segs.empty();
  for (const auto &sg : segs) all_rows &= (sg.sr == 1);
  if (all_rows) {
    // row strips innermost: CTAs scheduled together read whole source k-rows (contiguous
    // runs of rows * 8 bytes) instead of the same 256-byte strip of many k-rows
    for (size_t i = 0; i < segs.size(); ++i) {
      const int nkc = (segs[i].cols + E - 1) / E;
      const PackSeg &sg = segs[i];
      for (int kc = 0; kc < nkc; kc += 8)
        for (int r0 = 0; r0 < sg.rows; r0 += 32) {
          PackTileItemH t;
          t.src = sg.src_off + (int64_t)r0 * sg.sr + (int64_t)kc * E * sg.sk;
          t.sk = sg.sk;
          t.panel_off = sg.panel_off;
          t.row0 = sg.row0 + r0;
          t.k0 = sg.k0 + kc * E;
          t.nrows = std::min(32, sg.rows - r0);
          t.ncols = std::min(8 * E, sg.cols - kc * E);
          t.tile_rows = sg.tile_rows;
          t.kb = sg.kb;
          tile_items.push_back(t);
        }
    }
  }
  // the transposing tile pack (32 rows x 8 chunks per item) pays off only when the
  // blocks fill most of its tiles; small blocks use the flattened chunk items
  transposing = all_rows && (double)nchunks >= 0.5 * 256.0 * (double)tile_items.size();
  if (!transposing) tile_items.clear();
}

ctn_status Packer::upload(cudaStream_t st) {
  int dev = 0;
  CTN_CUDA(cudaGetDevice(&dev));
  if (d_mem && d_dev == dev) return CTN_OK;
  if (d_mem) cudaFree(d_mem);
  d_mem = nullptr;
  const size_t bytes = segs.size() * sizeof(PackSeg) + items.size() * sizeof(PackItem) +
                       tile_items.size() * sizeof(PackTileItem) + seg_chunk_begin.size() * sizeof(int64_t) + 64;
  CTN_CUDA(cudaMalloc(&d_mem, bytes));
  d_dev = dev;
  char *q = (char *)d_mem;
  if (!segs.empty()) CTN_CUDA(cudaMemcpyAsync(q, segs.data(), segs.size() * sizeof(PackSeg), cudaMemcpyHostToDevice, st));
  q += segs.size() * sizeof(PackSeg);
  if (!items.empty()) CTN_CUDA(cudaMemcpyAsync(q, items.data(), items.size() * sizeof(PackItem), cudaMemcpyHostToDevice, st));
  q += items.size() * sizeof(PackItem);
  if (!tile_items.empty())
    CTN_CUDA(cudaMemcpyAsync(q, tile_items.data(), tile_items.size() * sizeof(PackTileItem), cudaMemcpyHostToDevice, st));
  q += tile_items.size() * sizeof(PackTileItem);
  if (!seg_chunk_begin.empty())
    CTN_CUDA(cudaMemcpyAsync(q, seg_chunk_begin.data(), seg_chunk_begin.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  return CTN_OK;
}

ctn_status Packer::run(const void *src, int src_is_f32, uint8_t *panel, cudaStream_t st) {
  if (nchunks == 0) return CTN_OK;
  CTN_TRY(upload(st));
  // every segment of one packer fills the same panel: one tile height
  if (transposing ? tile_items.empty() : segs.empty()) return CTN_OK;
  const int rows = transposing ? tile_items[0].tile_rows : segs[0].tile_rows;
  uint8_t *hi = panel, *lo = panel + tc_lo_delta(rows);
  if (transposing) {
    PackTileParams tp;
    tp.segs = (const PackSeg *)d_mem;
    tp.items = (const PackTileItem *)((const char *)d_mem + segs.size() * sizeof(PackSeg) + items.size() * sizeof(PackItem));
    tp.nitems = (int64_t)tile_items.size();
    tp.kind = kind;
    tp.src_f32 = src_is_f32;
    tp.src = src;
    tp.hi = hi;
    tp.lo = lo;
    // one wave of resident CTAs, each walking several items with the next item's loads in
    // flight (PACK_TILE_WAVES_X2 / 2 waves)
    auto launch = [&](auto kern) -> void {
      const int64_t g2 =
          std::min<int64_t>(tp.nitems, (int64_t)nsm_count() * resident_ctas(kern, 256) * PACK_TILE_WAVES_X2 / 2);
      kern<<<(unsigned)std::max<int64_t>(g2, 1), 256, 0, st>>>(tp);
    };
    if (kind == TC_TF32) {
      if (src_is_f32) launch(k_pack_tile<TC_TF32, true>);
      else launch(k_pack_tile<TC_TF32, false>);
    } else {
      if (src_is_f32) launch(k_pack_tile<TC_BF16, true>);
      else launch(k_pack_tile<TC_BF16, false>);
    }
    CTN_CHECK_LAUNCH();
    return CTN_OK;
  }
  PackItemParams prm;
  const char *q = (const char *)d_mem;
  prm.segs = (const PackSeg *)q;
  prm.items = (const PackItem *)(q + segs.size() * sizeof(PackSeg));
  prm.begin = (const int64_t *)(q + segs.size() * sizeof(PackSeg) + items.size() * sizeof(PackItem) +
                                tile_items.size() * sizeof(PackTileItem));
  prm.nitems = (int64_t)items.size();
  prm.nchunks = nchunks;
  prm.kind = kind;
  prm.src_f32 = src_is_f32;
  prm.src = src;
  prm.hi = hi;
  prm.lo = lo;
  auto launch = [&](auto kern) -> void {
    const int64_t grid = std::min<int64_t>(prm.nitems, (int64_t)nsm_count() * resident_ctas(kern, PACK_THREADS) * 4);
    kern<<<(unsigned)grid, PACK_THREADS, 0, st>>>(prm);
  };
  if (kind == TC_TF32) {
    if (src_is_f32) launch(k_pack_items<TC_TF32, true>);
    else launch(k_pack_items<TC_TF32, false>);
  } else {
    if (src_is_f32) launch(k_pack_items<TC_BF16, true>);
    else launch(k_pack_items<TC_BF16, false>);
  }
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}

Packer::~Packer() {
  if (d_mem) cudaFree(d_mem);
}

}  // namespace ctn

// ------------------------------------------------------------------ dense split GEMM (C ABI)
// C[M][N] (FP64, row-major) = A[M][K] * B[K][N] computed with the tcgen05 split kernel:
// the packing, the tcgen05 GEMM and the FP64 epilogue in one call.  Workspace:
// ctn_split_gemm_workspace_bytes.  Mostly a building block and a test vehicle.
namespace {
struct SplitDense {
  ctn::TcGemm g;
  ctn::Packer pa, pb;
};
int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
}  // namespace

extern "C" size_t ctn_split_gemm_workspace_bytes(int64_t M, int64_t N, int64_t K, int precision) {
  const int kind = precision == CTN_PREC_BF16X3 ? ctn::TC_BF16 : ctn::TC_TF32;
  const int ks = ctn::tc_k_per_slice(kind);
  const int64_t kb = (K + ks - 1) / ks;
  const int64_t a = round_up(M, 128) * kb * ctn::TC_ROW_BYTES;
  const int64_t b = round_up(N, 128) * kb * ctn::TC_ROW_BYTES;
  return (size_t)(2 * a + 2 * b + 256 + 64);
}

extern "C" ctn_status ctn_selftest_wait_timeout(int precision, long long spin_limit, void *stream) {
  CTN_REQUIRE(precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3,
              "ctn_selftest_wait_timeout: precision must be split");
  CTN_REQUIRE(spin_limit > 0, "ctn_selftest_wait_timeout: spin_limit must be positive");
  cudaStream_t st = ctn::as_stream(stream);
  SplitDense s;
  const int kind = precision == CTN_PREC_BF16X3 ? ctn::TC_BF16 : ctn::TC_TF32;
  s.g.kind = kind;
  s.g.bn = 128;
  const int64_t n = 128;
  std::vector<int64_t> rows(n);
  for (int64_t r = 0; r < n; ++r) rows[r] = r * n;
  s.g.rowmap = rows;
  s.g.add_group((int)n, (int)n, (int)n, 1, 0, (int)n, 0);
  s.g.finalize();
  s.g.spin_limit = spin_limit;
  s.g.skip_copies = 1;  // the producer issues nothing: the MMA warp's first wait runs out
  uint8_t *ws = nullptr;
  const size_t bytes = (size_t)(s.g.a_bytes + s.g.b_bytes + 64 + (int64_t)n * n * 8);
  CTN_CUDA(cudaMalloc(&ws, bytes));
  CTN_CUDA(cudaMemsetAsync(ws, 0, bytes, st));
  int *err = (int *)(ws + s.g.a_bytes + s.g.b_bytes);
  double *C = (double *)(ws + s.g.a_bytes + s.g.b_bytes + 64);
  ctn_status rc = s.g.run(ws, ws + s.g.a_bytes, nullptr, C, err, st);
  int herr = 0;
  if (rc == CTN_OK) {
    if (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) rc = CTN_ERR_CUDA;
  }
  cudaFree(ws);
  if (rc != CTN_OK) return rc;
  if (herr) {
    ctn::set_error("tcgen05 GEMM: a bounded wait expired (code %d)", herr);
    return CTN_ERR_TIMEOUT;
  }
  ctn::set_error("ctn_selftest_wait_timeout: the kernel finished without a timeout");
  return CTN_ERR_INVALID;
}

extern "C" ctn_status ctn_split_gemm_f64(int64_t M, int64_t N, int64_t K, const double *A, const double *B, double *C,
                                         int precision, void *workspace, void *stream) {
  CTN_REQUIRE(M > 0 && N > 0 && K > 0 && A && B && C && workspace, "ctn_split_gemm_f64: bad argument");
  CTN_REQUIRE(precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3, "ctn_split_gemm_f64: precision must be split");
  CTN_REQUIRE(M < (1 << 30) && N < (1 << 30) && K < (1 << 30), "ctn_split_gemm_f64: too large");
  cudaStream_t st = ctn::as_stream(stream);
  SplitDense s;
  const int kind = precision == CTN_PREC_BF16X3 ? ctn::TC_BF16 : ctn::TC_TF32;
  s.g.kind = kind;
  s.g.bn = 128;
  s.pa.kind = s.pb.kind = kind;
  std::vector<int64_t> rows(M);
  for (int64_t r = 0; r < M; ++r) rows[r] = r * N;
  s.g.rowmap = rows;
  s.g.add_group((int)M, (int)N, (int)K, 1, 0, (int)N, 0);
  s.g.finalize();
  const ctn::TcGroup &g = s.g.groups[0];
  ctn::PackSeg sa{0, K, 1, (int32_t)M, (int32_t)K, 0, 0, g.a_off, 128, g.kb};
  ctn::PackSeg sb{0, 1, N, (int32_t)N, (int32_t)K, 0, 0, g.b_off, 128, g.kb};  // B^T rows = n, k stride N
  s.pa.segs.push_back(sa);
  s.pb.segs.push_back(sb);
  s.pa.finalize();
  s.pb.finalize();
  uint8_t *ws = (uint8_t *)workspace;
  uint8_t *pa = ws, *pb = pa + s.g.a_bytes;  // panels (hi and lo tiles interleaved)
  int *err = (int *)(pb + s.g.b_bytes);
  CTN_CUDA(cudaMemsetAsync(ws, 0, s.g.a_bytes + s.g.b_bytes + 64, st));
  CTN_TRY(s.pa.run(A, 0, pa, st));
  CTN_TRY(s.pb.run(B, 0, pb, st));
  CTN_TRY(s.g.run(pa, pb, nullptr, C, err, st));
  int herr = 0;
  CTN_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  if (herr) {
    ctn::set_error("tcgen05 GEMM: a bounded wait expired (code %d)", herr);
    return CTN_ERR_TIMEOUT;
  }
  return CTN_OK;
}
