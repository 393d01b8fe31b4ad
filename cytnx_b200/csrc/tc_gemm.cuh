// Split-precision grouped GEMM on the 5th-generation tensor cores (tcgen05 + TMEM).
//
// Operands are stored "pre-tiled": every group's A (M x K) and B^T (N x K) matrices are
// cut into tiles of 128 (A) or BN (B) rows by one 64-byte K slice (16 TF32 or 32 BF16
// values), each tile laid out exactly as the UMMA K-major SWIZZLE_64B canonical layout
// expects in shared memory (8-row x 64-byte atoms, 16-byte chunk index XOR (row / 2) % 4).
// Each operand is split as x = hi + lo (both exactly representable in TF32 or BF16), and a
// tile is stored as its hi half followed by its lo half: the hi and lo tiles of one K slice
// move global -> shared with ONE contiguous bulk copy (TMA engine, cp.async.bulk +
// mbarrier complete_tx), no tensor map needed, for any block shape.  64-byte slices keep a
// pipeline stage small (48 KiB for a 128 x 256 tile), so four to eight stages fit in shared
// memory: the ring depth sets the operand stream rate of these GEMMs, whose blocks have
// short K (a few hundred) and whose three products read every stage three times.  Padding
// rows/columns are zeros written once.  Every 32-byte K step issues three MMAs
// lo*hi + hi*lo + hi*hi into one FP32 TMEM accumulator.
#pragma once
#include <cstdint>
#include <algorithm>
#include <vector>

#include "ctn_common.h"

namespace ctn {

constexpr int TC_BM = 128;            // UMMA M (rows of an A tile, TMEM lanes)
constexpr int TC_ROW_BYTES = 64;      // one swizzle row = one K slice
constexpr int TC_ATOM_BYTES = 8 * TC_ROW_BYTES;  // 8-row swizzle atom (the UMMA stride byte offset)
constexpr int TC_A_TILE = TC_BM * TC_ROW_BYTES;  // 8 KiB
constexpr long long TC_SPIN_LIMIT = 1ll << 24;   // try_wait probes of a bounded wait (~seconds)
// mean K slices per tile from which a plan stages two slices per pipeline stage
constexpr double TC_SPS2_MEAN_SLICES = 16.0;

enum TcKind { TC_TF32 = 0, TC_BF16 = 1 };

inline int tc_k_per_slice(int kind) { return kind == TC_TF32 ? 16 : 32; }
inline int tc_elem_bytes(int kind) { return kind == TC_TF32 ? 4 : 2; }

// One stacked GEMM: C[M][N] = A[M][K] * B[K][N] over pre-tiled panels.
struct TcGroup {
  int64_t a_off;      // byte offset of tile (0,0) in the A panels (hi and lo identical layout)
  int64_t b_off;      // byte offset of tile (0,0) in the B panels
  int32_t M, N, K;    // logical sizes
  int32_t mt, nt, kb; // tile counts (128-row A tiles, BN-row B tiles, K slices)
  int32_t mode;       // 0: C32[c_off + r*ldc + c], 1: C64[rowmap[rm_off + r] + c], 2: C32[rowmap[rm_off + r] + c]
  int32_t ldc;
  int64_t c_off;
  int64_t rm_off;
};
struct TcTile {
  int32_t group, mt, nt, pad_;
};

struct TcParams {
  const TcGroup *groups;
  const TcTile *tiles;
  int64_t ntiles;
  const uint8_t *a, *b;  // operand panels (hi/lo interleaved per tile)
  float *c32;
  double *c64;
  const int64_t *rowmap;
  int *err;  // device error word: 0 ok, else the code of the wait that gave up
  int epi_staged;  // epilogue form: 1 through shared memory (whole row segments / TMA stores),
                   // 2 from 16-lane TMEM fragments straight to global memory, 0 one row per lane
  int64_t a_bytes, b_bytes;  // panel sizes, hi and lo (2-CTA form: extents of its TMA views)
  // one 2-D FP32 tensor map per group (CUtensorMap, 128 bytes each) over the row-strided
  // output of mode-0 groups, or null: the staged epilogue then stores 32 x 32 pieces by TMA
  const void *cmaps;
  long long spin_limit;  // try_wait probes of every bounded wait before it gives up
  int skip_copies;       // error-path self-test: the producer issues no copies (waits run out)
};

// byte offset of (row rr, byte b) of a tile, K-major SWIZZLE_64B: 8-row x 64-byte atoms, the
// 16-byte chunk index XORed with address bits 7-8, i.e. (row / 2) % 4
__host__ __device__ inline int tc_tile_byte(int rr, int byte) {
  return (rr >> 3) * TC_ATOM_BYTES + (rr & 7) * TC_ROW_BYTES + ((((byte >> 4) ^ (rr >> 1)) & 3) << 4) + (byte & 15);
}
// byte offset of the hi element (r, k) inside a panel of tiles with `rows` rows per tile
// (tile index = (r / rows) * kb + k / kslice); every tile is its hi half (rows x 64 bytes)
// followed by its lo half, so the lo element is rows * 64 bytes further (tc_lo_delta)
__host__ __device__ inline int64_t tc_panel_offset(int64_t r, int64_t k, int rows, int kb, int kind) {
  const int ks = kind == TC_TF32 ? 16 : 32;
  const int eb = kind == TC_TF32 ? 4 : 2;
  const int64_t tile = (r / rows) * kb + k / ks;
  return tile * 2 * (int64_t)rows * TC_ROW_BYTES + tc_tile_byte((int)(r % rows), (int)(k % ks) * eb);
}
// distance from a hi element to its lo element in a panel with `rows` rows per tile
__host__ __device__ inline int64_t tc_lo_delta(int rows) { return (int64_t)rows * TC_ROW_BYTES; }

// Host plan object for one grouped GEMM (device tables uploaded on first use).
struct TcGemm {
  int kind = TC_TF32;
  int bn = 128;
  bool pair = false;  // 2-CTA (cta_group::2) tiles of 256 rows
  // upload the tiles in a load-balanced round-robin order (off for the DRAM-bound batched
  // plans, whose panels stay in L2 longer when a group's tiles run together)
  bool balance = true;
  // signed width: bn for 1-CTA tiles, -bn for 2-CTA tiles
  void set_width(int w) {
    pair = w < 0;
    bn = w < 0 ? -w : w;
  }
  int width() const { return pair ? -bn : bn; }
  int sps = 1;  // K slices per pipeline stage of the 1-CTA kernel (chosen in finalize)
  // rows per B panel tile: the 2-CTA form stores each BN-wide tile as two BN/2-row tiles, so
  // that the half a CTA of the pair loads (hi and lo) is one contiguous copy
  int b_tile_rows() const { return pair ? bn / 2 : bn; }
  int epi_staged = 0;  // epilogue form (TcParams::epi_staged), chosen in finalize from the tile fill
  int epi_auto = 0;    // finalize's choice (restored by an automatic setting)
  std::vector<TcGroup> groups;
  std::vector<TcTile> tiles;
  std::vector<int64_t> rowmap;
  int64_t a_bytes = 0, b_bytes = 0;  // panel sizes (hi and lo together)
  void *d_mem = nullptr;
  int d_dev = -1;
  double flops = 0.0;  // 2*M*N*K summed over groups (useful flops, one product)
  long long spin_limit = TC_SPIN_LIMIT;  // probes of every bounded wait in the kernel
  int skip_copies = 0;                   // error-path self-test only (ctn_selftest_wait_timeout)

  // append a group; returns its index.  Panels are laid out back to back.
  int add_group(int M, int N, int K, int mode, int64_t c_off, int ldc, int64_t rm_off);
  void finalize();  // builds the tile list (largest K first)
  // out[0] useful flops (2*M*N*K, one product), out[1] executed MMA flops of the tiles (one
  // product: 128 (256 for 2-CTA) rows x the tile's N rounded to 16 x its K slices), out[2] operand
  // panel bytes the tiles copy into shared memory per launch (hi and lo, all products), out[3]
  // the operands' own bytes (M*K + N*K elements, hi and lo, each once)
  void stats(double *out) const;
  ctn_status upload(cudaStream_t st);
  // encode (once per output buffer) the TMA store maps of the mode-0 groups over c32; run()
  // with the same c32 then stores those groups' tiles by TMA
  ctn_status bind_c32(float *c32, cudaStream_t st);
  ctn_status run(const uint8_t *a, const uint8_t *b, float *c32,
                 double *c64, int *err, cudaStream_t st);
  void *d_cmaps = nullptr;
  const float *cmaps_for = nullptr;
  int cmaps_dev = -1;
  ~TcGemm();
};

// Pack segments: a source FP64 (or FP32) matrix region -> hi/lo panel tiles.
struct PackSeg {
  int64_t src_off;      // element offset of (0,0)
  int64_t sr, sk;       // source strides of rows and of k
  int32_t rows, cols;   // region size (cols = K extent)
  int32_t row0, k0;     // destination row / k of (0,0) inside the group panel
  int64_t panel_off;    // byte offset of the group's tile (0,0)
  int32_t tile_rows;    // 128 (A) or BN (B)
  int32_t kb;           // K slices of the group
};

struct PackItem {
  int32_t seg0, seg1;  // first and last segment overlapping the item's chunks
  int64_t chunk0;      // first chunk of this CTA work item (global chunk index)
};

// one 32-row x 8-chunk tile of a row-contiguous segment, self-contained so that a CTA needs
// a single descriptor load before it issues the tile's source loads
struct PackTileItemH {
  int64_t src;         // element offset of the tile's (row 0, k 0); rows are stride 1
  int64_t sk;          // source stride of k
  int64_t panel_off;   // byte offset of the group's tile (0,0)
  int32_t row0, k0;    // destination row / k of the tile's (0,0) inside the group panel
  int32_t nrows, ncols;  // valid rows (<= 32) and k values (<= 8 chunks) of the tile
  int32_t tile_rows, kb;
};

struct Packer {
  int kind = TC_TF32;
  std::vector<struct PackTileItemH> tile_items;  // transposing work items (all segments row-contiguous)
  bool transposing = false;
  std::vector<PackSeg> segs;
  std::vector<int64_t> seg_chunk_begin;  // prefix sums of 16-byte chunks per segment
  std::vector<PackItem> items;           // CTA work items: PACK_ITEM consecutive chunks (may span segments)
  int64_t nchunks = 0;
  void *d_mem = nullptr;
  int d_dev = -1;
  void finalize();
  ctn_status upload(cudaStream_t st);
  // src is FP64 (src_is_f32 == 0) or FP32; panel receives hi and lo tiles interleaved
  ctn_status run(const void *src, int src_is_f32, uint8_t *panel, cudaStream_t st);
  ~Packer();
};


// compiled tile widths: positive = 1-CTA tile of 128 x bn, negative = 2-CTA tile of 256 x |bn|
bool tc_tile_width_supported(int width);
// SM count of the current device (148 when it cannot be queried)
int nsm_count();
// resident CTAs per SM of a kernel at a block size (queried once per kernel)
template <class K>
int resident_ctas(K kernel, int threads) {
  static int occ = 0;
  if (!occ) {
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kernel, threads, 0) != cudaSuccess) cudaGetLastError();
    occ = o > 0 ? o : 4;
  }
  return occ;
}

// Work items of `per_item` consecutive chunks over segments with chunk prefix sums
// `begin`; each item records the first and last segment it overlaps (seg0, seg1).
template <class Item>
inline void chunk_items(const std::vector<int64_t> &begin, int64_t per_item, std::vector<Item> &items) {
  items.clear();
  const int64_t total = begin.back();
  const int nseg = (int)begin.size() - 1;
  int s = 0;
  for (int64_t c0 = 0; c0 < total; c0 += per_item) {
    while (s + 1 < nseg && begin[s + 1] <= c0) ++s;
    int e = s;
    const int64_t last = std::min(c0 + per_item, total) - 1;
    while (e + 1 < nseg && begin[e + 1] <= last) ++e;
    Item it{};
    it.seg0 = s;
    it.seg1 = e;
    it.chunk0 = c0;
    items.push_back(it);
  }
}

// Launch helpers over device-resident tables (the caller owns every buffer).
ctn_status tc_launch_tables(int kind, int bn, const TcGroup *d_groups, const TcTile *d_tiles, int64_t ntiles,
                            const int64_t *d_rowmap, const uint8_t *a, const uint8_t *b, float *c32, double *c64,
                            int *err, cudaStream_t st);
// `panel` receives hi and lo tiles interleaved; `tile_rows` is its rows per tile (128 or BN)
ctn_status pack_launch_tables(int kind, const PackSeg *d_segs, const int64_t *d_begin, int nseg, int64_t nchunks,
                              const void *src, int src_is_f32, uint8_t *panel, int tile_rows, cudaStream_t st);
}  // namespace ctn
