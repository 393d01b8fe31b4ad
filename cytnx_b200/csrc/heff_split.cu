// Split-precision (3xTF32 / BF16x3) form of the two-site H_eff matvec on tcgen05.
//
// Same algorithm as the FP64 plan (heff.cu), re-laid out for the tensor cores:
//   step 1: one stacked GEMM per left sector a:
//           X1_a[(w,a') rows][(s1,s2,b) cols] = L_a^T (rows of every L block (w,a,a'))
//                                             x psi_a (columns of every psi block (a,..))
//           A = L (packed once per environment), B = psi (packed per matvec),
//           FP32 result in a dense per-group matrix;
//   steps 2+3: X3 blocks = MPO-weighted sums of X1 blocks, written directly as the
//           split, swizzled A panels of step 4 (no intermediate FP32 X3 array);
//   step 4: one stacked GEMM per right sector b':
//           out[(a',s1',s2') rows][b'] = X3_b'[rows][(w2,b) K] x R_b'[(w2,b)][b'],
//           B = R (packed once), FP64 stores straight into the out blocks.
// The K offsets of the R blocks inside a step-4 group are padded to multiples of 8 so
// that every 8-element chunk of the fold (16 bytes of BF16, 32 of TF32) belongs to one X3 block.
#include <cuda_bf16.h>

#include <algorithm>
#include <map>
#include <memory>
#include <vector>

#include "ctn_common.h"
#include "gemm_f64.cuh"
#include "heff.cuh"
#include "tc_gemm.cuh"

namespace ctn {

struct MpoSegS {
  int32_t rows, cols;
  int32_t row0, k0;
  int64_t panel_off;
  int32_t kb, pad_;
  int32_t term_begin, term_count;
};
struct MpoTermS {
  int64_t x1_off;  // FP32 element offset of the X1 block's (0,0)
  int64_t ld;
  double coef;
};

struct WorkItem {
  int32_t seg0, seg1;  // first and last segment overlapping the item's chunks
  int64_t chunk0;      // global chunk index of the item's first chunk
};
// A work item inside one X3 block, with that block's descriptor and its first two terms inline
// (term_count < 0: the item spans several blocks and takes the table path)
struct alignas(16) MpoFat {
  int64_t seg_chunk0;  // global chunk index of the block's first chunk
  int64_t panel_off;
  int32_t cols, row0, k0, kb;
  int32_t term_begin, term_count;
  int64_t x1_off[2];
  int32_t ld[2];
  float coef[2];
};


struct HeffSplit {
  int kind = TC_TF32;
  std::vector<WorkItem> items;
  std::vector<MpoFat> fat;  // one per item
  TcGemm g1, g4;
  Packer pk_L, pk_P, pk_R;
  std::vector<MpoSegS> segs;
  std::vector<MpoTermS> terms;
  std::vector<int64_t> seg_begin;  // chunk prefix sums per segment
  int64_t nchunks = 0;
  void *d_mpo = nullptr;
  int d_dev = -1;
  int64_t x1_elems = 0;
  // workspace layout (bytes)
  int64_t o_a1, o_b1, o_x1, o_a4, o_b4, o_err, total;  // panels hold hi and lo tiles interleaved
  std::vector<std::pair<int64_t, int64_t>> uncovered;  // out ranges no group writes (zero them)
  uint8_t *ws = nullptr;
  int in_f32 = 0;   // psi / L / R given in FP32 (batched form) instead of FP64
  int out_f32 = 0;  // out written in FP32 (step-4 groups in mode 2)
  ~HeffSplit() {
    if (d_mpo) cudaFree(d_mpo);
  }
};

void heff_split_free(HeffSplit *s) { delete s; }

namespace {
constexpr int KALIGN = 8;

int64_t up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Inline descriptors of the work items that lie inside one X3 block (D=4096 fold 37.9 -> 35.8 us
// BF16x3, 49.2 -> 47.1 us 3xTF32: a thread's X1 reads then wait on the item alone, not on the
// block and term tables).  Kept only when at least half of the items are such: with many small
// blocks (the Hubbard batch) most items span several blocks and the extra 80-byte read per item
// cost 1.5 %.
void build_fat(HeffSplit *s) {
  size_t single = 0;
  for (const WorkItem &wi : s->items) single += wi.seg0 == wi.seg1;
  s->fat.clear();
  if (2 * single < s->items.size()) return;
  s->fat.assign(s->items.size(), MpoFat{});
  for (size_t i = 0; i < s->items.size(); ++i) {
    const WorkItem &wi = s->items[i];
    MpoFat &f = s->fat[i];
    f.term_count = -1;
    if (wi.seg0 != wi.seg1) continue;
    const MpoSegS &sg = s->segs[wi.seg0];
    f.seg_chunk0 = s->seg_begin[wi.seg0];
    f.panel_off = sg.panel_off;
    f.cols = sg.cols;
    f.row0 = sg.row0;
    f.k0 = sg.k0;
    f.kb = sg.kb;
    f.term_begin = sg.term_begin;
    f.term_count = sg.term_count;
    for (int t = 0; t < 2 && t < sg.term_count; ++t) {
      const MpoTermS &tm = s->terms[sg.term_begin + t];
      f.x1_off[t] = tm.x1_off;
      f.ld[t] = (int32_t)tm.ld;
      f.coef[t] = (float)tm.coef;
    }
  }
}

// workspace layout (bytes): [A1 panel][B1 panel][X1 f32][A4 panel][B4 panel][error word]
void split_layout(HeffSplit *s) {
  int64_t o = 0;
  auto take = [&](int64_t bytes) {
    const int64_t at = o;
    o = up(o + bytes, 1024);
    return at;
  };
  s->o_a1 = take(s->g1.a_bytes);
  s->o_b1 = take(s->g1.b_bytes);
  s->o_x1 = take(s->x1_elems * 4);
  s->o_a4 = take(s->g4.a_bytes);
  s->o_b4 = take(s->g4.b_bytes);
  s->o_err = take(256);
  s->total = o;
}

struct MpoSParams {
  const MpoFat *fat;
  const MpoSegS *segs;
  const MpoTermS *terms;
  const WorkItem *items;
  const int64_t *begin;  // chunk prefix sums per segment
  int64_t nitems, nchunks;
  int kind;
  const float *x1;
  uint8_t *hi, *lo;
};

constexpr int MPO_THREADS = 256;
constexpr int MPO_UNROLL = 1;
constexpr int MPO_ITEM = MPO_THREADS * MPO_UNROLL;  // chunks per work item
#ifndef MPO_TERMS
#define MPO_TERMS 1  // terms whose X1 loads are issued together (most X3 chunks have one or two)
#endif

// round-to-nearest (ties away) to TF32 / round-to-nearest-even to BF16 with integer ops
// (ALU pipe; the conversion unit is the bottleneck of a cvt-based version)
__device__ __forceinline__ float tf32_rna(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
__device__ __forceinline__ uint32_t bf16_rne_bits(float x) {
  const uint32_t u = __float_as_uint(x);
  return (u + 0x7FFFu + ((u >> 16) & 1u)) >> 16;
}

// split of one X3 chunk into its hi/lo panel chunks (integer rounding on the ALU pipe)
template <int KIND>
__device__ __forceinline__ void mpo_store(const float (&x)[8], const MpoSegS &s, int r, int kloc, uint8_t *hi,
                                          uint8_t *lo) {
  constexpr bool TF = KIND == TC_TF32;
  // panel offset (32-bit index math except the final byte offset)
  const int row = s.row0 + r, kabs = s.k0 + kloc;
  const int rr = row & (TC_BM - 1);
  const int kslice = TF ? (kabs >> 4) : (kabs >> 5);  // 64-byte K slices: 16 TF32 / 32 BF16
  const int byte = TF ? ((kabs & 15) << 2) : ((kabs & 31) << 1);
  const int64_t off = s.panel_off + ((int64_t)(row >> 7) * s.kb + kslice) * (2 * TC_A_TILE) +
                      tc_tile_byte(rr, byte);  // hi tile; lo = hi + TC_A_TILE
  if (TF) {  // 8 TF32 = two 16-byte chunks of one 64-byte slice row (kabs is a multiple of 8)
    const int64_t off1 = off - tc_tile_byte(rr, byte) + tc_tile_byte(rr, byte + 16);
    float h[8], l[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      h[e] = tf32_rna(x[e]);
      l[e] = tf32_rna(x[e] - h[e]);  // exact in FP32
    }
    *(float4 *)(hi + off) = make_float4(h[0], h[1], h[2], h[3]);
    *(float4 *)(lo + off) = make_float4(l[0], l[1], l[2], l[3]);
    *(float4 *)(hi + off1) = make_float4(h[4], h[5], h[6], h[7]);
    *(float4 *)(lo + off1) = make_float4(l[4], l[5], l[6], l[7]);
  } else {
    uint32_t hw[4], lw[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const uint32_t h0 = bf16_rne_bits(x[2 * e]), h1 = bf16_rne_bits(x[2 * e + 1]);
      const uint32_t l0 = bf16_rne_bits(x[2 * e] - __uint_as_float(h0 << 16));
      const uint32_t l1 = bf16_rne_bits(x[2 * e + 1] - __uint_as_float(h1 << 16));
      hw[e] = h0 | (h1 << 16);
      lw[e] = l0 | (l1 << 16);
    }
    *(uint4 *)(hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    *(uint4 *)(lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
  }
}

// One CTA per work item of MPO_ITEM consecutive chunks (E = 8 elements of one row; 4-element
// TF32 chunks made the 3xTF32 fold slower, its chunk count and table lookups being twice BF16's)
// of the flattened X3 blocks; an item may span several small blocks (each thread then finds its
// block by a binary search over the blocks the item overlaps; items inside one block carry it
// inline).  Blocks are ordered by (a', b), so the blocks that read the same X1 inputs run
// together and share them in L2.  X1 block rows start on 16-byte boundaries (padded step-1
// columns), so full chunks load as float4.  Each thread computes MPO_UNROLL chunks together,
// MPO_TERMS terms per round (one: with 1.4 terms per chunk on average wider rounds mostly issue
// predicated-off loads and multiplies by zero; 0.0386 -> 0.0371 ms at D=4096 BF16x3 against
// four).
// Six CTAs per SM (40 registers): occupancy over registers, the loads are latency-bound
// (39 vs 43 us at D=4096 BF16x3 against the unconstrained 44-register build).
template <int KIND>
__global__ void __launch_bounds__(MPO_THREADS, 6) k_mpo_split(MpoSParams p) {
  constexpr int E = 8;  // elements per chunk (a thread's share): 32 bytes of X1 per term
  constexpr int U = MPO_UNROLL;
  for (int64_t it = blockIdx.x; it < p.nitems; it += gridDim.x) {
    if (p.fat && p.fat[it].term_count >= 0) {  // the item lies in one block: item -> X1, no table lookups
      const MpoFat f = p.fat[it];
      const int64_t g = it * MPO_ITEM + threadIdx.x;
      if (g >= p.nchunks) continue;
      const int nkc = (f.cols + E - 1) / E;
      const int cl = (int)(g - f.seg_chunk0);
      const int r = cl / nkc;
      const int kloc = (cl - r * nkc) * E;
      const int nv = min(E, f.cols - kloc);
      float x[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) x[e] = 0.f;
      auto add = [&](float cf, const float *src) {
        if (nv == E) {
          const float4 v = __ldg(reinterpret_cast<const float4 *>(src));
          x[0] = fmaf(cf, v.x, x[0]);
          x[1] = fmaf(cf, v.y, x[1]);
          x[2] = fmaf(cf, v.z, x[2]);
          x[3] = fmaf(cf, v.w, x[3]);
          const float4 w = __ldg(reinterpret_cast<const float4 *>(src) + 1);
          x[4] = fmaf(cf, w.x, x[4]);
          x[5] = fmaf(cf, w.y, x[5]);
          x[6] = fmaf(cf, w.z, x[6]);
          x[7] = fmaf(cf, w.w, x[7]);
        } else {
#pragma unroll
          for (int e = 0; e < E; ++e)
            if (e < nv) x[e] = fmaf(cf, __ldg(src + e), x[e]);
        }
      };
      if (f.term_count > 0) add(f.coef[0], p.x1 + f.x1_off[0] + (int64_t)r * f.ld[0] + kloc);
      if (f.term_count > 1) add(f.coef[1], p.x1 + f.x1_off[1] + (int64_t)r * f.ld[1] + kloc);
      for (int t = 2; t < f.term_count; ++t) {
        const MpoTermS tm = p.terms[f.term_begin + t];
        add((float)tm.coef, p.x1 + tm.x1_off + (int64_t)r * tm.ld + kloc);
      }
      MpoSegS sg;
      sg.row0 = f.row0;
      sg.k0 = f.k0;
      sg.panel_off = f.panel_off;
      sg.kb = f.kb;
      mpo_store<KIND>(x, sg, r, kloc, p.hi, p.lo);
      continue;
    }
    const WorkItem wi = p.items[it];
    MpoSegS sg[U];
    int r[U], kloc[U], nv[U], nt[U];
#pragma unroll
    for (int j = 0; j < U; ++j) {
      const int64_t g = wi.chunk0 + threadIdx.x + j * MPO_THREADS;
      const bool ok = g < p.nchunks;
      int si = wi.seg0, hi_s = wi.seg1;  // last block with begin <= g
      while (ok && si < hi_s) {
        const int mid = (si + hi_s + 1) >> 1;
        if (__ldg(p.begin + mid) <= g) si = mid;
        else hi_s = mid - 1;
      }
      sg[j] = p.segs[si];
      const int nkc = (sg[j].cols + E - 1) / E;
      const int cl = ok ? (int)(g - __ldg(p.begin + si)) : 0;
      r[j] = cl / nkc;
      kloc[j] = (cl - r[j] * nkc) * E;
      nv[j] = ok ? min(E, sg[j].cols - kloc[j]) : 0;
      nt[j] = ok ? sg[j].term_count : 0;
    }
    float x[U][8];
#pragma unroll
    for (int j = 0; j < U; ++j)
#pragma unroll
      for (int e = 0; e < 8; ++e) x[j][e] = 0.f;
    int tmax = 0;
#pragma unroll
    for (int j = 0; j < U; ++j) tmax = max(tmax, nv[j] == E ? nt[j] : 0);
    for (int t0 = 0; t0 < tmax; t0 += MPO_TERMS) {
      float4 v[U][MPO_TERMS], w[U][MPO_TERMS];
      float cf[U][MPO_TERMS];
#pragma unroll
      for (int j = 0; j < U; ++j)
#pragma unroll
        for (int u = 0; u < MPO_TERMS; ++u) {
          v[j][u] = w[j][u] = make_float4(0.f, 0.f, 0.f, 0.f);
          cf[j][u] = 0.f;
          if (nv[j] == E && t0 + u < nt[j]) {
            const MpoTermS tm = p.terms[sg[j].term_begin + t0 + u];
            cf[j][u] = (float)tm.coef;
            const float4 *src = reinterpret_cast<const float4 *>(p.x1 + tm.x1_off + (int64_t)r[j] * tm.ld + kloc[j]);
            v[j][u] = __ldg(src);
            w[j][u] = __ldg(src + 1);
          }
        }
#pragma unroll
      for (int j = 0; j < U; ++j)
#pragma unroll
        for (int u = 0; u < MPO_TERMS; ++u) {
          x[j][0] = fmaf(cf[j][u], v[j][u].x, x[j][0]);
          x[j][1] = fmaf(cf[j][u], v[j][u].y, x[j][1]);
          x[j][2] = fmaf(cf[j][u], v[j][u].z, x[j][2]);
          x[j][3] = fmaf(cf[j][u], v[j][u].w, x[j][3]);
          x[j][4] = fmaf(cf[j][u], w[j][u].x, x[j][4]);
          x[j][5] = fmaf(cf[j][u], w[j][u].y, x[j][5]);
          x[j][6] = fmaf(cf[j][u], w[j][u].z, x[j][6]);
          x[j][7] = fmaf(cf[j][u], w[j][u].w, x[j][7]);
        }
    }
#pragma unroll
    for (int j = 0; j < U; ++j) {
      if (nv[j] <= 0) continue;
      if (nv[j] < E) {  // ragged end of a block row: scalar loads
        for (int t = 0; t < nt[j]; ++t) {
          const MpoTermS tm = p.terms[sg[j].term_begin + t];
          const float cf = (float)tm.coef;
          const float *src = p.x1 + tm.x1_off + (int64_t)r[j] * tm.ld + kloc[j];
#pragma unroll
          for (int e = 0; e < E; ++e)
            if (e < nv[j]) x[j][e] = fmaf(cf, __ldg(src + e), x[j][e]);
        }
      }
      mpo_store<KIND>(x[j], sg[j], r[j], kloc[j], p.hi, p.lo);
    }
  }
}
}  // namespace

ctn_status heff_split_prepare(ctn_heff2_plan *p, int kind) {
  if (p->split[kind]) return CTN_OK;
  std::unique_ptr<HeffSplit> s(new HeffSplit());
  s->kind = kind;
  s->g1.kind = s->g4.kind = kind;
  s->g1.set_width(p->split_bn[kind][0]);
  s->g4.set_width(p->split_bn[kind][1]);
  s->pk_L.kind = s->pk_P.kind = s->pk_R.kind = kind;
  const int bn = s->g1.bn;
  // ---------------- step 1 groups: one per left sector a
  std::map<int64_t, std::vector<int64_t>> Lg, Pg;
  for (size_t l = 0; l < p->Lb.size(); ++l) Lg[p->Lb[l].q[1]].push_back((int64_t)l);
  for (size_t q = 0; q < p->Pb.size(); ++q) Pg[p->Pb[q].q[0]].push_back((int64_t)q);
  std::vector<int64_t> l_group(p->Lb.size(), -1), l_row(p->Lb.size(), 0);
  std::vector<int64_t> p_group(p->Pb.size(), -1), p_col(p->Pb.size(), 0);
  std::vector<int64_t> g1_coff, g1_ldc;
  int64_t x1 = 0;
  for (auto &kv : Lg) {
    auto jt = Pg.find(kv.first);
    if (jt == Pg.end()) continue;
    int64_t M = 0, N = 0;
    const int64_t K = p->Lb[kv.second[0]].d[1];
    for (int64_t l : kv.second) {
      l_row[l] = M;
      M += p->Lb[l].d[0] * p->Lb[l].d[2];
    }
    for (int64_t q : jt->second) {  // each psi block's X1 columns start on a 16-byte boundary
      p_col[q] = N;
      N = up(N + p->Pb[q].d[1] * p->Pb[q].d[2] * p->Pb[q].d[3], 4);
    }
    if (M == 0 || N == 0 || K == 0) continue;
    const int64_t ldc = up(N, 4);  // FP32 rows start on 16-byte boundaries (TMA bulk stores)
    const int gi = s->g1.add_group((int)M, (int)N, (int)K, 0, x1, (int)ldc, 0);
    for (int64_t l : kv.second) l_group[l] = gi;
    for (int64_t q : jt->second) p_group[q] = gi;
    g1_coff.push_back(x1);
    g1_ldc.push_back(ldc);
    x1 += M * ldc;
  }
  s->x1_elems = x1;
  s->g1.finalize();
  for (size_t l = 0; l < p->Lb.size(); ++l) {
    if (l_group[l] < 0) continue;
    const TcGroup &g = s->g1.groups[l_group[l]];
    const BlkInfo &b = p->Lb[l];  // [w][a][a'] with d[0] == 1: element (row a', k a) at off + k*d2 + row
    PackSeg sg{b.off, 1, b.d[2], (int32_t)b.d[2], (int32_t)b.d[1], (int32_t)l_row[l], 0, g.a_off, TC_BM, g.kb};
    s->pk_L.segs.push_back(sg);
  }
  for (size_t q = 0; q < p->Pb.size(); ++q) {
    if (p_group[q] < 0) continue;
    const TcGroup &g = s->g1.groups[p_group[q]];
    const BlkInfo &b = p->Pb[q];  // [a][1][1][b]: element (row b, k a) at off + k*d3 + row
    PackSeg sg{b.off, 1, b.d[3], (int32_t)b.d[3], (int32_t)b.d[0], (int32_t)p_col[q], 0, g.b_off,
               s->g1.b_tile_rows(), g.kb};
    s->pk_P.segs.push_back(sg);
  }
  s->pk_L.finalize();
  s->pk_P.finalize();
  // ---------------- step 4 groups: one per right sector b'
  std::map<int64_t, std::vector<int64_t>> Og, Rg;
  for (size_t o = 0; o < p->Ob.size(); ++o) Og[p->Ob[o].q[3]].push_back((int64_t)o);
  for (size_t r = 0; r < p->Rb.size(); ++r) Rg[p->Rb[r].q[2]].push_back((int64_t)r);
  std::vector<int64_t> o_group(p->Ob.size(), -1), o_row(p->Ob.size(), 0);
  std::vector<int64_t> r_group(p->Rb.size(), -1), r_k(p->Rb.size(), 0);
  for (auto &kv : Og) {
    auto jt = Rg.find(kv.first);
    if (jt == Rg.end()) continue;
    int64_t M = 0, K = 0;
    const int64_t N = p->Ob[kv.second[0]].d[3];
    for (int64_t o : kv.second) {
      o_row[o] = M;
      M += p->Ob[o].d[0];
    }
    for (int64_t r : jt->second) {
      r_k[r] = K;
      K = up(K + p->Rb[r].d[1], KALIGN);
    }
    if (M == 0 || N == 0 || K == 0) continue;
    const int64_t rm = (int64_t)s->g4.rowmap.size();
    for (int64_t o : kv.second)
      for (int64_t i = 0; i < p->Ob[o].d[0]; ++i)
        s->g4.rowmap.push_back(p->Ob[o].off + i * p->Ob[o].d[1] * p->Ob[o].d[2] * p->Ob[o].d[3]);
    const int gi = s->g4.add_group((int)M, (int)N, (int)K, 1, 0, (int)N, rm);
    for (int64_t o : kv.second) o_group[o] = gi;
    for (int64_t r : jt->second) r_group[r] = gi;
  }
  s->g4.finalize();
  for (size_t r = 0; r < p->Rb.size(); ++r) {
    if (r_group[r] < 0) continue;
    const TcGroup &g = s->g4.groups[r_group[r]];
    const BlkInfo &b = p->Rb[r];  // [w2][b][b']: element (row b', k b) at off + k*d2 + row
    PackSeg sg{b.off, 1, b.d[2], (int32_t)b.d[2], (int32_t)b.d[1], 0, (int32_t)r_k[r], g.b_off,
               s->g4.b_tile_rows(), g.kb};
    s->pk_R.segs.push_back(sg);
  }
  s->pk_R.finalize();
  // out blocks no step-4 group writes must read as zeros
  for (size_t o = 0; o < p->Ob.size(); ++o)
    if (o_group[o] < 0) {
      const BlkInfo &b = p->Ob[o];
      s->uncovered.push_back({b.off, b.d[0] * b.d[1] * b.d[2] * b.d[3]});
    }
  // ---------------- MPO segments: X3 blocks into the step-4 A panels, ordered by (a', b)
  // (the blocks of one (a', b) read the same X1 blocks)
  const int E = 8;  // fold chunk: 8 elements (16 bytes of BF16 or 32 bytes of TF32 per panel)
  std::map<std::pair<int64_t, int64_t>, std::vector<size_t>> by_ab;
  for (size_t i = 0; i < p->x3.size(); ++i) {
    const X3Info &xi = p->x3[i];
    by_ab[{p->Ob[xi.o].q[0], p->Rb[xi.r].q[1]}].push_back(i);
  }
  s->seg_begin.push_back(0);
  for (auto &kv : by_ab) {
    for (size_t i : kv.second) {
      const X3Info &xi = p->x3[i];
      if (o_group[xi.o] < 0 || r_group[xi.r] < 0 || o_group[xi.o] != r_group[xi.r]) {
        set_error("heff split plan: inconsistent step-4 grouping");
        return CTN_ERR_INVALID;
      }
      const TcGroup &g = s->g4.groups[o_group[xi.o]];
      MpoSegS sg;
      sg.rows = (int32_t)xi.rows;
      sg.cols = (int32_t)xi.cols;
      sg.row0 = (int32_t)o_row[xi.o];
      sg.k0 = (int32_t)r_k[xi.r];
      sg.panel_off = g.a_off;
      sg.kb = g.kb;
      sg.pad_ = 0;
      sg.term_begin = (int32_t)s->terms.size();
      sg.term_count = (int32_t)xi.terms.size();
      for (auto &tm : xi.terms) {
        const int64_t l = p->x1_lp[tm.first].first, q = p->x1_lp[tm.first].second;
        const int64_t gi = l_group[l];
        if (gi < 0 || p_group[q] != gi) {
          set_error("heff split plan: X1 block outside the step-1 groups");
          return CTN_ERR_INVALID;
        }
        MpoTermS t;
        t.ld = g1_ldc[gi];
        t.x1_off = g1_coff[gi] + l_row[l] * t.ld + p_col[q];
        t.coef = tm.second;
        s->terms.push_back(t);
      }
      s->segs.push_back(sg);
      s->seg_begin.push_back(s->seg_begin.back() + (int64_t)xi.rows * ((xi.cols + E - 1) / E));
    }
  }
  s->nchunks = s->seg_begin.back();
  chunk_items(s->seg_begin, MPO_ITEM, s->items);
  build_fat(s.get());
  split_layout(s.get());
  p->split[kind] = s.release();
  heff_split_apply_epilogue(p, kind);
  return CTN_OK;
}

void heff_split_apply_epilogue(ctn_heff2_plan *p, int kind) {
  HeffSplit *s = p->split[kind];
  if (!s) return;
  s->g1.epi_staged = p->split_epi[kind][0] < 0 ? s->g1.epi_auto : p->split_epi[kind][0];
  s->g4.epi_staged = p->split_epi[kind][1] < 0 ? s->g4.epi_auto : p->split_epi[kind][1];
}

ctn_status heff_split_stats(const ctn_heff2_plan *p, int kind, double *out) {
  const HeffSplit *s = p->split[kind];
  CTN_REQUIRE(s, "ctn_heff2_split_stats: precision not prepared");
  s->g1.stats(out);
  s->g4.stats(out + 4);
  return CTN_OK;
}

double heff_split_gemm_flops(const ctn_heff2_plan *p, int kind, int step) {
  const HeffSplit *s = p->split[kind];
  if (!s) return 0.0;
  return step == 1 ? s->g1.flops : step == 4 ? s->g4.flops : 0.0;
}

size_t heff_split_ws_bytes(const ctn_heff2_plan *p, int kind) {
  return p->split[kind] ? (size_t)p->split[kind]->total : 0;
}

ctn_status split_set_env(HeffSplit *s, const void *L, const void *R, void *ws, cudaStream_t st) {
  CTN_REQUIRE(s, "heff split: not prepared");
  s->ws = (uint8_t *)ws;
  CTN_CUDA(cudaMemsetAsync(ws, 0, s->total, st));
  CTN_TRY(s->pk_L.run(L, s->in_f32, s->ws + s->o_a1, st));
  CTN_TRY(s->pk_R.run(R, s->in_f32, s->ws + s->o_b4, st));
  // device copy of the MPO segment tables
  int dev = 0;
  CTN_CUDA(cudaGetDevice(&dev));
  if (!s->d_mpo || s->d_dev != dev) {
    if (s->d_mpo) cudaFree(s->d_mpo);
    const size_t bytes = s->fat.size() * sizeof(MpoFat) + s->segs.size() * sizeof(MpoSegS) +
                         s->terms.size() * sizeof(MpoTermS) + s->items.size() * sizeof(WorkItem) +
                         s->seg_begin.size() * sizeof(int64_t) + 64;
    CTN_CUDA(cudaMalloc(&s->d_mpo, bytes));
    s->d_dev = dev;
    char *q = (char *)s->d_mpo;
    if (!s->fat.empty()) CTN_CUDA(cudaMemcpyAsync(q, s->fat.data(), s->fat.size() * sizeof(MpoFat), cudaMemcpyHostToDevice, st));
    q += s->fat.size() * sizeof(MpoFat);
    if (!s->segs.empty()) CTN_CUDA(cudaMemcpyAsync(q, s->segs.data(), s->segs.size() * sizeof(MpoSegS), cudaMemcpyHostToDevice, st));
    q += s->segs.size() * sizeof(MpoSegS);
    if (!s->terms.empty()) CTN_CUDA(cudaMemcpyAsync(q, s->terms.data(), s->terms.size() * sizeof(MpoTermS), cudaMemcpyHostToDevice, st));
    q += s->terms.size() * sizeof(MpoTermS);
    if (!s->items.empty()) CTN_CUDA(cudaMemcpyAsync(q, s->items.data(), s->items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice, st));
    q += s->items.size() * sizeof(WorkItem);
    if (!s->seg_begin.empty())
      CTN_CUDA(cudaMemcpyAsync(q, s->seg_begin.data(), s->seg_begin.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    CTN_CUDA(cudaStreamSynchronize(st));
  }
  CTN_TRY(s->g1.upload(st));
  CTN_TRY(s->g4.upload(st));
  CTN_TRY(s->g1.bind_c32((float *)(s->ws + s->o_x1), st));
  CTN_TRY(s->pk_P.upload(st));
  return CTN_OK;
}

ctn_status heff_split_set_env(ctn_heff2_plan *p, int kind, const double *L, const double *R, void *ws,
                              cudaStream_t st) {
  return split_set_env(p->split[kind], L, R, ws, st);
}

ctn_status split_matvec(HeffSplit *s, const void *psi, void *out, cudaStream_t st, double *ms4, bool f32_out) {
  CTN_REQUIRE(s && s->ws, "heff split: environments not bound");
  const int kind = s->kind;
  const bool o32 = s->out_f32 || f32_out;
  const size_t oes = o32 ? 4 : 8;
  uint8_t *w = s->ws;
  cudaEvent_t ev[5];
  if (ms4)
    for (auto &e : ev) CTN_CUDA(cudaEventCreate(&e));
  if (ms4) CTN_CUDA(cudaEventRecord(ev[0], st));
  for (auto &u : s->uncovered) CTN_CUDA(cudaMemsetAsync((char *)out + u.first * oes, 0, u.second * oes, st));
  CTN_TRY(s->pk_P.run(psi, s->in_f32, w + s->o_b1, st));
  if (ms4) CTN_CUDA(cudaEventRecord(ev[1], st));
  int *err = (int *)(w + s->o_err);
  CTN_TRY(s->g1.run(w + s->o_a1, w + s->o_b1, (float *)(w + s->o_x1), nullptr, err, st));
  if (ms4) CTN_CUDA(cudaEventRecord(ev[2], st));
  if (!s->items.empty()) {
    MpoSParams prm;
    const char *q = (const char *)s->d_mpo;
    prm.fat = s->fat.empty() ? nullptr : (const MpoFat *)q;
    q += s->fat.size() * sizeof(MpoFat);
    prm.segs = (const MpoSegS *)q;
    prm.terms = (const MpoTermS *)(q + s->segs.size() * sizeof(MpoSegS));
    const size_t o_items = s->segs.size() * sizeof(MpoSegS) + s->terms.size() * sizeof(MpoTermS);
    prm.items = (const WorkItem *)(q + o_items);
    prm.begin = (const int64_t *)(q + o_items + s->items.size() * sizeof(WorkItem));
    prm.nitems = (int64_t)s->items.size();
    prm.nchunks = s->nchunks;
    prm.kind = kind;
    prm.x1 = (const float *)(w + s->o_x1);
    prm.hi = w + s->o_a4;
    prm.lo = w + s->o_a4 + tc_lo_delta(TC_BM);
    // four waves of resident CTAs: items of uneven size balance through the CTA scheduler
    auto launch = [&](auto kern) -> void {
      const int64_t grid = std::min<int64_t>(prm.nitems, (int64_t)nsm_count() * resident_ctas(kern, MPO_THREADS) * 4);
      kern<<<(unsigned)grid, MPO_THREADS, 0, st>>>(prm);
    };
    if (kind == TC_TF32) launch(k_mpo_split<TC_TF32>);
    else launch(k_mpo_split<TC_BF16>);
    CTN_CHECK_LAUNCH();
  }
  if (ms4) CTN_CUDA(cudaEventRecord(ev[3], st));
  if (o32)
    CTN_TRY(s->g4.run(w + s->o_a4, w + s->o_b4, (float *)out, nullptr, err, st));
  else
    CTN_TRY(s->g4.run(w + s->o_a4, w + s->o_b4, nullptr, (double *)out, err, st));
  if (ms4) {
    CTN_CUDA(cudaEventRecord(ev[4], st));
    CTN_CUDA(cudaEventSynchronize(ev[4]));
    for (int k = 0; k < 4; ++k) {
      float ms = 0.f;
      CTN_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      ms4[k] += ms;
    }
    for (auto &e : ev) cudaEventDestroy(e);
  }
  return CTN_OK;
}

ctn_status heff_split_matvec(ctn_heff2_plan *p, int kind, const double *psi, double *out, cudaStream_t st,
                             double *ms4) {
  return split_matvec(p->split[kind], psi, out, st, ms4, false);
}

ctn_status heff_split_matvec_f32out(ctn_heff2_plan *p, int kind, const double *psi, float *out, cudaStream_t st) {
  return split_matvec(p->split[kind], psi, out, st, nullptr, true);
}

// ---------------------------------------------------------------- batches of independent problems
// The split tables of every problem are concatenated with their operand, panel, X1 and
// output offsets shifted, so each phase of all problems is ONE launch (the tcgen05 GEMMs
// schedule the union of all tiles, largest K first).
HeffSplit *split_batch(std::vector<ctn_heff2_plan *> &plans, const int64_t *psi_offs, const int64_t *L_offs,
                       const int64_t *R_offs, int kind, int bn1, int bn4, int fp32_io, ctn_status *st) {
  *st = CTN_OK;
  std::unique_ptr<HeffSplit> B(new HeffSplit());
  B->kind = kind;
  B->g1.kind = B->g4.kind = kind;
  B->g1.set_width(bn1);
  B->g4.set_width(bn4);
  B->g1.balance = B->g4.balance = false;
  B->pk_L.kind = B->pk_P.kind = B->pk_R.kind = kind;
  B->in_f32 = fp32_io;
  B->out_f32 = fp32_io;
  int64_t a1 = 0, b1 = 0, x1 = 0, a4 = 0, b4 = 0;
  B->seg_begin.push_back(0);
  for (size_t i = 0; i < plans.size(); ++i) {
    ctn_heff2_plan *p = plans[i];
    p->split_bn[kind][0] = bn1;
    p->split_bn[kind][1] = bn4;
    if (p->split[kind] && (p->split[kind]->g1.width() != bn1 || p->split[kind]->g4.width() != bn4)) {
      delete p->split[kind];
      p->split[kind] = nullptr;
    }
    *st = heff_split_prepare(p, kind);
    if (*st != CTN_OK) return nullptr;
    const HeffSplit *S = p->split[kind];
    for (TcGroup g : S->g1.groups) {
      g.a_off += a1;
      g.b_off += b1;
      g.c_off += x1;
      B->g1.groups.push_back(g);
    }
    for (PackSeg sg : S->pk_L.segs) {
      sg.src_off += L_offs[i];
      sg.panel_off += a1;
      B->pk_L.segs.push_back(sg);
    }
    for (PackSeg sg : S->pk_P.segs) {
      sg.src_off += psi_offs[i];
      sg.panel_off += b1;
      B->pk_P.segs.push_back(sg);
    }
    const int64_t rm_base = (int64_t)B->g4.rowmap.size();
    for (TcGroup g : S->g4.groups) {
      g.a_off += a4;
      g.b_off += b4;
      g.rm_off += rm_base;
      if (fp32_io) g.mode = 2;
      B->g4.groups.push_back(g);
    }
    for (int64_t r : S->g4.rowmap) B->g4.rowmap.push_back(r + psi_offs[i]);
    for (PackSeg sg : S->pk_R.segs) {
      sg.src_off += R_offs[i];
      sg.panel_off += b4;
      B->pk_R.segs.push_back(sg);
    }
    const int32_t tbase = (int32_t)B->terms.size();
    for (MpoSegS sg : S->segs) {
      sg.panel_off += a4;
      sg.term_begin += tbase;
      B->segs.push_back(sg);
    }
    for (MpoTermS t : S->terms) {
      t.x1_off += x1;
      B->terms.push_back(t);
    }
    for (size_t k = 0; k + 1 < S->seg_begin.size(); ++k)
      B->seg_begin.push_back(B->seg_begin.back() + (S->seg_begin[k + 1] - S->seg_begin[k]));
    for (auto u : S->uncovered) B->uncovered.push_back({u.first + psi_offs[i], u.second});
    a1 += S->g1.a_bytes;
    b1 += S->g1.b_bytes;
    x1 += S->x1_elems;
    a4 += S->g4.a_bytes;
    b4 += S->g4.b_bytes;
    B->g1.flops += S->g1.flops;
    B->g4.flops += S->g4.flops;
  }
  B->g1.a_bytes = a1;
  B->g1.b_bytes = b1;
  B->g4.a_bytes = a4;
  B->g4.b_bytes = b4;
  B->x1_elems = x1;
  B->g1.finalize();
  B->g4.finalize();
  B->pk_L.finalize();
  B->pk_P.finalize();
  B->pk_R.finalize();
  B->nchunks = B->seg_begin.back();
  chunk_items(B->seg_begin, MPO_ITEM, B->items);
  build_fat(B.get());
  split_layout(B.get());
  return B.release();
}

}  // namespace ctn

struct ctn_heff2_batch {
  ctn::HeffSplit *s = nullptr;
  ~ctn_heff2_batch() { delete s; }
};

extern "C" ctn_status ctn_heff2_batch_create(ctn_heff2_plan *const *plans, int nprob, const int64_t *psi_offs,
                                             const int64_t *L_offs, const int64_t *R_offs, int precision,
                                             int bn_step1, int bn_step4, int fp32_io, ctn_heff2_batch **out) {
  CTN_REQUIRE(plans && nprob > 0 && psi_offs && L_offs && R_offs && out, "ctn_heff2_batch_create: bad argument");
  CTN_REQUIRE(precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3,
              "ctn_heff2_batch_create: split precisions only (3xTF32 or BF16x3)");
  CTN_REQUIRE(ctn::tc_tile_width_supported(bn_step1) && ctn::tc_tile_width_supported(bn_step4),
              "ctn_heff2_batch_create: unsupported tile width");
  for (int i = 0; i < nprob; ++i) CTN_REQUIRE(plans[i], "ctn_heff2_batch_create: null plan");
  std::vector<ctn_heff2_plan *> v(plans, plans + nprob);
  ctn_status st = CTN_OK;
  const int kind = precision == CTN_PREC_BF16X3 ? ctn::TC_BF16 : ctn::TC_TF32;
  ctn::HeffSplit *s = ctn::split_batch(v, psi_offs, L_offs, R_offs, kind, bn_step1, bn_step4, fp32_io ? 1 : 0, &st);
  if (!s) return st;
  auto *b = new ctn_heff2_batch();
  b->s = s;
  *out = b;
  return CTN_OK;
}
extern "C" size_t ctn_heff2_batch_workspace_bytes(const ctn_heff2_batch *b) { return b ? (size_t)b->s->total : 0; }
extern "C" ctn_status ctn_heff2_batch_stats(const ctn_heff2_batch *b, double *out) {
  CTN_REQUIRE(b && out, "ctn_heff2_batch_stats: null argument");
  b->s->g1.stats(out);
  b->s->g4.stats(out + 4);
  return CTN_OK;
}
extern "C" double ctn_heff2_batch_gemm_flops(const ctn_heff2_batch *b) {
  return b ? b->s->g1.flops + b->s->g4.flops : 0.0;
}
extern "C" ctn_status ctn_heff2_batch_set_env(ctn_heff2_batch *b, const void *L_all, const void *R_all,
                                              void *workspace, void *stream) {
  CTN_REQUIRE(b && L_all && R_all && workspace, "ctn_heff2_batch_set_env: null argument");
  return ctn::split_set_env(b->s, L_all, R_all, workspace, ctn::as_stream(stream));
}
extern "C" ctn_status ctn_heff2_batch_matvec(ctn_heff2_batch *b, const void *psi_all, void *out_all, void *stream) {
  CTN_REQUIRE(b && psi_all && out_all, "ctn_heff2_batch_matvec: null argument");
  return ctn::split_matvec(b->s, psi_all, out_all, ctn::as_stream(stream), nullptr, false);
}
extern "C" ctn_status ctn_heff2_batch_profile(ctn_heff2_batch *b, const void *psi_all, void *out_all, int reps,
                                              double *ms4, void *stream) {
  CTN_REQUIRE(b && psi_all && out_all && reps > 0 && ms4, "ctn_heff2_batch_profile: bad argument");
  double acc[4] = {0, 0, 0, 0};
  for (int r = 0; r < reps; ++r) CTN_TRY(ctn::split_matvec(b->s, psi_all, out_all, ctn::as_stream(stream), acc, false));
  for (int i = 0; i < 4; ++i) ms4[i] = acc[i] / reps;
  return CTN_OK;
}
extern "C" void ctn_heff2_batch_destroy(ctn_heff2_batch *b) { delete b; }
