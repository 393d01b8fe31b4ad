// Host side of the block-sparse engine: block enumeration and contraction planning.
//
// BlockUniTensor::Init (src/BlockUniTensor.cpp:190-230) enumerates the blocks of a
// symmetric tensor with a lexicographic odometer over the bonds' qnum indices (last
// leg fastest), keeping a tuple when the total flux (ket: +q, bra: reverse(q),
// include/UniTensor.hpp:1139-1165) vanishes for every symmetry.  BlockUniTensor::contract
// (:777-1235) pairs left and right blocks through a hash of their common-leg qnum
// indices and accumulates Lmat * Rmat into the output block found by its qnum tuple.
//
// Here the pairing happens ONCE per plan, on the host, and is frozen into the task
// tables of one grouped GEMM (gemm_f64.cu): each output block is a task that sums
// over all of its block pairs, so no per-call hashing, no per-pair allocation, and
// no per-pair kernel launch remain on the device path.  Operand blocks whose
// legs are already grouped as [noncomm | comm] (or [comm | noncomm]) are read in
// place (optionally transposed); otherwise all blocks of that operand are permuted
// once per call into the caller's scratch by the permute kernel.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <unordered_map>
#include <vector>

#include "ctn_common.h"
#include "gemm_f64.cuh"

namespace ctn {

static int64_t sym_combine(int stype, int64_t n, int64_t a, int64_t b) {
  return stype == 0 ? (a + b) % n : a + b;  // Symmetry.cpp:33-50 (U1), :64-108 (Zn)
}
static int64_t sym_reverse(int stype, int64_t n, int64_t a) { return stype == 0 ? (n - a) % n : -a; }

struct TupleHash {
  size_t operator()(const std::vector<int64_t> &v) const {
    size_t h = 1469598103934665603ull;
    for (int64_t x : v) {
      h ^= (size_t)x + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    }
    return h;
  }
};

}  // namespace ctn

extern "C" ctn_status ctn_blocks_enumerate(int rank, int nsym, const int32_t *sym_types,
                                           const int64_t *sym_n, const int32_t *bond_types,
                                           const int64_t *nqs, const int64_t *const *qnums,
                                           int64_t *out_itoi, int64_t capacity, int64_t *out_count) {
  CTN_REQUIRE(rank > 0 && rank <= 64, "ctn_blocks_enumerate: rank %d out of range", rank);
  CTN_REQUIRE(nsym >= 0, "ctn_blocks_enumerate: nsym < 0");
  for (int s = 0; s < nsym; ++s)
    CTN_REQUIRE(sym_types[s] == -1 || (sym_types[s] == 0 && sym_n[s] > 0),
                "ctn_blocks_enumerate: unsupported symmetry type %d", sym_types[s]);
  std::vector<int64_t> loc(rank, 0);
  int64_t count = 0;
  for (int i = 0; i < rank; ++i)
    if (nqs[i] <= 0) {
      *out_count = 0;
      return CTN_OK;
    }
  // per-bond, per-symmetry contribution tables (bra legs reversed once)
  std::vector<std::vector<int64_t>> contrib(rank);
  for (int i = 0; i < rank; ++i) {
    contrib[i].resize(nqs[i] * nsym);
    for (int64_t q = 0; q < nqs[i]; ++q)
      for (int s = 0; s < nsym; ++s) {
        int64_t v = qnums[i][q * nsym + s];
        contrib[i][q * nsym + s] = bond_types[i] == 1 ? ctn::sym_reverse(sym_types[s], sym_n[s], v) : v;
      }
  }
  for (;;) {
    bool ok = true;
    for (int s = 0; s < nsym && ok; ++s) {
      int64_t tot = contrib[0][loc[0] * nsym + s];
      for (int j = 1; j < rank; ++j) tot = ctn::sym_combine(sym_types[s], sym_n[s], tot, contrib[j][loc[j] * nsym + s]);
      ok = (tot == 0);
    }
    if (ok) {
      if (count >= capacity) {
        ctn::set_error("ctn_blocks_enumerate: capacity %lld exceeded", (long long)capacity);
        return CTN_ERR_INVALID;
      }
      std::memcpy(out_itoi + count * rank, loc.data(), sizeof(int64_t) * rank);
      ++count;
    }
    int i = rank - 1;
    while (i >= 0) {
      if (loc[i] == nqs[i] - 1) {
        loc[i] = 0;
        --i;
      } else {
        ++loc[i];
        break;
      }
    }
    if (i < 0) break;
  }
  *out_count = count;
  return CTN_OK;
}

// ------------------------------------------------------------------ contract plan
struct ctn_contract_plan {
  // operand staging (copy into scratch with a permutation when the layout needs it)
  struct Stage {
    bool copy = false;
    int rank = 0;
    std::vector<uint64_t> old_shapes;  // physical shapes, per block
    std::vector<int64_t> src_offs, dst_offs;
    std::vector<uint64_t> mapper;      // new axis i = physical axis mapper[i]
    int64_t elems = 0;                 // elements of the staged copy
  } sl, sr;
  ctn::GroupedGemmF64 gemm;
};

namespace {
// classify an operand: need logical order `need` (first group then second group)
// returns 0 = in place (physical == need), 1 = in place transposed (physical ==
// second ++ first), 2 = needs a permuted copy.
int classify(const ctn_block_desc &d, const std::vector<int64_t> &first, const std::vector<int64_t> &second) {
  auto phys = [&](int64_t logical) { return d.perm ? d.perm[logical] : logical; };
  bool same = true, swapped = true;
  int pos = 0;
  for (int64_t x : first) same &= (phys(x) == pos++);
  for (int64_t x : second) same &= (phys(x) == pos++);
  pos = 0;
  for (int64_t x : second) swapped &= (phys(x) == pos++);
  for (int64_t x : first) swapped &= (phys(x) == pos++);
  if (same) return 0;
  if (swapped) return 1;
  return 2;
}

void make_stage(ctn_contract_plan::Stage &s, const ctn_block_desc &d, const std::vector<int64_t> &need) {
  s.copy = true;
  s.rank = d.rank;
  std::vector<int64_t> inv(d.rank);
  for (int i = 0; i < d.rank; ++i) inv[d.perm ? d.perm[i] : i] = i;  // physical -> logical
  s.mapper.resize(d.rank);
  for (int i = 0; i < d.rank; ++i) s.mapper[i] = (uint64_t)(d.perm ? d.perm[need[i]] : need[i]);
  int64_t off = 0;
  for (int64_t b = 0; b < d.nblocks; ++b) {
    int64_t sz = 1;
    for (int j = 0; j < d.rank; ++j) {
      // physical axis j holds logical axis inv[j]
      uint64_t e = (uint64_t)d.shapes[b * d.rank + inv[j]];
      s.old_shapes.push_back(e);
      sz *= (int64_t)e;
    }
    s.src_offs.push_back(d.offs[b]);
    s.dst_offs.push_back(off);
    off += sz;
  }
  s.elems = off;
}
}  // namespace

extern "C" ctn_status ctn_contract_plan_create(const ctn_block_desc *L, const ctn_block_desc *R, int ncomm,
                                               const int64_t *comm_l, const int64_t *comm_r,
                                               const ctn_block_desc *out, ctn_contract_plan **plan) {
  CTN_REQUIRE(L && R && out && plan, "ctn_contract_plan_create: null argument");
  CTN_REQUIRE(ncomm > 0 && ncomm <= L->rank && ncomm <= R->rank, "ctn_contract_plan_create: bad ncomm");
  CTN_REQUIRE(out->perm == nullptr, "ctn_contract_plan_create: output must be contiguous");
  std::vector<int64_t> cl(comm_l, comm_l + ncomm), cr(comm_r, comm_r + ncomm), nl, nr;
  for (int i = 0; i < L->rank; ++i)
    if (std::find(cl.begin(), cl.end(), i) == cl.end()) nl.push_back(i);
  for (int i = 0; i < R->rank; ++i)
    if (std::find(cr.begin(), cr.end(), i) == cr.end()) nr.push_back(i);
  CTN_REQUIRE((int)(nl.size() + nr.size()) == out->rank, "ctn_contract_plan_create: output rank mismatch");
  CTN_REQUIRE(!nl.empty() || !nr.empty(), "ctn_contract_plan_create: full contraction is a dot product");

  std::unique_ptr<ctn_contract_plan> p(new ctn_contract_plan());
  const int cls_l = classify(*L, nl, cl);  // want [M | K]
  const int cls_r = classify(*R, cr, nr);  // want [K | N]
  if (cls_l == 2) {
    std::vector<int64_t> need(nl);
    need.insert(need.end(), cl.begin(), cl.end());
    make_stage(p->sl, *L, need);
  }
  if (cls_r == 2) {
    std::vector<int64_t> need(cr);
    need.insert(need.end(), nr.begin(), nr.end());
    make_stage(p->sr, *R, need);
  }

  // right blocks hashed by their common qindex tuple (BlockUniTensor.cpp:994-1006)
  std::unordered_map<std::vector<int64_t>, std::vector<int64_t>, ctn::TupleHash> mp;
  for (int64_t b = 0; b < R->nblocks; ++b) {
    std::vector<int64_t> key(ncomm);
    for (int c = 0; c < ncomm; ++c) key[c] = R->itoi[b * R->rank + cr[c]];
    mp[key].push_back(b);
  }
  std::unordered_map<std::vector<int64_t>, int64_t, ctn::TupleHash> mpC;
  for (int64_t t = 0; t < out->nblocks; ++t)
    mpC[std::vector<int64_t>(out->itoi + t * out->rank, out->itoi + (t + 1) * out->rank)] = t;

  std::vector<std::vector<ctn::GemmPairD>> per_task(out->nblocks);
  auto prod = [](const int64_t *sh, const std::vector<int64_t> &idx) {
    int64_t v = 1;
    for (int64_t i : idx) v *= sh[i];
    return v;
  };
  for (int64_t a = 0; a < L->nblocks; ++a) {
    const int64_t *itl = L->itoi + a * L->rank;
    const int64_t *shl = L->shapes + a * L->rank;
    std::vector<int64_t> key(ncomm);
    for (int c = 0; c < ncomm; ++c) key[c] = itl[cl[c]];
    auto it = mp.find(key);
    if (it == mp.end()) continue;
    const int64_t M = prod(shl, nl), K = prod(shl, cl);
    for (int64_t b : it->second) {
      const int64_t *itr = R->itoi + b * R->rank;
      const int64_t *shr = R->shapes + b * R->rank;
      const int64_t N = prod(shr, nr), K2 = prod(shr, cr);
      CTN_REQUIRE(K == K2, "ctn_contract_plan_create: contracted dimensions differ (%lld vs %lld)",
                  (long long)K, (long long)K2);
      std::vector<int64_t> tup;
      for (int64_t i : nl) tup.push_back(itl[i]);
      for (int64_t i : nr) tup.push_back(itr[i]);
      auto jt = mpC.find(tup);
      CTN_REQUIRE(jt != mpC.end(), "ctn_contract_plan_create: target block not found");
      const int64_t t = jt->second;
      CTN_REQUIRE(M < (1ll << 31) && N < (1ll << 31) && K < (1ll << 31), "block too large");
      ctn::GemmPairD pr;
      pr.k = (int32_t)K;
      pr.flags = 0;
      if (p->sl.copy) {
        pr.a_off = p->sl.dst_offs[a];
        pr.lda = (int32_t)K;
      } else if (cls_l == 0) {
        pr.a_off = L->offs[a];
        pr.lda = (int32_t)K;
      } else {
        pr.a_off = L->offs[a];
        pr.lda = (int32_t)M;
        pr.flags |= 1;
      }
      if (p->sr.copy) {
        pr.b_off = p->sr.dst_offs[b];
        pr.ldb = (int32_t)N;
      } else if (cls_r == 0) {
        pr.b_off = R->offs[b];
        pr.ldb = (int32_t)N;
      } else {
        pr.b_off = R->offs[b];
        pr.ldb = (int32_t)K;
        pr.flags |= 2;
      }
      per_task[t].push_back(pr);
    }
  }
  for (int64_t t = 0; t < out->nblocks; ++t) {
    const int64_t *sho = out->shapes + t * out->rank;
    int64_t M = 1, N = 1;
    for (size_t i = 0; i < nl.size(); ++i) M *= sho[i];
    for (size_t i = nl.size(); i < (size_t)out->rank; ++i) N *= sho[i];
    if (M == 0 || N == 0) continue;
    ctn::GemmTaskD tk;
    tk.c_off = out->offs[t];
    tk.m = (int32_t)M;
    tk.n = (int32_t)N;
    tk.ldc = (int32_t)N;
    tk.pair_begin = (int32_t)p->gemm.pairs.size();
    tk.pair_count = (int32_t)per_task[t].size();
    tk.pad_ = 0;
    p->gemm.pairs.insert(p->gemm.pairs.end(), per_task[t].begin(), per_task[t].end());
    p->gemm.tasks.push_back(tk);
  }
  p->gemm.finalize();
  *plan = p.release();
  return CTN_OK;
}

extern "C" size_t ctn_contract_plan_scratch_bytes(const ctn_contract_plan *p) {
  return (size_t)(p->sl.elems + p->sr.elems) * sizeof(double) + 256;
}

extern "C" double ctn_contract_plan_flops(const ctn_contract_plan *p) { return p->gemm.flops; }

extern "C" ctn_status ctn_contract_execute(ctn_contract_plan *p, int dtype, const void *L, const void *R,
                                           void *out, void *scratch, void *stream) {
  CTN_REQUIRE(p, "ctn_contract_execute: null plan");
  if (dtype != CTN_FLOAT64) {
    ctn::set_error("ctn_contract_execute: dtype %d not supported on the device path (FP64 only)", dtype);
    return CTN_ERR_UNSUPPORTED;
  }
  cudaStream_t st = ctn::as_stream(stream);
  const double *A = (const double *)L;
  const double *B = (const double *)R;
  double *sc = (double *)scratch;
  if (p->sl.copy) {
    CTN_REQUIRE(scratch, "ctn_contract_execute: scratch required");
    CTN_TRY(ctn_permute_blocks(L, sc, CTN_FLOAT64, p->sl.rank, (int64_t)p->sl.src_offs.size(),
                               p->sl.old_shapes.data(), p->sl.src_offs.data(), p->sl.dst_offs.data(),
                               p->sl.mapper.data(), stream));
    A = sc;
  }
  if (p->sr.copy) {
    CTN_REQUIRE(scratch, "ctn_contract_execute: scratch required");
    double *dst = sc + p->sl.elems;
    CTN_TRY(ctn_permute_blocks(R, dst, CTN_FLOAT64, p->sr.rank, (int64_t)p->sr.src_offs.size(),
                               p->sr.old_shapes.data(), p->sr.src_offs.data(), p->sr.dst_offs.data(),
                               p->sr.mapper.data(), stream));
    B = dst;
  }
  return p->gemm.run(A, B, (double *)out, st);
}

extern "C" void ctn_contract_plan_destroy(ctn_contract_plan *p) { delete p; }

// ------------------------------------------------------------------ grouped GEMM C ABI
struct ctn_gemm_plan {
  ctn::GroupedGemmF64 g;
};

extern "C" ctn_status ctn_gemm_grouped_plan_create(int64_t ntasks, const ctn_gemm_task *tasks, int64_t npairs,
                                                   const ctn_gemm_pair *pairs, ctn_gemm_plan **plan) {
  CTN_REQUIRE(plan && ntasks >= 0 && npairs >= 0, "ctn_gemm_grouped_plan_create: bad argument");
  std::unique_ptr<ctn_gemm_plan> p(new ctn_gemm_plan());
  static_assert(sizeof(ctn_gemm_task) == sizeof(ctn::GemmTaskD), "task layout");
  static_assert(sizeof(ctn_gemm_pair) == sizeof(ctn::GemmPairD), "pair layout");
  p->g.tasks.resize(ntasks);
  p->g.pairs.resize(npairs);
  if (ntasks) std::memcpy(p->g.tasks.data(), tasks, ntasks * sizeof(ctn_gemm_task));
  if (npairs) std::memcpy(p->g.pairs.data(), pairs, npairs * sizeof(ctn_gemm_pair));
  for (const auto &t : p->g.tasks) {
    CTN_REQUIRE(t.m >= 0 && t.n >= 0 && t.ldc >= t.n && t.pair_begin >= 0 && t.pair_count >= 0 &&
                    (int64_t)t.pair_begin + t.pair_count <= npairs,
                "ctn_gemm_grouped_plan_create: invalid task");
    for (int q = 0; q < t.pair_count; ++q) {
      const auto &pr = p->g.pairs[t.pair_begin + q];
      const bool ta = pr.flags & 1, tb = pr.flags & 2;
      CTN_REQUIRE(pr.k >= 0 && pr.lda >= (ta ? t.m : pr.k) && pr.ldb >= (tb ? pr.k : t.n),
                  "ctn_gemm_grouped_plan_create: invalid pair");
    }
  }
  p->g.finalize();
  *plan = p.release();
  return CTN_OK;
}
extern "C" double ctn_gemm_grouped_plan_flops(const ctn_gemm_plan *p) { return p->g.flops; }
extern "C" ctn_status ctn_gemm_grouped_f64(ctn_gemm_plan *p, const double *A, const double *B, double *C,
                                           void *stream) {
  CTN_REQUIRE(p, "ctn_gemm_grouped_f64: null plan");
  return p->g.run(A, B, C, ctn::as_stream(stream));
}
extern "C" void ctn_gemm_grouped_plan_destroy(ctn_gemm_plan *p) { delete p; }
