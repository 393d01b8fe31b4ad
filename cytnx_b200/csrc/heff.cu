// Two-site DMRG effective-Hamiltonian matvec, planned once and run as three launches.
//
// The reference reaches this through Network::Launch (src/RegularNetwork.cpp:901-1007)
// on the network of example/DMRG/dmrg_two_sites_U1.py:25-41
//     psi[a,s1,s2,b] L[w,a,a'] M1[w,w1,s1,s1'] M2[w1,w2,s2,s2'] R[w2,b,b'] -> out[a',s1',s2',b']
// i.e. four pairwise BlockUniTensor::contract calls, each re-hashing blocks and
// issuing one GEMM (plus permute copies and temporaries) per block pair.
//
// Plan (order L -> M1 -> M2 -> R, the cheapest order):
//   step 1  X1(w,a',s1,s2,b)  = L(w,a,a')^T psi(a,s1,s2,b)        grouped GEMM, K = D_a
//   step 2+3 X3(a',w2,s1',s2',b) = sum_{w,s1,s2} C[w,s1,s2;w2,s1',s2'] X1(w,a',s1,s2,b)
//            with C = sum_w1 M1[w,w1,s1,s1'] M2[w1,w2,s2,s2'] folded on the host:
//            both MPO contractions become one bandwidth-bound linear combination of
//            D_a' x D_b matrices (one launch instead of two GEMM sweeps over K = 1 pairs)
//   step 4  out(a',s1',s2',b') = sum_{w2} X3(a',w2,s1',s2',b) R(w2,b,b')  grouped GEMM
// X1 blocks that no X3 term reads are not computed.  The MPO and physical sectors
// must have degeneracy 1 (true for the spin and Hubbard MPOs the DMRG examples use).
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <unordered_map>
#include <vector>

#include "blas1.cuh"
#include "ctn_common.h"
#include "gemm_f64.cuh"
#include "heff.cuh"
#include "tc_gemm.cuh"

namespace ctn {

namespace {
struct VecHash {
  size_t operator()(const std::vector<int64_t> &v) const {
    size_t h = 1469598103934665603ull;
    for (int64_t x : v) h ^= (size_t)x + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    return h;
  }
};
using Key = std::vector<int64_t>;

constexpr int MPO_CHUNK = 2048;

__global__ void __launch_bounds__(256) k_mpo_apply(const double *__restrict__ X1, double *__restrict__ X3,
                                                   const MpoTask *__restrict__ tasks,
                                                   const MpoTerm *__restrict__ terms,
                                                   const MpoChunk *__restrict__ chunks, int64_t nchunks) {
  // each thread owns MPO_CHUNK / 256 elements of the chunk, 256 apart; the terms run outside
  // so a term's loads for all of them are in flight together (per element the sum order over
  // the terms is unchanged)
  constexpr int PER = MPO_CHUNK / 256;
  for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const MpoChunk ch = chunks[c];
    const MpoTask tk = tasks[ch.task];
    const int64_t end = tk.size < ch.start + MPO_CHUNK ? tk.size : ch.start + MPO_CHUNK;
    const int64_t e0 = ch.start + threadIdx.x;
    double s[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) s[j] = 0.0;
    for (int t = 0; t < tk.term_count; ++t) {
      const MpoTerm tm = terms[tk.term_begin + t];
      const double *src = X1 + tm.x1_off;
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        const int64_t e = e0 + (int64_t)j * 256;
        if (e < end) s[j] = fma(tm.coef, __ldg(src + e), s[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int64_t e = e0 + (int64_t)j * 256;
      if (e < end) X3[tk.x3_off + e] = s[j];
    }
  }
}
}  // namespace

ctn_status MpoApply::upload(cudaStream_t st) {
  int dev = 0;
  CTN_CUDA(cudaGetDevice(&dev));
  if (d_mem && d_dev == dev) return CTN_OK;
  if (d_mem) cudaFree(d_mem);
  d_mem = nullptr;
  const size_t bytes = tasks.size() * sizeof(MpoTask) + terms.size() * sizeof(MpoTerm) +
                       chunks.size() * sizeof(MpoChunk) + 64;
  CTN_CUDA(cudaMalloc(&d_mem, bytes));
  d_dev = dev;
  char *p = (char *)d_mem;
  if (!tasks.empty()) CTN_CUDA(cudaMemcpyAsync(p, tasks.data(), tasks.size() * sizeof(MpoTask), cudaMemcpyHostToDevice, st));
  p += tasks.size() * sizeof(MpoTask);
  if (!terms.empty()) CTN_CUDA(cudaMemcpyAsync(p, terms.data(), terms.size() * sizeof(MpoTerm), cudaMemcpyHostToDevice, st));
  p += terms.size() * sizeof(MpoTerm);
  if (!chunks.empty()) CTN_CUDA(cudaMemcpyAsync(p, chunks.data(), chunks.size() * sizeof(MpoChunk), cudaMemcpyHostToDevice, st));
  CTN_CUDA(cudaStreamSynchronize(st));
  return CTN_OK;
}

ctn_status MpoApply::run(const double *X1, double *X3, cudaStream_t st) {
  CTN_TRY(upload(st));
  if (chunks.empty()) return CTN_OK;
  const char *p = (const char *)d_mem;
  const MpoTask *dt = (const MpoTask *)p;
  const MpoTerm *dm = (const MpoTerm *)(p + tasks.size() * sizeof(MpoTask));
  const MpoChunk *dc = (const MpoChunk *)(p + tasks.size() * sizeof(MpoTask) + terms.size() * sizeof(MpoTerm));
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int64_t grid = std::min<int64_t>((int64_t)chunks.size(), (int64_t)nsm * 8);
  k_mpo_apply<<<(unsigned)grid, 256, 0, st>>>(X1, X3, dt, dm, dc, (int64_t)chunks.size());
  CTN_CHECK_LAUNCH();
  return CTN_OK;
}

void MpoApply::finalize() {
  chunks.clear();
  bytes = 0.0;
  for (size_t t = 0; t < tasks.size(); ++t) {
    for (int64_t s = 0; s < tasks[t].size; s += MPO_CHUNK) chunks.push_back({(int32_t)t, 0, s});
    bytes += 8.0 * tasks[t].size * (1 + tasks[t].term_count);
  }
}

}  // namespace ctn

extern "C" ctn_status ctn_heff2_plan_create(const ctn_heff2_desc *d, ctn_heff2_plan **plan) {
  using namespace ctn;
  CTN_REQUIRE(d && d->psi && d->L && d->R && d->M1 && d->M2 && d->out && plan, "ctn_heff2_plan_create: null argument");
  const ctn_block_desc &P = *d->psi, &L = *d->L, &R = *d->R, &M1 = *d->M1, &M2 = *d->M2, &O = *d->out;
  CTN_REQUIRE(P.rank == 4 && L.rank == 3 && R.rank == 3 && M1.rank == 4 && M2.rank == 4 && O.rank == 4,
              "ctn_heff2_plan_create: expected psi[4] L[3] R[3] M1[4] M2[4] out[4]");
  CTN_REQUIRE(!P.perm && !L.perm && !R.perm && !M1.perm && !M2.perm && !O.perm,
              "ctn_heff2_plan_create: operands must be contiguous");
  std::unique_ptr<ctn_heff2_plan> p(new ctn_heff2_plan());
  auto blk_size = [](const ctn_block_desc &t, int64_t b) {
    int64_t s = 1;
    for (int i = 0; i < t.rank; ++i) s *= t.shapes[b * t.rank + i];
    return s;
  };
  auto total = [&](const ctn_block_desc &t) {
    int64_t m = 0;
    for (int64_t b = 0; b < t.nblocks; ++b) m = std::max(m, t.offs[b] + blk_size(t, b));
    return m;
  };
  p->psi_elems = total(P);
  p->out_elems = total(O);
  p->L_elems = total(L);
  p->R_elems = total(R);
  auto sh = [](const ctn_block_desc &t, int64_t b, int i) { return t.shapes[b * t.rank + i]; };
  auto it_ = [](const ctn_block_desc &t, int64_t b, int i) { return t.itoi[b * t.rank + i]; };
  // degeneracy-1 checks on MPO and physical legs
  for (int64_t b = 0; b < M1.nblocks; ++b)
    for (int i = 0; i < 4; ++i) CTN_REQUIRE(sh(M1, b, i) == 1, "ctn_heff2: MPO sectors must have degeneracy 1");
  for (int64_t b = 0; b < M2.nblocks; ++b)
    for (int i = 0; i < 4; ++i) CTN_REQUIRE(sh(M2, b, i) == 1, "ctn_heff2: MPO sectors must have degeneracy 1");
  for (int64_t b = 0; b < P.nblocks; ++b)
    CTN_REQUIRE(sh(P, b, 1) == 1 && sh(P, b, 2) == 1, "ctn_heff2: physical sectors must have degeneracy 1");
  for (int64_t b = 0; b < L.nblocks; ++b) CTN_REQUIRE(sh(L, b, 0) == 1, "ctn_heff2: MPO sectors must have degeneracy 1");
  for (int64_t b = 0; b < R.nblocks; ++b) CTN_REQUIRE(sh(R, b, 0) == 1, "ctn_heff2: MPO sectors must have degeneracy 1");

  auto info = [&](const ctn_block_desc &t, std::vector<BlkInfo> &v) {
    for (int64_t b = 0; b < t.nblocks; ++b) {
      BlkInfo bi{};
      for (int i = 0; i < t.rank && i < 4; ++i) {
        bi.q[i] = t.itoi[b * t.rank + i];
        bi.d[i] = t.shapes[b * t.rank + i];
      }
      bi.off = t.offs[b];
      v.push_back(bi);
    }
  };
  info(L, p->Lb);
  info(P, p->Pb);
  info(R, p->Rb);
  info(O, p->Ob);
  // MPO scalars by tuple
  std::unordered_map<Key, double, VecHash> m1v, m2v;
  for (int64_t b = 0; b < M1.nblocks; ++b)
    m1v[Key(M1.itoi + b * 4, M1.itoi + b * 4 + 4)] = d->M1_host[M1.offs[b]];
  for (int64_t b = 0; b < M2.nblocks; ++b)
    m2v[Key(M2.itoi + b * 4, M2.itoi + b * 4 + 4)] = d->M2_host[M2.offs[b]];
  // w1 index range (M1 leg 1 / M2 leg 0)
  int64_t nw1 = 0;
  for (int64_t b = 0; b < M1.nblocks; ++b) nw1 = std::max(nw1, it_(M1, b, 1) + 1);

  // L blocks grouped by a ; psi blocks grouped by a
  std::map<int64_t, std::vector<int64_t>> L_by_a, P_by_a;
  for (int64_t b = 0; b < L.nblocks; ++b) L_by_a[it_(L, b, 1)].push_back(b);
  for (int64_t b = 0; b < P.nblocks; ++b) P_by_a[it_(P, b, 0)].push_back(b);
  // candidate X1 blocks (w,a',s1,s2,b) -> (L block, psi block)
  struct X1c {
    int64_t l, p;
  };
  std::unordered_map<Key, X1c, VecHash> x1cand;
  std::unordered_map<Key, std::vector<Key>, VecHash> x1_by_ab;  // (a', b) -> list of X1 keys
  for (auto &kv : L_by_a) {
    auto jt = P_by_a.find(kv.first);
    if (jt == P_by_a.end()) continue;
    for (int64_t l : kv.second)
      for (int64_t q : jt->second) {
        Key k = {it_(L, l, 0), it_(L, l, 2), it_(P, q, 1), it_(P, q, 2), it_(P, q, 3)};
        x1cand[k] = {l, q};
        x1_by_ab[Key{k[1], k[4]}].push_back(k);
      }
  }
  for (auto &kv : x1_by_ab) std::sort(kv.second.begin(), kv.second.end());
  // step 4 pairs: out block o=(a',s1',s2',b') with R blocks r=(w2,b,b')
  std::map<int64_t, std::vector<int64_t>> R_by_bp;
  for (int64_t b = 0; b < R.nblocks; ++b) R_by_bp[it_(R, b, 2)].push_back(b);
  std::map<Key, int64_t> x3_off;  // X3 key (a',w2,s1',s2',b) -> offset (ordered for determinism)
  std::vector<Key> x3_keys;
  std::vector<int64_t> x3_rows, x3_cols;
  std::map<Key, int64_t> x1_off;
  std::vector<Key> x1_keys;
  std::vector<std::vector<GemmPairD>> out_pairs(O.nblocks);
  std::vector<MpoTask> mtasks;
  std::vector<MpoTerm> mterms;
  std::vector<std::vector<std::pair<Key, double>>> x3_terms;
  std::vector<std::pair<int64_t, int64_t>> x3_or;
  for (int64_t o = 0; o < O.nblocks; ++o) {
    const int64_t ap = it_(O, o, 0), s1p = it_(O, o, 1), s2p = it_(O, o, 2), bp = it_(O, o, 3);
    CTN_REQUIRE(sh(O, o, 1) == 1 && sh(O, o, 2) == 1, "ctn_heff2: physical sectors must have degeneracy 1");
    auto rt = R_by_bp.find(bp);
    if (rt == R_by_bp.end()) continue;
    for (int64_t r : rt->second) {
      const int64_t w2 = it_(R, r, 0), bb = it_(R, r, 1);
      Key xk = {ap, w2, s1p, s2p, bb};
      auto xt = x3_off.find(xk);
      if (xt == x3_off.end()) {
        // build terms for this X3 block
        std::vector<std::pair<Key, double>> terms;
        auto lt = x1_by_ab.find(Key{ap, bb});
        if (lt != x1_by_ab.end()) {
          for (const Key &k1 : lt->second) {
            const int64_t w = k1[0], s1 = k1[2], s2 = k1[3];
            double c = 0.0;
            for (int64_t w1 = 0; w1 < nw1; ++w1) {
              auto a1 = m1v.find(Key{w, w1, s1, s1p});
              if (a1 == m1v.end()) continue;
              auto a2 = m2v.find(Key{w1, w2, s2, s2p});
              if (a2 == m2v.end()) continue;
              c += a1->second * a2->second;
            }
            if (c != 0.0) terms.push_back({k1, c});
          }
        }
        if (terms.empty()) continue;  // X3 block identically zero: contributes nothing
        const int64_t rows = sh(O, o, 0), cols = sh(R, r, 1);
        x3_off[xk] = p->x3_elems;
        xt = x3_off.find(xk);
        x3_keys.push_back(xk);
        x3_rows.push_back(rows);
        x3_cols.push_back(cols);
        MpoTask mt;
        mt.x3_off = p->x3_elems;
        mt.size = rows * cols;
        mt.term_begin = (int32_t)mterms.size();
        mt.term_count = (int32_t)terms.size();
        for (auto &tm : terms) {
          auto ot = x1_off.find(tm.first);
          if (ot == x1_off.end()) {
            x1_off[tm.first] = -1;  // placeholder, offsets assigned below
            x1_keys.push_back(tm.first);
          }
          MpoTerm term;
          term.x1_off = -1;
          term.coef = tm.second;
          mterms.push_back(term);
        }
        x3_terms.push_back(terms);
        x3_or.push_back({o, r});
        mtasks.push_back(mt);
        p->x3_elems += rows * cols;
      }
      GemmPairD pr;
      pr.a_off = xt->second;
      pr.b_off = R.offs[r];
      pr.k = (int32_t)sh(R, r, 1);
      pr.lda = (int32_t)sh(R, r, 1);
      pr.ldb = (int32_t)sh(R, r, 2);
      pr.flags = 0;
      out_pairs[o].push_back(pr);
    }
  }
  // X1 layout + step-1 tasks (only X1 blocks that some X3 term reads)
  std::sort(x1_keys.begin(), x1_keys.end());
  // L staging table [a][w][a']
  {
    int64_t off = 0;
    for (int64_t b = 0; b < L.nblocks; ++b) {
      for (int i = 0; i < 3; ++i) p->L_shapes.push_back((uint64_t)sh(L, b, i));
      p->L_src.push_back(L.offs[b]);
      p->L_dst.push_back(off);
      off += blk_size(L, b);
    }
  }
  for (const Key &k : x1_keys) {
    const X1c c = x1cand.at(k);
    const int64_t M = sh(L, c.l, 0) * sh(L, c.l, 2);
    const int64_t N = sh(P, c.p, 1) * sh(P, c.p, 2) * sh(P, c.p, 3);
    const int64_t K = sh(L, c.l, 1);
    x1_off[k] = p->x1_elems;
    GemmTaskD tk;
    tk.c_off = p->x1_elems;
    tk.m = (int32_t)M;
    tk.n = (int32_t)N;
    tk.ldc = (int32_t)N;
    tk.pair_begin = (int32_t)p->g1.pairs.size();
    tk.pair_count = 1;
    tk.pad_ = 0;
    GemmPairD pr;
    pr.a_off = p->L_dst[c.l];
    pr.b_off = P.offs[c.p];
    pr.k = (int32_t)K;
    pr.lda = (int32_t)M;  // staged [a][w a'] = A^T
    pr.ldb = (int32_t)N;
    pr.flags = 1;
    p->g1.pairs.push_back(pr);
    p->g1.tasks.push_back(tk);
    p->x1_elems += M * N;
  }
  // resolve term offsets
  {
    size_t ti = 0;
    for (auto &terms : x3_terms)
      for (auto &tm : terms) mterms[ti++].x1_off = x1_off.at(tm.first);
  }
  {
    std::map<Key, int64_t> x1_index;
    for (size_t i = 0; i < x1_keys.size(); ++i) {
      x1_index[x1_keys[i]] = (int64_t)i;
      const X1c c = x1cand.at(x1_keys[i]);
      p->x1_lp.push_back({c.l, c.p});
    }
    for (size_t j = 0; j < x3_terms.size(); ++j) {
      X3Info xi;
      xi.o = x3_or[j].first;
      xi.r = x3_or[j].second;
      xi.rows = sh(O, xi.o, 0);
      xi.cols = sh(R, xi.r, 1);
      for (auto &tm : x3_terms[j]) xi.terms.push_back({x1_index.at(tm.first), tm.second});
      p->x3.push_back(std::move(xi));
    }
  }
  p->mpo.tasks = std::move(mtasks);
  p->mpo.terms = std::move(mterms);
  p->mpo.finalize();
  // step-4 tasks: one per out block
  for (int64_t o = 0; o < O.nblocks; ++o) {
    GemmTaskD tk;
    tk.c_off = O.offs[o];
    tk.m = (int32_t)sh(O, o, 0);
    tk.n = (int32_t)(sh(O, o, 1) * sh(O, o, 2) * sh(O, o, 3));
    tk.ldc = tk.n;
    tk.pair_begin = (int32_t)p->g4.pairs.size();
    tk.pair_count = (int32_t)out_pairs[o].size();
    tk.pad_ = 0;
    for (auto &pr : out_pairs[o]) p->g4.pairs.push_back(pr);
    if (tk.m > 0 && tk.n > 0) p->g4.tasks.push_back(tk);
  }
  p->g1.finalize();
  p->g4.finalize();
  p->gemm_flops = p->g1.flops + p->g4.flops;
  p->n_x1 = (int64_t)x1_keys.size();
  p->n_x3 = (int64_t)x3_keys.size();
  *plan = p.release();
  return CTN_OK;
}

extern "C" double ctn_heff2_flops(const ctn_heff2_plan *p) {
  return p->gemm_flops + 2.0 * [&] {
    double t = 0;
    for (auto &tk : p->mpo.tasks) t += (double)tk.size * tk.term_count;
    return t;
  }();
}
extern "C" size_t ctn_heff2_psi_elems(const ctn_heff2_plan *p) { return (size_t)p->psi_elems; }

static int split_kind(int precision) { return precision == CTN_PREC_BF16X3 ? ctn::TC_BF16 : ctn::TC_TF32; }

extern "C" size_t ctn_heff2_workspace_bytes(const ctn_heff2_plan *p, int precision) {
  if (precision == CTN_PREC_F64) return (size_t)(p->L_elems + p->x1_elems + p->x3_elems) * sizeof(double) + 256;
  if (precision != CTN_PREC_3XTF32 && precision != CTN_PREC_BF16X3) return 0;
  auto *pp = const_cast<ctn_heff2_plan *>(p);
  if (ctn::heff_split_prepare(pp, split_kind(precision)) != CTN_OK) return 0;
  return ctn::heff_split_ws_bytes(p, split_kind(precision));
}

extern "C" ctn_status ctn_heff2_set_env(ctn_heff2_plan *p, const double *L, const double *R, void *workspace,
                                        int precision, void *stream) {
  CTN_REQUIRE(p && L && R && workspace, "ctn_heff2_set_env: null argument");
  if (precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3) {
    const int k = split_kind(precision);
    CTN_TRY(ctn::heff_split_prepare(p, k));
    CTN_TRY(ctn::heff_split_set_env(p, k, L, R, workspace, ctn::as_stream(stream)));
    p->split_bound[k] = true;
    return CTN_OK;
  }
  CTN_REQUIRE(precision == CTN_PREC_F64, "ctn_heff2_set_env: unknown precision %d", precision);
  const uint64_t mapper[3] = {1, 0, 2};
  p->ws = (double *)workspace;
  CTN_TRY(ctn_permute_blocks(L, p->ws, CTN_FLOAT64, 3, (int64_t)p->L_src.size(), p->L_shapes.data(),
                             p->L_src.data(), p->L_dst.data(), mapper, stream));
  p->R = R;
  p->bound = true;
  return CTN_OK;
}

extern "C" ctn_status ctn_heff2_matvec(ctn_heff2_plan *p, const double *psi, double *out, int precision,
                                       void *stream) {
  CTN_REQUIRE(p, "ctn_heff2_matvec: null plan");
  cudaStream_t st = ctn::as_stream(stream);
  if (precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3) {
    const int k = split_kind(precision);
    CTN_REQUIRE(p->split_bound[k], "ctn_heff2_matvec: environments not bound for this precision (ctn_heff2_set_env)");
    return ctn::heff_split_matvec(p, k, psi, out, st, nullptr);
  }
  CTN_REQUIRE(precision == CTN_PREC_F64, "ctn_heff2_matvec: unknown precision %d", precision);
  CTN_REQUIRE(p->bound, "ctn_heff2_matvec: environments not bound (call ctn_heff2_set_env)");
  double *Lt = p->ws;
  double *X1 = Lt + p->L_elems;
  double *X3 = X1 + p->x1_elems;
  CTN_TRY(p->g1.run(Lt, psi, X1, st));
  CTN_TRY(p->mpo.run(X1, X3, st));
  CTN_TRY(p->g4.run(X3, p->R, out, st));
  return CTN_OK;
}

extern "C" void ctn_heff2_plan_destroy(ctn_heff2_plan *p) { delete p; }

extern "C" ctn_status ctn_heff2_set_tiles(ctn_heff2_plan *p, int precision, int bn_step1, int bn_step4) {
  CTN_REQUIRE(p, "ctn_heff2_set_tiles: null plan");
  CTN_REQUIRE(precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3, "ctn_heff2_set_tiles: split precision only");
  CTN_REQUIRE(ctn::tc_tile_width_supported(bn_step1) && ctn::tc_tile_width_supported(bn_step4),
              "ctn_heff2_set_tiles: tile widths must be one of 32, 48, 64, 96, 128, 144, 160, 192, 256 "
              "or -128, -192, -256 (2-CTA tiles)");
  const int k = split_kind(precision);
  if (p->split_bn[k][0] == bn_step1 && p->split_bn[k][1] == bn_step4) return CTN_OK;
  p->split_bn[k][0] = bn_step1;
  p->split_bn[k][1] = bn_step4;
  ctn::heff_split_free(p->split[k]);
  p->split[k] = nullptr;
  p->split_bound[k] = false;  // the panels depend on the tile widths: bind again
  return CTN_OK;
}

extern "C" ctn_status ctn_heff2_set_epilogue(ctn_heff2_plan *p, int precision, int epi_step1, int epi_step4) {
  CTN_REQUIRE(p, "ctn_heff2_set_epilogue: null plan");
  CTN_REQUIRE(precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3,
              "ctn_heff2_set_epilogue: split precision only");
  CTN_REQUIRE(epi_step1 >= -1 && epi_step1 <= 2 && epi_step4 >= -1 && epi_step4 <= 2,
              "ctn_heff2_set_epilogue: -1 (automatic), 0 (direct), 1 (staged) or 2 (fragments)");
  const int k = split_kind(precision);
  p->split_epi[k][0] = epi_step1;
  p->split_epi[k][1] = epi_step4;
  ctn::heff_split_apply_epilogue(p, k);  // the panels do not depend on it: no rebind
  return CTN_OK;
}

namespace {
struct HeffUser {
  ctn_heff2_plan *plan;
  int precision;
};
int heff_mv(void *u, const double *x, double *y, void *stream) {
  HeffUser *h = (HeffUser *)u;
  return ctn_heff2_matvec(h->plan, x, y, h->precision, stream) == CTN_OK ? 0 : 1;
}
// split-precision matvec with its result rounded to FP32 into y (n floats)
int heff_mv_f32(void *u, const double *x, double *y, void *stream) {
  HeffUser *h = (HeffUser *)u;
  return ctn::heff_split_matvec_f32out(h->plan, split_kind(h->precision), x, reinterpret_cast<float *>(y),
                                       ctn::as_stream(stream)) == CTN_OK
             ? 0
             : 1;
}
}  // namespace

extern "C" ctn_status ctn_heff2_lanczos_gnd(ctn_heff2_plan *plan, int precision, const double *psi0, int maxiter,
                                            double cvgcrit, double *krylov, double *work, double *eigvec,
                                            double *energy, int *iters, void *stream) {
  CTN_REQUIRE(plan && psi0 && krylov && work && eigvec && energy && iters, "ctn_heff2_lanczos_gnd: null argument");
  HeffUser u{plan, precision};
  // split-precision matvecs hand their result over in FP32 (the matvec's own error is far above it)
  const bool split = precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3;
  if (split)
    CTN_REQUIRE(plan->split_bound[split_kind(precision)],
                "ctn_heff2_lanczos_gnd: environments not bound for this precision (ctn_heff2_set_env)");
  return ctn::lanczos_gnd(split ? heff_mv_f32 : heff_mv, &u, psi0, plan->psi_elems, maxiter, cvgcrit, krylov, work,
                          eigvec, energy, iters, ctn::as_stream(stream), /*speculate=*/true, /*w_f32=*/split);
}

extern "C" ctn_status ctn_heff2_lanczos_refined(ctn_heff2_plan *plan, int precision, const double *psi0, int krydim,
                                                int max_restarts, double tol, double *krylov, double *work,
                                                double *eigvec, double *energy, double *residual, int *restarts,
                                                int64_t *matvecs, void *stream) {
  CTN_REQUIRE(plan && plan->bound, "ctn_heff2_lanczos_refined: the FP64 environments must be bound (ctn_heff2_set_env "
                                   "with CTN_PREC_F64) for the refinement matvecs");
  HeffUser lo{plan, precision}, hi{plan, CTN_PREC_F64};
  // split-precision Krylov steps take the matvec result in FP32 (half the bytes through the
  // step-4 epilogue and the two vector passes that read it)
  const bool split = precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3;
  if (split)
    CTN_REQUIRE(plan->split_bound[split_kind(precision)],
                "ctn_heff2_lanczos_refined: environments not bound for this precision (ctn_heff2_set_env)");
  CTN_REQUIRE(psi0 && krylov && work && eigvec && energy, "ctn_heff2_lanczos_refined: null argument");
  return ctn::lanczos_refined(split ? heff_mv_f32 : heff_mv, &lo, heff_mv, &hi, psi0, plan->psi_elems, krydim,
                              max_restarts, tol, krylov, work, eigvec, energy, residual, restarts, matvecs,
                              ctn::as_stream(stream), /*w_f32=*/split);
}

// median of per-repetition phase times: a repetition that the host was slow to launch (the
// first phase of each repetition holds the launch latency) does not move it
static double median_of(std::vector<double> v) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const size_t n = v.size();
  return n % 2 ? v[n / 2] : 0.5 * (v[n / 2 - 1] + v[n / 2]);
}

extern "C" ctn_status ctn_heff2_profile(ctn_heff2_plan *p, const double *psi, double *out, int precision, int reps,
                                        double *ms_out, int *launches_out, void *stream) {
  CTN_REQUIRE(p && reps > 0 && ms_out, "ctn_heff2_profile: bad argument");
  cudaStream_t st = ctn::as_stream(stream);
  if (precision == CTN_PREC_3XTF32 || precision == CTN_PREC_BF16X3) {
    const int k = split_kind(precision);
    CTN_REQUIRE(p->split_bound[k], "ctn_heff2_profile: environments not bound for this precision");
    std::vector<double> t[4];
    CTN_TRY(ctn::heff_split_matvec(p, k, psi, out, st, nullptr));  // warm
    for (int r = 0; r < reps; ++r) {
      double one[4] = {0, 0, 0, 0};
      CTN_TRY(ctn::heff_split_matvec(p, k, psi, out, st, one));
      for (int i = 0; i < 4; ++i) t[i].push_back(one[i]);
    }
    for (int i = 0; i < 4; ++i) ms_out[i] = median_of(t[i]);
    if (launches_out) *launches_out = 4;
    return CTN_OK;
  }
  CTN_REQUIRE(p->bound, "ctn_heff2_profile: environments not bound");
  double *Lt = p->ws;
  double *X1 = Lt + p->L_elems;
  double *X3 = X1 + p->x1_elems;
  // warm the table uploads outside the timed region
  CTN_TRY(p->g1.upload(st));
  CTN_TRY(p->mpo.upload(st));
  CTN_TRY(p->g4.upload(st));
  cudaEvent_t ev[4];
  for (auto &e : ev) CTN_CUDA(cudaEventCreate(&e));
  std::vector<double> acc[3];
  for (int r = 0; r < reps; ++r) {
    CTN_CUDA(cudaEventRecord(ev[0], st));
    CTN_TRY(p->g1.run(Lt, psi, X1, st));
    CTN_CUDA(cudaEventRecord(ev[1], st));
    CTN_TRY(p->mpo.run(X1, X3, st));
    CTN_CUDA(cudaEventRecord(ev[2], st));
    CTN_TRY(p->g4.run(X3, p->R, out, st));
    CTN_CUDA(cudaEventRecord(ev[3], st));
    CTN_CUDA(cudaEventSynchronize(ev[3]));
    for (int k = 0; k < 3; ++k) {
      float ms = 0.f;
      CTN_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      acc[k].push_back(ms);
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  ms_out[0] = 0.0;
  for (int k = 0; k < 3; ++k) ms_out[k + 1] = median_of(acc[k]);
  if (launches_out) *launches_out = 3;
  return CTN_OK;
}

extern "C" double ctn_heff2_gemm_flops(const ctn_heff2_plan *p, int step) {
  return step == 1 ? p->g1.flops : step == 4 ? p->g4.flops : 0.0;
}

extern "C" ctn_status ctn_heff2_split_stats(ctn_heff2_plan *p, int precision, double *out) {
  CTN_REQUIRE(p && out, "ctn_heff2_split_stats: null argument");
  const int k = split_kind(precision);
  CTN_TRY(ctn::heff_split_prepare(p, k));
  return ctn::heff_split_stats(p, k, out);
}
extern "C" double ctn_heff2_split_gemm_flops(ctn_heff2_plan *p, int precision, int step) {
  const int k = split_kind(precision);
  if (ctn::heff_split_prepare(p, k) != CTN_OK) return 0.0;
  return ctn::heff_split_gemm_flops(p, k, step);
}
