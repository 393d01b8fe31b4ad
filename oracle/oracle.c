/*
 * CPU oracle for the cytnx tensor-network hot path.  TEST INFRASTRUCTURE ONLY:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * this library, and only as the checker / the timed CPU restatement.  The
 * product (cytnx_b200) never calls it.
 *
 * Each function restates the reference's CPU algorithm, citing the file:line it
 * follows (paths relative to the Cytnx source tree):
 *
 *   orc_permute          src/backend/utils_internal_cpu/Movemem_cpu.cpp:152-191
 *                        (the non-HPTT odometer loop; HPTT is not vendored)
 *   orc_blocks_enumerate src/BlockUniTensor.cpp:190-230 (lexicographic odometer)
 *                        include/UniTensor.hpp:1139-1165 (_fx_get_total_fluxs)
 *                        src/Symmetry.cpp:33-50 (U1), :64-108 (Zn)
 *   orc_bs_contract      src/BlockUniTensor.cpp:1180-1223 (non-MKL branch of
 *                        BlockUniTensor::contract): per left block a permuted to
 *                        [noncomm, comm]; right blocks hashed by their common
 *                        qnum indices (:994-1006), permuted to [comm, noncomm];
 *                        out[targ] += Lmat * Rmat via dgemm/zgemm with the
 *                        row-major trick of src/backend/linalg_internal_cpu/
 *                        Matmul_internal.cpp:49-60.
 *
 * BLAS comes from the container's OpenBLAS (scipy's bundled build); the Python
 * wrapper injects the dgemm/zgemm symbols through orc_set_blas().
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>

typedef void (*dgemm_fn)(const char *, const char *, const int *, const int *, const int *,
                         const double *, const double *, const int *, const double *, const int *,
                         const double *, double *, const int *);
typedef void (*zgemm_fn)(const char *, const char *, const int *, const int *, const int *,
                         const void *, const void *, const int *, const void *, const int *,
                         const void *, void *, const int *);

static dgemm_fn g_dgemm = 0;
static zgemm_fn g_zgemm = 0;

void orc_set_blas(void *dgemm, void *zgemm) {
  g_dgemm = (dgemm_fn)dgemm;
  g_zgemm = (zgemm_fn)zgemm;
}

/* Movemem_cpu.cpp:152-191.  des[sum_j shifter_new[j] * old_idx[mapper[j]]] = src[n],
 * walking src in row-major order with an odometer over old_shape. */
int orc_permute(const void *src_, void *des_, int64_t esize, int rank, const uint64_t *old_shape,
                const uint64_t *mapper, const uint64_t *invmapper) {
  const char *src = (const char *)src_;
  char *des = (char *)des_;
  int64_t newshape[16], shifter_new[16], old_inds[16];
  int64_t accu_old = 1, accu_new = 1;
  if (rank > 16) return 1;
  if (rank == 0) {
    memcpy(des, src, esize);
    return 0;
  }
  for (int i = 0; i < rank; i++) newshape[i] = old_shape[mapper[i]];
  for (int i = rank - 1; i >= 0; i--) {
    shifter_new[i] = accu_new;
    accu_old *= old_shape[i];
    accu_new *= newshape[i];
  }
  for (int i = 0; i < rank; i++) old_inds[i] = 0;
  int64_t new_loc = 0;
  for (int64_t n = 0; n < accu_old; n++) {
    int recalc = 0;
    for (int i = rank - 1; i >= 0; i--) {
      if (old_inds[i] >= (int64_t)old_shape[i]) {
        recalc = 1;
        old_inds[i - 1]++;
        old_inds[i] = 0;
      } else
        break;
    }
    if (recalc) {
      new_loc = 0;
      for (int j = 0; j < rank; j++) new_loc += shifter_new[j] * old_inds[mapper[j]];
    } else {
      if (n != 0) new_loc += shifter_new[invmapper[rank - 1]];
    }
    if (esize == 8)
      ((uint64_t *)des)[new_loc] = ((const uint64_t *)src)[n];
    else
      memcpy(des + new_loc * esize, src + n * esize, esize);
    old_inds[rank - 1]++;
  }
  return 0;
}

/* Symmetry.cpp:33-50 (U1: combine = add, reverse = negate) and :64-108
 * (Zn: combine = (a+b) mod n, reverse = (n - q) mod n).  stype -1 = U1, 0 = Zn
 * (include/Symmetry.hpp:30). */
static int64_t sym_combine(int stype, int64_t n, int64_t a, int64_t b) {
  if (stype == 0) return (a + b) % n;
  return a + b;
}
static int64_t sym_reverse(int stype, int64_t n, int64_t a) {
  if (stype == 0) return (n - a) % n;
  return -a;
}

/* BlockUniTensor.cpp:190-230 with the flux rule of UniTensor.hpp:1139-1165.
 * qnums[i] points at bond i's table [nq_i][nsym]; bond_types: -1 ket, +1 bra.
 * Writes the qnum-index tuples of all allowed blocks (last leg fastest) into
 * out_itoi (capacity tuples); returns the block count (or -1 on overflow). */
int64_t orc_blocks_enumerate(int rank, int nsym, const int32_t *stype, const int64_t *symn,
                             const int32_t *bond_types, const int64_t *nqs,
                             const int64_t *const *qnums, int64_t *out_itoi, int64_t capacity) {
  int64_t loc[32];
  int64_t count = 0;
  if (rank <= 0 || rank > 32) return -1;
  for (int i = 0; i < rank; i++) {
    loc[i] = 0;
    if (nqs[i] <= 0) return 0;
  }
  for (;;) {
    int ok = 1;
    for (int s = 0; s < nsym && ok; s++) {
      int64_t tot;
      int64_t q0 = qnums[0][loc[0] * nsym + s];
      tot = (bond_types[0] == 1) ? sym_reverse(stype[s], symn[s], q0) : q0;
      for (int j = 1; j < rank; j++) {
        int64_t q = qnums[j][loc[j] * nsym + s];
        if (bond_types[j] == 1) q = sym_reverse(stype[s], symn[s], q);
        tot = sym_combine(stype[s], symn[s], tot, q);
      }
      if (tot != 0) ok = 0;
    }
    if (ok) {
      if (count >= capacity) return -1;
      for (int i = 0; i < rank; i++) out_itoi[count * rank + i] = loc[i];
      count++;
    }
    /* odometer: advance the last leg; carry leftwards */
    int i = rank - 1;
    while (i >= 0) {
      if (loc[i] == nqs[i] - 1) {
        loc[i] = 0;
        i--;
      } else {
        loc[i]++;
        break;
      }
    }
    if (i < 0) break;
  }
  return count;
}

/* A block-sparse tensor as seen by the oracle: blocks stored contiguously
 * (row-major in their logical leg order) at element offsets into data. */
typedef struct {
  int rank;
  int64_t nblocks;
  const int64_t *itoi;   /* [nblocks][rank] */
  const int64_t *shapes; /* [nblocks][rank] */
  const int64_t *offs;   /* [nblocks] */
} orc_layout;

static int tuple_eq(const int64_t *a, const int64_t *b, int n) {
  for (int i = 0; i < n; i++)
    if (a[i] != b[i]) return 0;
  return 1;
}

static uint64_t tuple_hash(const int64_t *a, int n) {
  uint64_t h = 1469598103934665603ull;
  for (int i = 0; i < n; i++) {
    h ^= (uint64_t)a[i] + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
  }
  return h;
}

/* open-addressing table: tuple -> block index (mpC of BlockUniTensor.cpp:1003-1006) */
typedef struct {
  int64_t cap;
  int64_t *slot; /* block index or -1 */
} tmap;

static void tmap_build(tmap *m, const int64_t *itoi, int64_t nb, int rank) {
  m->cap = 16;
  while (m->cap < 2 * nb + 16) m->cap <<= 1;
  m->slot = (int64_t *)malloc(sizeof(int64_t) * m->cap);
  for (int64_t i = 0; i < m->cap; i++) m->slot[i] = -1;
  for (int64_t b = 0; b < nb; b++) {
    uint64_t h = tuple_hash(itoi + b * rank, rank) & (m->cap - 1);
    while (m->slot[h] >= 0) h = (h + 1) & (m->cap - 1);
    m->slot[h] = b;
  }
}

static int64_t tmap_find(const tmap *m, const int64_t *itoi, int rank, const int64_t *key) {
  uint64_t h = tuple_hash(key, rank) & (m->cap - 1);
  while (m->slot[h] >= 0) {
    if (tuple_eq(itoi + m->slot[h] * rank, key, rank)) return m->slot[h];
    h = (h + 1) & (m->cap - 1);
  }
  return -1;
}

/* dtype: 3 = float64, 1 = complex128 (reference dtype ids).
 * Pair sampling (for bounded CPU timings): the block pairs are numbered in the order the
 * loops below meet them; with stride >= 1 only pairs p with p % stride == offset are
 * multiplied (stride 1: every pair, the reference's contract), and the output is cleared
 * only when offset == 0.  stride <= 0 counts without computing or touching Odata.
 * *flops (if not NULL) receives 2*M*N*K summed over the pairs taken. */
int orc_bs_contract_ex(int dtype, orc_layout L, const void *Ldata, orc_layout R, const void *Rdata,
                       int ncomm, const int64_t *comm1, const int64_t *comm2, orc_layout O,
                       void *Odata, int64_t stride, int64_t offset, double *flops) {
  const int64_t es = (dtype == 1) ? 16 : 8;
  int rl = L.rank, rr = R.rank;
  int ncl = rl - ncomm, ncr = rr - ncomm;
  int64_t nonc1[32], nonc2[32];
  uint64_t mapL[32], invL[32], mapR[32], invR[32];
  if (rl > 32 || rr > 32) return 1;
  if ((dtype == 3 && !g_dgemm) || (dtype == 1 && !g_zgemm)) return 2;
  /* non_comm_idx = vec_erase(range(rank), comm_idx) (BlockUniTensor.cpp:884-885) */
  {
    int c = 0;
    for (int i = 0; i < rl; i++) {
      int isc = 0;
      for (int k = 0; k < ncomm; k++) isc |= (comm1[k] == i);
      if (!isc) nonc1[c++] = i;
    }
    c = 0;
    for (int i = 0; i < rr; i++) {
      int isc = 0;
      for (int k = 0; k < ncomm; k++) isc |= (comm2[k] == i);
      if (!isc) nonc2[c++] = i;
    }
  }
  /* mapperL = non_comm_idx1 ++ comm_idx1 ; mapperR = comm_idx2 ++ non_comm_idx2 (:1024-1026) */
  for (int i = 0; i < ncl; i++) mapL[i] = nonc1[i];
  for (int i = 0; i < ncomm; i++) mapL[ncl + i] = comm1[i];
  for (int i = 0; i < ncomm; i++) mapR[i] = comm2[i];
  for (int i = 0; i < ncr; i++) mapR[ncomm + i] = nonc2[i];
  for (int i = 0; i < rl; i++) invL[mapL[i]] = i;
  for (int i = 0; i < rr; i++) invR[mapR[i]] = i;

  const int count_only = stride <= 0;
  double fl = 0.0;
  int64_t pair = -1;
  /* Init() allocates every output block as zeros (BlockUniTensor.cpp:213-216). */
  if (!count_only && offset == 0) {
    int64_t tot = 0;
    for (int64_t b = 0; b < O.nblocks; b++) {
      int64_t sz = 1;
      for (int i = 0; i < O.rank; i++) sz *= O.shapes[b * O.rank + i];
      int64_t end = O.offs[b] + sz;
      if (end > tot) tot = end;
    }
    memset(Odata, 0, tot * es);
  }

  tmap mpC;
  tmap_build(&mpC, O.itoi, O.nblocks, O.rank);
  char *Lbuf = 0, *Rbuf = 0;
  int64_t lcap = 0, rcap = 0;
  int64_t ktup[32], gbuf[64];
  for (int64_t a = 0; a < L.nblocks; a++) {
    const int64_t *itl = L.itoi + a * rl;
    const int64_t *shl = L.shapes + a * rl;
    int64_t comm_dim = 1, lsz = 1;
    for (int k = 0; k < ncomm; k++) comm_dim *= shl[comm1[k]];
    for (int i = 0; i < rl; i++) lsz *= shl[i];
    if (!count_only && lsz > lcap) {
      free(Lbuf);
      Lbuf = (char *)malloc(lsz * es);
      lcap = lsz;
    }
    /* Lmat = block[a].permute(mapperL).reshape({-1, comm_dim}) */
    uint64_t oshape[32];
    for (int i = 0; i < rl; i++) oshape[i] = shl[i];
    /* Lmat is built up front like the reference; a sampled call builds it on the first
     * pair it takes for this left block */
    int l_done = 0;
    if (!count_only && stride <= 1) {
      orc_permute((const char *)Ldata + L.offs[a] * es, Lbuf, es, rl, oshape, mapL, invL);
      l_done = 1;
    }
    int64_t mrows = comm_dim ? lsz / comm_dim : 0;
    for (int k = 0; k < ncomm; k++) ktup[k] = itl[comm1[k]];
    /* right blocks whose common qindices match, in ascending b (the hash-map push order) */
    for (int64_t b = 0; b < R.nblocks; b++) {
      const int64_t *itr = R.itoi + b * rr;
      int match = 1;
      for (int k = 0; k < ncomm && match; k++) match = (itr[comm2[k]] == ktup[k]);
      if (!match) continue;
      const int64_t *shr = R.shapes + b * rr;
      int64_t rsz = 1;
      for (int i = 0; i < rr; i++) rsz *= shr[i];
      ++pair;
      const int take = count_only || stride <= 1 || (pair % stride) == offset;
      if (!take) continue;
      if (count_only) {
        const int64_t nc = comm_dim ? rsz / comm_dim : 0;
        if (mrows && nc && comm_dim) fl += 2.0 * (double)mrows * (double)nc * (double)comm_dim;
        continue;
      }
      if (!l_done) {
        orc_permute((const char *)Ldata + L.offs[a] * es, Lbuf, es, rl, oshape, mapL, invL);
        l_done = 1;
      }
      if (rsz > rcap) {
        free(Rbuf);
        Rbuf = (char *)malloc(rsz * es);
        rcap = rsz;
      }
      uint64_t rshape[32];
      for (int i = 0; i < rr; i++) rshape[i] = shr[i];
      orc_permute((const char *)Rdata + R.offs[b] * es, Rbuf, es, rr, rshape, mapR, invR);
      int64_t ncols = comm_dim ? rsz / comm_dim : 0;
      /* Lgbuffer: output qindex tuple = nonc of a ++ nonc of b */
      for (int i = 0; i < ncl; i++) gbuf[i] = itl[nonc1[i]];
      for (int i = 0; i < ncr; i++) gbuf[ncl + i] = itr[nonc2[i]];
      int64_t targ = tmap_find(&mpC, O.itoi, O.rank, gbuf);
      if (targ < 0) {
        free(Lbuf);
        free(Rbuf);
        free(mpC.slot);
        return 3;
      }
      if (mrows == 0 || ncols == 0) continue;
      /* out[targ] += Lmat(M x K) * Rmat(K x N), row-major via C^T = R^T L^T. */
      int M = (int)mrows, N = (int)ncols, K = (int)comm_dim;
      char *C = (char *)Odata + O.offs[targ] * es;
      if (K == 0) continue;
      fl += 2.0 * (double)M * (double)N * (double)K;
      if (dtype == 3) {
        double one = 1.0;
        g_dgemm("N", "N", &N, &M, &K, &one, (double *)Rbuf, &N, (double *)Lbuf, &K, &one,
                (double *)C, &N);
      } else {
        double one[2] = {1.0, 0.0};
        g_zgemm("N", "N", &N, &M, &K, one, Rbuf, &N, Lbuf, &K, one, C, &N);
      }
    }
  }
  free(Lbuf);
  free(Rbuf);
  free(mpC.slot);
  if (flops) *flops = fl;
  return 0;
}

int orc_bs_contract(int dtype, orc_layout L, const void *Ldata, orc_layout R, const void *Rdata,
                    int ncomm, const int64_t *comm1, const int64_t *comm2, orc_layout O,
                    void *Odata) {
  return orc_bs_contract_ex(dtype, L, Ldata, R, Rdata, ncomm, comm1, comm2, O, Odata, 1, 0, NULL);
}
