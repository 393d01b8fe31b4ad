// Tables of the MPO linear-combination kernel of the two-site H_eff plan.
#pragma once
#include <vector>

#include "ctn_common.h"

namespace ctn {
struct MpoTask {
  int64_t x3_off;
  int64_t size;  // elements of the X3 block (rows * cols, contiguous)
  int32_t term_begin, term_count;
};
struct MpoTerm {
  int64_t x1_off;
  double coef;
};
struct MpoChunk {
  int32_t task;
  int32_t pad_;
  int64_t start;
};
struct MpoApply {
  std::vector<MpoTask> tasks;
  std::vector<MpoTerm> terms;
  std::vector<MpoChunk> chunks;
  void *d_mem = nullptr;
  int d_dev = -1;
  double bytes = 0.0;
  void finalize();
  ctn_status upload(cudaStream_t st);
  ctn_status run(const double *X1, double *X3, cudaStream_t st);
  ~MpoApply() {
    if (d_mem) cudaFree(d_mem);
  }
};

// host metadata of one block: qnum-index tuple, shape (rank <= 4), element offset
struct BlkInfo {
  int64_t q[4];
  int64_t d[4];
  int64_t off;
};
// an X3 block of the plan: (a', w2, s1', s2', b) fed to out block `o` with R block `r`
struct X3Info {
  int64_t o, r;
  int64_t rows, cols;
  std::vector<std::pair<int64_t, double>> terms;  // (X1 key index, coefficient)
};

struct HeffSplit;  // split-precision (tcgen05) state, heff_split.cu

ctn_status heff_split_prepare(struct ::ctn_heff2_plan *p, int kind);
size_t heff_split_ws_bytes(const struct ::ctn_heff2_plan *p, int kind);
ctn_status heff_split_set_env(struct ::ctn_heff2_plan *p, int kind, const double *L, const double *R, void *ws,
                              cudaStream_t st);
ctn_status heff_split_matvec(struct ::ctn_heff2_plan *p, int kind, const double *psi, double *out, cudaStream_t st,
                             double *ms3);
// the same with the result rounded to FP32 (n floats at out)
ctn_status heff_split_matvec_f32out(struct ::ctn_heff2_plan *p, int kind, const double *psi, float *out,
                                    cudaStream_t st);
void heff_split_free(HeffSplit *s);
double heff_split_gemm_flops(const struct ::ctn_heff2_plan *p, int kind, int step);
ctn_status heff_split_stats(const struct ::ctn_heff2_plan *p, int kind, double *out);
void heff_split_apply_epilogue(struct ::ctn_heff2_plan *p, int kind);
}  // namespace ctn

struct ctn_heff2_plan {
  int64_t psi_elems = 0, out_elems = 0, L_elems = 0, R_elems = 0;
  int64_t x1_elems = 0, x3_elems = 0;
  // L staged as [a][w][a'] per block (transposed operand of step 1)
  std::vector<uint64_t> L_shapes;
  std::vector<int64_t> L_src, L_dst;
  ctn::GroupedGemmF64 g1, g4;
  ctn::MpoApply mpo;
  // bound environment (FP64 form)
  const double *R = nullptr;
  double *ws = nullptr;  // [Lt | X1 | X3]
  bool bound = false;
  double gemm_flops = 0.0;
  int64_t n_x1 = 0, n_x3 = 0;
  // host metadata for the split builder
  std::vector<ctn::BlkInfo> Lb, Pb, Rb, Ob;
  std::vector<std::pair<int64_t, int64_t>> x1_lp;  // X1 key index -> (L block, psi block)
  std::vector<ctn::X3Info> x3;
  // split-precision state per kind (0: 3xTF32, 1: BF16x3)
  ctn::HeffSplit *split[2] = {nullptr, nullptr};
  int split_bn[2][2] = {{128, 128}, {128, 128}};  // tile widths of steps 1 and 4 per split kind
  int split_epi[2][2] = {{-1, -1}, {-1, -1}};     // epilogue form per GEMM: -1 automatic, 0 direct, 1 staged
  bool split_bound[2] = {false, false};
  ~ctn_heff2_plan() {
    for (auto *s : split) ctn::heff_split_free(s);
  }
};
