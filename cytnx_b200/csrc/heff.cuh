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
}  // namespace ctn
