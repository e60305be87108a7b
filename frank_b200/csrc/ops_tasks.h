// Task table of the batched LowRank addition (ops.cu) for callers that add
// blocks of different sizes in one launch (the H-LU driver, hodlr.cu).
#pragma once
#include <cstdint>

namespace frank {
namespace ops {

// One LowRank addition A += B: A = ua sa va (rank *ka, updated in place),
// B = ub sb vb (rank *kb), m x n, scratch at scratch_off doubles.
struct LrAddTask {
  double *ua, *sa, *va;
  const double *ub, *sb, *vb;
  int64_t ldua, ldsa, ldva, ldub, ldsb, ldvb;
  int64_t scratch_off;
  int* ka;
  const int* kb;
  int m, n;
};

}  // namespace ops
}  // namespace frank
