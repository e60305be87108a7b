// The reference's own BLR test sequences (test/blr_fixed_acc_test.cpp:67-83,
// test/blr_fixed_rank_test.cpp, test/lowrank_test.cpp, test/dense_id_test.cpp,
// test/dense_qr_test.cpp) written against FRANK's API and compiled against
// the engine's C++ layer (frank_b200/FRANK.hpp): every call runs on the GPU.
// Prints one line per check; exit status 0 only if every check passes.
#include "frank_b200/FRANK.hpp"

#include <cmath>
#include <cstdio>
#include <string>
#include <tuple>
#include <vector>

static int failures = 0;

static void expect(bool ok, const std::string& what, double v) {
  std::printf("%s %s %.3e\n", ok ? "PASS" : "FAIL", what.c_str(), v);
  if (!ok) ++failures;
}

// test/blr_fixed_acc_test.cpp:67-83 (FRANK_LRA=rounded_addition)
static void blr_fixed_accuracy(int64_t n, int64_t nleaf, double eps, double admis, FRANK::AdmisType at) {
  FRANK::setGlobalValue("FRANK_LRA", "rounded_addition");
  const int64_t nb = n / nleaf;
  std::vector<std::vector<double>> randx{FRANK::get_sorted_random_vector(n)};
  FRANK::Hierarchical A(FRANK::laplacend, randx, n, n, nleaf, eps, admis, nb, nb, at);
  const FRANK::Dense x(FRANK::random_uniform, {}, n, 1);
  FRANK::Dense b(n);
  FRANK::gemm(A, x, b, 1, 1);
  FRANK::Hierarchical L, U;
  std::tie(L, U) = FRANK::getrf(A);
  FRANK::trsm(L, b, FRANK::Mode::Lower);
  FRANK::trsm(U, b, FRANK::Mode::Upper);
  const double err = FRANK::l2_error(x, b);
  expect(err <= eps, "blr_fixed_acc n=" + std::to_string(n) + " eps=" + std::to_string(eps) + " admis=" +
                         std::to_string(admis) + (at == FRANK::AdmisType::GeometryBased ? " geometry" : " position"),
         err);
}

// test/blr_fixed_rank_test.cpp (default LowRank addition: fast_rounded_addition)
static void blr_fixed_rank(int64_t n, int64_t nleaf, int64_t rank, double admis) {
  FRANK::setGlobalValue("FRANK_LRA", "");
  const int64_t nb = n / nleaf;
  std::vector<std::vector<double>> randx{FRANK::get_sorted_random_vector(n)};
  FRANK::Hierarchical A(FRANK::laplacend, randx, n, n, rank, nleaf, admis, nb, nb);
  bool ranks_ok = true;
  for (int64_t i = 0; i < nb; ++i)
    for (int64_t j = 0; j < nb; ++j)
      if (auto* lr = dynamic_cast<const FRANK::LowRank*>(&static_cast<const FRANK::Matrix&>(A(i, j))))
        ranks_ok = ranks_ok && lr->rank == rank;
  expect(ranks_ok, "blr_fixed_rank uniform ranks n=" + std::to_string(n) + " rank=" + std::to_string(rank), 0.0);
  const FRANK::Dense x(FRANK::random_uniform, {}, n, 1);
  FRANK::Dense b(n);
  FRANK::gemm(A, x, b, 1, 1);
  FRANK::Hierarchical L, U;
  std::tie(L, U) = FRANK::getrf(A);
  FRANK::trsm(L, b, FRANK::Mode::Lower);
  FRANK::trsm(U, b, FRANK::Mode::Upper);
  const double err = FRANK::l2_error(x, b);
  expect(err < 1e-2, "blr_fixed_rank solve n=" + std::to_string(n) + " rank=" + std::to_string(rank), err);
}

// test/lowrank_test.cpp:28-61: LowRank += LowRank keeps the fixed-rank error
static void lowrank_addition(const char* lra) {
  FRANK::setGlobalValue("FRANK_LRA", lra);
  const int64_t m = 64, n = 64, rank = 8;
  std::vector<std::vector<double>> randx{FRANK::get_sorted_random_vector(2 * n)};
  const FRANK::Dense D(FRANK::laplacend, randx, m, n, 0, n);
  FRANK::LowRank A(D, rank);
  const FRANK::LowRank B(D, rank);
  A += B;
  FRANK::Dense sum(m, n), two(m, n);
  FRANK::Dense US(m, rank);
  FRANK::gemm(A.U, A.S, US, 1, 0);
  FRANK::gemm(US, A.V, sum, 1, 0);
  for (int64_t i = 0; i < m; ++i)
    for (int64_t j = 0; j < n; ++j) two(i, j) = 2 * D(i, j);
  const double err = FRANK::l2_error(two, sum);
  expect(err < 1e-4 && A.rank == rank, std::string("lowrank += lowrank ") + lra, err);
}

// FRANK_LRA=naive (addition.cpp:68-89): rank + rank < min(m, n) concatenates
// (rank 2 * rank, the sum represented exactly)
static void lowrank_naive() {
  FRANK::setGlobalValue("FRANK_LRA", "naive");
  const int64_t m = 64, n = 64, rank = 8;
  std::vector<std::vector<double>> randx{FRANK::get_sorted_random_vector(2 * n)};
  const FRANK::Dense D(FRANK::laplacend, randx, m, n, 0, n);
  FRANK::LowRank A(D, rank);
  const FRANK::LowRank B(D, rank);
  A += B;
  FRANK::Dense sum(m, n), two(m, n), US(m, A.rank);
  FRANK::gemm(A.U, A.S, US, 1, 0);
  FRANK::gemm(US, A.V, sum, 1, 0);
  for (int64_t i = 0; i < m; ++i)
    for (int64_t j = 0; j < n; ++j) two(i, j) = 2 * D(i, j);
  const double err = FRANK::l2_error(two, sum);
  expect(err < 1e-4 && A.rank == 2 * rank, "lowrank += lowrank naive", err);
  FRANK::setGlobalValue("FRANK_LRA", "");
}

// test/dense_qr_test.cpp, dense_svd_test.cpp, dense_id_test.cpp (reduced n)
static void dense_ops() {
  const int64_t n = 256, k = 16;
  std::vector<std::vector<double>> randx{FRANK::get_sorted_random_vector(2 * n)};
  FRANK::Dense A(FRANK::laplacend, randx, n, n, 0, n);
  FRANK::Dense Q(n, n), R(n, n), QR(n, n);
  FRANK::Dense Acopy(A);
  FRANK::qr(Acopy, Q, R);
  FRANK::gemm(Q, R, QR, 1, 0);
  expect(FRANK::l2_error(A, QR) < 1e-13, "qr", FRANK::l2_error(A, QR));
  FRANK::Dense R2(n, n), Q2(n, n), RQ(n, n);
  FRANK::rq(Acopy, R2, Q2);
  FRANK::gemm(R2, Q2, RQ, 1, 0);
  expect(FRANK::l2_error(A, RQ) < 1e-13, "rq", FRANK::l2_error(A, RQ));
  FRANK::Dense U, S, V;
  std::tie(U, S, V) = FRANK::svd(Acopy);
  FRANK::Dense US(n, n), USV(n, n);
  FRANK::gemm(U, S, US, 1, 0);
  FRANK::gemm(US, V, USV, 1, 0);
  expect(FRANK::l2_error(A, USV) < 1e-11, "svd", FRANK::l2_error(A, USV));
  std::tie(U, S, V) = FRANK::id(Acopy, k);
  FRANK::Dense US2(n, k), A2(n, n);
  FRANK::gemm(U, S, US2, 1, 0);
  FRANK::gemm(US2, V, A2, 1, 0);
  expect(FRANK::l2_error(A, A2) < 1e-7, "id", FRANK::l2_error(A, A2));
  std::tie(U, S, V) = FRANK::rid(A, k + 5, k);
  FRANK::gemm(U, S, US2, 1, 0);
  FRANK::gemm(US2, V, A2, 1, 0);
  expect(FRANK::l2_error(A, A2) < 1e-7, "rid", FRANK::l2_error(A, A2));
}

// Dispatch: an operation without an overload reports the reference's error
// (print + abort there, FRANK::Error here).
static void dispatch_errors() {
  FRANK::Dense D(8, 8);
  bool thrown = false;
  try {
    FRANK::getrf(D);
  } catch (const FRANK::Error& e) {
    thrown = std::string(e.what()).find("getrf") != std::string::npos;
  }
  expect(thrown, "getrf(Dense) has no overload", 0.0);
  thrown = false;
  FRANK::Empty E(8, 8);
  FRANK::Dense B(8, 1), C(8, 1);
  try {
    FRANK::gemm(E, B, C, 1, 1);
  } catch (const FRANK::Error&) {
    thrown = true;
  }
  expect(thrown, "gemm(Empty, Dense, Dense) has no overload", 0.0);
}

int main() {
  FRANK::initialize();
  for (int64_t n : {128, 256})
    for (double eps : {1e-6, 1e-8, 1e-10})
      for (double admis : {0.0, 1.0, 4.0})
        for (auto at : {FRANK::AdmisType::PositionBased, FRANK::AdmisType::GeometryBased})
          blr_fixed_accuracy(n, 32, eps, admis, at);
  for (int64_t n : {128, 256})
    for (int64_t rank : {4, 8}) blr_fixed_rank(n, 32, rank, 0.0);
  lowrank_addition("rounded_addition");
  lowrank_addition("fast_rounded_addition");
  lowrank_naive();
  dense_ops();
  dispatch_errors();
  std::printf("%d failures\n", failures);
  return failures == 0 ? 0 : 1;
}
