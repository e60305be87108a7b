// C++ layer of the B200 engine with FRANK's operator API.
//
// The classes and free functions in namespace FRANK mirror the reference's
// public interface for the factor-and-solve path (include/FRANK/classes/*.h,
// include/FRANK/operations/{BLAS,LAPACK,arithmetic,randomized_factorizations}.h):
// a program written against FRANK's getrf / trsm / gemm / operator+= / qr /
// rq / svd / rsvd / id / rid compiles against this header.  Every operation
// dispatches on the dynamic types of its matrix arguments through the
// open multimethods of frank_b200/multimethod.hpp (the declare_method /
// define_method surface FRANK uses with yomm2), and every overload runs on the
// GPU through the C ABI of include/frank_b200.h; there is no host arithmetic
// behind these calls.
//
// Differences from the reference, by design:
// * matrices keep FRANK's host-side representation (row-major Dense, LowRank
//   U S V, block grids of MatrixProxy); a Hierarchical built from a kernel
//   or factored by getrf also holds its GPU plan, which trsm and gemm use;
// * getrf applies partial pivoting inside the diagonal blocks (the reference
//   drops LAPACK's pivots): trsm on the returned L applies them, and the
//   host copy of L(i, i) is the unit lower factor of the pivoted block;
// * a Hierarchical is one level of blocks (BLR) on the GPU; deeper trees are
//   reported as unsupported;
// * an operation without an overload, or one the engine does not support,
//   throws FRANK::Error where the reference prints and aborts.
#ifndef FRANK_B200_FRANK_HPP
#define FRANK_B200_FRANK_HPP

#include <array>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace FRANK {

enum class Mode { Upper, Lower };
enum class Side { Left, Right };
enum class AdmisType { PositionBased, GeometryBased };

// Status of the C ABI (FRANK_ERR_*) with its text.
class Error : public std::runtime_error {
 public:
  int status;
  Error(int status_, const std::string& msg) : std::runtime_error(msg), status(status_) {}
};

// Abstract base of every matrix type (classes/matrix.h).
class Matrix {
 public:
  virtual ~Matrix() = default;
};

// The kernel plugin signature (functions.h): fills A (rows x cols, row
// stride) with the kernel evaluated on the points `params` (params[d][i])
// for rows starting at row_start and columns at col_start.
using Kernel = void (*)(double* A, const uint64_t A_rows, const uint64_t A_cols, const uint64_t A_stride,
                        const std::vector<std::vector<double>>& params, const int64_t row_start,
                        const int64_t col_start);

// Dense matrix in host memory, row-major (classes/dense.h).
class Dense : public Matrix {
 public:
  std::array<int64_t, 2> dim = {0, 0};
  int64_t stride = 0;
  Dense() = default;
  Dense(const int64_t n_rows, const int64_t n_cols = 1);
  Dense(Kernel kernel, const std::vector<std::vector<double>>& params, const int64_t n_rows,
        const int64_t n_cols = 1, const int64_t row_start = 0, const int64_t col_start = 0);
  double& operator()(const int64_t i, const int64_t j) { return data_[i * stride + j]; }
  const double& operator()(const int64_t i, const int64_t j) const { return data_[i * stride + j]; }
  double* data() { return data_.data(); }
  const double* data() const { return data_.data(); }
  // column-major copy (ld = rows) and its inverse
  std::vector<double> col_major() const;
  void set_col_major(const double* a, int64_t ld);

 private:
  std::vector<double> data_;
};

// Low-rank matrix U S V (classes/low_rank.h).
class LowRank : public Matrix {
 public:
  std::array<int64_t, 2> dim = {0, 0};
  int64_t rank = 0;
  double eps = 0;
  Dense U, S, V;
  LowRank() = default;
  LowRank(const Dense& U_, const Dense& S_, const Dense& V_);
  // LowRank(Dense, rank): randomized SVD with oversample 5 and the
  // reference's Omega (classes/low_rank.cpp:40-48), on the GPU.
  LowRank(const Dense& A, const int64_t rank_);
};

// A block that only has dimensions (classes/empty.h).
class Empty : public Matrix {
 public:
  std::array<int64_t, 2> dim = {0, 0};
  Empty() = default;
  Empty(const int64_t n_rows, const int64_t n_cols) : dim{n_rows, n_cols} {}
};

// Owner of any matrix type, used for the blocks of a Hierarchical
// (classes/matrix_proxy.h).
class MatrixProxy {
 public:
  MatrixProxy() = default;
  MatrixProxy(const MatrixProxy& A);
  MatrixProxy& operator=(const MatrixProxy& A);
  MatrixProxy(MatrixProxy&&) = default;
  MatrixProxy& operator=(MatrixProxy&&) = default;
  explicit MatrixProxy(const Matrix& A);
  MatrixProxy(Dense&& A);
  MatrixProxy(LowRank&& A);
  MatrixProxy(Empty&& A);
  MatrixProxy& operator=(Dense&& A);
  MatrixProxy& operator=(LowRank&& A);
  MatrixProxy& operator=(Empty&& A);
  operator Matrix&();
  operator const Matrix&() const;
  Matrix* get() const { return ptr_.get(); }

 private:
  std::unique_ptr<Matrix> ptr_;
  friend class Hierarchical;
};

namespace detail {
struct Plan;   // a frank_blr plan of the C ABI
}

// Block grid (classes/hierarchical.h), one level on the GPU.
class Hierarchical : public Matrix {
 public:
  std::array<int64_t, 2> dim = {0, 0};   // blocks per side
  Hierarchical() = default;
  Hierarchical(const int64_t n_row_blocks, const int64_t n_col_blocks = 1);
  Hierarchical(MatrixProxy&& A);
  // Fixed accuracy (hierarchical.cpp:89-109): diagonal and inadmissible
  // blocks dense, admissible blocks compressed to eps on the GPU.
  Hierarchical(Kernel kernel, std::vector<std::vector<double>> params, const int64_t n_rows, const int64_t n_cols,
               const int64_t nleaf, const double eps, const double admis = 0, const int64_t n_row_blocks = 2,
               const int64_t n_col_blocks = 2, const AdmisType admis_type = AdmisType::PositionBased);
  // Fixed rank (hierarchical.cpp:67-87), randomized SVD on the GPU.
  Hierarchical(Kernel kernel, std::vector<std::vector<double>> params, const int64_t n_rows, const int64_t n_cols,
               const int64_t rank, const int64_t nleaf, const double admis = 0, const int64_t n_row_blocks = 2,
               const int64_t n_col_blocks = 2, const AdmisType admis_type = AdmisType::PositionBased);
  MatrixProxy& operator()(const int64_t i, const int64_t j) { return data_[i * dim[1] + j]; }
  const MatrixProxy& operator()(const int64_t i, const int64_t j) const { return data_[i * dim[1] + j]; }

  // GPU plan holding this matrix (role 0) or the factor it is part of
  // (role 1: L, role 2: U); empty for a matrix assembled on the host, which
  // getrf / gemm upload on first use.
  std::shared_ptr<detail::Plan> plan;
  int role = 0;

 private:
  std::vector<MatrixProxy> data_;
};

// Global settings (util/global_key_value.h): "FRANK_LRA" selects the LowRank
// addition ("naive" -- LowRank += LowRank only, the BLR plans reject it --,
// "rounded_addition", else fast_rounded_addition, which falls back to
// rounded_addition at a tolerance); "FRANK_PRECISION" ("fp64", default, or
// "mixed": FP32 factor, meant for iterative refinement) the plans' arithmetic.
void setGlobalValue(const std::string key, const std::string value);
std::string getGlobalValue(const std::string key);

// Finalises the dispatch tables (util/initialize.cpp:14-16).
void initialize();

// Kernels and inputs (functions.cpp, util/experiment_setup.cpp), evaluated
// on the host to create input matrices; Hierarchical(kernel, ...) recognises
// laplacend and helmholtznd and evaluates them on the GPU.
void laplacend(double* A, const uint64_t A_rows, const uint64_t A_cols, const uint64_t A_stride,
               const std::vector<std::vector<double>>& x, const int64_t row_start, const int64_t col_start);
void helmholtznd(double* A, const uint64_t A_rows, const uint64_t A_cols, const uint64_t A_stride,
                 const std::vector<std::vector<double>>& x, const int64_t row_start, const int64_t col_start);
void random_uniform(double* A, const uint64_t A_rows, const uint64_t A_cols, const uint64_t A_stride,
                    const std::vector<std::vector<double>>& x, const int64_t row_start, const int64_t col_start);
void random_normal(double* A, const uint64_t A_rows, const uint64_t A_cols, const uint64_t A_stride,
                   const std::vector<std::vector<double>>& x, const int64_t row_start, const int64_t col_start);
std::vector<double> get_sorted_random_vector(const int64_t N);

// Operations (operations/*.h).
std::tuple<MatrixProxy, MatrixProxy> getrf(Matrix& A);
void trsm(const Matrix& A, Matrix& B, const Mode uplo, const Side side = Side::Left);
void gemm(const Matrix& A, const Matrix& B, Matrix& C, const double alpha = 1, const double beta = 1,
          const bool TransA = false, const bool TransB = false);
Matrix& operator+=(Matrix& A, const Matrix& B);
void qr(Matrix& A, Matrix& Q, Matrix& R);
void rq(Matrix& A, Matrix& R, Matrix& Q);
std::tuple<Dense, Dense, Dense> svd(Dense& A);
std::tuple<Dense, Dense, Dense> rsvd(const Dense& A, const int64_t sample_size);
std::tuple<Dense, Dense, Dense> id(Matrix& A, const int64_t k);
std::tuple<Dense, std::vector<int64_t>> one_sided_id(Matrix& A, const int64_t k);
std::tuple<Dense, Dense, Dense> rid(const Dense& A, const int64_t sample_size, const int64_t rank);

// Relative error ||A - B||_F / ||A||_F of two Dense matrices (util/l2_error.h).
double l2_error(const Matrix& A, const Matrix& B);

}  // namespace FRANK

#endif  // FRANK_B200_FRANK_HPP
