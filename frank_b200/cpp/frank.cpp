// C++ layer of the B200 engine: FRANK's classes and operations over the C ABI.
// Every operation below is an open multimethod (frank_b200/multimethod.hpp)
// whose overloads call the GPU entry points of include/frank_b200.h.
#include "frank_b200/FRANK.hpp"

#include "frank_b200/multimethod.hpp"
#include "../../include/frank_b200.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <random>
#include <utility>

namespace FRANK {

using frank_mm::virtual_;

// ---------------------------------------------------------------------------
// C ABI plumbing
// ---------------------------------------------------------------------------
namespace {

void check(int rc, const char* what) {
  if (rc != FRANK_OK) throw Error(rc, std::string(what) + ": " + frank_last_error());
}

[[noreturn]] void unsupported(const std::string& what) { throw Error(FRANK_ERR_UNSUPPORTED, what); }

// Device buffer of doubles or ints owned by a scope.
template <typename T>
struct DeviceBuffer {
  T* p = nullptr;
  size_t n = 0;
  explicit DeviceBuffer(size_t count) : n(count) {
    void* v = nullptr;
    check(frank_device_alloc(count * sizeof(T), &v), "frank_device_alloc");
    p = static_cast<T*>(v);
  }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() { frank_device_free(p); }
  void upload(const T* h) { check(frank_copy(p, h, n * sizeof(T), 1), "frank_copy"); }
  void download(T* h) const { check(frank_copy(h, p, n * sizeof(T), 0), "frank_copy"); }
};

std::map<std::string, std::string>& globals() {
  static std::map<std::string, std::string> g;
  return g;
}
std::mutex& globals_mutex() {
  static std::mutex m;
  return m;
}

// FRANK_LRA as addition.cpp:191-203 reads it: "naive", "rounded_addition",
// anything else fast_rounded_addition.  Plans reject "naive" (set_lra fails).
std::string lra_name() {
  const std::string v = getGlobalValue("FRANK_LRA");
  if (v == "rounded_addition" || v == "naive") return v;
  return "fast_rounded_addition";
}

// Device copy of a Dense (column-major, ld = rows).
struct DevDense {
  DeviceBuffer<double> buf;
  int64_t m, n;
  explicit DevDense(const Dense& A) : buf((size_t)std::max<int64_t>(1, A.dim[0] * A.dim[1])), m(A.dim[0]), n(A.dim[1]) {
    std::vector<double> c = A.col_major();
    if (!c.empty()) buf.upload(c.data());
  }
  DevDense(int64_t rows, int64_t cols) : buf((size_t)std::max<int64_t>(1, rows * cols)), m(rows), n(cols) {}
  void to(Dense& A) const {
    std::vector<double> c((size_t)std::max<int64_t>(1, m * n));
    buf.download(c.data());
    A = Dense(m, n);
    A.set_col_major(c.data(), m);
  }
};

}  // namespace

namespace detail {

// A frank_blr plan: one BLR matrix on the GPU (A_H and, after getrf, its factor).
struct Plan {
  frank_blr* h = nullptr;
  int64_t n = 0;
  int nb = 0;
  double eps = 0.0;   // truncation tolerance (0: fixed rank)
  bool factored = false;
  ~Plan() {
    if (h) frank_blr_destroy(h);
  }
};

}  // namespace detail

// ---------------------------------------------------------------------------
// Classes
// ---------------------------------------------------------------------------

Dense::Dense(const int64_t n_rows, const int64_t n_cols)
    : dim{n_rows, n_cols}, stride(n_cols), data_((size_t)(n_rows * n_cols), 0.0) {}

Dense::Dense(Kernel kernel, const std::vector<std::vector<double>>& params, const int64_t n_rows, const int64_t n_cols,
             const int64_t row_start, const int64_t col_start)
    : Dense(n_rows, n_cols) {
  kernel(data_.data(), n_rows, n_cols, stride, params, row_start, col_start);
}

std::vector<double> Dense::col_major() const {
  std::vector<double> c((size_t)(dim[0] * dim[1]));
  for (int64_t j = 0; j < dim[1]; ++j)
    for (int64_t i = 0; i < dim[0]; ++i) c[i + j * dim[0]] = (*this)(i, j);
  return c;
}

void Dense::set_col_major(const double* a, int64_t ld) {
  for (int64_t j = 0; j < dim[1]; ++j)
    for (int64_t i = 0; i < dim[0]; ++i) (*this)(i, j) = a[i + j * ld];
}

LowRank::LowRank(const Dense& U_, const Dense& S_, const Dense& V_)
    : dim{U_.dim[0], V_.dim[1]}, rank(S_.dim[0]), U(U_), S(S_), V(V_) {}

LowRank::LowRank(const Dense& A, const int64_t rank_) : dim{A.dim[0], A.dim[1]}, rank(rank_) {
  const int m = (int)A.dim[0], n = (int)A.dim[1], k = (int)rank_;
  DevDense dA(A), dU(m, k), dS(k, k), dV(k, n);
  check(frank_rsvd_batched(m, n, 1, k, 5, 0, dA.buf.p, m, 0, dU.buf.p, m, 0, dS.buf.p, k, 0, dV.buf.p, k, 0,
                           nullptr),
        "frank_rsvd_batched");
  dU.to(U);
  dS.to(S);
  dV.to(V);
}

MatrixProxy::MatrixProxy(const MatrixProxy& A) {
  if (A.ptr_) *this = MatrixProxy(static_cast<const Matrix&>(A));
}

MatrixProxy& MatrixProxy::operator=(const MatrixProxy& A) {
  if (this != &A) {
    MatrixProxy t(A);
    ptr_ = std::move(t.ptr_);
  }
  return *this;
}

MatrixProxy::MatrixProxy(const Matrix& A) {
  if (auto* d = dynamic_cast<const Dense*>(&A)) ptr_ = std::make_unique<Dense>(*d);
  else if (auto* l = dynamic_cast<const LowRank*>(&A)) ptr_ = std::make_unique<LowRank>(*l);
  else if (auto* e = dynamic_cast<const Empty*>(&A)) ptr_ = std::make_unique<Empty>(*e);
  else if (auto* h = dynamic_cast<const Hierarchical*>(&A)) ptr_ = std::make_unique<Hierarchical>(*h);
  else unsupported("MatrixProxy of an unknown matrix type");
}

MatrixProxy::MatrixProxy(Dense&& A) : ptr_(std::make_unique<Dense>(std::move(A))) {}
MatrixProxy::MatrixProxy(LowRank&& A) : ptr_(std::make_unique<LowRank>(std::move(A))) {}
MatrixProxy::MatrixProxy(Empty&& A) : ptr_(std::make_unique<Empty>(std::move(A))) {}
MatrixProxy& MatrixProxy::operator=(Dense&& A) { ptr_ = std::make_unique<Dense>(std::move(A)); return *this; }
MatrixProxy& MatrixProxy::operator=(LowRank&& A) { ptr_ = std::make_unique<LowRank>(std::move(A)); return *this; }
MatrixProxy& MatrixProxy::operator=(Empty&& A) { ptr_ = std::make_unique<Empty>(std::move(A)); return *this; }

MatrixProxy::operator Matrix&() {
  if (!ptr_) unsupported("empty MatrixProxy");
  return *ptr_;
}

MatrixProxy::operator const Matrix&() const {
  if (!ptr_) unsupported("empty MatrixProxy");
  return *ptr_;
}

Hierarchical::Hierarchical(const int64_t n_row_blocks, const int64_t n_col_blocks)
    : dim{n_row_blocks, n_col_blocks}, data_((size_t)(n_row_blocks * n_col_blocks)) {}

Hierarchical::Hierarchical(MatrixProxy&& A) {
  auto* h = dynamic_cast<Hierarchical*>(A.ptr_.get());
  if (!h) unsupported("Hierarchical from a MatrixProxy that holds another type");
  *this = std::move(*h);
}

namespace {

int kernel_id(Kernel k) {
  if (k == laplacend) return FRANK_KERNEL_LAPLACE;
  if (k == helmholtznd) return FRANK_KERNEL_HELMHOLTZ;
  unsupported("Hierarchical: on-device construction knows laplacend and helmholtznd only");
}

int precision_value() {
  return getGlobalValue("FRANK_PRECISION") == "mixed" ? FRANK_PREC_MIXED : FRANK_PREC_FP64;
}

// Host blocks of the plan (which = 0: A_H, 1: the factor) into H.
void download_blocks(const detail::Plan& P, int which, Hierarchical& H, int role) {
  std::vector<int64_t> off(P.nb + 1);
  check(frank_blr_offsets(P.h, off.data()), "frank_blr_offsets");
  for (int i = 0; i < P.nb; ++i)
    for (int j = 0; j < P.nb; ++j) {
      const int64_t bi = off[i + 1] - off[i], bj = off[j + 1] - off[j];
      if ((role == 1 && j > i) || (role == 2 && j < i)) {
        H(i, j) = Empty(bi, bj);
        continue;
      }
      int type = 0, rank = 0;
      check(frank_blr_block_info(P.h, which, i, j, &type, &rank), "frank_blr_block_info");
      if (type == FRANK_BLOCK_DENSE) {
        Dense D(bi, bj);
        check(frank_blr_get_dense(P.h, which, i, j, D.data(), bj, 1), "frank_blr_get_dense");
        if (i == j && role == 1) {        // unit lower factor of the pivoted block
          for (int64_t r = 0; r < bi; ++r)
            for (int64_t c = r; c < bj; ++c) D(r, c) = r == c ? 1.0 : 0.0;
        } else if (i == j && role == 2) {
          for (int64_t r = 0; r < bi; ++r)
            for (int64_t c = 0; c < r; ++c) D(r, c) = 0.0;
        }
        H(i, j) = std::move(D);
      } else {
        Dense U(bi, rank), S(rank, rank), V(rank, bj);
        check(frank_blr_get_lowrank(P.h, which, i, j, U.data(), std::max(rank, 1), S.data(), std::max(rank, 1),
                                    V.data(), bj, 1),
              "frank_blr_get_lowrank");
        LowRank L(U, S, V);
        L.eps = P.eps;
        H(i, j) = std::move(L);
      }
    }
}

// A plan holding H (uploaded from its host blocks): one level of Dense /
// LowRank blocks, square block grid.
std::shared_ptr<detail::Plan> upload(const Hierarchical& H) {
  if (H.dim[0] != H.dim[1] || H.dim[0] < 1) unsupported("getrf / gemm: the GPU plans take a square block grid");
  const int nb = (int)H.dim[0];
  int64_t n = 0;
  int max_rank = 0;
  double eps = 0.0;   // the LowRank blocks' own tolerance (0: fixed rank), as FRANK keeps it per block
  for (int i = 0; i < nb; ++i) {
    const Matrix& d = H(i, i);
    auto* D = dynamic_cast<const Dense*>(&d);
    if (!D) unsupported("getrf / gemm: the diagonal blocks must be Dense (one level of blocks on the GPU)");
    n += D->dim[0];
    for (int j = 0; j < nb; ++j) {
      const Matrix& b = H(i, j);
      if (auto* L = dynamic_cast<const LowRank*>(&b)) {
        max_rank = std::max<int>(max_rank, (int)L->rank);
        eps = std::max(eps, L->eps);
      } else if (!dynamic_cast<const Dense*>(&b)) {
        unsupported("getrf / gemm: blocks must be Dense or LowRank");
      }
    }
  }
  // the block-low-rank blocks decide admissibility: a plan whose
  // position-based rule reproduces them exactly
  int admis = -1;
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      const Matrix& b = H(i, j);
      if (i != j && dynamic_cast<const Dense*>(&b)) admis = std::max(admis, std::abs(i - j));
    }
  frank_blr_desc d{};
  d.n = n;
  d.nb = nb;
  d.precision = precision_value();
  d.admis = admis < 0 ? 0.0 : (double)admis;
  d.eps = eps;
  if (d.eps <= 0.0) d.fixed_rank = std::max(1, max_rank);
  auto P = std::make_shared<detail::Plan>();
  check(frank_blr_create(&d, &P->h), "frank_blr_create");
  P->n = n;
  P->nb = nb;
  P->eps = d.eps;
  std::vector<int64_t> off(nb + 1);
  check(frank_blr_offsets(P->h, off.data()), "frank_blr_offsets");
  for (int i = 0; i < nb; ++i) {
    const Matrix& dd = H(i, i);
    if (dynamic_cast<const Dense&>(dd).dim[0] != off[i + 1] - off[i])
      unsupported("getrf / gemm: block sizes must follow IndexRange::split (ceil(n / nb))");
  }
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      const Matrix& b = H(i, j);
      int type = 0;
      check(frank_blr_block_info(P->h, 0, i, j, &type, nullptr), "frank_blr_block_info");
      if (auto* D = dynamic_cast<const Dense*>(&b)) {
        if (type != FRANK_BLOCK_DENSE) unsupported("getrf / gemm: a Dense block where admissibility expects LowRank");
        check(frank_blr_set_dense(P->h, i, j, D->data(), D->stride, 1), "frank_blr_set_dense");
      } else {
        auto* L = dynamic_cast<const LowRank*>(&b);
        if (type != FRANK_BLOCK_LOWRANK) unsupported("getrf / gemm: a LowRank block where admissibility expects Dense");
        check(frank_blr_set_lowrank(P->h, i, j, (int)L->rank, L->U.data(), L->U.stride, L->S.data(), L->S.stride,
                                    L->V.data(), L->V.stride, 1),
              "frank_blr_set_lowrank");
      }
    }
  check(frank_blr_set_lra(P->h, lra_name().c_str(), 0.0), "frank_blr_set_lra");
  return P;
}

std::shared_ptr<detail::Plan> plan_of(const Hierarchical& H) { return H.plan ? H.plan : upload(H); }

Hierarchical build(Kernel kernel, const std::vector<std::vector<double>>& params, int64_t n_rows, int64_t n_cols,
                   int64_t rank, int64_t nleaf, double eps, double admis, int64_t nrb, int64_t ncb, AdmisType at) {
  if (n_rows != n_cols || nrb != ncb) unsupported("Hierarchical: the GPU plans are square");
  if ((n_rows + nrb - 1) / nrb > std::max<int64_t>(nleaf, 1))
    unsupported("Hierarchical: blocks above nleaf would recurse; the GPU plans are one level of blocks");
  const int kid = kernel_id(kernel);
  frank_blr_desc d{};
  d.n = n_rows;
  d.nb = (int)nrb;
  d.precision = precision_value();
  d.fixed_rank = (int)rank;
  d.eps = eps;
  d.admis = admis;
  const int dim = (int)params.size();
  std::vector<double> pts((size_t)dim * n_rows);
  for (int a = 0; a < dim; ++a)
    for (int64_t i = 0; i < n_rows; ++i) pts[a * n_rows + i] = params[a][i];
  auto P = std::make_shared<detail::Plan>();
  if (at == AdmisType::GeometryBased) check(frank_blr_create_geometric(&d, pts.data(), dim, &P->h), "frank_blr_create_geometric");
  else check(frank_blr_create(&d, &P->h), "frank_blr_create");
  P->n = n_rows;
  P->nb = (int)nrb;
  P->eps = rank > 0 ? 0.0 : eps;
  check(frank_blr_set_lra(P->h, lra_name().c_str(), 0.0), "frank_blr_set_lra");
  check(frank_blr_build_kernel(P->h, kid, pts.data(), dim, nullptr, rank > 0 ? 0.0 : eps, nullptr),
        "frank_blr_build_kernel");
  Hierarchical H(nrb, ncb);
  download_blocks(*P, 0, H, 0);
  H.plan = P;
  H.role = 0;
  return H;
}

}  // namespace

Hierarchical::Hierarchical(Kernel kernel, std::vector<std::vector<double>> params, const int64_t n_rows,
                           const int64_t n_cols, const int64_t nleaf, const double eps, const double admis,
                           const int64_t n_row_blocks, const int64_t n_col_blocks, const AdmisType admis_type) {
  *this = build(kernel, params, n_rows, n_cols, 0, nleaf, eps, admis, n_row_blocks, n_col_blocks, admis_type);
}

Hierarchical::Hierarchical(Kernel kernel, std::vector<std::vector<double>> params, const int64_t n_rows,
                           const int64_t n_cols, const int64_t rank, const int64_t nleaf, const double admis,
                           const int64_t n_row_blocks, const int64_t n_col_blocks, const AdmisType admis_type) {
  *this = build(kernel, params, n_rows, n_cols, rank, nleaf, 0.0, admis, n_row_blocks, n_col_blocks, admis_type);
}

// ---------------------------------------------------------------------------
// Globals, kernels, inputs
// ---------------------------------------------------------------------------

void setGlobalValue(const std::string key, const std::string value) {
  std::lock_guard<std::mutex> lock(globals_mutex());
  globals()[key] = value;
}

std::string getGlobalValue(const std::string key) {
  std::lock_guard<std::mutex> lock(globals_mutex());
  auto it = globals().find(key);
  return it == globals().end() ? std::string() : it->second;
}

register_class(Matrix)
register_class(Dense, Matrix)
register_class(LowRank, Matrix)
register_class(Empty, Matrix)
register_class(Hierarchical, Matrix)

void initialize() { frank_mm::update_methods(); }

namespace {
double dist2(const std::vector<std::vector<double>>& x, int64_t i, int64_t j) {
  double r = 0.0;
  for (const auto& a : x) r += (a[i] - a[j]) * (a[i] - a[j]);
  return r;
}
}  // namespace

void laplacend(double* A, const uint64_t rows, const uint64_t cols, const uint64_t stride,
               const std::vector<std::vector<double>>& x, const int64_t r0, const int64_t c0) {
  for (uint64_t i = 0; i < rows; ++i)
    for (uint64_t j = 0; j < cols; ++j) A[i * stride + j] = 1.0 / (std::sqrt(dist2(x, r0 + i, c0 + j)) + 1e-3);
}

void helmholtznd(double* A, const uint64_t rows, const uint64_t cols, const uint64_t stride,
                 const std::vector<std::vector<double>>& x, const int64_t r0, const int64_t c0) {
  for (uint64_t i = 0; i < rows; ++i)
    for (uint64_t j = 0; j < cols; ++j) {
      const double r2 = dist2(x, r0 + i, c0 + j);
      A[i * stride + j] = std::exp(-r2) / (std::sqrt(r2) + 1e-3);
    }
}

void random_uniform(double* A, const uint64_t rows, const uint64_t cols, const uint64_t stride,
                    const std::vector<std::vector<double>>&, const int64_t, const int64_t) {
  std::mt19937 gen;
  gen.seed(0);
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  for (uint64_t i = 0; i < rows; ++i)
    for (uint64_t j = 0; j < cols; ++j) A[i * stride + j] = dist(gen);
}

void random_normal(double* A, const uint64_t rows, const uint64_t cols, const uint64_t stride,
                   const std::vector<std::vector<double>>&, const int64_t, const int64_t) {
  std::mt19937 gen;
  gen.seed(0);
  std::normal_distribution<double> dist(0.0, 1.0);
  for (uint64_t i = 0; i < rows; ++i)
    for (uint64_t j = 0; j < cols; ++j) A[i * stride + j] = dist(gen);
}

std::vector<double> get_sorted_random_vector(const int64_t N) {
  std::vector<double> v((size_t)N);
  std::mt19937 gen;
  gen.seed(0);
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  for (auto& a : v) a = dist(gen);
  std::sort(v.begin(), v.end());
  return v;
}

// ---------------------------------------------------------------------------
// Operations (multimethods)
// ---------------------------------------------------------------------------

using MatrixPair = std::tuple<MatrixProxy, MatrixProxy>;

declare_method(MatrixPair, getrf_omm, (virtual_<Matrix&>))

define_method(MatrixPair, getrf_omm, (Hierarchical& A)) {
  auto P = plan_of(A);
  check(frank_blr_getrf(P->h, nullptr), "frank_blr_getrf");
  P->factored = true;
  Hierarchical L(A.dim[0], A.dim[1]), U(A.dim[0], A.dim[1]);
  download_blocks(*P, 1, L, 1);
  download_blocks(*P, 1, U, 2);
  L.plan = P;
  L.role = 1;
  U.plan = P;
  U.role = 2;
  A.plan = P;
  return MatrixPair(MatrixProxy(static_cast<const Matrix&>(L)), MatrixProxy(static_cast<const Matrix&>(U)));
}

define_method(MatrixPair, getrf_omm, (Matrix&)) { unsupported("getrf: no overload for this matrix type"); }

std::tuple<MatrixProxy, MatrixProxy> getrf(Matrix& A) { return getrf_omm(A); }

declare_method(void, trsm_omm, (virtual_<const Matrix&>, virtual_<Matrix&>, const Mode, const Side))

define_method(void, trsm_omm, (const Hierarchical& A, Dense& B, const Mode uplo, const Side side)) {
  if (side != Side::Left) unsupported("trsm: right-side substitution with a Hierarchical factor");
  if (!A.plan || !A.plan->factored || A.role == 0) unsupported("trsm: the Hierarchical is not a factor from getrf");
  if ((uplo == Mode::Lower) != (A.role == 1)) unsupported("trsm: Mode does not match the factor (L: Lower, U: Upper)");
  if (B.dim[0] != A.plan->n) throw Error(FRANK_ERR_INVALID, "trsm: right-hand side has the wrong number of rows");
  std::vector<double> b = B.col_major();
  check(frank_blr_trsm(A.plan->h, uplo == Mode::Lower ? FRANK_LOWER : FRANK_UPPER, b.data(), B.dim[0],
                       (int)B.dim[1], nullptr),
        "frank_blr_trsm");
  B.set_col_major(b.data(), B.dim[0]);
}

define_method(void, trsm_omm, (const Matrix&, Matrix&, const Mode, const Side)) {
  unsupported("trsm: no overload for these matrix types");
}

void trsm(const Matrix& A, Matrix& B, const Mode uplo, const Side side) { trsm_omm(A, B, uplo, side); }

declare_method(void, gemm_omm,
               (virtual_<const Matrix&>, virtual_<const Matrix&>, virtual_<Matrix&>, double, double, bool, bool))

define_method(void, gemm_omm,
              (const Hierarchical& A, const Dense& B, Dense& C, double alpha, double beta, bool ta, bool tb)) {
  if (ta || tb) unsupported("gemm: transposed Hierarchical products");
  if (A.role != 0) unsupported("gemm: products with a factor L or U");
  auto P = plan_of(A);
  if (B.dim[0] != P->n || C.dim[0] != P->n || B.dim[1] != C.dim[1])
    throw Error(FRANK_ERR_INVALID, "gemm: dimension mismatch");
  std::vector<double> x = B.col_major(), y = C.col_major();
  check(frank_blr_gemv(P->h, alpha, x.data(), B.dim[0], beta, y.data(), C.dim[0], (int)B.dim[1], nullptr),
        "frank_blr_gemv");
  C.set_col_major(y.data(), C.dim[0]);
}

define_method(void, gemm_omm,
              (const Dense& A, const Dense& B, Dense& C, double alpha, double beta, bool ta, bool tb)) {
  const int64_t m = ta ? A.dim[1] : A.dim[0], k = ta ? A.dim[0] : A.dim[1];
  const int64_t n = tb ? B.dim[0] : B.dim[1], kb = tb ? B.dim[1] : B.dim[0];
  if (k != kb || C.dim[0] != m || C.dim[1] != n) throw Error(FRANK_ERR_INVALID, "gemm: dimension mismatch");
  DevDense dA(A), dB(B), dC(C);
  check(frank_gemm_batched((int)m, (int)n, (int)k, 1, alpha, dA.buf.p, A.dim[0], 0, ta, dB.buf.p, B.dim[0], 0, tb,
                           beta, dC.buf.p, C.dim[0], 0, nullptr),
        "frank_gemm_batched");
  dC.to(C);
}

define_method(void, gemm_omm,
              (const Matrix&, const Matrix&, Matrix&, double, double, bool, bool)) {
  unsupported("gemm: no overload for these matrix types");
}

void gemm(const Matrix& A, const Matrix& B, Matrix& C, const double alpha, const double beta, const bool TransA,
          const bool TransB) {
  gemm_omm(A, B, C, alpha, beta, TransA, TransB);
}

declare_method(Matrix&, addition_omm, (virtual_<Matrix&>, virtual_<const Matrix&>))

define_method(Matrix&, addition_omm, (LowRank& A, const LowRank& B)) {
  const int m = (int)A.dim[0], n = (int)A.dim[1], ka = (int)A.rank, kb = (int)B.rank;
  if (B.dim[0] != m || B.dim[1] != n) throw Error(FRANK_ERR_INVALID, "operator+=: dimension mismatch");
  const int kmax = std::min(ka + kb, std::min(m, n));
  Dense Ua(m, kmax), Sa(kmax, kmax), Va(kmax, n);
  for (int i = 0; i < m; ++i) for (int c = 0; c < ka; ++c) Ua(i, c) = A.U(i, c);
  for (int i = 0; i < ka; ++i) for (int c = 0; c < ka; ++c) Sa(i, c) = A.S(i, c);
  for (int i = 0; i < ka; ++i) for (int c = 0; c < n; ++c) Va(i, c) = A.V(i, c);
  DevDense dUa(Ua), dSa(Sa), dVa(Va), dUb(B.U), dSb(B.S), dVb(B.V);
  DeviceBuffer<int> dka(1), dkb(1);
  dka.upload(&ka);
  dkb.upload(&kb);
  check(frank_lowrank_add_batched(m, n, 1, kmax, lra_name().c_str(), A.eps, dUa.buf.p, m, 0, dSa.buf.p, kmax, 0,
                                  dVa.buf.p, kmax, 0, dka.p, dUb.buf.p, m, 0, dSb.buf.p, kb, 0, dVb.buf.p, kb, 0,
                                  dkb.p, kb, nullptr),
        "frank_lowrank_add_batched");
  int r = 0;
  dka.download(&r);
  Dense U2, S2, V2;
  dUa.to(U2);
  dSa.to(S2);
  dVa.to(V2);
  A.rank = r;
  A.U = Dense(m, r);
  A.S = Dense(r, r);
  A.V = Dense(r, n);
  for (int i = 0; i < m; ++i) for (int c = 0; c < r; ++c) A.U(i, c) = U2(i, c);
  for (int i = 0; i < r; ++i) for (int c = 0; c < r; ++c) A.S(i, c) = S2(i, c);
  for (int i = 0; i < r; ++i) for (int c = 0; c < n; ++c) A.V(i, c) = V2(i, c);
  return A;
}

define_method(Matrix&, addition_omm, (Matrix&, const Matrix&)) {
  unsupported("operator+=: no overload for these matrix types");
}

Matrix& operator+=(Matrix& A, const Matrix& B) { return addition_omm(A, B); }

declare_method(void, qr_omm, (virtual_<Matrix&>, virtual_<Matrix&>, virtual_<Matrix&>))

define_method(void, qr_omm, (Dense& A, Dense& Q, Dense& R)) {
  const int m = (int)A.dim[0], n = (int)A.dim[1], k = std::min(m, n);
  if (Q.dim[0] != m || Q.dim[1] != k || R.dim[0] != k || R.dim[1] != n)
    throw Error(FRANK_ERR_INVALID, "qr: Q must be m x min(m, n) and R min(m, n) x n");
  DevDense dA(A), dQ(m, k), dR(k, n);
  check(frank_qr_batched(m, n, 1, dA.buf.p, m, 0, dQ.buf.p, m, 0, dR.buf.p, k, 0, nullptr), "frank_qr_batched");
  dQ.to(Q);
  dR.to(R);
}

define_method(void, qr_omm, (Matrix&, Matrix&, Matrix&)) { unsupported("qr: no overload for these matrix types"); }

void qr(Matrix& A, Matrix& Q, Matrix& R) { qr_omm(A, Q, R); }

declare_method(void, rq_omm, (virtual_<Matrix&>, virtual_<Matrix&>, virtual_<Matrix&>))

define_method(void, rq_omm, (Dense& A, Dense& R, Dense& Q)) {
  const int m = (int)A.dim[0], n = (int)A.dim[1], k = std::min(m, n);
  if (R.dim[0] != m || R.dim[1] != k || Q.dim[0] != k || Q.dim[1] != n)
    throw Error(FRANK_ERR_INVALID, "rq: R must be m x min(m, n) and Q min(m, n) x n");
  DevDense dA(A), dR(m, k), dQ(k, n);
  check(frank_rq_batched(m, n, 1, dA.buf.p, m, 0, dR.buf.p, m, 0, dQ.buf.p, k, 0, nullptr), "frank_rq_batched");
  dR.to(R);
  dQ.to(Q);
}

define_method(void, rq_omm, (Matrix&, Matrix&, Matrix&)) { unsupported("rq: no overload for these matrix types"); }

void rq(Matrix& A, Matrix& R, Matrix& Q) { rq_omm(A, R, Q); }

std::tuple<Dense, Dense, Dense> svd(Dense& A) {
  const int m = (int)A.dim[0], n = (int)A.dim[1], k = std::min(m, n);
  DevDense dA(A), dU(m, k), dS(k, 1), dV(k, n);
  check(frank_svd_batched(m, n, 1, dA.buf.p, m, 0, dU.buf.p, m, 0, dS.buf.p, 0, dV.buf.p, k, 0, nullptr),
        "frank_svd_batched");
  Dense U, s, V;
  dU.to(U);
  dS.to(s);
  dV.to(V);
  Dense S(k, k);   // svd.cpp returns S as a diagonal Dense
  for (int i = 0; i < k; ++i) S(i, i) = s(i, 0);
  return {std::move(U), std::move(S), std::move(V)};
}

std::tuple<Dense, Dense, Dense> rsvd(const Dense& A, const int64_t sample_size) {
  const int m = (int)A.dim[0], n = (int)A.dim[1], s = (int)std::min<int64_t>(sample_size, std::min(m, n));
  DevDense dA(A), dU(m, s), dS(s, s), dV(s, n);
  check(frank_rsvd_batched(m, n, 1, s, 0, 0, dA.buf.p, m, 0, dU.buf.p, m, 0, dS.buf.p, s, 0, dV.buf.p, s, 0, nullptr),
        "frank_rsvd_batched");
  Dense U, S, V;
  dU.to(U);
  dS.to(S);
  dV.to(V);
  return {std::move(U), std::move(S), std::move(V)};
}

namespace {
std::tuple<Dense, Dense, Dense, std::vector<int64_t>, std::vector<int64_t>> id_impl(const Dense& A, int64_t k) {
  const int m = (int)A.dim[0], n = (int)A.dim[1], kk = (int)k;
  DevDense dA(A), dU(m, kk), dS(kk, kk), dV(kk, n);
  DeviceBuffer<int> rows(kk), cols(kk);
  check(frank_id_batched(m, n, 1, kk, dA.buf.p, m, 0, dU.buf.p, m, 0, dS.buf.p, kk, 0, dV.buf.p, kk, 0, rows.p,
                         cols.p, nullptr),
        "frank_id_batched");
  std::vector<int> r(kk), c(kk);
  rows.download(r.data());
  cols.download(c.data());
  Dense U, S, V;
  dU.to(U);
  dS.to(S);
  dV.to(V);
  return {std::move(U), std::move(S), std::move(V), std::vector<int64_t>(r.begin(), r.end()),
          std::vector<int64_t>(c.begin(), c.end())};
}
}  // namespace

using DenseTriplet = std::tuple<Dense, Dense, Dense>;
using DenseIndexSetPair = std::tuple<Dense, std::vector<int64_t>>;

declare_method(DenseTriplet, id_omm, (virtual_<Matrix&>, const int64_t))

define_method(DenseTriplet, id_omm, (Dense& A, const int64_t k)) {
  auto t = id_impl(A, k);
  return DenseTriplet(std::move(std::get<0>(t)), std::move(std::get<1>(t)), std::move(std::get<2>(t)));
}

define_method(DenseTriplet, id_omm, (Matrix&, const int64_t)) { unsupported("id: no overload for this matrix type"); }

std::tuple<Dense, Dense, Dense> id(Matrix& A, const int64_t k) { return id_omm(A, k); }

declare_method(DenseIndexSetPair, one_sided_id_omm, (virtual_<Matrix&>, const int64_t))

define_method(DenseIndexSetPair, one_sided_id_omm, (Dense& A, const int64_t k)) {
  auto t = id_impl(A, k);   // the column ID is the first half of the two-sided one
  return DenseIndexSetPair(std::move(std::get<2>(t)), std::move(std::get<4>(t)));
}

define_method(DenseIndexSetPair, one_sided_id_omm, (Matrix&, const int64_t)) {
  unsupported("one_sided_id: no overload for this matrix type");
}

std::tuple<Dense, std::vector<int64_t>> one_sided_id(Matrix& A, const int64_t k) { return one_sided_id_omm(A, k); }

std::tuple<Dense, Dense, Dense> rid(const Dense& A, const int64_t sample_size, const int64_t rank) {
  const int m = (int)A.dim[0], n = (int)A.dim[1], s = (int)sample_size, k = (int)rank;
  DevDense dA(A), dU(m, k), dS(k, k), dV(k, n);
  check(frank_rid_batched(m, n, 1, s, k, dA.buf.p, m, 0, dU.buf.p, m, 0, dS.buf.p, k, 0, dV.buf.p, k, 0, nullptr),
        "frank_rid_batched");
  Dense U, S, V;
  dU.to(U);
  dS.to(S);
  dV.to(V);
  return {std::move(U), std::move(S), std::move(V)};
}

double l2_error(const Matrix& A, const Matrix& B) {
  auto* a = dynamic_cast<const Dense*>(&A);
  auto* b = dynamic_cast<const Dense*>(&B);
  if (!a || !b || a->dim != b->dim) unsupported("l2_error: two Dense matrices of equal shape");
  double num = 0.0, den = 0.0;
  for (int64_t i = 0; i < a->dim[0]; ++i)
    for (int64_t j = 0; j < a->dim[1]; ++j) {
      const double d = (*a)(i, j) - (*b)(i, j);
      num += d * d;
      den += (*a)(i, j) * (*a)(i, j);
    }
  return std::sqrt(num / den);
}

}  // namespace FRANK
