// TEST INFRASTRUCTURE ONLY.  Driver of the reference itself: the FRANK
// sources, compiled unmodified into oracle/_ref by oracle/build_ref.py, run
// through FRANK's own public API on the BLR / H-LU factor-and-solve path the
// engine replaces.  Used to pin the CPU oracle and the GPU path to the
// reference's actual outputs (fixtures under tests/golden) and as the timed
// CPU baseline of bench.py (`--impl reference`).  Nothing in the engine links
// or runs it.
//
// The sequence mirrors examples/h_lu.cpp:19-54 and
// test/blr_fixed_acc_test.cpp:67-83:
//   Hierarchical A(kernel, points, n, n, rank | eps, nleaf, admis, nb, nb);
//   b = A x  (x = random_uniform, as the tests do) or b from a file;
//   std::tie(L, U) = getrf(A); trsm(L, b, Lower); trsm(U, b, Upper);
// and reports (one JSON line on stdout) the timings (std::chrono), the solve
// error l2_error(x, x_hat), the residual ||b - A_H x_hat|| / ||b|| and the
// factorization error ||A_H V - L (U V)||_F / ||A_H V||_F on random probes,
// the ranks of A_H and of the factor, and optionally binary dumps of the
// factor blocks and of x_hat.
//
// Usage: frank_ref --n N --nb NB (--rank K | --eps E) [--nleaf L] [--admis A]
//   [--lra naive|rounded_addition|fast] [--kernel laplace|neglog|exp]
//   [--kparams p0,p1] [--points FILE --dim D] [--rhs FILE --nrhs K]
//   [--admis-type position|geometry] [--residual] [--factor-error]
//   [--dump-factor FILE] [--dump-x FILE] [--threads T] [--repeat R] [--no-solve]
//   [--write-json FILE]   (write_JSON of A_H, util/print.cpp:124-128)
#include "FRANK/FRANK.h"

#include <cblas.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <tuple>
#include <vector>

using namespace FRANK;

namespace {

// Kernels of the batched / adjoint workloads, passed through the reference's
// kernel plugin signature (functions.h:192-201); their parameters travel in
// this side channel because the signature carries only the coordinates.
double g_p0 = 0.0, g_p1 = 0.0;

double dist(const std::vector<std::vector<double>>& x, int64_t i, int64_t j) {
  double r2 = 0.0;
  for (const auto& ax : x) {
    const double d = ax[i] - ax[j];
    r2 += d * d;
  }
  return std::sqrt(r2);
}

void neglog_kernel(double* A, const uint64_t rows, const uint64_t cols, const uint64_t stride,
                   const std::vector<std::vector<double>>& x, const int64_t r0, const int64_t c0) {
  for (uint64_t i = 0; i < rows; ++i)
    for (uint64_t j = 0; j < cols; ++j) {
      const int64_t gi = r0 + (int64_t)i, gj = c0 + (int64_t)j;
      A[i * stride + j] = -std::log(dist(x, gi, gj) + 1e-3) + (gi == gj ? g_p0 : 0.0);
    }
}

void exp_kernel(double* A, const uint64_t rows, const uint64_t cols, const uint64_t stride,
                const std::vector<std::vector<double>>& x, const int64_t r0, const int64_t c0) {
  for (uint64_t i = 0; i < rows; ++i)
    for (uint64_t j = 0; j < cols; ++j) {
      const int64_t gi = r0 + (int64_t)i, gj = c0 + (int64_t)j;
      A[i * stride + j] = std::exp(-dist(x, gi, gj) / g_p0) + (gi == gj ? g_p1 : 0.0);
    }
}

struct Args {
  int64_t n = 0, nb = 0, rank = 0, nleaf = 0, nrhs = 1;
  double eps = 0.0, admis = 0.0;
  int dim = 1, threads = 0, repeat = 1;
  std::string lra, kernel = "laplace", points, rhs, dump_factor, dump_x, write_json;
  bool residual = false, factor_error = false, solve = true, geometry = false;
};

[[noreturn]] void usage(const char* msg) {
  std::fprintf(stderr, "frank_ref: %s\n", msg);
  std::exit(2);
}

Args parse(int argc, char** argv) {
  Args a;
  for (int k = 1; k < argc; ++k) {
    const std::string f = argv[k];
    auto val = [&]() -> std::string {
      if (k + 1 >= argc) usage(("missing value for " + f).c_str());
      return argv[++k];
    };
    if (f == "--n") a.n = std::atoll(val().c_str());
    else if (f == "--nb") a.nb = std::atoll(val().c_str());
    else if (f == "--rank") a.rank = std::atoll(val().c_str());
    else if (f == "--eps") a.eps = std::atof(val().c_str());
    else if (f == "--nleaf") a.nleaf = std::atoll(val().c_str());
    else if (f == "--admis") a.admis = std::atof(val().c_str());
    else if (f == "--lra") a.lra = val();
    else if (f == "--kernel") a.kernel = val();
    else if (f == "--kparams") {
      const std::string v = val();
      std::sscanf(v.c_str(), "%lf,%lf", &g_p0, &g_p1);
    } else if (f == "--points") a.points = val();
    else if (f == "--dim") a.dim = std::atoi(val().c_str());
    else if (f == "--rhs") a.rhs = val();
    else if (f == "--nrhs") a.nrhs = std::atoll(val().c_str());
    else if (f == "--residual") a.residual = true;
    else if (f == "--factor-error") a.factor_error = true;
    else if (f == "--dump-factor") a.dump_factor = val();
    else if (f == "--dump-x") a.dump_x = val();
    else if (f == "--threads") a.threads = std::atoi(val().c_str());
    else if (f == "--repeat") a.repeat = std::atoi(val().c_str());
    else if (f == "--no-solve") a.solve = false;
    else if (f == "--write-json") a.write_json = val();
    else if (f == "--admis-type") {
      const std::string v = val();
      if (v == "geometry") a.geometry = true;
      else if (v != "position") usage("--admis-type is position or geometry");
    }
    else usage(("unknown flag " + f).c_str());
  }
  if (a.n <= 0 || a.nb <= 0) usage("need --n and --nb");
  if ((a.rank > 0) == (a.eps > 0.0)) usage("need exactly one of --rank and --eps");
  if (a.nleaf <= 0) a.nleaf = (a.n + a.nb - 1) / a.nb;
  return a;
}

std::vector<double> read_doubles(const std::string& path, size_t count) {
  std::vector<double> v(count);
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) usage(("cannot open " + path).c_str());
  if (std::fread(v.data(), sizeof(double), count, f) != count) usage(("short file " + path).c_str());
  std::fclose(f);
  return v;
}

double fro(const Dense& A) {
  double s = 0.0;
  for (int64_t i = 0; i < A.dim[0]; ++i)
    for (int64_t j = 0; j < A.dim[1]; ++j) s += A(i, j) * A(i, j);
  return std::sqrt(s);
}

// Ranks of the blocks of a one-level BLR matrix (-1: dense), row-major nb x nb.
std::vector<int64_t> block_ranks(const Hierarchical& H) {
  std::vector<int64_t> r;
  for (int64_t i = 0; i < H.dim[0]; ++i)
    for (int64_t j = 0; j < H.dim[1]; ++j) {
      const Matrix& m = H(i, j);
      const auto* lr = dynamic_cast<const LowRank*>(&m);
      r.push_back(lr ? lr->rank : -1);
    }
  return r;
}

void write_dense(FILE* f, const Dense& D) {
  for (int64_t i = 0; i < D.dim[0]; ++i)
    for (int64_t j = 0; j < D.dim[1]; ++j) {
      const double v = D(i, j);
      std::fwrite(&v, sizeof v, 1, f);
    }
}

// Block (i, j) as: int64 i, j, type (0 dense, 1 low rank, 2 other), rows,
// cols, rank; then dense data (row-major) or U (rows x rank), S (rank x
// rank), V (rank x cols), row-major.
void dump_block(FILE* f, int64_t i, int64_t j, const Matrix& m) {
  int64_t hdr[6] = {i, j, 2, 0, 0, 0};
  if (const auto* d = dynamic_cast<const Dense*>(&m)) {
    hdr[2] = 0; hdr[3] = d->dim[0]; hdr[4] = d->dim[1];
    std::fwrite(hdr, sizeof hdr, 1, f);
    write_dense(f, *d);
  } else if (const auto* lr = dynamic_cast<const LowRank*>(&m)) {
    hdr[2] = 1; hdr[3] = lr->dim[0]; hdr[4] = lr->dim[1]; hdr[5] = lr->rank;
    std::fwrite(hdr, sizeof hdr, 1, f);
    write_dense(f, lr->U);
    write_dense(f, lr->S);
    write_dense(f, lr->V);
  } else {
    std::fwrite(hdr, sizeof hdr, 1, f);
  }
}

// y (n x c, row-major, zeroed by the caller) += H x for a one-level block
// matrix whose blocks are Dense, LowRank or Empty (the factors L and U);
// block offsets from the row counts of the diagonal blocks.
void block_apply(const Hierarchical& H, const std::vector<double>& x, std::vector<double>& y, int64_t c) {
  std::vector<int64_t> off(1, 0);
  for (int64_t i = 0; i < H.dim[0]; ++i) {
    const Matrix& m = H(i, i);
    int64_t rows = 0;
    if (const auto* d = dynamic_cast<const Dense*>(&m)) rows = d->dim[0];
    else if (const auto* lr = dynamic_cast<const LowRank*>(&m)) rows = lr->dim[0];
    off.push_back(off.back() + rows);
  }
  for (int64_t i = 0; i < H.dim[0]; ++i)
    for (int64_t j = 0; j < H.dim[1]; ++j) {
      const Matrix& m = H(i, j);
      const double* xj = x.data() + off[j] * c;
      double* yi = y.data() + off[i] * c;
      if (const auto* d = dynamic_cast<const Dense*>(&m)) {
        for (int64_t r = 0; r < d->dim[0]; ++r)
          for (int64_t k = 0; k < d->dim[1]; ++k)
            for (int64_t h = 0; h < c; ++h) yi[r * c + h] += (*d)(r, k) * xj[k * c + h];
      } else if (const auto* lr = dynamic_cast<const LowRank*>(&m)) {
        std::vector<double> t1(lr->rank * c, 0.0), t2(lr->rank * c, 0.0);
        for (int64_t a = 0; a < lr->rank; ++a)
          for (int64_t k = 0; k < lr->dim[1]; ++k)
            for (int64_t h = 0; h < c; ++h) t1[a * c + h] += lr->V(a, k) * xj[k * c + h];
        for (int64_t a = 0; a < lr->rank; ++a)
          for (int64_t e = 0; e < lr->rank; ++e)
            for (int64_t h = 0; h < c; ++h) t2[a * c + h] += lr->S(a, e) * t1[e * c + h];
        for (int64_t r = 0; r < lr->dim[0]; ++r)
          for (int64_t a = 0; a < lr->rank; ++a)
            for (int64_t h = 0; h < c; ++h) yi[r * c + h] += lr->U(r, a) * t2[a * c + h];
      }
    }
}

std::string join(const std::vector<int64_t>& v) {
  std::string s = "[";
  for (size_t k = 0; k < v.size(); ++k) s += (k ? "," : "") + std::to_string(v[k]);
  return s + "]";
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

int main(int argc, char** argv) {
  const Args a = parse(argc, argv);
  if (a.threads > 0) scipy_openblas_set_num_threads(a.threads);
  initialize();
  if (a.lra == "naive") setGlobalValue("FRANK_LRA", "naive");
  else if (a.lra == "rounded_addition") setGlobalValue("FRANK_LRA", "rounded_addition");
  else if (!a.lra.empty() && a.lra != "fast") usage("unknown --lra");

  std::vector<std::vector<double>> x;
  if (a.points.empty()) {
    x.emplace_back(get_sorted_random_vector(a.n));   // util/experiment_setup.cpp:12-23
  } else {
    const std::vector<double> flat = read_doubles(a.points, (size_t)a.dim * a.n);
    for (int d = 0; d < a.dim; ++d) x.emplace_back(flat.begin() + (size_t)d * a.n, flat.begin() + (size_t)(d + 1) * a.n);
  }
  auto kernel = a.kernel == "laplace" ? laplacend : a.kernel == "neglog" ? neglog_kernel
              : a.kernel == "exp" ? exp_kernel : nullptr;
  if (!kernel) usage("unknown --kernel");

  auto t0 = std::chrono::steady_clock::now();
  const AdmisType at = a.geometry ? AdmisType::GeometryBased : AdmisType::PositionBased;
  Hierarchical A = a.rank > 0 ? Hierarchical(kernel, x, a.n, a.n, a.rank, a.nleaf, a.admis, a.nb, a.nb, at)
                              : Hierarchical(kernel, x, a.n, a.n, a.nleaf, a.eps, a.admis, a.nb, a.nb, at);
  const double t_build = seconds_since(t0);
  const std::vector<int64_t> ranks_h = block_ranks(A);
  if (!a.write_json.empty()) write_JSON(A, a.write_json);

  // right-hand sides: b = A x with x = random_uniform (the tests' choice) or from a file
  Dense xtrue, b;
  if (a.rhs.empty()) {
    xtrue = Dense(random_uniform, {}, a.n, 1);
    b = Dense(a.n, 1);
    gemm(A, xtrue, b, 1, 1);
  } else {
    const std::vector<double> flat = read_doubles(a.rhs, (size_t)a.n * a.nrhs);  // column-major n x nrhs
    b = Dense(a.n, a.nrhs);
    for (int64_t c = 0; c < a.nrhs; ++c)
      for (int64_t r = 0; r < a.n; ++r) b(r, c) = flat[(size_t)c * a.n + r];
  }
  // probes for the factorization error, and the copy of A_H for the residual
  Dense probe, ap;
  if (a.factor_error) {
    probe = Dense(random_normal, {}, a.n, 4);
    ap = Dense(a.n, 4);
    gemm(A, probe, ap, 1, 0);
  }
  Hierarchical Acopy;
  if (a.residual) Acopy = Hierarchical(A);

  std::vector<double> t_getrf, t_solve;
  Hierarchical L, U;
  Dense xs;
  for (int rep = 0; rep < a.repeat; ++rep) {
    Hierarchical Aw = rep + 1 < a.repeat ? Hierarchical(A) : std::move(A);
    t0 = std::chrono::steady_clock::now();
    std::tie(L, U) = getrf(Aw);
    t_getrf.push_back(seconds_since(t0));
    if (a.solve) {
      xs = Dense(b);
      t0 = std::chrono::steady_clock::now();
      trsm(L, xs, Mode::Lower);
      trsm(U, xs, Mode::Upper);
      t_solve.push_back(seconds_since(t0));
    }
  }

  std::printf("{\"n\": %lld, \"nb\": %lld, \"nleaf\": %lld, \"rank\": %lld, \"eps\": %.3e, \"admis\": %g, "
              "\"lra\": \"%s\", \"kernel\": \"%s\", \"build_s\": %.6f, \"getrf_s\": [",
              (long long)a.n, (long long)a.nb, (long long)a.nleaf, (long long)a.rank, a.eps, a.admis,
              getGlobalValue("FRANK_LRA").c_str(), a.kernel.c_str(), t_build);
  for (size_t k = 0; k < t_getrf.size(); ++k) std::printf("%s%.6f", k ? ", " : "", t_getrf[k]);
  std::printf("], \"solve_s\": [");
  for (size_t k = 0; k < t_solve.size(); ++k) std::printf("%s%.6f", k ? ", " : "", t_solve[k]);
  std::printf("]");
  if (a.solve && a.rhs.empty()) std::printf(", \"solve_error\": %.6e", l2_error(xtrue, xs));
  if (a.solve && a.residual) {
    Dense r(b);
    gemm(Acopy, xs, r, -1, 1);
    std::printf(", \"residual\": %.6e", fro(r) / fro(b));
  }
  if (a.factor_error) {
    const int64_t c = probe.dim[1];
    std::vector<double> v((size_t)a.n * c), uv(v.size(), 0.0), luv(v.size(), 0.0);
    for (int64_t r = 0; r < a.n; ++r)
      for (int64_t h = 0; h < c; ++h) v[r * c + h] = probe(r, h);
    block_apply(U, v, uv, c);
    block_apply(L, uv, luv, c);
    double num = 0.0, den = 0.0;
    for (int64_t r = 0; r < a.n; ++r)
      for (int64_t h = 0; h < c; ++h) {
        const double d = ap(r, h) - luv[r * c + h];
        num += d * d;
        den += ap(r, h) * ap(r, h);
      }
    std::printf(", \"factor_error\": %.6e", std::sqrt(num / den));
  }
  std::printf(", \"ranks_h\": %s", join(ranks_h).c_str());
  std::printf(", \"ranks_l\": %s, \"ranks_u\": %s", join(block_ranks(L)).c_str(), join(block_ranks(U)).c_str());
  std::printf("}\n");

  if (!a.dump_factor.empty()) {
    FILE* f = std::fopen(a.dump_factor.c_str(), "wb");
    if (!f) usage("cannot write the factor dump");
    for (int64_t i = 0; i < L.dim[0]; ++i)
      for (int64_t j = 0; j < L.dim[1]; ++j) {
        if (i >= j) dump_block(f, i, j, L(i, j));
        if (i <= j) dump_block(f, i, j, U(i, j));
      }
    std::fclose(f);
  }
  if (!a.dump_x.empty() && a.solve) {
    FILE* f = std::fopen(a.dump_x.c_str(), "wb");
    if (!f) usage("cannot write x");
    for (int64_t c = 0; c < xs.dim[1]; ++c)
      for (int64_t r = 0; r < xs.dim[0]; ++r) {
        const double v = xs(r, c);
        std::fwrite(&v, sizeof v, 1, f);
      }
    std::fclose(f);
  }
  return 0;
}
