// Per-operation entry points of the C ABI (batched, FP64, device buffers,
// column-major): the dense factorizations and low-rank operations of FRANK's
// operator set that the factor-and-solve path is built from, exposed one
// operation at a time for callers that work on individual blocks (FRANK's
// multimethods qr, rq, svd, rsvd, id, rid and LowRank += LowRank).
//
// One CTA per matrix of the batch; every routine is the cooperative CTA code
// of common.cuh (Householder QR, Q application, column-pivoted QR, one-sided
// Jacobi, CTA GEMM) working on a per-matrix FP64 scratch slot in global
// memory, allocated from the stream-ordered pool for the call.
#include "common.cuh"
#include "ops_tasks.h"
#include "../../include/frank_b200.h"

#include <algorithm>
#include <random>
#include <string>
#include <vector>

namespace frank {
// defined in api.cu: sets the calling thread's error text, returns `code`
int set_error(int code, const std::string& msg);
}  // namespace frank

namespace frank {
namespace ops {

constexpr int OT = 256;                // threads per CTA
constexpr int GSM = 2 * 16 * 64;       // cta_gemm tile buffer (doubles)

enum { OPS_ERR_JACOBI = 0, OPS_ERR_SLOTS = 2 };

// ---------------------------------------------------------------------------
// Device building blocks (all threads of the CTA; each ends with a barrier)
// ---------------------------------------------------------------------------

// Explicit Q (m x k, ldq) = H_0 ... H_{k-1} [I; 0] from reflectors V (ldv).
FRANK_D void form_q(int m, int k, const double* V, int64_t ldv, const double* tau, double* Q, int64_t ldq) {
  for (int64_t e = threadIdx.x; e < (int64_t)m * k; e += blockDim.x) {
    const int r = e % m, c = e / m;
    Q[r + (int64_t)c * ldq] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  cta_apply_q(m, k, V, ldv, tau, k, Q, ldq);
}

// Thin SVD of G's leading m x n (ld m + n, m >= n) by one-sided Jacobi with
// the right singular vectors accumulated in rows m .. m+n-1 (which the caller
// fills with the identity).  On return sig[c] (unsorted) is the norm of
// column c of the rotated G(0:m, :), ord[j] the column of the j-th largest.
// Returns false when the sweeps did not converge.
FRANK_D bool jacobi_svd(int m, int n, double* G, double* sig, int* ord, int* flag) {
  const int sweeps = cta_jacobi_columns(m, n, G, m + n, 60, flag, m + n);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c = wid; c < n; c += nw) {
    double s = 0.0;
    for (int r = lane; r < m; r += 32) s += G[r + (int64_t)c * (m + n)] * G[r + (int64_t)c * (m + n)];
    s = warp_sum(s);
    if (lane == 0) sig[c] = sqrt(s);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    const double v = sig[c];
    int pos = 0;
    for (int d = 0; d < n; ++d) pos += (sig[d] > v) || (sig[d] == v && d < c);
    ord[pos] = c;
  }
  __syncthreads();
  return sweeps >= 0;
}

// Load a (m x n, lda) as G = [a; I] or, transposed, G = [a^T; I] into a
// (rows + cols) x cols slot, so that jacobi_svd factors the tall side.
FRANK_D void load_svd(int m, int n, const double* a, int64_t lda, bool trans, double* G) {
  const int mm = trans ? n : m, nn = trans ? m : n;
  for (int64_t e = threadIdx.x; e < (int64_t)(mm + nn) * nn; e += blockDim.x) {
    const int r = e % (mm + nn), c = e / (mm + nn);
    double v;
    if (r < mm) v = trans ? a[c + (int64_t)r * lda] : a[r + (int64_t)c * lda];
    else v = (r - mm == c) ? 1.0 : 0.0;
    G[e] = v;
  }
  __syncthreads();
}

// SVD of a (m x n, lda): U (m x k, ldu), s (k), Vt (k x n, ldvt), k = min(m, n),
// singular values descending; columns with a zero singular value get a zero
// left vector.  Scratch: (m + n) * k + 2 k doubles.  Returns false on a
// Jacobi sweep limit.  When shm holds at least (max(m, n) + k) k doubles the
// rotated matrix lives there instead of in the scratch (the sweeps are a
// chain of dependent column loads, so shared memory's latency sets their
// pace; the scratch layout is unchanged).
FRANK_D bool cta_svd(int m, int n, const double* a, int64_t lda, double* U, int64_t ldu, double* s, double* Vt,
                     int64_t ldvt, double* scratch, int* flag, double* shm = nullptr, int64_t shm_cap = 0) {
  const bool trans = m < n;
  const int mm = trans ? n : m, k = trans ? m : n;
  double* G = (shm && (int64_t)(mm + k) * k <= shm_cap) ? shm : scratch;
  double* sig = scratch + (int64_t)(mm + k) * k;
  int* ord = reinterpret_cast<int*>(sig + k);
  load_svd(m, n, a, lda, trans, G);
  const bool ok = jacobi_svd(mm, k, G, sig, ord, flag);
  const int64_t ldg = mm + k;
  // tall side: left vectors of the factored matrix; short side: the rotations
  for (int64_t e = threadIdx.x; e < (int64_t)mm * k; e += blockDim.x) {
    const int r = e % mm, j = e / mm, c = ord[j];
    const double sv = sig[c];
    const double v = sv > 0.0 ? G[r + (int64_t)c * ldg] / sv : 0.0;
    if (!trans) U[r + (int64_t)j * ldu] = v;
    else Vt[j + (int64_t)r * ldvt] = v;
  }
  for (int64_t e = threadIdx.x; e < (int64_t)k * k; e += blockDim.x) {
    const int r = e % k, j = e / k, c = ord[j];
    const double v = G[mm + r + (int64_t)c * ldg];
    if (!trans) Vt[j + (int64_t)r * ldvt] = v;
    else U[r + (int64_t)j * ldu] = v;
  }
  for (int j = threadIdx.x; j < k; j += blockDim.x) s[j] = sig[ord[j]];
  __syncthreads();
  return ok;
}

// SVD of a square a (n x n, lda) preconditioned by column-pivoted QR
// (Drmac and Veselic, "New fast and accurate Jacobi SVD algorithm", 2008):
// a P = Q R, one-sided Jacobi on the columns of R^T with the rotations V
// accumulated, R^T V = Y; then a = (Q V) diag(sigma) (P Y diag(1/sigma))^T.
// The pivoted R is graded, so the sweeps converge in a few passes.  All of it
// in shared memory shm (3 n^2 doubles); sc: 4 n doubles + 2 n ints (global).
// Outputs as cta_svd.
FRANK_D bool cta_svd_pqr(int n, const double* a, int64_t lda, double* U, int64_t ldu, double* s, double* Vt,
                         int64_t ldvt, double* sc, double* shm, int* flag, double* red, int* redi) {
  double* W = shm;                                  // n x n: R above, reflectors below
  double* G = shm + (int64_t)n * n;                 // 2n x n (ld 2n): [R^T; I], rotated
  double* tau = sc;
  double* cn = tau + n;
  double* pn = cn + n;
  double* sig = pn + n;
  int* jpvt = reinterpret_cast<int*>(sig + n);
  int* ord = jpvt + n;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) W[e] = a[e % n + (int64_t)(e / n) * lda];
  __syncthreads();
  cta_truncated_geqp3(n, n, W, n, -1.0, n, tau, cn, pn, jpvt, red, redi);
  __syncthreads();
  const int ldg = 2 * n;
  for (int e = threadIdx.x; e < ldg * n; e += blockDim.x) {
    const int r = e % ldg, c = e / ldg;
    G[e] = r < n ? (c <= r ? W[c + r * n] : 0.0) : (r - n == c ? 1.0 : 0.0);
  }
  __syncthreads();
  const bool ok = jacobi_svd(n, n, G, sig, ord, flag);
  cta_apply_q(n, n, W, n, tau, n, G + n, ldg);     // rows n..2n-1 become Q V
  __syncthreads();
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e % n, j = e / n, c = ord[j];
    U[r + (int64_t)j * ldu] = G[n + r + c * ldg];
    const double sv = sig[c];
    Vt[j + (int64_t)jpvt[r] * ldvt] = sv > 0.0 ? G[r + c * ldg] / sv : 0.0;
  }
  for (int j = threadIdx.x; j < n; j += blockDim.x) s[j] = sig[ord[j]];
  __syncthreads();
  return ok;
}

// The first k steps of the column-pivoted QR of W (m x n, ld m) in place;
// jpvt (n): original column at pivoted position.  geqp3
// (operations/LAPACK/geqp3.cpp:36-69: LAPACKE_dgeqp3) pivots greedily on the
// largest remaining column norm, so its first k pivots and the first k rows
// of R are those of the first k steps; the ID uses nothing else.
FRANK_D void cta_geqp3(int m, int n, int k, double* W, double* tau, double* cn, double* pn, int* jpvt, double* red,
                       int* redi) {
  cta_truncated_geqp3(m, n, W, m, -1.0, k, tau, cn, pn, jpvt, red, redi);
}

// one_sided_id (operations/LAPACK/id.cpp:49-73) of a (m x n, lda), rank k:
// V (k x n, ldv) with V(:, P(j)) = e_j (j < k), (R11^{-1} R12)(:, j - k)
// (j >= k); cols[0..k) = P(0..k).  Scratch: m n + 3 n + k n doubles + n ints.
FRANK_D void cta_one_sided_id(int m, int n, int k, const double* a, int64_t lda, bool trans, double* V, int64_t ldv,
                              int* cols, double* scratch, double* red, int* redi) {
  double* W = scratch;                         // m x n (ld m)
  double* tau = W + (int64_t)m * n;
  double* cn = tau + n;
  double* pn = cn + n;
  double* X = pn + n;                          // k x (n - k), ld k
  int* jpvt = reinterpret_cast<int*>(X + (int64_t)k * n);
  for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) {
    const int r = e % m, c = e / m;
    W[e] = trans ? a[c + (int64_t)r * lda] : a[r + (int64_t)c * lda];
  }
  __syncthreads();
  cta_geqp3(m, n, k, W, tau, cn, pn, jpvt, red, redi);
  const bool solve = k < min(m, n) || n > m;
  if (solve) {
    for (int64_t e = threadIdx.x; e < (int64_t)k * (n - k); e += blockDim.x) {
      const int r = e % k, c = e / k;
      X[e] = W[r + (int64_t)(k + c) * m];
    }
    __syncthreads();
    cta_upper_solve(k, W, m, n - k, X, k);
  }
  for (int64_t e = threadIdx.x; e < (int64_t)k * n; e += blockDim.x) {
    const int r = e % k, j = e / k;
    const double v = j < k ? (r == j ? 1.0 : 0.0) : (solve ? X[r + (int64_t)(j - k) * k] : 0.0);
    V[r + (int64_t)jpvt[j] * ldv] = v;
  }
  for (int j = threadIdx.x; j < k; j += blockDim.x) cols[j] = jpvt[j];
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Kernels (grid = batch count)
// ---------------------------------------------------------------------------

struct Mat {
  double* p;
  int64_t ld, stride;
  FRANK_D double* at(int b) const { return p + (int64_t)b * stride; }
};

// qr (operations/LAPACK/qr.cpp:65-90): Q (m x k), R (k x n), k = min(m, n).
__global__ void __launch_bounds__(OT) k_op_qr(int m, int n, Mat A, Mat Q, Mat R, double* scratch, int64_t ws) {
  __shared__ double red[32];
  const int b = blockIdx.x, k = min(m, n);
  double* W = scratch + (int64_t)b * ws;
  double* tau = W + (int64_t)m * n;
  const double* a = A.at(b);
  for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) W[e] = a[e % m + (e / m) * A.ld];
  __syncthreads();
  cta_householder_qr(m, n, W, m, tau, red);
  double* r = R.at(b);
  for (int64_t e = threadIdx.x; e < (int64_t)k * n; e += blockDim.x) {
    const int i = e % k, c = e / k;
    r[i + (int64_t)c * R.ld] = i <= c ? W[i + (int64_t)c * m] : 0.0;
  }
  form_q(m, k, W, m, tau, Q.at(b), Q.ld);
}

// rq (operations/LAPACK/rq.cpp:43-70): A = R Q, R (m x k), Q (k x n) with
// orthonormal rows.  From the QR of B = (J_m A)^T = Q1 R1 (J = reversal):
// R = J_m R1^T J_k, Q = J_k Q1^T.
__global__ void __launch_bounds__(OT) k_op_rq(int m, int n, Mat A, Mat R, Mat Q, double* scratch, int64_t ws) {
  __shared__ double red[32];
  const int b = blockIdx.x, k = min(m, n);
  double* W = scratch + (int64_t)b * ws;       // n x m, ld n
  double* tau = W + (int64_t)m * n;
  double* Q1 = tau + k;                         // n x k, ld n
  const double* a = A.at(b);
  for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) {
    const int r = e % n, c = e / n;             // B(r, c) = A(m-1-c, r)
    W[e] = a[(m - 1 - c) + (int64_t)r * A.ld];
  }
  __syncthreads();
  cta_householder_qr(n, m, W, n, tau, red);
  form_q(n, k, W, n, tau, Q1, n);
  double* rr = R.at(b);
  for (int64_t e = threadIdx.x; e < (int64_t)m * k; e += blockDim.x) {
    const int i = e % m, c = e / m;             // R(i, c) = R1(k-1-c, m-1-i)
    const int p = k - 1 - c, q = m - 1 - i;
    rr[i + (int64_t)c * R.ld] = p <= q ? W[p + (int64_t)q * n] : 0.0;
  }
  double* qq = Q.at(b);
  for (int64_t e = threadIdx.x; e < (int64_t)k * n; e += blockDim.x) {
    const int i = e % k, c = e / k;             // Q(i, c) = Q1(c, k-1-i)
    qq[i + (int64_t)c * Q.ld] = Q1[c + (int64_t)(k - 1 - i) * n];
  }
}

// svd (operations/LAPACK/svd.cpp:23-44): U (m x k), s (k), Vt (k x n).
__global__ void __launch_bounds__(OT) k_op_svd(int m, int n, Mat A, Mat U, Mat S, Mat Vt, double* scratch, int64_t ws,
                                               int* err) {
  __shared__ int flag;
  const int b = blockIdx.x;
  if (!cta_svd(m, n, A.at(b), A.ld, U.at(b), U.ld, S.at(b), Vt.at(b), Vt.ld, scratch + (int64_t)b * ws, &flag) &&
      threadIdx.x == 0)
    atomicAdd(err + OPS_ERR_JACOBI, 1);
}

// Randomized range finder shared by rsvd / rid: Q (m x s, ld m) orthonormal
// basis of A Omega (plus `power` subspace iterations), B = Q^T A (s x n, ld s).
// Omega: n x s row-major (the reference's random_uniform fill order).
FRANK_D void range_finder(int m, int n, int s, int power, const double* a, int64_t lda, const double* omega,
                          double* Q, double* B, double* Z, double* tau, double* gsm, double* red) {
  // Y = A Omega into Q
  cta_gemm<double, OT>(m, s, n, 1.0, a, lda, false, omega, s, true, 0.0, Q, m, gsm);
  cta_householder_qr(m, s, Q, m, tau, red);
  form_q(m, s, Q, m, tau, B, m);               // B as scratch for the explicit Q (m x s)
  for (int64_t e = threadIdx.x; e < (int64_t)m * s; e += blockDim.x) Q[e] = B[e];
  __syncthreads();
  for (int it = 0; it < power; ++it) {
    // Z = A^T Q (n x s), orthonormalise, Y = A Z, orthonormalise
    cta_gemm<double, OT>(n, s, m, 1.0, a, lda, true, Q, m, false, 0.0, Z, n, gsm);
    cta_householder_qr(n, s, Z, n, tau, red);
    form_q(n, s, Z, n, tau, B, n);
    cta_gemm<double, OT>(m, s, n, 1.0, a, lda, false, B, n, false, 0.0, Q, m, gsm);
    cta_householder_qr(m, s, Q, m, tau, red);
    form_q(m, s, Q, m, tau, B, m);
    for (int64_t e = threadIdx.x; e < (int64_t)m * s; e += blockDim.x) Q[e] = B[e];
    __syncthreads();
  }
  // B = Q^T A (s x n)
  cta_gemm<double, OT>(s, n, m, 1.0, Q, m, true, a, lda, false, 0.0, B, s, gsm);
}

// rsvd (operations/randomized/rsvd.cpp:17-29, via LowRank(Dense, rank),
// low_rank.cpp:40-48): U (m x rank), S (rank x rank, diagonal), V (rank x n).
__global__ void __launch_bounds__(OT) k_op_rsvd(int m, int n, int s, int rank, int power, Mat A, const double* omega,
                                                Mat U, Mat S, Mat V, double* scratch, int64_t ws, int* err) {
  __shared__ double gsm[GSM];
  __shared__ double red[32];
  __shared__ int flag;
  const int b = blockIdx.x;
  double* Q = scratch + (int64_t)b * ws;       // m x s
  double* B = Q + (int64_t)m * s;               // max(m, n) x s
  double* Z = B + (int64_t)max(m, n) * s;       // n x s
  double* tau = Z + (int64_t)n * s;             // s
  double* Ub = tau + s;                         // s x s
  double* sv = Ub + (int64_t)s * s;             // s
  double* Vbt = sv + s;                         // s x n
  double* sc = Vbt + (int64_t)s * n;            // svd scratch
  range_finder(m, n, s, power, A.at(b), A.ld, omega, Q, B, Z, tau, gsm, red);
  if (!cta_svd(s, n, B, s, Ub, s, sv, Vbt, s, sc, &flag) && threadIdx.x == 0) atomicAdd(err + OPS_ERR_JACOBI, 1);
  // U = Q Ub(:, :rank), S = diag(sv), V = Vbt(:rank, :)
  cta_gemm<double, OT>(m, rank, s, 1.0, Q, m, false, Ub, s, false, 0.0, U.at(b), U.ld, gsm);
  double* sp = S.at(b);
  for (int64_t e = threadIdx.x; e < (int64_t)rank * rank; e += blockDim.x) {
    const int i = e % rank, c = e / rank;
    sp[i + (int64_t)c * S.ld] = i == c ? sv[i] : 0.0;
  }
  double* vp = V.at(b);
  for (int64_t e = threadIdx.x; e < (int64_t)rank * n; e += blockDim.x) {
    const int i = e % rank, c = e / rank;
    vp[i + (int64_t)c * V.ld] = Vbt[i + (int64_t)c * s];
  }
}

// id (operations/LAPACK/id.cpp:75-116) of a (m x n) at rank k: A ~= U S V with
// S = A(rows, cols) (k x k), U (m x k), V (k x n).  rid
// (operations/randomized/rid.cpp:18-31) runs it on Q^T A of the range
// finder and returns U = Q Ub.
FRANK_D void cta_id(int m, int n, int k, const double* a, int64_t lda, double* U, int64_t ldu, double* S, int64_t lds,
                    double* V, int64_t ldv, int* rows, int* cols, double* AC, double* Ut, double* scratch, double* red,
                    int* redi) {
  cta_one_sided_id(m, n, k, a, lda, false, V, ldv, cols, scratch, red, redi);
  // AC = A(:, cols) (m x k); one_sided_id of AC^T (k x m)
  for (int64_t e = threadIdx.x; e < (int64_t)m * k; e += blockDim.x) {
    const int r = e % m, c = e / m;
    AC[e] = a[r + (int64_t)cols[c] * lda];
  }
  __syncthreads();
  cta_one_sided_id(k, m, k, AC, m, true, Ut, k, rows, scratch, red, redi);
  for (int64_t e = threadIdx.x; e < (int64_t)m * k; e += blockDim.x) {
    const int r = e % m, c = e / m;
    U[r + (int64_t)c * ldu] = Ut[c + (int64_t)r * k];
  }
  for (int64_t e = threadIdx.x; e < (int64_t)k * k; e += blockDim.x) {
    const int r = e % k, c = e / k;
    S[r + (int64_t)c * lds] = AC[rows[r] + (int64_t)c * m];
  }
  __syncthreads();
}

__global__ void __launch_bounds__(OT) k_op_id(int m, int n, int k, Mat A, Mat U, Mat S, Mat V, int* rows, int* cols,
                                              double* scratch, int64_t ws) {
  __shared__ double red[32];
  __shared__ int redi[32];
  const int b = blockIdx.x;
  double* AC = scratch + (int64_t)b * ws;      // m x k
  double* Ut = AC + (int64_t)m * k;             // k x m
  double* sc = Ut + (int64_t)k * m;
  cta_id(m, n, k, A.at(b), A.ld, U.at(b), U.ld, S.at(b), S.ld, V.at(b), V.ld, rows + (int64_t)b * k,
         cols + (int64_t)b * k, AC, Ut, sc, red, redi);
}

__global__ void __launch_bounds__(OT) k_op_rid(int m, int n, int s, int k, Mat A, const double* omega, Mat U, Mat S,
                                               Mat V, double* scratch, int64_t ws) {
  __shared__ double gsm[GSM];
  __shared__ double red[32];
  __shared__ int redi[32];
  const int b = blockIdx.x;
  double* Q = scratch + (int64_t)b * ws;       // m x s
  double* B = Q + (int64_t)m * s;               // max(m, n) x s
  double* Z = B + (int64_t)max(m, n) * s;       // n x s
  double* tau = Z + (int64_t)n * s;
  double* Ub = tau + s;                         // s x k
  double* AC = Ub + (int64_t)s * k;             // s x k
  double* Ut = AC + (int64_t)s * k;             // k x s
  int* rw = reinterpret_cast<int*>(Ut + (int64_t)k * s);
  int* cl = rw + k;
  double* sc = reinterpret_cast<double*>(cl + k + (k & 1));
  range_finder(m, n, s, 0, A.at(b), A.ld, omega, Q, B, Z, tau, gsm, red);
  cta_id(s, n, k, B, s, Ub, s, S.at(b), S.ld, V.at(b), V.ld, rw, cl, AC, Ut, sc, red, redi);
  cta_gemm<double, OT>(m, k, s, 1.0, Q, m, false, Ub, s, false, 0.0, U.at(b), U.ld, gsm);
}

// LowRank += LowRank (operations/arithmetic/addition.cpp:93-127 rounded,
// 133-189 fast).  A = Ua Sa Va (m x ka, ka x ka, ka x n; written in place
// with the new rank, capacity kmax), B = Ub Sb Vb (kb).  rounded: QR of
// [Ua Sa | Ub Sb] and of [Va; Vb]^T, core M = Ru Rv^T, SVD, rank by
// find_svd_truncation_rank (misc.cpp:133-146, quirk included) when eps > 0,
// else ka.  fast (fixed rank, Ua and Va^T orthonormal): the projections
// Zu = Ua^T Ub, Zv = Va Vb^T, QR of the remainders only, core
// [I Zu; 0 Ru] blockdiag(Sa, Sb) [I Zv; 0 Rv]^T.
// Optional phase counters of the LowRank addition (build with
// -DFRANK_LRA_TIMING; off by default): [0] operands and projections,
// [1] QR of the remainders, [2] core and its SVD, [3] new bases, [4] count.
#ifdef FRANK_LRA_TIMING
__device__ unsigned long long g_lra_cycles[8];
#define LRA_MARK(k)                                                                          \
  do {                                                                                       \
    if (threadIdx.x == 0) {                                                                  \
      const long long _t = clock64();                                                        \
      atomicAdd(&g_lra_cycles[(k)], (unsigned long long)(_t - _lra_t0));                     \
      _lra_t0 = _t;                                                                          \
    }                                                                                        \
  } while (0)
#define LRA_BEGIN() long long _lra_t0 = clock64()
#else
#define LRA_MARK(k) do {} while (0)
#define LRA_BEGIN() do {} while (0)
#endif

FRANK_D void lr_add_body(int m, int n, int kmax, int fast, double eps, double* ua_out, int64_t ldua, double* sa_out,
                         int64_t ldsa, double* va_out, int64_t ldva, int* ka_io, const double* ub, int64_t ldub,
                         const double* sb, int64_t ldsb, const double* vb, int64_t ldvb, int kb, double* X, int* err,
                         double* shm, int64_t shm_cap) {
  __shared__ double gsm[GSM];
  __shared__ double red[32];
  __shared__ int redi[32];
  __shared__ int flag, s_rank;
  const int ka = *ka_io;
  const int kt = ka + kb;
  double* Y = X + (int64_t)m * kt;              // n x kt stacked V side (V^T columns)
  double* tu = Y + (int64_t)n * kt;             // kt
  double* tv = tu + kt;                         // kt
  double* Rc = tv + kt;                         // kt x kt
  double* Rv = Rc + (int64_t)kt * kt;           // kt x kt
  double* M = Rv + (int64_t)kt * kt;            // kt x kt
  double* Um = M + (int64_t)kt * kt;            // kt x kt
  double* sv = Um + (int64_t)kt * kt;           // kt
  double* Vmt = sv + kt;                        // kt x kt
  double* T = Vmt + (int64_t)kt * kt;           // max(m, n) x kt
  double* sc = T + (int64_t)max(m, n) * kt;     // svd scratch (2 kt + 2) kt
  const double *ua = ua_out, *sa = sa_out, *va = va_out;
  struct LD { int64_t ld; } Ua{ldua}, Sa{ldsa}, Va{ldva}, Ub{ldub}, Sb{ldsb}, Vb{ldvb};
  LRA_BEGIN();
  const bool use_fast = fast && eps == 0.0 && kt <= m && kt <= n;
  int mu, mv;
  if (!use_fast) {
    // X = [Ua Sa | Ub Sb], Y = [Va^T | Vb^T]
    cta_gemm<double, OT>(m, ka, ka, 1.0, ua, Ua.ld, false, sa, Sa.ld, false, 0.0, X, m, gsm);
    cta_gemm<double, OT>(m, kb, kb, 1.0, ub, Ub.ld, false, sb, Sb.ld, false, 0.0, X + (int64_t)ka * m, m, gsm);
    for (int64_t e = threadIdx.x; e < (int64_t)n * kt; e += blockDim.x) {
      const int r = e % n, c = e / n;
      Y[e] = c < ka ? va[c + (int64_t)r * Va.ld] : vb[(c - ka) + (int64_t)r * Vb.ld];
    }
    __syncthreads();
    cta_householder_qr(m, kt, X, m, tu, red);
    cta_householder_qr(n, kt, Y, n, tv, red);
    mu = min(m, kt);
    mv = min(n, kt);
    for (int64_t e = threadIdx.x; e < (int64_t)mu * kt; e += blockDim.x) {
      const int r = e % mu, c = e / mu;
      Rc[e] = r <= c ? X[r + (int64_t)c * m] : 0.0;
    }
    for (int64_t e = threadIdx.x; e < (int64_t)mv * kt; e += blockDim.x) {
      const int r = e % mv, c = e / mv;
      Rv[e] = r <= c ? Y[r + (int64_t)c * n] : 0.0;
    }
    __syncthreads();
    // M (mu x mv) = Rc Rv^T
    cta_gemm<double, OT>(mu, mv, kt, 1.0, Rc, mu, false, Rv, mv, true, 0.0, M, mu, gsm);
  } else {
    mu = kt;
    mv = kt;
    // X = [Ua | Ub], Y = [Va^T | Vb^T]
    for (int64_t e = threadIdx.x; e < (int64_t)m * kt; e += blockDim.x) {
      const int r = e % m, c = e / m;
      X[e] = c < ka ? ua[r + (int64_t)c * Ua.ld] : ub[r + (int64_t)(c - ka) * Ub.ld];
    }
    for (int64_t e = threadIdx.x; e < (int64_t)n * kt; e += blockDim.x) {
      const int r = e % n, c = e / n;
      Y[e] = c < ka ? va[c + (int64_t)r * Va.ld] : vb[(c - ka) + (int64_t)r * Vb.ld];
    }
    __syncthreads();
    // Zu into Rc(0:ka, ka:kt), Yu = Ub - Ua Zu; same for V
    cta_gemm<double, OT>(ka, kb, m, 1.0, X, m, true, X + (int64_t)ka * m, m, false, 0.0, Rc + (int64_t)ka * kt, kt,
                         gsm);
    cta_gemm<double, OT>(m, kb, ka, -1.0, X, m, false, Rc + (int64_t)ka * kt, kt, false, 1.0, X + (int64_t)ka * m, m,
                         gsm);
    cta_gemm<double, OT>(ka, kb, n, 1.0, Y, n, true, Y + (int64_t)ka * n, n, false, 0.0, Rv + (int64_t)ka * kt, kt,
                         gsm);
    cta_gemm<double, OT>(n, kb, ka, -1.0, Y, n, false, Rv + (int64_t)ka * kt, kt, false, 1.0, Y + (int64_t)ka * n, n,
                         gsm);
    LRA_MARK(0);
    cta_householder_qr(m, kb, X + (int64_t)ka * m, m, tu, red);
    cta_householder_qr(n, kb, Y + (int64_t)ka * n, n, tv, red);
    LRA_MARK(1);
    for (int64_t e = threadIdx.x; e < (int64_t)kt * kt; e += blockDim.x) {
      const int r = e % kt, c = e / kt;
      if (c < ka) { Rc[e] = r == c ? 1.0 : 0.0; Rv[e] = r == c ? 1.0 : 0.0; }
      else if (r >= ka) {
        Rc[e] = (r - ka <= c - ka) ? X[(r - ka) + (int64_t)c * m] : 0.0;
        Rv[e] = (r - ka <= c - ka) ? Y[(r - ka) + (int64_t)c * n] : 0.0;
      }
    }
    __syncthreads();
    // M = Rc blockdiag(Sa, Sb) Rv^T, through T = Rc blockdiag(Sa, Sb) (kt x kt)
    cta_gemm<double, OT>(kt, ka, ka, 1.0, Rc, kt, false, sa, Sa.ld, false, 0.0, T, kt, gsm);
    cta_gemm<double, OT>(kt, kb, kb, 1.0, Rc + (int64_t)ka * kt, kt, false, sb, Sb.ld, false, 0.0,
                         T + (int64_t)ka * kt, kt, gsm);
    cta_gemm<double, OT>(kt, kt, kt, 1.0, T, kt, false, Rv, kt, true, 0.0, M, kt, gsm);
  }
  const bool svd_ok = (mu == mv && shm && 3 * (int64_t)mu * mu <= shm_cap)
                          ? cta_svd_pqr(mu, M, mu, Um, mu, sv, Vmt, mu, sc, shm, &flag, red, redi)
                          : cta_svd(mu, mv, M, mu, Um, mu, sv, Vmt, min(mu, mv), sc, &flag, shm, shm_cap);
  if (!svd_ok && threadIdx.x == 0) atomicAdd(err + OPS_ERR_JACOBI, 1);
  LRA_MARK(2);
  const int nsv = min(mu, mv);
  if (threadIdx.x == 0) {
    int r;
    if (eps > 0.0) {
      double fro = 0.0;
      for (int j = 0; j < nsv; ++j) fro += sv[j] * sv[j];
      const double thr = eps * sqrt(fro);
      r = 0;
      double e2;
      do {
        ++r;
        e2 = 0.0;
        if (r < nsv)
          for (int j = r; j < nsv; ++j) e2 += sv[r] * sv[r];
      } while (r < nsv && sqrt(e2) > thr);
    } else {
      r = min(ka, nsv);
    }
    if (r > kmax) { atomicAdd(err + 1, 1); r = kmax; }
    s_rank = r;
  }
  __syncthreads();
  const int r = s_rank;
  const int ldvm = nsv;
  // U = [Q_u-side] Um(:, :r): rounded: Qu [Um; 0]; fast: [Ua | Qu] Um
  for (int side = 0; side < 2; ++side) {
    const int rows = side ? n : m;
    double* St = side ? Y : X;
    const double* tt = side ? tv : tu;
    // T (rows x r) = [Um(:, :r); 0] or [Vm^T(:, :r); 0] below the leading part
    if (!use_fast) {
      const int lead = side ? mv : mu;
      for (int64_t e = threadIdx.x; e < (int64_t)rows * r; e += blockDim.x) {
        const int i = e % rows, c = e / rows;
        T[e] = i < lead ? (side ? Vmt[c + (int64_t)i * ldvm] : Um[i + (int64_t)c * mu]) : 0.0;
      }
      __syncthreads();
      cta_apply_q(rows, lead, St, rows, tt, r, T, rows);
    } else {
      for (int64_t e = threadIdx.x; e < (int64_t)rows * r; e += blockDim.x) {
        const int i = e % rows, c = e / rows;
        T[e] = i < kb ? (side ? Vmt[c + (int64_t)(ka + i) * ldvm] : Um[(ka + i) + (int64_t)c * mu]) : 0.0;
      }
      __syncthreads();
      cta_apply_q(rows, kb, St + (int64_t)ka * rows, rows, tt, r, T, rows);
      // + [Ua | Va^T](:, :ka) times the leading ka rows
      for (int64_t e = threadIdx.x; e < (int64_t)rows * r; e += blockDim.x) {
        const int i = e % rows, c = e / rows;
        double acc = 0.0;
        for (int t = 0; t < ka; ++t)
          acc += (side ? va[t + (int64_t)i * Va.ld] : ua[i + (int64_t)t * Ua.ld]) *
                 (side ? Vmt[c + (int64_t)t * ldvm] : Um[t + (int64_t)c * mu]);
        T[e] += acc;
      }
      __syncthreads();
    }
    for (int64_t e = threadIdx.x; e < (int64_t)rows * r; e += blockDim.x) {
      const int i = e % rows, c = e / rows;
      if (side) va_out[c + (int64_t)i * Va.ld] = T[e];
      else ua_out[i + (int64_t)c * Ua.ld] = T[e];
    }
    __syncthreads();
  }
  LRA_MARK(3);
#ifdef FRANK_LRA_TIMING
  if (threadIdx.x == 0) atomicAdd(&g_lra_cycles[4], 1ull);
#endif
  double* sp = sa_out;
  for (int64_t e = threadIdx.x; e < (int64_t)r * r; e += blockDim.x) {
    const int i = e % r, c = e / r;
    sp[i + (int64_t)c * Sa.ld] = i == c ? sv[i] : 0.0;
  }
  if (threadIdx.x == 0) *ka_io = r;
}

__global__ void __launch_bounds__(OT) k_op_lr_add(int m, int n, int kmax, int fast, double eps, Mat Ua, Mat Sa, Mat Va,
                                                  int* ka_io, Mat Ub, Mat Sb, Mat Vb, const int* kb_in,
                                                  double* scratch, int64_t ws, int* err, int64_t shm_cap) {
  extern __shared__ double dyn[];
  const int b = blockIdx.x;
  lr_add_body(m, n, kmax, fast, eps, Ua.at(b), Ua.ld, Sa.at(b), Sa.ld, Va.at(b), Va.ld, ka_io + b, Ub.at(b), Ub.ld,
              Sb.at(b), Sb.ld, Vb.at(b), Vb.ld, kb_in[b], scratch + (int64_t)b * ws, err, dyn, shm_cap);
}

// One LowRank addition per CTA from a task table (blocks of different sizes
// in one launch).
__global__ void __launch_bounds__(OT) k_op_lr_add_tasks(const LrAddTask* tasks, int kmax, int fast, double* scratch,
                                                        int* err, int64_t shm_cap) {
  extern __shared__ double dyn[];
  const LrAddTask t = tasks[blockIdx.x];
  lr_add_body(t.m, t.n, kmax, fast, 0.0, t.ua, t.ldua, t.sa, t.ldsa, t.va, t.ldva, t.ka, t.ub, t.ldub, t.sb, t.ldsb,
              t.vb, t.ldvb, *t.kb, scratch + t.scratch_off, err, dyn, shm_cap);
}

// C = alpha op(A) op(B) + beta C (operations/BLAS/gemm.cpp:126-146,
// cblas_dgemm): grid (64 x 64 output tiles, batch), one CTA GEMM per tile.
__global__ void __launch_bounds__(OT) k_op_gemm(int m, int n, int k, double alpha, Mat A, bool ta, Mat B, bool tb,
                                                double beta, Mat Cm) {
  __shared__ double gsm[GSM];
  const int b = blockIdx.y;
  const int tm = (m + 63) / 64;
  const int r0 = (blockIdx.x % tm) * 64, c0 = (blockIdx.x / tm) * 64;
  const double* a = A.at(b) + (ta ? (int64_t)r0 * A.ld : r0);
  const double* bb = B.at(b) + (tb ? c0 : (int64_t)c0 * B.ld);
  cta_gemm<double, OT>(min(64, m - r0), min(64, n - c0), k, alpha, a, A.ld, ta, bb, B.ld, tb, beta,
                       Cm.at(b) + r0 + (int64_t)c0 * Cm.ld, Cm.ld, gsm);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

struct Scratch {
  double* p = nullptr;
  int* err = nullptr;
  cudaStream_t s = nullptr;
  ~Scratch() {
    if (p) cudaFreeAsync(p, s);
  }
};

#define OPS_TRY(expr)                                                                        \
  do {                                                                                       \
    cudaError_t _e = (expr);                                                                 \
    if (_e != cudaSuccess) return set_error(FRANK_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

int check_dims(int m, int n, int count, int maxdim = 4096) {
  if (m < 1 || n < 1 || count < 0 || m > maxdim || n > maxdim)
    return set_error(FRANK_ERR_INVALID, "batched op: need 1 <= m, n <= " + std::to_string(maxdim) + ", count >= 0");
  return FRANK_OK;
}

// naive_addition (addition.cpp:68-89), concatenation branch: U = [Ua Ub],
// S = blockdiag(Sa, Sb), V = [Va; Vb] in A's buffers (capacity >= ka + kb).
__global__ void k_op_lr_concat(int m, int n, int ka, int kb, Mat Ua, Mat Sa, Mat Va, Mat Ub, Mat Sb, Mat Vb,
                               int b) {
  double *ua = Ua.at(b), *sa = Sa.at(b), *va = Va.at(b);
  const double *ub = Ub.at(b), *sb = Sb.at(b), *vb = Vb.at(b);
  const int kt = ka + kb;
  for (int64_t e = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; e < (int64_t)m * kb;
       e += (int64_t)blockDim.x * gridDim.x) {
    const int r = e % m, c = e / m;
    ua[r + (int64_t)(ka + c) * Ua.ld] = ub[r + (int64_t)c * Ub.ld];
  }
  for (int64_t e = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; e < (int64_t)kb * n;
       e += (int64_t)blockDim.x * gridDim.x) {
    const int r = e % kb, c = e / kb;
    va[ka + r + (int64_t)c * Va.ld] = vb[r + (int64_t)c * Vb.ld];
  }
  // S: the new rows / columns (the old ka x ka block stays)
  for (int64_t e = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; e < (int64_t)kt * kt;
       e += (int64_t)blockDim.x * gridDim.x) {
    const int r = e % kt, c = e / kt;
    if (r < ka && c < ka) continue;
    sa[r + (int64_t)c * Sa.ld] = (r >= ka && c >= ka) ? sb[(r - ka) + (int64_t)(c - ka) * Sb.ld] : 0.0;
  }
}

// naive_addition, recompression branch: D = Ua Sa Va + Ub Sb Vb (m x n, ld m)
// for LowRank(Dense(A) + Dense(B), ka).
__global__ void __launch_bounds__(OT) k_op_lr_dense(int m, int n, int ka, int kb, Mat Ua, Mat Sa, Mat Va, Mat Ub,
                                                    Mat Sb, Mat Vb, int b, double* D, double* T) {
  __shared__ double gsm[GSM];
  // T = Ua Sa (m x ka), D = T Va; T = Ub Sb, D += T Vb
  cta_gemm<double, OT>(m, ka, ka, 1.0, Ua.at(b), Ua.ld, false, Sa.at(b), Sa.ld, false, 0.0, T, m, gsm);
  cta_gemm<double, OT>(m, n, ka, 1.0, T, m, false, Va.at(b), Va.ld, false, 0.0, D, m, gsm);
  cta_gemm<double, OT>(m, kb, kb, 1.0, Ub.at(b), Ub.ld, false, Sb.at(b), Sb.ld, false, 0.0, T, m, gsm);
  cta_gemm<double, OT>(m, n, kb, 1.0, T, m, false, Vb.at(b), Vb.ld, false, 1.0, D, m, gsm);
}

// Allocate `count` slots of `ws` doubles plus the error words, run, sync, read errors.
template <typename Launch>
int run(cudaStream_t s, int count, int64_t ws, Launch launch) {
  if (count == 0) return FRANK_OK;
  Scratch sc;
  sc.s = s;
  OPS_TRY(cudaMallocAsync(reinterpret_cast<void**>(&sc.p), sizeof(double) * ((size_t)count * ws + OPS_ERR_SLOTS), s));
  sc.err = reinterpret_cast<int*>(sc.p + (size_t)count * ws);
  OPS_TRY(cudaMemsetAsync(sc.err, 0, sizeof(int) * OPS_ERR_SLOTS, s));
  launch(sc.p, sc.err);
  OPS_TRY(cudaGetLastError());
  int errs[OPS_ERR_SLOTS];
  OPS_TRY(cudaMemcpyAsync(errs, sc.err, sizeof(errs), cudaMemcpyDeviceToHost, s));
  OPS_TRY(cudaStreamSynchronize(s));
  if (errs[OPS_ERR_JACOBI]) return set_error(FRANK_ERR_NOT_CONVERGED, "one-sided Jacobi reached its sweep limit");
  if (errs[1]) return set_error(FRANK_ERR_RANK_OVERFLOW, "a recompressed rank exceeded kmax and was clamped");
  return FRANK_OK;
}

// The reference's Omega: random_uniform (functions.cpp:52-66), std::mt19937
// seeded 0, uniform [0, 1), n x s row-major; a new Omega from the same seed
// at every call.
std::vector<double> omega(int n, int s) {
  std::mt19937 gen;
  gen.seed(0);
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  std::vector<double> om((size_t)n * s);
  for (auto& v : om) v = dist(gen);
  return om;
}

int64_t svd_scratch(int m, int n) {
  const int mm = std::max(m, n), k = std::min(m, n);
  return (int64_t)(mm + k) * k + 2 * (int64_t)k + 2;
}

// ---------------------------------------------------------------------------
// Stream-ordered launches for the H-matrix driver (hodlr.cu): the caller owns
// the scratch (count x ws doubles) and the error slots, nothing is allocated
// or synchronised, so a whole factorization can be captured into one graph.
// ---------------------------------------------------------------------------

int64_t qr_ws(int m, int n) { return (int64_t)m * n + std::min(m, n) + 2; }

int64_t lr_add_ws(int m, int n, int ka, int kb) {
  const int kt = ka + kb, mx = std::max(m, n);
  return (int64_t)(m + n) * kt + 2 * kt + 5 * (int64_t)kt * kt + kt + (int64_t)mx * kt + svd_scratch(kt, kt) + 2;
}

void launch_gemm(cudaStream_t s, int m, int n, int k, int count, double alpha, const double* a, int64_t lda,
                 int64_t sa, bool ta, const double* b, int64_t ldb, int64_t sb, bool tb, double beta, double* c,
                 int64_t ldc, int64_t sc) {
  const int64_t tiles = (int64_t)((m + 63) / 64) * ((n + 63) / 64);
  k_op_gemm<<<dim3((unsigned)tiles, count), OT, 0, s>>>(m, n, k, alpha, Mat{const_cast<double*>(a), lda, sa}, ta,
                                                       Mat{const_cast<double*>(b), ldb, sb}, tb, beta,
                                                       Mat{c, ldc, sc});
}

void launch_qr(cudaStream_t s, int m, int n, int count, const double* a, int64_t lda, int64_t sa, double* q,
               int64_t ldq, int64_t sq, double* r, int64_t ldr, int64_t sr, double* scratch, int64_t ws) {
  k_op_qr<<<count, OT, 0, s>>>(m, n, Mat{const_cast<double*>(a), lda, sa}, Mat{q, ldq, sq}, Mat{r, ldr, sr}, scratch,
                               ws);
}

void launch_svd(cudaStream_t s, int m, int n, int count, const double* a, int64_t lda, int64_t sa, double* u,
                int64_t ldu, int64_t su, double* sv, int64_t ss, double* vt, int64_t ldvt, int64_t svt,
                double* scratch, int64_t ws, int* err) {
  k_op_svd<<<count, OT, 0, s>>>(m, n, Mat{const_cast<double*>(a), lda, sa}, Mat{u, ldu, su}, Mat{sv, 1, ss},
                                Mat{vt, ldvt, svt}, scratch, ws, err);
}

// Shared memory (bytes) for the core SVD of an addition of ranks ka + kb
// (the pivoted-QR-preconditioned Jacobi: 3 kt^2 doubles), or 0 when it does
// not fit beside the kernel's static arrays.
int lr_add_shm_bytes(int ka, int kb) {
  const int64_t kt = ka + kb, b = (3 * kt) * kt * (int64_t)sizeof(double);
  return b <= 160 * 1024 ? (int)b : 0;
}

// Opt the addition kernels in to the shared memory of lr_add_shm_bytes (once,
// outside any stream capture).
int lr_add_prepare(int bytes) {
  if (cudaFuncSetAttribute(k_op_lr_add, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess ||
      cudaFuncSetAttribute(k_op_lr_add_tasks, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
    return set_error(FRANK_ERR_CUDA, "LowRank addition: shared memory attribute");
  return FRANK_OK;
}

void launch_lr_add_tasks(cudaStream_t s, int count, const LrAddTask* tasks, int kmax, int fast, double* scratch,
                         int* err, int shm_bytes) {
  k_op_lr_add_tasks<<<count, OT, shm_bytes, s>>>(tasks, kmax, fast, scratch, err, shm_bytes / (int)sizeof(double));
}

}  // namespace ops
}  // namespace frank

using namespace frank;
using namespace frank::ops;

extern "C" {

int frank_device_alloc(size_t bytes, void** out) {
  if (!out) return set_error(FRANK_ERR_INVALID, "null output pointer");
  *out = nullptr;
  if (bytes == 0) return FRANK_OK;
  OPS_TRY(cudaMalloc(out, bytes));
  return FRANK_OK;
}

int frank_device_free(void* ptr) {
  if (ptr) OPS_TRY(cudaFree(ptr));
  return FRANK_OK;
}

int frank_copy(void* dst, const void* src, size_t bytes, int to_device) {
  if ((!dst || !src) && bytes) return set_error(FRANK_ERR_INVALID, "null copy pointer");
  if (bytes) OPS_TRY(cudaMemcpy(dst, src, bytes, to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost));
  return FRANK_OK;
}

int frank_gemm_batched(int m, int n, int k, int count, double alpha, const double* d_a, int64_t lda, int64_t sa,
                       int trans_a, const double* d_b, int64_t ldb, int64_t sb, int trans_b, double beta, double* d_c,
                       int64_t ldc, int64_t sc, void* stream) {
  if (m < 1 || n < 1 || k < 1 || count < 0 || count > 65535 || !d_a || !d_b || !d_c ||
      lda < (trans_a ? k : m) || ldb < (trans_b ? n : k) || ldc < m)
    return set_error(FRANK_ERR_INVALID, "bad gemm arguments");
  if (count == 0) return FRANK_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t tiles = (int64_t)((m + 63) / 64) * ((n + 63) / 64);
  if (tiles > 2147483647) return set_error(FRANK_ERR_UNSUPPORTED, "gemm too large");
  k_op_gemm<<<dim3((unsigned)tiles, count), OT, 0, s>>>(m, n, k, alpha, Mat{const_cast<double*>(d_a), lda, sa},
                                                       trans_a != 0, Mat{const_cast<double*>(d_b), ldb, sb},
                                                       trans_b != 0, beta, Mat{d_c, ldc, sc});
  OPS_TRY(cudaGetLastError());
  OPS_TRY(cudaStreamSynchronize(s));
  return FRANK_OK;
}

int frank_qr_batched(int m, int n, int count, const double* d_a, int64_t lda, int64_t sa, double* d_q, int64_t ldq,
                     int64_t sq, double* d_r, int64_t ldr, int64_t sr, void* stream) {
  int rc = check_dims(m, n, count);
  if (rc) return rc;
  const int k = std::min(m, n);
  if (!d_a || !d_q || !d_r || lda < m || ldq < m || ldr < k) return set_error(FRANK_ERR_INVALID, "bad qr arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t ws = (int64_t)m * n + k + 2;
  return run(s, count, ws, [&](double* sc, int*) {
    k_op_qr<<<count, OT, 0, s>>>(m, n, Mat{const_cast<double*>(d_a), lda, sa}, Mat{d_q, ldq, sq}, Mat{d_r, ldr, sr}, sc, ws);
  });
}

int frank_rq_batched(int m, int n, int count, const double* d_a, int64_t lda, int64_t sa, double* d_r, int64_t ldr,
                     int64_t sr, double* d_q, int64_t ldq, int64_t sq, void* stream) {
  int rc = check_dims(m, n, count);
  if (rc) return rc;
  const int k = std::min(m, n);
  if (!d_a || !d_q || !d_r || lda < m || ldr < m || ldq < k) return set_error(FRANK_ERR_INVALID, "bad rq arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t ws = (int64_t)m * n + k + (int64_t)n * k + 2;
  return run(s, count, ws, [&](double* sc, int*) {
    k_op_rq<<<count, OT, 0, s>>>(m, n, Mat{const_cast<double*>(d_a), lda, sa}, Mat{d_r, ldr, sr}, Mat{d_q, ldq, sq}, sc, ws);
  });
}

int frank_svd_batched(int m, int n, int count, const double* d_a, int64_t lda, int64_t sa, double* d_u, int64_t ldu,
                      int64_t su, double* d_s, int64_t ss, double* d_vt, int64_t ldvt, int64_t svt, void* stream) {
  int rc = check_dims(m, n, count, 1024);
  if (rc) return rc;
  const int k = std::min(m, n);
  if (!d_a || !d_u || !d_s || !d_vt || lda < m || ldu < m || ldvt < k) return set_error(FRANK_ERR_INVALID, "bad svd arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t ws = svd_scratch(m, n);
  return run(s, count, ws, [&](double* sc, int* err) {
    k_op_svd<<<count, OT, 0, s>>>(m, n, Mat{const_cast<double*>(d_a), lda, sa}, Mat{d_u, ldu, su}, Mat{d_s, 1, ss},
                                  Mat{d_vt, ldvt, svt}, sc, ws, err);
  });
}

int frank_rsvd_batched(int m, int n, int count, int rank, int oversample, int power_its, const double* d_a,
                       int64_t lda, int64_t sa, double* d_u, int64_t ldu, int64_t su, double* d_s, int64_t lds,
                       int64_t ss, double* d_v, int64_t ldv, int64_t sv, void* stream) {
  int rc = check_dims(m, n, count);
  if (rc) return rc;
  const int smp = std::min(rank + oversample, std::min(m, n));
  if (rank < 1 || oversample < 0 || power_its < 0 || rank > smp || !d_a || !d_u || !d_s || !d_v || lda < m ||
      ldu < m || lds < rank || ldv < rank)
    return set_error(FRANK_ERR_INVALID, "bad rsvd arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const std::vector<double> om = omega(n, smp);
  double* d_om = nullptr;
  OPS_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d_om), sizeof(double) * om.size(), s));
  OPS_TRY(cudaMemcpyAsync(d_om, om.data(), sizeof(double) * om.size(), cudaMemcpyHostToDevice, s));
  const int64_t ws = (int64_t)m * smp + (int64_t)std::max(m, n) * smp + (int64_t)n * smp + smp + (int64_t)smp * smp +
                     smp + (int64_t)smp * n + svd_scratch(smp, n) + 2;
  rc = run(s, count, ws, [&](double* sc, int* err) {
    k_op_rsvd<<<count, OT, 0, s>>>(m, n, smp, rank, power_its, Mat{const_cast<double*>(d_a), lda, sa}, d_om,
                                   Mat{d_u, ldu, su}, Mat{d_s, lds, ss}, Mat{d_v, ldv, sv}, sc, ws, err);
  });
  cudaFreeAsync(d_om, s);
  cudaStreamSynchronize(s);
  return rc;
}

int frank_id_batched(int m, int n, int count, int k, const double* d_a, int64_t lda, int64_t sa, double* d_u,
                     int64_t ldu, int64_t su, double* d_s, int64_t lds, int64_t ss, double* d_v, int64_t ldv,
                     int64_t sv, int* d_rows, int* d_cols, void* stream) {
  int rc = check_dims(m, n, count);
  if (rc) return rc;
  if (k < 1 || k > std::min(m, n) || !d_a || !d_u || !d_s || !d_v || !d_rows || !d_cols || lda < m || ldu < m ||
      lds < k || ldv < k)
    return set_error(FRANK_ERR_INVALID, "bad id arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int mx = std::max(m, n);
  const int64_t ws = 2 * (int64_t)m * k + (int64_t)mx * mx + 4 * (int64_t)mx + (int64_t)k * mx + mx + 4;
  return run(s, count, ws, [&](double* sc, int*) {
    k_op_id<<<count, OT, 0, s>>>(m, n, k, Mat{const_cast<double*>(d_a), lda, sa}, Mat{d_u, ldu, su},
                                 Mat{d_s, lds, ss}, Mat{d_v, ldv, sv}, d_rows, d_cols, sc, ws);
  });
}

int frank_rid_batched(int m, int n, int count, int sample, int k, const double* d_a, int64_t lda, int64_t sa,
                      double* d_u, int64_t ldu, int64_t su, double* d_s, int64_t lds, int64_t ss, double* d_v,
                      int64_t ldv, int64_t sv, void* stream) {
  int rc = check_dims(m, n, count);
  if (rc) return rc;
  if (sample < 1 || sample > std::min(m, n) || k < 1 || k > sample || !d_a || !d_u || !d_s || !d_v || lda < m ||
      ldu < m || lds < k || ldv < k)
    return set_error(FRANK_ERR_INVALID, "bad rid arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const std::vector<double> om = omega(n, sample);
  double* d_om = nullptr;
  OPS_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d_om), sizeof(double) * om.size(), s));
  OPS_TRY(cudaMemcpyAsync(d_om, om.data(), sizeof(double) * om.size(), cudaMemcpyHostToDevice, s));
  const int mx = std::max(sample, n);
  const int64_t ws = (int64_t)m * sample + (int64_t)std::max(m, n) * sample + (int64_t)n * sample + sample +
                     3 * (int64_t)sample * k + 2 * (int64_t)k + 2 + (int64_t)mx * mx + 4 * (int64_t)mx +
                     (int64_t)k * mx + mx + 4;
  rc = run(s, count, ws, [&](double* sc, int*) {
    k_op_rid<<<count, OT, 0, s>>>(m, n, sample, k, Mat{const_cast<double*>(d_a), lda, sa}, d_om, Mat{d_u, ldu, su},
                                  Mat{d_s, lds, ss}, Mat{d_v, ldv, sv}, sc, ws);
  });
  cudaFreeAsync(d_om, s);
  cudaStreamSynchronize(s);
  return rc;
}

// naive_addition (addition.cpp:68-89) pair by pair: ranks are read to the
// host; ka + kb >= min(m, n) recompresses Dense(A) + Dense(B) to rank ka by
// rsvd with sample min(ka + 5, m, n) and the reference's Omega
// (LowRank(Dense, rank), low_rank.cpp:40-48), else the bases and S are
// concatenated (rank ka + kb, which must fit kmax).
static int lowrank_add_naive(int m, int n, int count, int kmax, double* d_ua, int64_t ldua, int64_t sua, double* d_sa,
                      int64_t ldsa, int64_t ssa, double* d_va, int64_t ldva, int64_t sva, int* d_ka,
                      const double* d_ub, int64_t ldub, int64_t sub, const double* d_sb, int64_t ldsb, int64_t ssb,
                      const double* d_vb, int64_t ldvb, int64_t svb, const int* d_kb, cudaStream_t s) {
  std::vector<int> ka(count), kb(count);
  OPS_TRY(cudaMemcpyAsync(ka.data(), d_ka, sizeof(int) * count, cudaMemcpyDeviceToHost, s));
  OPS_TRY(cudaMemcpyAsync(kb.data(), d_kb, sizeof(int) * count, cudaMemcpyDeviceToHost, s));
  OPS_TRY(cudaStreamSynchronize(s));
  const Mat Ua{d_ua, ldua, sua}, Sa{d_sa, ldsa, ssa}, Va{d_va, ldva, sva};
  const Mat Ub{const_cast<double*>(d_ub), ldub, sub}, Sb{const_cast<double*>(d_sb), ldsb, ssb},
      Vb{const_cast<double*>(d_vb), ldvb, svb};
  for (int b = 0; b < count; ++b) {
    if (ka[b] < 1 || kb[b] < 1 || ka[b] > kmax) return set_error(FRANK_ERR_INVALID, "bad lowrank_add ranks");
    if (ka[b] + kb[b] < std::min(m, n)) {
      if (ka[b] + kb[b] > kmax)
        return set_error(FRANK_ERR_RANK_OVERFLOW, "naive_addition: rank ka + kb exceeds the capacity kmax");
      k_op_lr_concat<<<std::max(1, std::min(64, (int)(((int64_t)(m + n) * (ka[b] + kb[b]) + 255) / 256))), 256, 0,
                       s>>>(m, n, ka[b], kb[b], Ua, Sa, Va, Ub, Sb, Vb, b);
      OPS_TRY(cudaGetLastError());
      ka[b] += kb[b];
      continue;
    }
    const int rank = ka[b], smp = std::min(rank + 5, std::min(m, n));
    const std::vector<double> om = omega(n, smp);
    double *d_om = nullptr, *d_dense = nullptr;
    OPS_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d_om), sizeof(double) * om.size(), s));
    OPS_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d_dense),
                            sizeof(double) * ((int64_t)m * n + (int64_t)m * std::max(ka[b], kb[b])), s));
    OPS_TRY(cudaMemcpyAsync(d_om, om.data(), sizeof(double) * om.size(), cudaMemcpyHostToDevice, s));
    k_op_lr_dense<<<1, OT, 0, s>>>(m, n, ka[b], kb[b], Ua, Sa, Va, Ub, Sb, Vb, b, d_dense, d_dense + (int64_t)m * n);
    const int64_t ws = (int64_t)m * smp + (int64_t)std::max(m, n) * smp + (int64_t)n * smp + smp +
                       (int64_t)smp * smp + smp + (int64_t)smp * n + svd_scratch(smp, n) + 2;
    int rc = run(s, 1, ws, [&](double* sc, int* err) {
      k_op_rsvd<<<1, OT, 0, s>>>(m, n, smp, rank, 0, Mat{d_dense, m, 0}, d_om, Mat{d_ua + b * sua, ldua, 0},
                                 Mat{d_sa + b * ssa, ldsa, 0}, Mat{d_va + b * sva, ldva, 0}, sc, ws, err);
    });
    cudaFreeAsync(d_om, s);
    cudaFreeAsync(d_dense, s);
    if (rc) return rc;
  }
  OPS_TRY(cudaMemcpyAsync(d_ka, ka.data(), sizeof(int) * count, cudaMemcpyHostToDevice, s));
  OPS_TRY(cudaStreamSynchronize(s));
  return FRANK_OK;
}

int frank_lowrank_add_batched(int m, int n, int count, int kmax, const char* lra, double eps, double* d_ua,
                              int64_t ldua, int64_t sua, double* d_sa, int64_t ldsa, int64_t ssa, double* d_va,
                              int64_t ldva, int64_t sva, int* d_ka, const double* d_ub, int64_t ldub, int64_t sub,
                              const double* d_sb, int64_t ldsb, int64_t ssb, const double* d_vb, int64_t ldvb,
                              int64_t svb, const int* d_kb, int kb_max, void* stream) {
  int rc = check_dims(m, n, count);
  if (rc) return rc;
  if (!lra || kmax < 1 || kb_max < 1 || eps < 0.0 || !d_ua || !d_sa || !d_va || !d_ka || !d_ub || !d_sb || !d_vb ||
      !d_kb || ldua < m || ldub < m || ldsa < kmax || ldva < kmax || ldvb < kb_max || kmax + kb_max > 2048)
    return set_error(FRANK_ERR_INVALID, "bad lowrank_add arguments");
  const std::string name(lra);
  int fast;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (name == "naive" || name == "naive_addition") return lowrank_add_naive(m, n, count, kmax, d_ua, ldua, sua, d_sa, ldsa, ssa, d_va,
                                                         ldva, sva, d_ka, d_ub, ldub, sub, d_sb, ldsb, ssb, d_vb,
                                                         ldvb, svb, d_kb, s);
  if (name == "rounded_addition") fast = 0;
  else if (name == "fast_rounded_addition") fast = 1;
  else return set_error(FRANK_ERR_UNSUPPORTED, "lowrank_add: unknown LowRank addition " + name);
  const int kt = kmax + kb_max, mx = std::max(m, n);
  const int64_t ws = (int64_t)(m + n) * kt + 2 * kt + 5 * (int64_t)kt * kt + kt + (int64_t)mx * kt +
                     svd_scratch(kt, kt) + 2;
  return run(s, count, ws, [&](double* sc, int* err) {
    k_op_lr_add<<<count, OT, 0, s>>>(m, n, kmax, fast, eps, Mat{d_ua, ldua, sua}, Mat{d_sa, ldsa, ssa},
                                     Mat{d_va, ldva, sva}, d_ka, Mat{const_cast<double*>(d_ub), ldub, sub},
                                     Mat{const_cast<double*>(d_sb), ldsb, ssb},
                                     Mat{const_cast<double*>(d_vb), ldvb, svb}, d_kb, sc, ws, err, 0);
  });
}

#ifdef FRANK_LRA_TIMING
int frank_debug_lra_cycles(unsigned long long* out) {
  OPS_TRY(cudaMemcpyFromSymbol(out, g_lra_cycles, sizeof(unsigned long long) * 8));
  return FRANK_OK;
}
#endif

}  // extern "C"
