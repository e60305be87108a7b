// Kernels of the BLR-LU factor-and-solve path (sm_100a).
//
// Storage (all column-major):
//   * dense block (i,j): bmax x bmax slot, ld = bmax, of which bs(i) x bs(j) used;
//   * low-rank block (i,j) = U S V: U (bmax x kcap, ld bmax), S (kcap x kcap,
//     ld kcap), Vt = V^T (bmax x kcap, ld bmax); rank r = rank[i*nb+j] columns used.
// T is the working precision (double for the plain FP64 path, float for the
// mixed path); every small factorization (leaf getrf, stacked-basis QR, core
// SVD) is computed in FP64.
#pragma once

#include "common.cuh"

#include <cooperative_groups.h>

namespace frank {

template <typename T>
struct BlrView {
  int nb, bmax, kcap;
  const int* off;    // [nb+1] block offsets
  const int* dslot;  // [nb*nb] dense slot or -1
  const int* lslot;  // [nb*nb] low-rank slot or -1
  int* rank;         // [nb*nb] current ranks (low-rank blocks)
  T* D;
  T* U;
  T* S;
  T* Vt;
  FRANK_D int bs(int i) const { return off[i + 1] - off[i]; }
  FRANK_D bool is_lr(int i, int j) const { return lslot[i * nb + j] >= 0; }
  FRANK_D T* dense(int i, int j) const { return D + (int64_t)dslot[i * nb + j] * bmax * bmax; }
  FRANK_D T* u(int i, int j) const { return U + (int64_t)lslot[i * nb + j] * bmax * kcap; }
  FRANK_D T* s(int i, int j) const { return S + (int64_t)lslot[i * nb + j] * kcap * kcap; }
  FRANK_D T* vt(int i, int j) const { return Vt + (int64_t)lslot[i * nb + j] * bmax * kcap; }
};

// Optional per-phase cycle counters of the recompression kernels (build with
// -DFRANK_PHASE_TIMING; off by default).  Slots: [size class][phase], the
// classes stacked sizes <= 64, <= 160 and larger.
#ifdef FRANK_PHASE_TIMING
__device__ unsigned long long g_getrf_cycles[8];
#define GPHASE(k)                                                                           \
  do {                                                                                      \
    if (threadIdx.x == 0) {                                                                 \
      const long long _t = clock64();                                                      \
      atomicAdd(&g_getrf_cycles[(k)], (unsigned long long)(_t - _g_t0));                    \
      _g_t0 = _t;                                                                           \
    }                                                                                       \
  } while (0)
#define GPHASE_BEGIN() long long _g_t0 = clock64()
#else
#define GPHASE(k) do {} while (0)
#define GPHASE_BEGIN() do {} while (0)
#endif
#ifdef FRANK_PHASE_TIMING
__device__ unsigned long long g_phase_cycles[3][8];
__device__ unsigned long long g_phase_count[3];
#define PHASE_BEGIN() long long _ph_t0 = clock64(); int _ph_last = 0
#define PHASE_MARK(cls, k)                                                                  \
  do {                                                                                      \
    if (threadIdx.x == 0) {                                                                 \
      const long long _t = clock64();                                                      \
      atomicAdd(&g_phase_cycles[(cls)][(k)], (unsigned long long)(_t - _ph_t0));            \
      _ph_t0 = _t;                                                                          \
    }                                                                                       \
    (void)_ph_last;                                                                         \
  } while (0)
#else
#define PHASE_BEGIN() do {} while (0)
#define PHASE_MARK(cls, k) do {} while (0)
#endif
#ifdef FRANK_PHASE_TIMING
__device__ unsigned long long g_tlog_n;
__device__ long long g_tlog[200000][6];
FRANK_D long long gtimer() { long long t; asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t)); return t; }
#endif

// Per-factorization workspace (device pointers).
template <typename T>
struct FactorWs {
  int* perm;      // [nb][bmax]: row i of P*B is row perm[i] of B, per diagonal block
  int* ipiv;      // [nb][bmax]: LAPACK-style 0-based pivots per diagonal block
  T* Linv;        // [nb][bmax*bmax]: unit-lower inverse per diagonal block
  T* Uinv;        // [nb][bmax*bmax]: upper inverse per diagonal block
  T* WL;          // [nb][bmax*bmax]: (S V)^T of column-panel blocks, by block row
  T* WU;          // [nb][bmax*bmax]: U S of row-panel blocks, by block column
  double* getrf_scratch;  // bmax*bmax + 32*bmax
  double* dscratch;       // dense-update scratch, per CTA slot
  int64_t dscratch_stride;
  double* rscratch;       // recompression scratch, per CTA slot
  int64_t rscratch_stride;
  int* err;
  int* work;                  // [nb] per-step work counters of the recompression
  unsigned long long* flops;  // [FLOP_SLOTS]
  int fixed_rank;
  double eps;
};

// Algorithmic FLOPs of one rounded LowRank addition as the reference issues it
// (gemm.cpp:253-272 then addition.cpp:93-127), counted with the LAWN 41
// operation counts: the inner product S_A V_A U_B S_B, U_C S_C and U_B S_B,
// geqrf + orgqr of Uc (m x s), gerqf + orgrq of VcT (s x n), the core gemm,
// dgesvd of the s x s core (22 s^3) and the two basis gemms.
FRANK_HD double rounded_addition_flops(double m, double n, double bi, double kc, double p, double q, double r) {
  const double s = fmin(kc + q, fmin(m, n));
  double f = 2.0 * p * p * bi + 2.0 * bi * q * q + 2.0 * p * bi * q;   // core of the product
  f += 2.0 * m * kc * kc + 2.0 * m * p * q;                               // U_C S_C, U_B S_B
  f += 4.0 * m * s * s - 4.0 / 3.0 * s * s * s;                           // geqrf + orgqr
  f += 4.0 * n * s * s - 4.0 / 3.0 * s * s * s;                           // gerqf + orgrq
  f += 2.0 * s * s * s + 22.0 * s * s * s;                                // Ru RvT, gesvd
  f += 2.0 * m * s * r + 2.0 * n * s * r;                                 // new U, V
  return f;
}

// Algorithmic FLOPs of one fast rounded addition (addition.cpp:133-189) as
// the reference issues it: projections Zu = U_C^T U_B, Zv, the residual bases,
// their QR / RQ with explicit factors, the (kc+p) x (kc+q) core, its SVD and
// the new bases [U_C | Q_u] U_m, V_m [V_C; Q_v].
FRANK_HD double fast_rounded_addition_flops(double m, double n, double bi, double kc, double p, double q, double r) {
  double f = 2.0 * p * p * bi + 2.0 * bi * q * q + 2.0 * p * bi * q;   // core of the product
  f += 4.0 * m * kc * p + 4.0 * n * kc * q;                               // Zu, Yu; Zv, Yv
  f += 4.0 * m * p * p - 4.0 / 3.0 * p * p * p;                           // geqrf + orgqr of Yu
  f += 4.0 * n * q * q - 4.0 / 3.0 * q * q * q;                           // gerqf + orgrq of Yv^T
  const double s = fmax(kc + p, kc + q);
  f += 4.0 * s * s * s + 22.0 * s * s * s;                                // core M, gesvd
  f += 2.0 * m * (kc + p) * r + 2.0 * n * (kc + q) * r;                   // new U, V
  return f;
}

// ---------------------------------------------------------------------------
// Reset the working copy from A_H (FP64) -- only the used parts are copied.
// One CTA per block.
// ---------------------------------------------------------------------------
template <typename T>
FRANK_D void k_reset_impl(BlrView<double> H, BlrView<T> W) {
  const int blk = blockIdx.x;
  const int i = blk / H.nb, j = blk % H.nb;
  const int bi = H.bs(i), bj = H.bs(j);
  if (H.lslot[blk] >= 0) {
    const int r = H.rank[blk];
    const double* hu = H.u(i, j); const double* hs = H.s(i, j); const double* hv = H.vt(i, j);
    T* wu = W.u(i, j); T* ws = W.s(i, j); T* wv = W.vt(i, j);
    for (int64_t e = threadIdx.x; e < (int64_t)bi * r; e += blockDim.x) {
      const int rr = e % bi, c = e / bi;
      wu[rr + (int64_t)c * W.bmax] = T(hu[rr + (int64_t)c * H.bmax]);
    }
    for (int64_t e = threadIdx.x; e < (int64_t)bj * r; e += blockDim.x) {
      const int rr = e % bj, c = e / bj;
      wv[rr + (int64_t)c * W.bmax] = T(hv[rr + (int64_t)c * H.bmax]);
    }
    for (int64_t e = threadIdx.x; e < (int64_t)r * r; e += blockDim.x) {
      const int rr = e % r, c = e / r;
      ws[rr + (int64_t)c * W.kcap] = T(hs[rr + (int64_t)c * H.kcap]);
    }
    if (threadIdx.x == 0) W.rank[blk] = r;
  } else if (H.dslot[blk] >= 0) {
    const double* hd = H.dense(i, j);
    T* wd = W.dense(i, j);
    for (int64_t e = threadIdx.x; e < (int64_t)bi * bj; e += blockDim.x) {
      const int rr = e % bi, c = e / bi;
      wd[rr + (int64_t)c * W.bmax] = T(hd[rr + (int64_t)c * H.bmax]);
    }
  }
}

template <typename T>
__global__ void k_reset(BlrView<double> H, BlrView<T> W) {
  k_reset_impl<T>(H, W);
}

// ---------------------------------------------------------------------------
// K0': truncation of the working copy's low-rank blocks to the factor
// tolerance (mixed plans, whose factor is computed at a looser tolerance
// than A_H).  Block U S V^T of A_H with orthonormal U, V: truncated pivoted
// QR of S to thr_scale * ||S||_F (the core truncation of the recompression,
// geqp3.cpp:71-192), S P = Q R, then RQ of the kept rows R P^T = S' Q', so
// W = (U Q_r) S' (V Q'^T)^T with rank r.  Blocks whose rank does not drop
// keep the copy k_reset made.  One CTA per block (grid-stride), FP64
// scratch slot per CTA (4 k^2 + 8 k doubles).
// ---------------------------------------------------------------------------
constexpr int TRUNC_THREADS = 256;

// Orthonormal bases for low-rank blocks given by the caller
// (frank_blr_set_lowrank): U = Qu Ru and V^T = Qv Rv by Householder QR, stored
// as U <- Qu, V^T <- Qv, S <- Ru S Rv^T -- the same matrix, with the
// orthonormal bases that the reset truncation and the projected additions
// assume (the on-device constructions produce them already).  One CTA per
// block at a time; scratch per CTA: 2 (bmax + kcap) kcap + 3 kcap^2 doubles.
constexpr int ORTH_THREADS = 256;
__global__ void __launch_bounds__(ORTH_THREADS) k_orthonormalize_lr(BlrView<double> H, double* scratch,
                                                                   int64_t stride) {
  __shared__ double gsm[2 * 16 * 64];
  __shared__ double red[32];
  double* base = scratch + (int64_t)blockIdx.x * stride;
  const int nblk = H.nb * H.nb;
  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    if (H.lslot[blk] < 0) continue;
    const int k = H.rank[blk];
    const int i = blk / H.nb, j = blk % H.nb;
    const int bi = H.bs(i), bj = H.bs(j);
    if (k < 1 || k > bi || k > bj) continue;
    double* A1 = base;                        // bi x k, then its reflectors
    double* A2 = A1 + (int64_t)bi * k;        // bj x k
    double* Q = A2 + (int64_t)bj * k;         // max(bi, bj) x k
    double* Ru = Q + (int64_t)max(bi, bj) * k;
    double* Rv = Ru + (int64_t)k * k;
    double* Tmp = Rv + (int64_t)k * k;
    double* tu = Tmp + (int64_t)k * k;
    double* tv = tu + k;
    double* hu = H.u(i, j);
    double* hv = H.vt(i, j);
    double* hs = H.s(i, j);
    for (int64_t e = threadIdx.x; e < (int64_t)bi * k; e += blockDim.x) A1[e] = hu[(e % bi) + (e / bi) * H.bmax];
    for (int64_t e = threadIdx.x; e < (int64_t)bj * k; e += blockDim.x) A2[e] = hv[(e % bj) + (e / bj) * H.bmax];
    __syncthreads();
    cta_householder_qr(bi, k, A1, bi, tu, red);
    cta_householder_qr(bj, k, A2, bj, tv, red);
    for (int64_t e = threadIdx.x; e < (int64_t)k * k; e += blockDim.x) {
      const int r = e % k, c = e / k;
      Ru[e] = r <= c ? A1[r + (int64_t)c * bi] : 0.0;
      Rv[e] = r <= c ? A2[r + (int64_t)c * bj] : 0.0;
    }
    __syncthreads();
    // S <- Ru S Rv^T
    cta_gemm<double, ORTH_THREADS>(k, k, k, 1.0, Ru, k, false, hs, H.kcap, false, 0.0, Tmp, k, gsm);
    cta_gemm<double, ORTH_THREADS>(k, k, k, 1.0, Tmp, k, false, Rv, k, true, 0.0, hs, H.kcap, gsm);
    // U <- Qu, V^T <- Qv (explicit, from the reflectors)
    for (int side = 0; side < 2; ++side) {
      const int m = side ? bj : bi;
      const double* R = side ? A2 : A1;
      for (int64_t e = threadIdx.x; e < (int64_t)m * k; e += blockDim.x) Q[e] = ((e % m) == (e / m)) ? 1.0 : 0.0;
      __syncthreads();
      cta_apply_q(m, k, R, m, side ? tv : tu, k, Q, (int64_t)m);
      double* out = side ? hv : hu;
      for (int64_t e = threadIdx.x; e < (int64_t)m * k; e += blockDim.x) out[(e % m) + (e / m) * H.bmax] = Q[e];
      __syncthreads();
    }
  }
}

template <typename T>
FRANK_D void k_truncate_lr_impl(BlrView<double> H, BlrView<T> W, FactorWs<T> ws,
                                                              double thr_scale, double* scratch, int64_t stride) {
  __shared__ double gsm[2 * 16 * 64];
  __shared__ double red[32];
  __shared__ int redi[32];
  double* base = scratch + (int64_t)blockIdx.x * stride;
  const int nblk = H.nb * H.nb;
  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    if (H.lslot[blk] < 0) continue;
    const int k = H.rank[blk];
    if (k <= 1) continue;
    const int i = blk / H.nb, j = blk % H.nb;
    const int bi = H.bs(i), bj = H.bs(j);
    double* M = base;                          // k x k
    double* Xo = M + (int64_t)k * k;           // k x r
    double* X2 = Xo + (int64_t)k * k;          // k x r
    double* Qt = X2 + (int64_t)k * k;          // k x r
    double* tau = Qt + (int64_t)k * k;
    double* tau2 = tau + k;
    double* cn = tau2 + k;
    double* pn = cn + k;
    int* jpvt = reinterpret_cast<int*>(pn + k);
    int* jinv = jpvt + k;
    const double* hs = H.s(i, j);
    double f = 0.0;
    for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
      const double v = hs[(e % k) + (int64_t)(e / k) * H.kcap];
      M[e] = v;
      f += v * v;
    }
    f = block_sum(f, red);
    const int r = cta_truncated_geqp3(k, k, M, k, thr_scale * sqrt(f), W.kcap, tau, cn, pn, jpvt, red, redi);
    if (r >= k) continue;
    T* wu = W.u(i, j); T* wsm = W.s(i, j); T* wv = W.vt(i, j);
    if (r == 0) {
      for (int e = threadIdx.x; e < bi; e += blockDim.x) wu[e] = T(e == 0 ? 1.0 : 0.0);
      for (int e = threadIdx.x; e < bj; e += blockDim.x) wv[e] = T(e == 0 ? 1.0 : 0.0);
      if (threadIdx.x == 0) { wsm[0] = T(0); W.rank[blk] = 1; }
      __syncthreads();
      continue;
    }
    // Xo = Q[:, :r]
    for (int e = threadIdx.x; e < k * r; e += blockDim.x) Xo[e] = ((e % k) == (e / k)) ? 1.0 : 0.0;
    for (int c = threadIdx.x; c < k; c += blockDim.x) jinv[jpvt[c]] = c;
    __syncthreads();
    cta_apply_q(k, r, M, k, tau, r, Xo, (int64_t)k);
    // RQ of R P^T (r x k): QR of X2 = (R P^T)^T J
    for (int e = threadIdx.x; e < k * r; e += blockDim.x) {
      const int c = e % k, a = e / k;
      const int row = r - 1 - a, src = jinv[c];
      X2[e] = (row <= src) ? M[row + (int64_t)src * k] : 0.0;
    }
    __syncthreads();
    cta_householder_qr(k, r, X2, k, tau2, red);
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
      const int a = e % r, c = e / r;
      const int ra = r - 1 - c, ca = r - 1 - a;
      wsm[a + (int64_t)c * W.kcap] = T((ra <= ca) ? X2[ra + (int64_t)ca * k] : 0.0);
    }
    for (int e = threadIdx.x; e < k * r; e += blockDim.x) Qt[e] = ((e % k) == (e / k)) ? 1.0 : 0.0;
    __syncthreads();
    cta_apply_q(k, r, X2, k, tau2, r, Qt, (int64_t)k);
    // new U = U Xo; then Xo := Qt with its columns reversed, new V = V Xo
    cta_gemm<double, TRUNC_THREADS>(bi, r, k, 1.0, H.u(i, j), H.bmax, false, Xo, k, false, 0.0, wu, W.bmax, gsm);
    for (int e = threadIdx.x; e < k * r; e += blockDim.x) {
      const int rr = e % k, a = e / k;
      Xo[e] = Qt[rr + (int64_t)(r - 1 - a) * k];
    }
    __syncthreads();
    cta_gemm<double, TRUNC_THREADS>(bj, r, k, 1.0, H.vt(i, j), H.bmax, false, Xo, k, false, 0.0, wv, W.bmax, gsm);
    if (threadIdx.x == 0) W.rank[blk] = r;
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(TRUNC_THREADS) k_truncate_lr(BlrView<double> H, BlrView<T> W, FactorWs<T> ws,
                                                              double thr_scale, double* scratch, int64_t stride) {
  k_truncate_lr_impl<T>(H, W, ws, thr_scale, scratch, stride);
}

// ---------------------------------------------------------------------------
// K1: leaf getrf of diagonal block i with partial pivoting, FP64, one CTA
// (512 threads).  Blocked right-looking LU (panel width 32): the panel is
// factored column by column (idamax pivot, row swap across the whole block,
// reciprocal scaling and rank-1 update as in LAPACK dgetf2), then the row
// block is solved with the unit-lower 32x32 triangle and the trailing matrix
// updated by a CTA GEMM.  Writes the packed LU back into the block and the
// pivots/permutation; the explicit inverses Linv, Uinv are formed by k_trinv.
// ---------------------------------------------------------------------------
constexpr int GETRF_THREADS = 512;

// One 32-column panel step of the leaf LU of a b x b FP64 matrix Wm (ld b):
// partial-pivoted factorization of columns jb .. jb+jn-1 (in registers, one
// row per thread, when b <= GETRF_THREADS; column steps on the global copy
// otherwise), the panel's interchanges applied to every other column, and
// U12 = L11^{-1} A12 (through the 32 x bmax scratch panel Gp).  Pivots into
// piv[jb ..]; returns the first column with a zero pivot, or -1.  Called by
// all threads of a GETRF_THREADS CTA.
FRANK_D int getrf_panel_step(int b, int jb, double* Wm, double* Gp, int* piv, double* red, int* redi, double* gsm,
                             double* tri, double* prow, double* xrow) {
  const int jn = min(32, b - jb);
  int zero = -1;
  if (b <= GETRF_THREADS) {
    // Panel in registers: thread t owns row t (t >= jb) and its jn panel
    // entries; a column step is an arg-max, a row exchange through shared
    // memory and a rank-1 update, with no global traffic.
    const int t = threadIdx.x;
    const bool own = (t >= jb && t < b);
    double a[32];
#pragma unroll
    for (int c = 0; c < 32; ++c) a[c] = (own && c < jn) ? Wm[t + (int64_t)(jb + c) * b] : 0.0;
    for (int jj = 0; jj < jn; ++jj) {
      const int j = jb + jj;
      double v = -1.0;
      int vi = -1;
      if (t >= j && t < b) {
#pragma unroll
        for (int c = 0; c < 32; ++c) if (c == jj) v = fabs(a[c]);
        vi = t;
      }
      double amax;
      const int p = block_argmax_abs(v < 0.0 ? 0.0 : v, vi, red, redi, &amax);
      if (threadIdx.x == 0) piv[j] = p;
      if (amax == 0.0 && zero < 0) zero = j;
      // the pivot row goes to row j, row j to row p
      if (t == p) {
#pragma unroll
        for (int c = 0; c < 32; ++c) prow[c] = a[c];
      }
      if (t == j) {
#pragma unroll
        for (int c = 0; c < 32; ++c) xrow[c] = a[c];
      }
      __syncthreads();
      if (t == j) {
#pragma unroll
        for (int c = 0; c < 32; ++c) a[c] = prow[c];
      } else if (t == p) {
#pragma unroll
        for (int c = 0; c < 32; ++c) a[c] = xrow[c];
      }
      if (t > j && t < b && amax != 0.0) {
        const double rcp = 1.0 / prow[jj];
        double l = 0.0;
#pragma unroll
        for (int c = 0; c < 32; ++c) if (c == jj) { a[c] *= rcp; l = a[c]; }
#pragma unroll
        for (int c = 0; c < 32; ++c) if (c > jj) a[c] -= l * prow[c];
      }
      __syncthreads();
    }
    if (own) {
#pragma unroll
      for (int c = 0; c < 32; ++c) if (c < jn) Wm[t + (int64_t)(jb + c) * b] = a[c];
    }
    __syncthreads();
    // the panel's interchanges applied to the columns outside the panel
    for (int c = threadIdx.x; c < b; c += blockDim.x) {
      if (c >= jb && c < jb + jn) continue;
      double* col = Wm + (int64_t)c * b;
      for (int jj = 0; jj < jn; ++jj) {
        const int j = jb + jj, p = piv[j];
        if (p != j) { const double tmp = col[j]; col[j] = col[p]; col[p] = tmp; }
      }
    }
    __syncthreads();
  } else {
    // blocks larger than the thread count: column steps on the global copy
    for (int j = jb; j < jb + jn; ++j) {
      double best = -1.0;
      int bi = -1;
      for (int r = j + threadIdx.x; r < b; r += blockDim.x) {
        const double av = fabs(Wm[r + (int64_t)j * b]);
        if (av > best) { best = av; bi = r; }
      }
      double amax;
      const int p = block_argmax_abs(best < 0.0 ? 0.0 : best, bi, red, redi, &amax);
      if (threadIdx.x == 0) piv[j] = p;
      if (amax == 0.0 && zero < 0) zero = j;
      if (p != j && amax != 0.0) {
        for (int c = threadIdx.x; c < b; c += blockDim.x) {
          const double tt = Wm[j + (int64_t)c * b];
          Wm[j + (int64_t)c * b] = Wm[p + (int64_t)c * b];
          Wm[p + (int64_t)c * b] = tt;
        }
      }
      __syncthreads();
      if (amax != 0.0) {
        const double rcp = 1.0 / Wm[j + (int64_t)j * b];
        for (int r = j + 1 + threadIdx.x; r < b; r += blockDim.x) Wm[r + (int64_t)j * b] *= rcp;
      }
      __syncthreads();
      const int nr = b - j - 1, nc = jb + jn - j - 1;
      for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
        const int r = j + 1 + e % nr, c = j + 1 + e / nr;
        Wm[r + (int64_t)c * b] -= Wm[r + (int64_t)j * b] * Wm[j + (int64_t)c * b];
      }
      __syncthreads();
    }
  }
  // U12 = L11^{-1} A12: invert the unit-lower 32x32 L11 into tri, then a
  // CTA GEMM into the scratch panel and back.
  const int ncr = b - jb - jn;
  if (ncr > 0) {
    for (int e = threadIdx.x; e < 32 * 33; e += blockDim.x) tri[e] = 0.0;
    __syncthreads();
    if (threadIdx.x < jn) {
      const int c = threadIdx.x;
      tri[c + c * 33] = 1.0;
      for (int r = c + 1; r < jn; ++r) {
        double s = 0.0;
        for (int t = c; t < r; ++t) s += Wm[(jb + r) + (int64_t)(jb + t) * b] * tri[t + c * 33];
        tri[r + c * 33] = -s;
      }
    }
    __syncthreads();
    cta_gemm<double, GETRF_THREADS>(jn, ncr, jn, 1.0, tri, 33, false, Wm + jb + (int64_t)(jb + jn) * b, b, false,
                                    0.0, Gp, 32, gsm);
    for (int e = threadIdx.x; e < jn * ncr; e += blockDim.x) {
      const int r = e % jn, c = e / jn;
      Wm[(jb + r) + (int64_t)(jb + jn + c) * b] = Gp[r + (int64_t)c * 32];
    }
    __syncthreads();
  }
  return zero;
}

template <typename T>
__global__ void __launch_bounds__(GETRF_THREADS) k_getrf(BlrView<T> A, FactorWs<T> ws, int i) {
  __shared__ double red[32];
  __shared__ int redi[32];
  __shared__ double gsm[2 * 16 * 64];
  __shared__ double tri[32 * 33];
  const int b = A.bs(i);
  const int ldA = A.bmax;
  T* Dp = A.dense(i, i);
  double* Wm = ws.getrf_scratch;                       // b x b working matrix
  double* Gp = Wm + (int64_t)A.bmax * A.bmax;          // 32 x bmax product panel
  int* piv = ws.ipiv + (int64_t)i * A.bmax;
  int* perm = ws.perm + (int64_t)i * A.bmax;
  T* Li = ws.Linv + (int64_t)i * A.bmax * A.bmax;
  T* Ui = ws.Uinv + (int64_t)i * A.bmax * A.bmax;
  GPHASE_BEGIN();
  for (int64_t e = threadIdx.x; e < (int64_t)b * b; e += blockDim.x) {
    const int r = e % b, c = e / b;
    Wm[r + (int64_t)c * b] = double(Dp[r + (int64_t)c * ldA]);
  }
  __syncthreads();
  GPHASE(0);
  int first_zero = -1;
  __shared__ double prow[32];          // pivot row of the panel, broadcast
  __shared__ double xrow[32];          // row exchanged with the pivot row
  for (int jb = 0; jb < b; jb += 32) {
    const int jn = min(32, b - jb);
    {
      const int z = getrf_panel_step(b, jb, Wm, Gp, piv, red, redi, gsm, tri, prow, xrow);
      if (z >= 0 && first_zero < 0) first_zero = z;
    }
    GPHASE(1);
    const int m2 = b - jb - jn;
    if (m2 > 0)
      cta_gemm<double, GETRF_THREADS>(m2, m2, jn, -1.0, Wm + (jb + jn) + (int64_t)jb * b, b, false,
                                      Wm + jb + (int64_t)(jb + jn) * b, b, false, 1.0,
                                      Wm + (jb + jn) + (int64_t)(jb + jn) * b, b, gsm);
  }
  GPHASE(3);
  if (threadIdx.x == 0) {
    atomicAdd(ws.flops + FLOP_GETRF, (unsigned long long)(2.0 / 3.0 * (double)b * b * b));
    if (first_zero >= 0) atomicCAS(ws.err + ERR_SINGULAR_STEP, 0, i + 1);
    // permutation from the interchanges: (P B)[r] = B[perm[r]]
    for (int r = 0; r < b; ++r) perm[r] = r;
    for (int r = 0; r < b; ++r) {
      const int p = piv[r];
      const int t = perm[r]; perm[r] = perm[p]; perm[p] = t;
    }
  }
  // packed LU back into the block
  for (int64_t e = threadIdx.x; e < (int64_t)b * b; e += blockDim.x) {
    const int r = e % b, c = e / b;
    Dp[r + (int64_t)c * ldA] = T(Wm[r + (int64_t)c * b]);
  }
  __syncthreads();
  GPHASE(5);
}

// ---------------------------------------------------------------------------
// K1 as separate launches (the factorization path): the same leaf LU, with
// the trailing update of each 32-column panel spread over 64 x 64 tiles on
// many CTAs instead of one.  Sequence for diagonal block i:
//   k_getrf_load; for each panel: k_getrf_panel (one CTA: getrf_panel_step),
//   k_getrf_trail (tiles); k_getrf_store.
// Per element the same operations in the same order as k_getrf.
// ---------------------------------------------------------------------------
constexpr int GETRF_AUX_THREADS = 256;

template <typename T>
FRANK_D void k_getrf_load_impl(BlrView<T> A, FactorWs<T> ws, int i) {
  const int b = A.bs(i), ld = A.bmax;
  const T* Dp = A.dense(i, i);
  double* Wm = ws.getrf_scratch;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)b * b;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int r = e % b, c = e / b;
    Wm[r + (int64_t)c * b] = double(Dp[r + (int64_t)c * ld]);
  }
}

template <typename T>
__global__ void __launch_bounds__(GETRF_AUX_THREADS) k_getrf_load(BlrView<T> A, FactorWs<T> ws, int i) {
  k_getrf_load_impl<T>(A, ws, i);
}

template <typename T>
FRANK_D void k_getrf_panel_impl(BlrView<T> A, FactorWs<T> ws, int i, int jb) {
  __shared__ double red[32];
  __shared__ int redi[32];
  __shared__ double gsm[2 * 16 * 64];
  __shared__ double tri[32 * 33];
  __shared__ double prow[32];
  __shared__ double xrow[32];
  const int b = A.bs(i);
  if (jb >= b) return;
  double* Wm = ws.getrf_scratch;
  double* Gp = Wm + (int64_t)A.bmax * A.bmax;
  int* piv = ws.ipiv + (int64_t)i * A.bmax;
  const int z = getrf_panel_step(b, jb, Wm, Gp, piv, red, redi, gsm, tri, prow, xrow);
  if (z >= 0 && threadIdx.x == 0) atomicCAS(ws.err + ERR_SINGULAR_STEP, 0, i + 1);
}

template <typename T>
__global__ void __launch_bounds__(GETRF_THREADS) k_getrf_panel(BlrView<T> A, FactorWs<T> ws, int i, int jb) {
  k_getrf_panel_impl<T>(A, ws, i, jb);
}

template <typename T>
FRANK_D void k_getrf_trail_impl(BlrView<T> A, FactorWs<T> ws, int i, int jb) {
  __shared__ double gsm[2 * 16 * 64];
  const int b = A.bs(i);
  if (jb >= b) return;
  const int jn = min(32, b - jb), m2 = b - jb - jn;
  if (m2 <= 0) return;
  double* Wm = ws.getrf_scratch;
  const int nt = (m2 + 63) / 64;
  for (int tile = blockIdx.x; tile < nt * nt; tile += gridDim.x) {
    const int r0 = (tile / nt) * 64, c0 = (tile % nt) * 64;
    const int rn = min(64, m2 - r0), cn = min(64, m2 - c0);
    cta_gemm<double, GETRF_AUX_THREADS>(rn, cn, jn, -1.0, Wm + (jb + jn + r0) + (int64_t)jb * b, b, false,
                                        Wm + jb + (int64_t)(jb + jn + c0) * b, b, false, 1.0,
                                        Wm + (jb + jn + r0) + (int64_t)(jb + jn + c0) * b, b, gsm);
  }
}

template <typename T>
__global__ void __launch_bounds__(GETRF_AUX_THREADS) k_getrf_trail(BlrView<T> A, FactorWs<T> ws, int i, int jb) {
  k_getrf_trail_impl<T>(A, ws, i, jb);
}

template <typename T>
FRANK_D void k_getrf_store_impl(BlrView<T> A, FactorWs<T> ws, int i) {
  const int b = A.bs(i), ld = A.bmax;
  T* Dp = A.dense(i, i);
  const double* Wm = ws.getrf_scratch;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    atomicAdd(ws.flops + FLOP_GETRF, (unsigned long long)(2.0 / 3.0 * (double)b * b * b));
    const int* piv = ws.ipiv + (int64_t)i * ld;
    int* perm = ws.perm + (int64_t)i * ld;
    // permutation from the interchanges: (P B)[r] = B[perm[r]]
    for (int r = 0; r < b; ++r) perm[r] = r;
    for (int r = 0; r < b; ++r) {
      const int p = piv[r];
      const int t = perm[r]; perm[r] = perm[p]; perm[p] = t;
    }
  }
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)b * b;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int r = e % b, c = e / b;
    Dp[r + (int64_t)c * ld] = T(Wm[r + (int64_t)c * b]);
  }
}

template <typename T>
__global__ void __launch_bounds__(GETRF_AUX_THREADS) k_getrf_store(BlrView<T> A, FactorWs<T> ws, int i) {
  k_getrf_store_impl<T>(A, ws, i);
}

// ---------------------------------------------------------------------------
// K1': explicit inverses of the factors of diagonal block i, Uinv = U^{-1} and
// Linv = L^{-1} (L unit lower), in column blocks of width cw: CTA q < nblk
// forms column block q of Uinv, CTA nblk + q column block q of Linv.  The
// column blocks are independent, so all 2 * nblk CTAs run at once.  A CTA
// keeps its b x cw block X of the inverse in shared memory (FP64) and sweeps
// the 32-row blocks in substitution order (upper: from the diagonal up to
// row 0; lower: from the diagonal down): acc = E - T(rb, solved) X(solved)
// by a CTA GEMM, then X(rb) = T(rb, rb)^{-1} acc by warp substitution (one
// warp per column, lane = row, the solved value broadcast by shuffle).  The
// packed LU is read from the block (precision T).  (LAPACK dtrtri forms the
// same inverse, by column blocks in sequence.)
// ---------------------------------------------------------------------------
constexpr int TRINV_THREADS = 256;

// Column-block width for block order bmax: X (bmax x cw doubles) must fit in
// shared memory beside the static arrays.
inline int trinv_width(int bmax) { return bmax <= 640 ? 32 : 16; }
constexpr int TRINV_SMEM_MAX = 640 * 32 * (int)sizeof(double);   // covers 1024 x 16 too

template <typename T>
FRANK_D void k_trinv_impl(BlrView<T> A, FactorWs<T> ws, int i, int cw) {
  extern __shared__ double X[];        // b x cw (ld b), rows indexed absolutely
  __shared__ double tri[32 * 33];
  __shared__ double acc[32 * 32];
  __shared__ double gsm[2 * 16 * 64];
  const int b = A.bs(i), ld = A.bmax;
  const T* LU = A.dense(i, i);
  const int nblk = (b + cw - 1) / cw;
  const bool upper = (int)blockIdx.x < nblk;
  const int cb = upper ? blockIdx.x : blockIdx.x - nblk;
  const int c0 = cb * cw, cn = min(cw, b - c0);
  if (c0 >= b) return;
  T* out = (upper ? ws.Uinv : ws.Linv) + (int64_t)i * ld * ld;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nrb = (b + 31) / 32;
  // upper: rows at or above the last diagonal row c0+cn-1; lower: from c0 down
  const int rb_first = upper ? (c0 + cn - 1) / 32 : c0 / 32;
  const int rb_last = upper ? 0 : nrb - 1;
  const int rb_step = upper ? -1 : 1;
  for (int rb = rb_first;; rb += rb_step) {
    const int r0 = rb * 32, rn = min(32, b - r0);
    for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
      const int r = e % 32, c = e / 32;
      acc[e] = (r < rn && c < cn && r0 + r == c0 + c) ? 1.0 : 0.0;
      tri[r + c * 33] = (r < rn && c < rn) ? double(LU[(r0 + r) + (int64_t)(r0 + c) * ld]) : 0.0;
    }
    __syncthreads();
    if (upper) {
      const int k0 = r0 + rn, kn = c0 + cn - k0;   // solved rows of X below this block
      if (kn > 0)
        cta_gemm<double, TRINV_THREADS>(rn, cn, kn, -1.0, LU + r0 + (int64_t)k0 * ld, ld, false, X + k0, b, false,
                                        1.0, acc, 32, gsm);
    } else {
      const int k0 = c0, kn = r0 - c0;              // solved rows of X above this block
      if (kn > 0)
        cta_gemm<double, TRINV_THREADS>(rn, cn, kn, -1.0, LU + r0 + (int64_t)k0 * ld, ld, false, X + k0, b, false,
                                        1.0, acc, 32, gsm);
    }
    __syncthreads();
    for (int c = wid; c < cn; c += nw) {
      double v = lane < rn ? acc[lane + c * 32] : 0.0;
      if (upper) {
        for (int t = rn - 1; t >= 0; --t) {
          const double xt = __shfl_sync(0xffffffffu, v, t) / tri[t + t * 33];
          if (lane == t) v = xt;
          else if (lane < t) v -= tri[lane + t * 33] * xt;
        }
      } else {
        for (int t = 0; t < rn; ++t) {
          const double xt = __shfl_sync(0xffffffffu, v, t);
          if (lane > t) v -= tri[lane + t * 33] * xt;
        }
      }
      if (lane < rn) X[r0 + lane + (int64_t)c * b] = v;
    }
    __syncthreads();
    if (rb == rb_last) break;
  }
  // upper: rows below the last diagonal row are zero; lower: rows above c0
  const int rlo = upper ? 0 : c0, rhi = upper ? c0 + cn : b;
  for (int e = threadIdx.x; e < b * cn; e += blockDim.x) {
    const int r = e % b, c = e / b;
    out[r + (int64_t)(c0 + c) * ld] = (r >= rlo && r < rhi) ? T(X[r + (int64_t)c * b]) : T(0);
  }
  if (threadIdx.x == 0 && blockIdx.x == 0)
    atomicAdd(ws.flops + FLOP_GETRF, (unsigned long long)(2.0 / 3.0 * (double)b * b * b));
}

template <typename T>
__global__ void __launch_bounds__(TRINV_THREADS) k_trinv(BlrView<T> A, FactorWs<T> ws, int i, int cw) {
  k_trinv_impl<T>(A, ws, i, cw);
}

// ---------------------------------------------------------------------------
// K2: panel of step i (trsm.cpp:92-115 with the leaf inverse; the pivots of
// K1 applied).  Task t < m: column-panel block (i+1+t, i):
//   low rank: V <- V Uinv (Vt <- Uinv^T Vt), then WL = Vt S^T;
//   dense:    A <- A Uinv.
// Task t >= m: row-panel block (i, i+1+t-m):
//   low rank: U <- Linv P U, then WU = U S;   dense: A <- Linv P A.
// Three launches, each over (task, 64-row tile of the result), so that every
// block is spread over several CTAs and no tile reads rows another tile of
// the same launch writes:
//   k_panel_gather  row tasks:    tmp = P U  (P A)                 -> WU[k]
//   k_panel_mul     column tasks: tmp = Uinv^T Vt  (A Uinv)        -> WL[ic]
//                   row tasks:    U = Linv tmp  (A = Linv tmp)
//   k_panel_fin     column tasks: Vt = tmp, then WL = Vt S^T  (A = tmp)
//                   row tasks:    WU = U S
// ---------------------------------------------------------------------------
constexpr int PANEL_THREADS = 256;
constexpr int PANEL_TILE = 64;

template <typename T>
struct PanelTask {
  bool col;      // column-panel block (else row-panel block)
  bool lr;
  int blk, rows, cols, r;   // result rows x cols (cols = rank for low rank)
  T* tmp;
};

template <typename T>
FRANK_D PanelTask<T> panel_task(const BlrView<T>& A, const FactorWs<T>& ws, int i, int t) {
  const int m = A.nb - i - 1;
  const int bi = A.bs(i), ld = A.bmax;
  PanelTask<T> P;
  P.col = t < m;
  if (P.col) {
    const int ic = i + 1 + t;
    P.blk = ic * A.nb + i;
    P.tmp = ws.WL + (int64_t)ic * ld * ld;
    P.lr = A.lslot[P.blk] >= 0;
    P.r = P.lr ? A.rank[P.blk] : 0;
    P.rows = P.lr ? bi : A.bs(ic);
    P.cols = P.lr ? P.r : bi;
  } else {
    const int k = i + 1 + (t - m);
    P.blk = i * A.nb + k;
    P.tmp = ws.WU + (int64_t)k * ld * ld;
    P.lr = A.lslot[P.blk] >= 0;
    P.r = P.lr ? A.rank[P.blk] : 0;
    P.rows = bi;
    P.cols = P.lr ? P.r : A.bs(k);
  }
  return P;
}

template <typename T>
FRANK_D T* panel_data(const BlrView<T>& A, const PanelTask<T>& P) {
  const int bi_ = P.blk / A.nb, bj_ = P.blk % A.nb;
  if (!P.lr) return A.dense(bi_, bj_);
  return P.col ? A.vt(bi_, bj_) : A.u(bi_, bj_);
}

template <typename T>
FRANK_D void k_panel_gather_impl(BlrView<T> A, FactorWs<T> ws, int i) {
  const int m = A.nb - i - 1;
  const PanelTask<T> P = panel_task(A, ws, i, m + blockIdx.x);
  const int r0 = blockIdx.y * PANEL_TILE;
  if (r0 >= P.rows) return;
  const int rn = min(PANEL_TILE, P.rows - r0), ld = A.bmax;
  const int* perm = ws.perm + (int64_t)i * ld;
  const T* src = panel_data(A, P);
  for (int e = threadIdx.x; e < rn * P.cols; e += blockDim.x) {
    const int rr = r0 + e % rn, c = e / rn;
    P.tmp[rr + (int64_t)c * ld] = src[perm[rr] + (int64_t)c * ld];
  }
}

template <typename T>
__global__ void __launch_bounds__(PANEL_THREADS) k_panel_gather(BlrView<T> A, FactorWs<T> ws, int i) {
  k_panel_gather_impl<T>(A, ws, i);
}

template <typename T>
FRANK_D void k_panel_mul_impl(BlrView<T> A, FactorWs<T> ws, int i) {
  __shared__ T gsm[2 * 16 * 64];
  const int t = blockIdx.x;
  const PanelTask<T> P = panel_task(A, ws, i, t);
  const int r0 = blockIdx.y * PANEL_TILE;
  const int bi = A.bs(i), ld = A.bmax;
  if (threadIdx.x == 0 && blockIdx.y == 0) {
    const double kk = P.lr ? P.r : (P.col ? P.rows : P.cols);
    atomicAdd(ws.flops + FLOP_PANEL, (unsigned long long)((double)bi * bi * kk));
  }
  if (r0 >= P.rows) return;
  const int rn = min(PANEL_TILE, P.rows - r0);
  T* d = panel_data(A, P);
  const T* Li = ws.Linv + (int64_t)i * ld * ld;
  const T* Ui = ws.Uinv + (int64_t)i * ld * ld;
  if (P.col) {
    if (P.lr)   // tmp(rows) = Uinv^T(rows, :) Vt
      cta_gemm<T, PANEL_THREADS>(rn, P.cols, bi, T(1), Ui + (int64_t)r0 * ld, ld, true, d, ld, false, T(0), P.tmp + r0,
                                 ld, gsm);
    else        // tmp(rows) = A(rows, :) Uinv
      cta_gemm<T, PANEL_THREADS>(rn, P.cols, bi, T(1), d + r0, ld, false, Ui, ld, false, T(0), P.tmp + r0, ld, gsm);
  } else {      // U(rows) = Linv(rows, :) P U   (A likewise)
    cta_gemm<T, PANEL_THREADS>(rn, P.cols, bi, T(1), Li + r0, ld, false, P.tmp, ld, false, T(0), d + r0, ld, gsm);
  }
}

template <typename T>
__global__ void __launch_bounds__(PANEL_THREADS) k_panel_mul(BlrView<T> A, FactorWs<T> ws, int i) {
  k_panel_mul_impl<T>(A, ws, i);
}

template <typename T>
FRANK_D void k_panel_fin_impl(BlrView<T> A, FactorWs<T> ws, int i) {
  __shared__ T gsm[2 * 16 * 64];
  const int t = blockIdx.x;
  const PanelTask<T> P = panel_task(A, ws, i, t);
  const int r0 = blockIdx.y * PANEL_TILE;
  if (r0 >= P.rows) return;
  if (!P.col && !P.lr) return;
  const int rn = min(PANEL_TILE, P.rows - r0), ld = A.bmax;
  T* d = panel_data(A, P);
  const int bi_ = P.blk / A.nb, bj_ = P.blk % A.nb;
  if (P.col) {
    for (int e = threadIdx.x; e < rn * P.cols; e += blockDim.x) {
      const int rr = r0 + e % rn, c = e / rn;
      d[rr + (int64_t)c * ld] = P.tmp[rr + (int64_t)c * ld];
    }
    __syncthreads();
    if (P.lr)   // WL(rows) = Vt(rows) S^T
      cta_gemm<T, PANEL_THREADS>(rn, P.r, P.r, T(1), d + r0, ld, false, A.s(bi_, bj_), A.kcap, true, T(0),
                                 P.tmp + r0, ld, gsm);
  } else {      // WU(rows) = U(rows) S
    cta_gemm<T, PANEL_THREADS>(rn, P.r, P.r, T(1), d + r0, ld, false, A.s(bi_, bj_), A.kcap, false, T(0),
                               P.tmp + r0, ld, gsm);
  }
}

template <typename T>
__global__ void __launch_bounds__(PANEL_THREADS) k_panel_fin(BlrView<T> A, FactorWs<T> ws, int i) {
  k_panel_fin_impl<T>(A, ws, i);
}

// Task t (0 <= t < m*(m-1)) of step i's off-diagonal targets, ordered by
// band d = |ic - k| = 1, 2, ... (the near-diagonal targets carry the largest
// ranks, so they are handed out first), within a band by row.
FRANK_D void band_task(int m, int t, int& a, int& c) {
  int d = 1;
  while (t >= 2 * (m - d)) { t -= 2 * (m - d); ++d; }
  const int half = m - d;
  if (t < half) { a = t + d; c = t; } else { a = t - half; c = t - half + d; }
}

// Next task of the step for this CTA (dynamic scheduling through an atomic
// counter; all threads receive it).
FRANK_D int next_task(int* counter, int* slot) {
  __syncthreads();
  if (threadIdx.x == 0) *slot = atomicAdd(counter, 1);
  __syncthreads();
  return *slot;
}

// Operands of the update of target (ic, k) at step i:
//   update = - XL * (WL^T WU) * YR^T,
// XL = U(ic,i) (bc x p) or dense A(ic,i) (bc x bi, WL = I),
// YR = Vt(i,k) (bk x q) or A(i,k)^T (WU = I).
template <typename T>
struct UpdOps {
  const T* XL; int p; bool left_dense;
  const T* YR; int q; bool right_dense;   // right_dense: YR^T = A(i,k) (bi x bk, ld)
  const T* WL; const T* WU;
};

template <typename T>
FRANK_D UpdOps<T> update_operands(const BlrView<T>& A, const FactorWs<T>& ws, int i, int ic, int k) {
  UpdOps<T> o;
  const int ld = A.bmax;
  const int bi = A.bs(i);
  o.WL = ws.WL + (int64_t)ic * ld * ld;
  o.WU = ws.WU + (int64_t)k * ld * ld;
  if (A.is_lr(ic, i)) { o.XL = A.u(ic, i); o.p = A.rank[ic * A.nb + i]; o.left_dense = false; }
  else { o.XL = A.dense(ic, i); o.p = bi; o.left_dense = true; }
  if (A.is_lr(i, k)) { o.YR = A.vt(i, k); o.q = A.rank[i * A.nb + k]; o.right_dense = false; }
  else { o.YR = A.dense(i, k); o.q = bi; o.right_dense = true; }
  return o;
}

// core T (p x q) = -WL^T WU, FP64, into Tm (ld p).
template <typename T, int NT>
FRANK_D void form_core(const UpdOps<T>& o, int bi, int ld, double* Tm, double* gsm) {
  if (!o.left_dense && !o.right_dense) {
    // small cores: one warp per entry (lanes along the b-long inner dimension)
    if (o.p * o.q <= 1024) cta_gemm_tn_dot(o.p, o.q, bi, -1.0, o.WL, ld, o.WU, ld, Tm, o.p);
    else cta_gemm<double, NT>(o.p, o.q, bi, -1.0, o.WL, ld, true, o.WU, ld, false, 0.0, Tm, o.p, gsm);
  } else if (!o.left_dense && o.right_dense) {
    // -WL^T (p x bi)
    for (int64_t e = threadIdx.x; e < (int64_t)o.p * o.q; e += blockDim.x) {
      const int r = e % o.p, c = e / o.p;
      Tm[e] = -double(o.WL[c + (int64_t)r * ld]);
    }
    __syncthreads();
  } else if (o.left_dense && !o.right_dense) {
    for (int64_t e = threadIdx.x; e < (int64_t)o.p * o.q; e += blockDim.x) {
      const int r = e % o.p, c = e / o.p;
      Tm[e] = -double(o.WU[r + (int64_t)c * ld]);
    }
    __syncthreads();
  } else {
    for (int64_t e = threadIdx.x; e < (int64_t)o.p * o.q; e += blockDim.x) {
      const int r = e % o.p, c = e / o.p;
      Tm[e] = (r == c) ? -1.0 : 0.0;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// K5: update of dense targets (diagonal blocks and inadmissible blocks):
// C += XL * T * YR^T  (gemm.cpp:180-200 for LR.LR.D; 126-178 for the others).
// One task per (target, band of band_rows rows): the band's CTA forms the
// small core T (p x q) once, X = XL(band, :) T (rows x q) in its scratch slot,
// and updates its rows of C over the full width, so the core is formed
// ceil(b / band_rows) times per target and C is streamed in full rows.
// Modes: every dense target of the step, only the next diagonal block
// (i+1, i+1) (which the next leaf getrf waits for), or all but that block.
// ---------------------------------------------------------------------------
constexpr int DUPD_THREADS = 256;
constexpr int DUPD_BAND = 128;    // rows of a dense update task (default; the autotuner may change it)
enum DenseUpdateMode { DUPD_ALL = 0, DUPD_NEXT = 1, DUPD_REST = 2 };

template <typename T>
FRANK_D void k_update_dense_impl(BlrView<T> A, FactorWs<T> ws, int i, int band_rows,
                                                                int mode) {
  __shared__ double gsm[2 * 16 * 64];
  __shared__ T gsmt[2 * 16 * 64];
  const int m = A.nb - i - 1;
  const int ld = A.bmax;
  const int bi = A.bs(i);
  double* Tm = ws.dscratch + (int64_t)blockIdx.x * ws.dscratch_stride;
  // X (rn x q, ld ldx) in the second ld x ld half of the slot: ldx * q <= ld * ld
  T* X = reinterpret_cast<T*>(Tm + (int64_t)ld * ld);
  const int bandr = min(band_rows, ld);
  const int ldx = bandr;
  const int nbands = (ld + bandr - 1) / bandr;
  // pair 0 is the next diagonal block (i+1, i+1)
  const int ntask = mode == DUPD_NEXT ? nbands : m * m * nbands;
  for (int tsk = blockIdx.x; tsk < ntask; tsk += gridDim.x) {
    const int pair = tsk / nbands, band = tsk % nbands;
    if (mode == DUPD_REST && pair == 0) continue;
    const int ic = i + 1 + pair / m, k = i + 1 + pair % m;
    if (A.is_lr(ic, k)) continue;
    const int bc = A.bs(ic), bk = A.bs(k);
    const int r0 = band * bandr;
    if (r0 >= bc) continue;
    const int rn = min(bandr, bc - r0);
    T* C = A.dense(ic, k) + r0;
    UpdOps<T> o = update_operands(A, ws, i, ic, k);
    if (threadIdx.x == 0 && band == 0)
      atomicAdd(ws.flops + FLOP_DENSE, (unsigned long long)(2.0 * bc * bk * o.q + 2.0 * bc * o.p * o.q +
                                                            2.0 * bi * o.p * o.q));
    if (o.left_dense && o.right_dense) {
      // C -= A(ic,i) A(i,k)
      cta_gemm<T, DUPD_THREADS>(rn, bk, bi, T(-1), o.XL + r0, ld, false, o.YR, ld, false, T(1), C, ld, gsmt);
      continue;
    }
    form_core<T, DUPD_THREADS>(o, bi, ld, Tm, gsm);
    // X = XL(r0 : r0+rn, :) T  (rn x q), accumulate in the working precision
    cta_gemm<T, DUPD_THREADS>(rn, o.q, o.p, T(1), o.XL + r0, ld, false, Tm, o.p, false, T(0), X, ldx, gsmt);
    // C(band) += X * YR^T
    if (!o.right_dense)
      cta_gemm<T, DUPD_THREADS>(rn, bk, o.q, T(1), X, ldx, false, o.YR, ld, true, T(1), C, ld, gsmt);
    else
      cta_gemm<T, DUPD_THREADS>(rn, bk, o.q, T(1), X, ldx, false, o.YR, ld, false, T(1), C, ld, gsmt);
  }
}

template <typename T>
__global__ void __launch_bounds__(DUPD_THREADS) k_update_dense(BlrView<T> A, FactorWs<T> ws, int i, int band_rows,
                                                                int mode) {
  k_update_dense_impl<T>(A, ws, i, band_rows, mode);
}

// ---------------------------------------------------------------------------
// K4: recompression of the update into every low-rank target of the step
// (rounded LowRank addition, operations/arithmetic/addition.cpp:93-127,
// Bebendorf p.16):
//   C + W = [U_C | XL] blockdiag(S_C, T) [Vt_C | YR]^T,
//   blocked Householder QR of the stacked U bases and of the stacked V bases
//   (FP64), core M = Ru blockdiag(S_C, T) Rv^T (FP64),
//   core truncation, either
//     RRQR: truncated column-pivoted QR of M to core_scale * eps * ||M||_F,
//           then RQ of the kept rows, i.e. the reference's own fixed-accuracy
//           compressor LowRank(Dense, eps) (low_rank.cpp:50-59, geqp3.cpp:71-192)
//           applied to the core; S comes out upper triangular;
//     SVD:  one-sided Jacobi of M with the rank of find_svd_truncation_rank
//           (misc.cpp:133-146, quirk included) or the fixed rank; S diagonal;
//   new U = Qu [Q_core; 0], new V^T = Qv [V_core; 0].
// Persistent grid, one target per CTA at a time, FP64 scratch slot per CTA.
// The core lives in shared memory when it fits (RECOMP_SMEM_CORE doubles).
// ---------------------------------------------------------------------------
constexpr int RECOMP_THREADS = 512;
constexpr int SPLIT_P = 32;       // split band-1 targets whose operand rank exceeds this (default)
constexpr int SPLIT_MAX = 128;    // band-1 tasks eligible for the split (scratch slots)
constexpr int RECOMP_SMEM_BYTES = 227 * 1024 - 512;     // dynamic shared memory (all but the static part)
constexpr int RECOMP_GSM = 2 * 16 * 64;                 // cta_gemm tiles (doubles)
constexpr int RECOMP_REGION = RECOMP_SMEM_BYTES / 8 - RECOMP_GSM;  // doubles for panels / core
// Core of the recompression: RRQR (truncated pivoted QR + RQ of the core),
// SVD (one-sided Jacobi, find_svd_truncation_rank or the fixed rank), FAST
// (fast_rounded_addition, addition.cpp:133-189: fixed-rank targets with
// orthonormal bases; the update's bases are projected out of the target's and
// only the remainders are QR-factored; SVD core as above).
enum CoreMethod { CORE_RRQR = 0, CORE_SVD = 1, CORE_FAST = 2 };

// SVD of the recompression core Mm (mu x mv, ld mu), preconditioned
// one-sided Jacobi: column-pivoted QR M P = Q R (in place in Mm), then
// one-sided Jacobi on the columns of A = R^T (mv x k) with the rotations
// accumulated in Z (k x k, appended rows); the pivoting leaves A's columns
// nearly orthogonal, so a few sweeps converge (Drmac & Veselic, "New fast and
// accurate Jacobi SVD algorithm", SIAM J. Matrix Anal. Appl. 29, 2008).
// With A Z = W S: M = (Q Z) S (P W)^T, so the left singular vectors are Q Z
// (the QR's reflectors applied to Z) and the right ones P W (the normalised
// columns of A Z, rows permuted back); both sets are orthonormal to working
// accuracy whatever the singular value, which the next projected addition
// into this target relies on.  Tolerance plans stop the QR once the
// remaining columns are below thr = 0.01 eps ||M||_F / sqrt(mv min(mu, mv)),
// so the dropped block R22 moves the truncation test below by at most 1 % of
// its threshold.  Rank: the fixed rank of the plan, else
// find_svd_truncation_rank (misc.cpp:133-146, quirk included: the tail error
// is (min_dim - r) sigma_r^2) at ws.eps with ||M||_F as the reference norm;
// capped at kcap (counted as a rank overflow).  Scratch: the Jacobi matrix
// ((mv + k) x k) in smem (region, cap doubles, after the core if the core is
// there) when it fits, else in Atmp (global, (mv + min(mu,mv)) x min(mu,mv));
// tau / cnorm / partial / jpvt (mv each), sig / ord (min(mu, mv)).  On return
// partial[c] is the c-th largest singular value (c < r), Xo (bc x r, ld bc) =
// [U_m(:, :r); 0] and Yo (bk x r, ld bk) = [V_m(:, :r); 0].  Returns r (all
// threads).
template <typename T, int NT>
FRANK_D int svd_core(int mu, int mv, double* Mm, const FactorWs<T>& ws, int kcap, double* region, int64_t cap,
                     double* Atmp, double* tau, double* cnorm, double* partial, int* jpvt, double* sig, int* ord,
                     double* Xo, int bc, double* Yo, int bk, double* gsm, double* red, int* redi, int* flag,
                     int* s_rank) {
  const int nsv = min(mu, mv);
  double f = 0.0;
  for (int64_t e = threadIdx.x; e < (int64_t)mu * mv; e += blockDim.x) f += Mm[e] * Mm[e];
  const double fro = sqrt(block_sum(f, red));
  const double thr = ws.fixed_rank > 0 ? 0.0 : 0.01 * ws.eps * fro / sqrt((double)mv * (double)nsv);
  // a core in L2 takes the blocked pivoted QR (F, mv x 32, in Atmp)
  const int k = Mm != region ? cta_truncated_geqp3_blocked<NT>(mu, mv, Mm, mu, thr, nsv, tau, cnorm, partial, jpvt,
                                                               red, redi, Atmp, gsm)
                             : cta_truncated_geqp3(mu, mv, Mm, mu, thr, nsv, tau, cnorm, partial, jpvt, red, redi);
  // [A; I] with A = R(0:k, :)^T (mv x k), ld mv + k
  const int ldj = mv + k;
  const int64_t off = (Mm == region) ? (int64_t)mu * mv : 0;
  double* Aj = off + (int64_t)ldj * k <= cap ? region + off : Atmp;
  for (int64_t e = threadIdx.x; e < (int64_t)ldj * k; e += blockDim.x) {
    const int c = e % ldj, j = e / ldj;
    Aj[e] = c < mv ? ((c >= j) ? Mm[j + (int64_t)c * mu] : 0.0) : (c - mv == j ? 1.0 : 0.0);
  }
  __syncthreads();
  const int sweeps = cta_jacobi_columns(mv, k, Aj, ldj, 60, flag, ldj);
  if (sweeps < 0 && threadIdx.x == 0) atomicAdd(ws.err + ERR_JACOBI, 1);
  for (int c = threadIdx.x >> 5; c < k; c += blockDim.x >> 5) {
    double sacc = 0.0;
    for (int rr = threadIdx.x & 31; rr < mv; rr += 32) sacc += Aj[rr + (int64_t)c * ldj] * Aj[rr + (int64_t)c * ldj];
    sacc = warp_sum(sacc);
    if ((threadIdx.x & 31) == 0) sig[c] = sqrt(sacc);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < k; c += blockDim.x) {
    const double v = sig[c];
    int pos = 0;
    for (int d = 0; d < k; ++d) {
      const double w = sig[d];
      pos += (w > v) || (w == v && d < c);
    }
    ord[pos] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int rr;
    if (ws.fixed_rank > 0) {
      rr = min(ws.fixed_rank, nsv);
    } else {
      // singular values beyond the k computed ones are below ||R22||, which
      // satisfies the test by the choice of thr: count them as zero
      const double thr_t = ws.eps * fro;
      rr = 0;
      double err;
      do {
        ++rr;
        err = 0.0;
        if (rr < nsv) {
          const double v = rr < k ? sig[ord[rr]] : 0.0;
          err = (double)(nsv - rr) * v * v;
        }
      } while (rr < nsv && sqrt(err) > thr_t);
    }
    if (rr > kcap) { atomicAdd(ws.err + ERR_RANK_OVERFLOW, 1); rr = kcap; }
    atomicMax(ws.err + ERR_MAX_RANK, rr);
    atomicAdd(ws.err + ERR_RECOMP, 1);
    *s_rank = rr;
  }
  __syncthreads();
  const int r = *s_rank;
  // Yo (bk x r): V_M = P W, row jpvt[i] of V_M = row i of W (columns of A Z
  // normalised); Xo (bc x r) = [Z(:, ord); 0], then Q applied below
  for (int64_t e = threadIdx.x; e < (int64_t)bk * r; e += blockDim.x) Yo[e] = 0.0;
  for (int64_t e = threadIdx.x; e < (int64_t)bc * r; e += blockDim.x) {
    const int i = e % bc, c = e / bc;
    Xo[e] = (i < k && c < k) ? Aj[mv + i + (int64_t)ord[c] * ldj] : 0.0;
  }
  __syncthreads();
  for (int64_t e = threadIdx.x; e < (int64_t)mv * r; e += blockDim.x) {
    const int i = e % mv, c = e / mv;
    const int src = c < k ? ord[c] : -1;
    const double sv_ = src >= 0 ? sig[src] : 0.0;
    Yo[jpvt[i] + (int64_t)c * bk] = sv_ > 0.0 ? Aj[i + (int64_t)src * ldj] / sv_ : 0.0;
  }
  __syncthreads();
  cta_apply_q(mu, k, Mm, mu, tau, r, Xo, (int64_t)bc);
  // the kept singular values in order, in partial (free after the QR)
  for (int c = threadIdx.x; c < r; c += blockDim.x) partial[c] = c < k ? sig[ord[c]] : 0.0;
  __syncthreads();
  return r;
}

struct RecompLayout {
  int64_t ash, bsh, tm, rc, rv, mtmp, mglob, m0, xo, yo, tfu, tfv, w, tau_u, tau_v, tau_c, tau2, cn, pn, jp, ji, total;
};

FRANK_HD RecompLayout recomp_layout(int bmax, int smax) {
  RecompLayout L;
  int64_t o = 0;
  auto take = [&](int64_t n) { int64_t r = o; o += (n + 31) & ~int64_t(31); return r; };
  const int mu = smax < bmax ? smax : bmax;
  const int64_t np = (smax + QRB - 1) / QRB;
  L.ash = take((int64_t)bmax * smax);
  L.bsh = take((int64_t)bmax * smax);
  L.tm = take((int64_t)bmax * bmax);
  L.rc = take((int64_t)mu * smax);
  L.rv = take((int64_t)mu * smax);
  L.mtmp = take((int64_t)mu * smax);
  L.mglob = take((int64_t)mu * mu);
  L.m0 = take((int64_t)mu * mu);
  L.xo = take((int64_t)bmax * mu);
  L.yo = take((int64_t)bmax * mu);
  L.tfu = take(np * QRB * QRB);
  L.tfv = take(np * QRB * QRB);
  L.w = take((int64_t)QRB * (smax > bmax ? smax : bmax));
  L.tau_u = take(smax);
  L.tau_v = take(smax);
  L.tau_c = take(mu);
  L.tau2 = take(mu);
  L.cn = take(mu);
  L.pn = take(mu);
  L.jp = take(mu);
  L.ji = take(mu);
  L.total = o;
  return L;
}

template <typename T>
FRANK_D void k_recompress_impl(BlrView<T> A, FactorWs<T> ws, int i, int smax,
                                                               int core_method, double core_scale,
                                                               int only_dense_operands, int* counter, int nsplit,
                                                               double* split_base, int* split_done, int proj_tol,
                                                               int split_p, int core_smem) {
  extern __shared__ double dsm[];
  double* gsm = dsm;
  double* region = dsm + RECOMP_GSM;
  __shared__ double red[32];
  __shared__ int redi[32];
  __shared__ int flag;
  __shared__ int s_rank;
  const int m = A.nb - i - 1;
  const int ld = A.bmax;
  const int bi = A.bs(i);
  const RecompLayout L = recomp_layout(A.bmax, smax);
  double* const cta_base = ws.rscratch + (int64_t)blockIdx.x * ws.rscratch_stride;
  double *Ash, *Bsh, *Tm, *Rc, *Rv, *Mtmp, *Mg, *M0, *Xo, *Yo, *Tfu, *Tfv, *Wq, *tau_u, *tau_v, *tau_c, *tau2, *cnorm,
      *pnorm;
  int *jpvt, *jinv;
  auto set_base = [&](double* base) {
    Ash = base + L.ash; Bsh = base + L.bsh; Tm = base + L.tm; Rc = base + L.rc; Rv = base + L.rv;
    Mtmp = base + L.mtmp; Mg = base + L.mglob; M0 = base + L.m0; Xo = base + L.xo; Yo = base + L.yo;
    Tfu = base + L.tfu; Tfv = base + L.tfv; Wq = base + L.w; tau_u = base + L.tau_u; tau_v = base + L.tau_v;
    tau_c = base + L.tau_c; tau2 = base + L.tau2; cnorm = base + L.cn; pnorm = base + L.pn;
    jpvt = reinterpret_cast<int*>(base + L.jp); jinv = reinterpret_cast<int*>(base + L.ji);
  };
  __shared__ int s_last;
  double* smP = region;
  double* smT = region + (int64_t)A.bmax * QRB;
  __shared__ int s_task;
  const int ntask = m * (m - 1);
  // Split targets: band-1 targets (the first 2(m-1) tasks, largest ranks)
  // whose operands have ranks above SPLIT_P get one task per side of the
  // stacked-basis QR, run on two CTAs into the target's own scratch slot;
  // the CTA that finishes second does the rest (no waiting).  The test uses
  // only operand ranks, which no CTA changes during the launch.
  const int nspl = split_base ? min(nsplit, 2 * (m - 1)) : 0;
  const int ntot = 2 * nspl + ntask;
  for (int q = next_task(counter, &s_task); q < ntot; q = next_task(counter, &s_task)) {
    const int side = q < 2 * nspl ? (q & 1) : -1;
    const int tsk = q < 2 * nspl ? (q >> 1) : q - 2 * nspl;
    int a_, c_;
    band_task(m, tsk, a_, c_);
    const int ic = i + 1 + a_, k = i + 1 + c_;
    if (!A.is_lr(ic, k)) continue;
    if (only_dense_operands && A.is_lr(ic, i) && A.is_lr(i, k)) continue;
    const bool split_t = tsk < nspl && split_p > 0 && A.is_lr(ic, i) && A.is_lr(i, k) &&
                         max(A.rank[ic * A.nb + i], A.rank[i * A.nb + k]) > split_p;
    if ((side >= 0) != split_t) continue;
    set_base(side >= 0 ? split_base + (int64_t)tsk * ws.rscratch_stride : cta_base);
    const bool do_u = side != 1, do_v = side != 0;
    const int blk = ic * A.nb + k;
    const int bc = A.bs(ic), bk = A.bs(k);
    const int kc = A.rank[blk];
    UpdOps<T> o = update_operands(A, ws, i, ic, k);
    const int su = kc + o.p, sv = kc + o.q;
    if (su > smax || sv > smax) {
      if (threadIdx.x == 0) atomicAdd(ws.err + ERR_BOUNDS, 1);
      continue;
    }
    const int cls = (su <= 64 && sv <= 64) ? 0 : (su <= 160 && sv <= 160 ? 1 : 2);
    PHASE_BEGIN();
#ifdef FRANK_PHASE_TIMING
    const long long t_start = gtimer();
#endif
#ifdef FRANK_PHASE_TIMING
    if (threadIdx.x == 0) atomicAdd(&g_phase_count[cls], 1ull);
#endif
    T* Uc = A.u(ic, k);
    T* Sc = A.s(ic, k);
    T* Vc = A.vt(ic, k);
    SUB_BEGIN();
    // stacked bases in FP64
    for (int64_t e = threadIdx.x; do_u && e < (int64_t)bc * su; e += blockDim.x) {
      const int r = e % bc, c = e / bc;
      Ash[r + (int64_t)c * bc] = (c < kc) ? double(Uc[r + (int64_t)c * ld]) : double(o.XL[r + (int64_t)(c - kc) * ld]);
    }
    for (int64_t e = threadIdx.x; do_v && e < (int64_t)bk * sv; e += blockDim.x) {
      const int r = e % bk, c = e / bk;
      double v;
      if (c < kc) v = double(Vc[r + (int64_t)c * ld]);
      else if (!o.right_dense) v = double(o.YR[r + (int64_t)(c - kc) * ld]);
      else v = double(o.YR[(c - kc) + (int64_t)r * ld]);  // A(i,k)^T
      Bsh[r + (int64_t)c * bk] = v;
    }
    // the stacked bases are read across threads below (the V side of a split
    // target forms no core, whose barrier would otherwise cover this)
    __syncthreads();
    SUB_MARK(9);
    if (do_u) form_core<T, RECOMP_THREADS>(o, bi, ld, Tm, gsm);
    SUB_MARK(10);
    PHASE_MARK(cls, 0);
    // Bases.  Stacked (rounded_addition, addition.cpp:93-127): Householder QR
    // of [U_C | U_B] and of [V_C | V_B].  Projected (fast_rounded_addition,
    // addition.cpp:133-189, the default of fixed-rank plans, and on request
    // for tolerance plans): U_C and V_C have orthonormal columns (every
    // target comes from construction, a core SVD / RRQR or the reset
    // truncation), so U_B is projected out of span(U_C) twice, Zu = U_C^T U_B,
    // and only the remainder Y_u = U_B - U_C Zu is QR-factored; the same on the
    // V side.  Both give the same sum C + B = [U_C | Q] M [V_C | Q']^T.
    const bool proj = (core_method == CORE_FAST ? ws.fixed_rank > 0 : proj_tol != 0) && kc > 0 && o.p > 0 &&
                      o.q > 0 && !o.left_dense && !o.right_dense && su <= bc && sv <= bk;
    if (proj) {
      if (do_u) {
        cta_project_out<RECOMP_THREADS>(bc, kc, o.p, Ash, bc, Ash + (int64_t)kc * bc, bc, Rc + (int64_t)kc * su, su,
                                        Xo, gsm);
        cta_qr_blocked<RECOMP_THREADS>(bc, o.p, Ash + (int64_t)kc * bc, bc, tau_u, Tfu, Wq, smP, smT, gsm, red);
      }
      PHASE_MARK(cls, 1);
      if (do_v) {
        cta_project_out<RECOMP_THREADS>(bk, kc, o.q, Bsh, bk, Bsh + (int64_t)kc * bk, bk, Rv + (int64_t)kc * sv, sv,
                                        Yo, gsm);
        cta_qr_blocked<RECOMP_THREADS>(bk, o.q, Bsh + (int64_t)kc * bk, bk, tau_v, Tfv, side == 1 ? Mtmp : Wq, smP,
                                       smT, gsm, red);
      }
    } else {
      if (do_u) cta_qr_blocked<RECOMP_THREADS>(bc, su, Ash, bc, tau_u, Tfu, Wq, smP, smT, gsm, red);
      PHASE_MARK(cls, 1);
      // the V side of a split target works in Mtmp (free until the core), so
      // that the two sides never share the W scratch
      if (do_v) cta_qr_blocked<RECOMP_THREADS>(bk, sv, Bsh, bk, tau_v, Tfv, side == 1 ? Mtmp : Wq, smP, smT, gsm, red);
    }
    PHASE_MARK(cls, 2);
    if (side >= 0) {
      // publish this side; the second of the two CTAs goes on with the target
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) s_last = atomicAdd(split_done + tsk, 1);
      __syncthreads();
      if (s_last == 0) continue;
      __threadfence();
    }
    const int mu = proj ? su : min(bc, su), mv = proj ? sv : min(bk, sv);
    if (!proj) {
      // clean upper-trapezoidal R factors
      for (int64_t e = threadIdx.x; e < (int64_t)mu * su; e += blockDim.x) {
        const int r = e % mu, c = e / mu;
        Rc[e] = (r <= c) ? Ash[r + (int64_t)c * bc] : 0.0;
      }
      for (int64_t e = threadIdx.x; e < (int64_t)mv * sv; e += blockDim.x) {
        const int r = e % mv, c = e / mv;
        Rv[e] = (r <= c) ? Bsh[r + (int64_t)c * bk] : 0.0;
      }
    } else {
      // Rc = [I Zu; 0 Ru] (su x su), Rv = [I Zv; 0 Rv'] (sv x sv); Zu, Zv are in place
      for (int64_t e = threadIdx.x; e < (int64_t)mu * su; e += blockDim.x) {
        const int r = e % mu, c = e / mu;
        if (c < kc) Rc[e] = (r == c) ? 1.0 : 0.0;
        else if (r >= kc) Rc[e] = (r - kc <= c - kc) ? Ash[(r - kc) + (int64_t)c * bc] : 0.0;
      }
      for (int64_t e = threadIdx.x; e < (int64_t)mv * sv; e += blockDim.x) {
        const int r = e % mv, c = e / mv;
        if (c < kc) Rv[e] = (r == c) ? 1.0 : 0.0;
        else if (r >= kc) Rv[e] = (r - kc <= c - kc) ? Bsh[(r - kc) + (int64_t)c * bk] : 0.0;
      }
    }
    __syncthreads();
    // Mtmp (mu x sv) = [Rc[:, :kc] S_C | Rc[:, kc:] T]
    cta_gemm<double, RECOMP_THREADS>(mu, kc, kc, 1.0, Rc, mu, false, Sc, A.kcap, false, 0.0, Mtmp, mu, gsm);
    cta_gemm<double, RECOMP_THREADS>(mu, o.q, o.p, 1.0, Rc + (int64_t)kc * mu, mu, false, Tm, o.p, false, 0.0,
                                     Mtmp + (int64_t)kc * mu, mu, gsm);
    // core M (mu x mv) = Mtmp Rv^T, in shared memory if it fits
    // the core in shared memory when it fits and is not above the tuned size
    // (small cores always: the L2 paths need mu >= 64 for their T scratch)
    const int64_t core_need = (int64_t)mu * mv + 4 * (int64_t)mv + 2 * mu;
    const bool in_smem = core_need <= RECOMP_REGION && (mu < 64 || core_need <= core_smem);
    double* Mm = in_smem ? region : Mg;
    cta_gemm<double, RECOMP_THREADS>(mu, mv, sv, 1.0, Mtmp, mu, false, Rv, mv, true, 0.0, Mm, mu, gsm);
    PHASE_MARK(cls, 3);
    int r = 0;
    if (core_method == CORE_RRQR && ws.fixed_rank == 0) {
      double f = 0.0;
      for (int64_t e = threadIdx.x; e < (int64_t)mu * mv; e += blockDim.x) f += Mm[e] * Mm[e];
      f = block_sum(f, red);
      double* cn = in_smem ? region + (int64_t)mu * mv : cnorm;
      double* pn = in_smem ? cn + mv : pnorm;
      double* tc = in_smem ? pn + mv : tau_c;
      // a core in L2 (too large for shared memory) takes the pivoted QR with
      // randomized block pivoting (panel GEMMs instead of one pass over the
      // core per column), its scratch in Mtmp (free until the RQ below)
      const double thr_c = core_scale * ws.eps * sqrt(f);
      r = (!in_smem && rqrcp_scratch(mu, mv) <= L.mglob - L.mtmp)
              ? cta_rand_qrcp<RECOMP_THREADS>(mu, mv, Mm, mu, thr_c, A.kcap, tc, jpvt, Mtmp, smP, smT, gsm, red,
                                              redi)
              : cta_truncated_geqp3(mu, mv, Mm, mu, thr_c, A.kcap, tc, cn, pn, jpvt, red, redi);
      if (r == 0) {
        // zero core: rank-1 zero block (geqp3.cpp:97-102)
        if (threadIdx.x == 0) { atomicMax(ws.err + ERR_MAX_RANK, 1); atomicAdd(ws.err + ERR_RECOMP, 1); }
        for (int64_t e = threadIdx.x; e < (int64_t)bc; e += blockDim.x) Uc[e] = T(e == 0 ? 1.0 : 0.0);
        for (int64_t e = threadIdx.x; e < (int64_t)bk; e += blockDim.x) Vc[e] = T(e == 0 ? 1.0 : 0.0);
        if (threadIdx.x == 0) { Sc[0] = T(0); A.rank[blk] = 1; }
        __syncthreads();
        continue;
      }
      if (threadIdx.x == 0) {
        if (r >= A.kcap && r < min(mu, mv)) atomicAdd(ws.err + ERR_RANK_OVERFLOW, 1);
        atomicMax(ws.err + ERR_MAX_RANK, r);
        atomicAdd(ws.err + ERR_RECOMP, 1);
      }
      // the small factors (Q_core, the RQ of its kept rows and its explicit Q)
      // stay in shared memory after the core when they fit
      const int64_t voff = (int64_t)mu * mv + 4 * (int64_t)mv + 2 * (int64_t)mu;
      const bool t_sm = in_smem && voff + 2 * (int64_t)mv * r + (int64_t)mu * r <= RECOMP_REGION;
      // Xo (bc x r) = [Q_core; 0]
      if (t_sm) {
        double* X1s = region + voff + 2 * (int64_t)mv * r;   // mu x r
        for (int64_t e = threadIdx.x; e < (int64_t)mu * r; e += blockDim.x) X1s[e] = ((e % mu) == (e / mu)) ? 1.0 : 0.0;
        __syncthreads();
        cta_apply_q(mu, r, Mm, mu, tc, r, X1s, (int64_t)mu);
        for (int64_t e = threadIdx.x; e < (int64_t)bc * r; e += blockDim.x) {
          const int rr = e % bc, c = e / bc;
          Xo[e] = rr < mu ? X1s[rr + (int64_t)c * mu] : 0.0;
        }
      } else {
        for (int64_t e = threadIdx.x; e < (int64_t)bc * r; e += blockDim.x) {
          const int rr = e % bc, c = e / bc;
          Xo[e] = (rr == c) ? 1.0 : 0.0;
        }
        __syncthreads();
        if (!in_smem) {
          // a core in L2: the reflectors in panels of QRB (T factors in M0,
          // free in this branch), applied as blocked WY -- one reflector at a
          // time would sweep the r x r block once per reflector
          cta_form_t(mu, r, Mm, mu, tc, M0, smP, smT);
          cta_apply_q_blocked<RECOMP_THREADS>(mu, r, Mm, mu, M0, r, Xo, (int64_t)bc, Wq, smP, smT, gsm, r);
        } else {
          cta_apply_q(mu, r, Mm, mu, tc, r, Xo, (int64_t)bc);
        }
      }
      // X2 (mv x r) = R_perm^T J, R_perm[:, jpvt[c']] = R[:, c']
      for (int c = threadIdx.x; c < mv; c += blockDim.x) jinv[jpvt[c]] = c;
      __syncthreads();
      double* X2 = t_sm ? region + voff : Mtmp;
      for (int64_t e = threadIdx.x; e < (int64_t)mv * r; e += blockDim.x) {
        const int c = e % mv, a = e / mv;
        const int row = r - 1 - a, src = jinv[c];
        X2[e] = (row <= src) ? Mm[row + (int64_t)src * mu] : 0.0;
      }
      __syncthreads();
      if (!in_smem) cta_qr_blocked<RECOMP_THREADS>(mv, r, X2, mv, tau2, M0, Wq, smP, smT, gsm, red);
      else cta_householder_qr(mv, r, X2, mv, tau2, red);
      // S = J Rt^T J (upper triangular)
      for (int64_t e = threadIdx.x; e < (int64_t)r * r; e += blockDim.x) {
        const int a = e % r, c = e / r;
        const int ra = r - 1 - c, ca = r - 1 - a;
        Sc[a + (int64_t)c * A.kcap] = T((ra <= ca) ? X2[ra + (int64_t)ca * mv] : 0.0);
      }
      // Qt (mv x r) explicit, then Yo[:, a] = [Qt[:, r-1-a]; 0]
      double* Qt = t_sm ? X2 + (int64_t)mv * r : Rc;
      for (int64_t e = threadIdx.x; e < (int64_t)mv * r; e += blockDim.x) {
        const int rr = e % mv, c = e / mv;
        Qt[e] = (rr == c) ? 1.0 : 0.0;
      }
      __syncthreads();
      if (!in_smem)
        cta_apply_q_blocked<RECOMP_THREADS>(mv, r, X2, mv, M0, r, Qt, (int64_t)mv, Wq, smP, smT, gsm, r);
      else
        cta_apply_q(mv, r, X2, mv, tau2, r, Qt, (int64_t)mv);
      for (int64_t e = threadIdx.x; e < (int64_t)bk * r; e += blockDim.x) {
        const int rr = e % bk, a = e / bk;
        Yo[e] = (rr < mv) ? Qt[rr + (int64_t)(r - 1 - a) * mv] : 0.0;
      }
      __syncthreads();
    } else {
      // SVD core (Rc / Rv are free once the core is formed: Jacobi scratch)
      r = svd_core<T, RECOMP_THREADS>(mu, mv, Mm, ws, A.kcap, region, RECOMP_REGION, Rc, tau_c, cnorm, pnorm, jpvt,
                                      tau2, jinv, Xo, bc, Yo, bk, gsm, red, redi, &flag, &s_rank);
      for (int64_t e = threadIdx.x; e < (int64_t)r * r; e += blockDim.x) {
        const int rr = e % r, c = e / r;
        Sc[rr + (int64_t)c * A.kcap] = T(rr == c ? pnorm[c] : 0.0);
      }
      __syncthreads();
    }
    PHASE_MARK(cls, 4);
    if (threadIdx.x == 0)
      atomicAdd(ws.flops + FLOP_RECOMP,
                (unsigned long long)(proj ? fast_rounded_addition_flops(bc, bk, bi, kc, o.p, o.q, r)
                                          : rounded_addition_flops(bc, bk, bi, kc, o.p, o.q, r)));
    if (!proj) {
      // U = Qu Xo ; Vt = Qv Yo  (blocked WY application)
      // Xo = [Q_core; 0], Yo = [V_core; 0]: rows at or below mu (mv) are zero
      cta_apply_q_blocked<RECOMP_THREADS>(bc, mu, Ash, bc, Tfu, r, Xo, (int64_t)bc, Wq, smP, smT, gsm, mu);
      cta_apply_q_blocked<RECOMP_THREADS>(bk, mv, Bsh, bk, Tfv, r, Yo, (int64_t)bk, Wq, smP, smT, gsm, mv);
      for (int64_t e = threadIdx.x; e < (int64_t)bc * r; e += blockDim.x) {
        const int rr = e % bc, c = e / bc;
        Uc[rr + (int64_t)c * ld] = T(Xo[e]);
      }
      for (int64_t e = threadIdx.x; e < (int64_t)bk * r; e += blockDim.x) {
        const int rr = e % bk, c = e / bk;
        Vc[rr + (int64_t)c * ld] = T(Yo[e]);
      }
    } else {
      // U = [U_C | Q_u] Xo = Q_u [Xo(kc:mu); 0] + U_C Xo(0:kc), through Tm
      // (bc x r); U_C is read from its FP64 copy in Ash, so Uc is written last
      for (int side2 = 0; side2 < 2; ++side2) {
        const int bb = side2 ? bk : bc, pp = side2 ? o.q : o.p;
        double* X = side2 ? Yo : Xo;
        double* Bs = side2 ? Bsh : Ash;
        T* out = side2 ? Vc : Uc;
        for (int64_t e = threadIdx.x; e < (int64_t)bb * r; e += blockDim.x) {
          const int rr = e % bb, c = e / bb;
          Tm[e] = rr < pp ? X[kc + rr + (int64_t)c * bb] : 0.0;
        }
        __syncthreads();
        cta_apply_q_blocked<RECOMP_THREADS>(bb, pp, Bs + (int64_t)kc * bb, bb, side2 ? Tfv : Tfu, r, Tm, (int64_t)bb,
                                            Wq, smP, smT, gsm, pp);
        if (r <= 16) cta_gemm_tall(bb, r, kc, Bs, bb, X, bb, Tm, bb, true);
        else cta_gemm<double, RECOMP_THREADS>(bb, r, kc, 1.0, Bs, bb, false, X, bb, false, 1.0, Tm, bb, gsm);
        for (int64_t e = threadIdx.x; e < (int64_t)bb * r; e += blockDim.x) {
          const int rr = e % bb, c = e / bb;
          out[rr + (int64_t)c * ld] = T(Tm[e]);
        }
        __syncthreads();
      }
    }
    if (threadIdx.x == 0) A.rank[blk] = r;
    __syncthreads();
    PHASE_MARK(cls, 5);
#ifdef FRANK_PHASE_TIMING
    if (threadIdx.x == 0) {
      const unsigned long long q = atomicAdd(&g_tlog_n, 1ull);
      if (q < 200000) {
        g_tlog[q][0] = i; g_tlog[q][1] = su; g_tlog[q][2] = sv; g_tlog[q][3] = r;
        g_tlog[q][4] = t_start; g_tlog[q][5] = gtimer();
      }
    }
#endif
  }
}

template <typename T>
__global__ void __launch_bounds__(RECOMP_THREADS) k_recompress(BlrView<T> A, FactorWs<T> ws, int i, int smax,
                                                               int core_method, double core_scale,
                                                               int only_dense_operands, int* counter, int nsplit,
                                                               double* split_base, int* split_done, int proj_tol,
                                                               int split_p, int core_smem) {
  k_recompress_impl<T>(A, ws, i, smax, core_method, core_scale, only_dense_operands, counter, nsplit, split_base,
                       split_done, proj_tol, split_p, core_smem);
}

// ---------------------------------------------------------------------------
// K4' (mixed path): recompression by Gram matrices.  Same update and the same
// core truncation (RRQR + RQ of the core, or its fixed rank) as k_recompress,
// but the stacked bases A = [U_C | U_L] and B = [Vt_C | V_U] are not
// factored along their b rows: their FP64 Gram matrices A^T A, B^T B (one
// GEMM pass over the FP32 bases) are factored by pivoted Cholesky,
// A Pa ~= Qa [Ra11 Ra12] with Qa = A Pa(:, :ra) Ra11^{-1}, dropping directions
// whose relative norm is below sqrt(gram_tol); the core is
// M = Ra Pa^T blockdiag(S_C, T) Pb Rb^T and the new bases are
// U = A Pa [Ra11^{-1} Q_core; 0], V^T = B Pb [Rb11^{-1} V_core; 0].
// A Gram matrix in FP64 resolves directions down to ~1e-8 of the basis norm,
// which is ample for the loose factor tolerance of the mixed path (the FP64
// path keeps the Householder kernel).  Targets with a dense operand are left
// to k_recompress.  256 threads; small matrices in shared memory when they fit.
// ---------------------------------------------------------------------------
constexpr int GRAM_THREADS = 256;
constexpr int GRAM_SMEM_BYTES = 110 * 1024;
constexpr int GRAM_REGION = GRAM_SMEM_BYTES / 8;

// Per-CTA global scratch of the Gram kernel (used for the small matrices when
// they do not fit shared memory, and for the tall outputs).
struct GramLayout {
  int64_t ga, gb, m1, m2, m3, m4, vec, uo, vo, tm, total;
};

FRANK_HD GramLayout gram_layout(int bmax, int smax) {
  GramLayout L;
  int64_t o = 0;
  auto take = [&](int64_t n) { int64_t r = o; o += (n + 31) & ~int64_t(31); return r; };
  L.ga = take((int64_t)smax * smax);
  L.gb = take((int64_t)smax * smax);
  L.m1 = take((int64_t)smax * smax);
  L.m2 = take((int64_t)smax * smax);
  L.m3 = take((int64_t)smax * smax);
  L.m4 = take((int64_t)smax * smax);
  L.vec = take(16 * (int64_t)smax);
  L.uo = take((int64_t)bmax * smax);
  L.vo = take((int64_t)bmax * smax);
  L.tm = take((int64_t)bmax * bmax);
  L.total = o;
  return L;
}

template <typename T>
__global__ void __launch_bounds__(GRAM_THREADS) k_recompress_gram(BlrView<T> A, FactorWs<T> ws, int i, int smax,
                                                                  double core_scale, double gram_tol, int* counter) {
  extern __shared__ double region[];
  __shared__ double gsm[2 * 16 * 64];
  __shared__ double red[32];
  __shared__ int s_redi[32];
  __shared__ int s_r[3];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int m = A.nb - i - 1;
  const int ld = A.bmax;
  const int bi = A.bs(i);
  const GramLayout L = gram_layout(A.bmax, smax);
  double* base = ws.rscratch + (int64_t)blockIdx.x * ws.rscratch_stride;
  __shared__ int s_task;
  const int ntask = m * (m - 1);
  for (int tsk = next_task(counter, &s_task); tsk < ntask; tsk = next_task(counter, &s_task)) {
    int a_, c_;
    band_task(m, tsk, a_, c_);
    const int ic = i + 1 + a_, k = i + 1 + c_;
    if (!A.is_lr(ic, k) || !A.is_lr(ic, i) || !A.is_lr(i, k)) continue;
    const int blk = ic * A.nb + k;
    const int bc = A.bs(ic), bk = A.bs(k);
    const int kc = A.rank[blk];
    const int p = A.rank[ic * A.nb + i], q = A.rank[i * A.nb + k];
    const int su = kc + p, sv = kc + q;
    if (su > smax || sv > smax) {
      if (threadIdx.x == 0) atomicAdd(ws.err + ERR_BOUNDS, 1);
      continue;
    }
    const T* Uc = A.u(ic, k);
    const T* Sc = A.s(ic, k);
    const T* Vc = A.vt(ic, k);
    const T* UL = A.u(ic, i);
    const T* VU = A.vt(i, k);
    const T* WL = ws.WL + (int64_t)ic * ld * ld;
    const T* WU = ws.WU + (int64_t)k * ld * ld;
    const int sm_ = su > sv ? su : sv;
    // small matrices: Ga (su^2), Gb (sv^2), M1, M2 (su*sv), M3, M4 (sv*sv), vec;
    // all in shared memory when they fit (then also the V-side temporaries)
    const int64_t sq = (int64_t)sm_ * sm_;
    const int64_t need = 6 * sq + 16 * (int64_t)sm_;
    const bool in_sm = need <= GRAM_REGION;
    double *Ga, *Gb, *M1, *M2, *M3, *M4, *vec;
    if (in_sm) {
      Ga = region; Gb = Ga + sq; M1 = Gb + sq; M2 = M1 + sq; M3 = M2 + sq; M4 = M3 + sq; vec = M4 + sq;
    } else {
      Ga = base + L.ga; Gb = base + L.gb; M1 = base + L.m1; M2 = base + L.m2; M3 = base + L.m3; M4 = base + L.m4;
      vec = base + L.vec;
    }
    int* pa = reinterpret_cast<int*>(vec);
    int* pb = pa + sm_;
    int* jp = pb + sm_;
    int* ji = jp + sm_;
    double* tc = vec + 2 * (int64_t)sm_;
    double* cn = tc + sm_;
    double* pn = cn + sm_;
    double* tc2 = pn + sm_;
    double* Tm = base + L.tm;
    double* Uo = base + L.uo;
    double* Vo = base + L.vo;
    // small targets: warp-level factorizations in shared memory; large ones:
    // CTA-level factorizations
    const bool small = in_sm && su <= 64 && sv <= 64;
    const int cls = small ? 0 : 1;
    PHASE_BEGIN();
#ifdef FRANK_PHASE_TIMING
    if (threadIdx.x == 0) atomicAdd(&g_phase_count[cls], 1ull);
#endif
    // T = -WL^T WU (p x q); Gram matrices of the stacked bases (upper blocks)
    // skinny products: warp dot products when small, tiled GEMM otherwise
    auto tn = [&](int mm_, int nn_, int kk_, double al, const T* Ap, const T* Bp, double* Cp, int ldc_) {
      if ((int64_t)mm_ * nn_ <= 1024) cta_gemm_tn_dot(mm_, nn_, kk_, al, Ap, ld, Bp, ld, Cp, ldc_);
      else cta_gemm<double, GRAM_THREADS>(mm_, nn_, kk_, al, Ap, ld, true, Bp, ld, false, 0.0, Cp, ldc_, gsm);
    };
    tn(p, q, bi, -1.0, WL, WU, Tm, p);
    tn(kc, kc, bc, 1.0, Uc, Uc, Ga, su);
    tn(kc, p, bc, 1.0, Uc, UL, Ga + (int64_t)kc * su, su);
    tn(p, p, bc, 1.0, UL, UL, Ga + kc + (int64_t)kc * su, su);
    tn(kc, kc, bk, 1.0, Vc, Vc, Gb, sv);
    tn(kc, q, bk, 1.0, Vc, VU, Gb + (int64_t)kc * sv, sv);
    tn(q, q, bk, 1.0, VU, VU, Gb + kc + (int64_t)kc * sv, sv);
    for (int e = threadIdx.x; e < kc * p; e += blockDim.x) {
      const int r = e % kc, c = e / kc;
      Ga[(kc + c) + (int64_t)r * su] = Ga[r + (int64_t)(kc + c) * su];
    }
    for (int e = threadIdx.x; e < kc * q; e += blockDim.x) {
      const int r = e % kc, c = e / kc;
      Gb[(kc + c) + (int64_t)r * sv] = Gb[r + (int64_t)(kc + c) * sv];
    }
    __syncthreads();
    PHASE_MARK(cls, 0);
    // pivoted Cholesky of both Gram matrices (one warp each when small)
    if (small) {
      if (wid == 0) {
        const int r_ = warp_pivoted_cholesky(su, Ga, su, pa, gram_tol, su);
        if (lane == 0) s_r[0] = r_;
      } else if (wid == 1) {
        const int r_ = warp_pivoted_cholesky(sv, Gb, sv, pb, gram_tol, sv);
        if (lane == 0) s_r[1] = r_;
      }
    } else {
      const int r0 = cta_pivoted_cholesky(su, Ga, su, pa, gram_tol, su, red, s_redi);
      const int r1 = cta_pivoted_cholesky(sv, Gb, sv, pb, gram_tol, sv, red, s_redi);
      if (threadIdx.x == 0) { s_r[0] = r0; s_r[1] = r1; }
    }
    __syncthreads();
    PHASE_MARK(cls, 1);
    const int ra = s_r[0], rb = s_r[1];
    // M1 = Pa^T blockdiag(S_C, T) Pb (su x sv); zero the lower parts of Ra, Rb
    for (int64_t e = threadIdx.x; e < (int64_t)su * sv; e += blockDim.x) {
      const int r = e % su, c = e / su;
      const int orr = pa[r], occ = pb[c];
      double v = 0.0;
      if (orr < kc && occ < kc) v = double(Sc[orr + (int64_t)occ * A.kcap]);
      else if (orr >= kc && occ >= kc) v = Tm[(orr - kc) + (int64_t)(occ - kc) * p];
      M1[e] = v;
    }
    for (int64_t e = threadIdx.x; e < (int64_t)ra * su; e += blockDim.x) {
      const int r = e % ra, c = e / ra;
      if (r > c) Ga[r + (int64_t)c * su] = 0.0;
    }
    for (int64_t e = threadIdx.x; e < (int64_t)rb * sv; e += blockDim.x) {
      const int r = e % rb, c = e / rb;
      if (r > c) Gb[r + (int64_t)c * sv] = 0.0;
    }
    __syncthreads();
    // M2 (ra x sv) = Ra M1 ; Core = M1 <- M2 Rb^T (ra x rb)
    for (int64_t e = threadIdx.x; e < (int64_t)ra * sv; e += blockDim.x) {
      const int r = e % ra, c = e / ra;
      double acc = 0.0;
      for (int t = r; t < su; ++t) acc += Ga[r + (int64_t)t * su] * M1[t + (int64_t)c * su];
      M2[e] = acc;
    }
    __syncthreads();
    double* Core = M1;  // ra x rb, ld ra
    for (int64_t e = threadIdx.x; e < (int64_t)ra * rb; e += blockDim.x) {
      const int r = e % ra, c = e / ra;
      double acc = 0.0;
      for (int t = c; t < sv; ++t) acc += M2[r + (int64_t)t * ra] * Gb[c + (int64_t)t * sv];
      Core[e] = acc;
    }
    double f = 0.0;
    __syncthreads();
    for (int64_t e = threadIdx.x; e < (int64_t)ra * rb; e += blockDim.x) f += Core[e] * Core[e];
    f = block_sum(f, red);
    const double thr = ws.fixed_rank > 0 ? 0.0 : core_scale * ws.eps * sqrt(f);
    const int maxr = ws.fixed_rank > 0 ? min(ws.fixed_rank, A.kcap) : A.kcap;
    PHASE_MARK(cls, 2);
    if (small) {
      if (wid == 0) {
        const int r_ = (ra > 0 && rb > 0) ? warp_truncated_geqp3(ra, rb, Core, ra, thr, maxr, tc, cn, pn, jp) : 0;
        if (lane == 0) s_r[2] = r_;
      }
    } else {
      const int r_ = (ra > 0 && rb > 0) ? cta_truncated_geqp3(ra, rb, Core, ra, thr, maxr, tc, cn, pn, jp, red, s_redi)
                                        : 0;
      if (threadIdx.x == 0) s_r[2] = r_;
    }
    __syncthreads();
    PHASE_MARK(cls, 3);
    const int r = s_r[2];
    if (r == 0) {
      T* Uw = A.u(ic, k); T* Vw = A.vt(ic, k); T* Sw = A.s(ic, k);
      for (int e = threadIdx.x; e < bc; e += blockDim.x) Uw[e] = T(e == 0 ? 1.0 : 0.0);
      for (int e = threadIdx.x; e < bk; e += blockDim.x) Vw[e] = T(e == 0 ? 1.0 : 0.0);
      if (threadIdx.x == 0) { Sw[0] = T(0); A.rank[blk] = 1; atomicAdd(ws.err + ERR_RECOMP, 1); }
      __syncthreads();
      continue;
    }
    if (threadIdx.x == 0) {
      if (ws.fixed_rank == 0 && r >= A.kcap && r < min(ra, rb)) atomicAdd(ws.err + ERR_RANK_OVERFLOW, 1);
      atomicMax(ws.err + ERR_MAX_RANK, r);
      atomicAdd(ws.err + ERR_RECOMP, 1);
      atomicAdd(ws.flops + FLOP_RECOMP, (unsigned long long)rounded_addition_flops(bc, bk, bi, kc, p, q, r));
    }
    double* X1 = M2;   // ra x r (M2 no longer needed)
    double* X2 = M3;   // rb x r
    double* Qt = M4;   // rb x r
    double* Yk = M4;   // Qt with its columns reversed in place
    T* Sw = A.s(ic, k);
    if (small) {
      if (wid == 0) {
        // X1 = Ra11^{-1} Q_core
        for (int e = lane; e < ra * r; e += 32) X1[e] = ((e % ra) == (e / ra)) ? 1.0 : 0.0;
        __syncwarp();
        warp_apply_q(ra, r, Core, ra, tc, r, X1, ra);
        warp_upper_solve(ra, Ga, su, r, X1, ra);
      } else if (wid == 1) {
        // RQ of the kept rows R_core Pcore^T (r x rb): QR of X2 = (R_perm)^T J
        for (int c = lane; c < rb; c += 32) ji[jp[c]] = c;
        __syncwarp();
        for (int e = lane; e < rb * r; e += 32) {
          const int c = e % rb, a = e / rb;
          const int row = r - 1 - a, src = ji[c];
          X2[e] = (row <= src) ? Core[row + (int64_t)src * ra] : 0.0;
        }
        __syncwarp();
        warp_householder_qr(rb, r, X2, rb, tc2);
        for (int e = lane; e < r * r; e += 32) {
          const int a = e % r, c = e / r;
          const int ra_ = r - 1 - c, ca = r - 1 - a;
          Sw[a + (int64_t)c * A.kcap] = T((ra_ <= ca) ? X2[ra_ + (int64_t)ca * rb] : 0.0);
        }
        for (int e = lane; e < rb * r; e += 32) Qt[e] = ((e % rb) == (e / rb)) ? 1.0 : 0.0;
        __syncwarp();
        warp_apply_q(rb, r, X2, rb, tc2, r, Qt, rb);
        for (int e = lane; e < rb * (r / 2); e += 32) {
          const int rr = e % rb, a = e / rb;
          const double t0 = Qt[rr + (int64_t)a * rb];
          Qt[rr + (int64_t)a * rb] = Qt[rr + (int64_t)(r - 1 - a) * rb];
          Qt[rr + (int64_t)(r - 1 - a) * rb] = t0;
        }
        __syncwarp();
        warp_upper_solve(rb, Gb, sv, r, Yk, rb);
      }
      __syncthreads();
    } else {
      for (int64_t e = threadIdx.x; e < (int64_t)ra * r; e += blockDim.x) X1[e] = ((e % ra) == (e / ra)) ? 1.0 : 0.0;
      for (int c = threadIdx.x; c < rb; c += blockDim.x) ji[jp[c]] = c;
      __syncthreads();
      cta_apply_q(ra, r, Core, ra, tc, r, X1, (int64_t)ra);
      for (int64_t e = threadIdx.x; e < (int64_t)rb * r; e += blockDim.x) {
        const int c = e % rb, a = e / rb;
        const int row = r - 1 - a, src = ji[c];
        X2[e] = (row <= src) ? Core[row + (int64_t)src * ra] : 0.0;
      }
      __syncthreads();
      cta_householder_qr(rb, r, X2, rb, tc2, red);
      for (int64_t e = threadIdx.x; e < (int64_t)r * r; e += blockDim.x) {
        const int a = e % r, c = e / r;
        const int ra_ = r - 1 - c, ca = r - 1 - a;
        Sw[a + (int64_t)c * A.kcap] = T((ra_ <= ca) ? X2[ra_ + (int64_t)ca * rb] : 0.0);
      }
      for (int64_t e = threadIdx.x; e < (int64_t)rb * r; e += blockDim.x) Qt[e] = ((e % rb) == (e / rb)) ? 1.0 : 0.0;
      __syncthreads();
      cta_apply_q(rb, r, X2, rb, tc2, r, Qt, (int64_t)rb);
      for (int64_t e = threadIdx.x; e < (int64_t)rb * (r / 2); e += blockDim.x) {
        const int rr = e % rb, a = e / rb;
        const double t0 = Qt[rr + (int64_t)a * rb];
        Qt[rr + (int64_t)a * rb] = Qt[rr + (int64_t)(r - 1 - a) * rb];
        Qt[rr + (int64_t)(r - 1 - a) * rb] = t0;
      }
      __syncthreads();
      cta_upper_solve(ra, Ga, su, r, X1, ra);
      cta_upper_solve(rb, Gb, sv, r, Yk, rb);
    }
    PHASE_MARK(cls, 4);
    // scatter to the stacked order: Xf (su x r) reuses M1, Yf (sv x r) M3
    double* Xf = M1;
    double* Yf = M3;
    for (int64_t e = threadIdx.x; e < (int64_t)su * r; e += blockDim.x) Xf[e] = 0.0;
    __syncthreads();
    for (int64_t e = threadIdx.x; e < (int64_t)ra * r; e += blockDim.x) {
      const int rr = e % ra, c = e / ra;
      Xf[pa[rr] + (int64_t)c * su] = X1[e];
    }
    for (int64_t e = threadIdx.x; e < (int64_t)sv * r; e += blockDim.x) Yf[e] = 0.0;
    __syncthreads();
    for (int64_t e = threadIdx.x; e < (int64_t)rb * r; e += blockDim.x) {
      const int rr = e % rb, c = e / rb;
      Yf[pb[rr] + (int64_t)c * sv] = Yk[e];
    }
    __syncthreads();
    // new bases into temporaries (the target's own U, Vt are operands):
    // U = Uc Xf[:kc] + UL Xf[kc:], V^T = Vc Yf[:kc] + VU Yf[kc:]
    if (r <= 16) {
      cta_gemm_tall(bc, r, kc, Uc, ld, Xf, su, Uo, bc, false);
      cta_gemm_tall(bc, r, p, UL, ld, Xf + kc, su, Uo, bc, true);
      cta_gemm_tall(bk, r, kc, Vc, ld, Yf, sv, Tm, bk, false);
      cta_gemm_tall(bk, r, q, VU, ld, Yf + kc, sv, Tm, bk, true);
    } else {
      cta_gemm<double, GRAM_THREADS>(bc, r, kc, 1.0, Uc, ld, false, Xf, su, false, 0.0, Uo, bc, gsm);
      cta_gemm<double, GRAM_THREADS>(bc, r, p, 1.0, UL, ld, false, Xf + kc, su, false, 1.0, Uo, bc, gsm);
      cta_gemm<double, GRAM_THREADS>(bk, r, kc, 1.0, Vc, ld, false, Yf, sv, false, 0.0, Tm, bk, gsm);
      cta_gemm<double, GRAM_THREADS>(bk, r, q, 1.0, VU, ld, false, Yf + kc, sv, false, 1.0, Tm, bk, gsm);
    }
    T* Uw = A.u(ic, k);
    T* Vw = A.vt(ic, k);
    for (int64_t e = threadIdx.x; e < (int64_t)bc * r; e += blockDim.x) {
      const int rr = e % bc, c = e / bc;
      Uw[rr + (int64_t)c * ld] = T(Uo[e]);
    }
    for (int64_t e = threadIdx.x; e < (int64_t)bk * r; e += blockDim.x) {
      const int rr = e % bk, c = e / bk;
      Vw[rr + (int64_t)c * ld] = T(Tm[e]);
    }
    PHASE_MARK(cls, 5);
    if (threadIdx.x == 0) A.rank[blk] = r;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Solve kernels.  z is the n x nrhs right-hand side / solution (T, ld n).
// Forward (trsm(L, b, Lower), trsm.cpp:163-174 for a block column B):
//   y_i = Linv_i P_i z_i ; z_j -= L(j,i) y_i for j > i.
// Backward (trsm(U, b, Upper), trsm.cpp:136-145):
//   x_i = Uinv_i z_i ; z_j -= U(j,i) x_i for j < i.
// ---------------------------------------------------------------------------
constexpr int SOLVE_THREADS = 256;
constexpr int SOLVE_ROWS = 16;   // rows of the diagonal solve per CTA (16 inner-index slices each)

// y = M * P(z_i) (which 0: Linv, permuted input; 1: Uinv),
// y = M^T z_i (2: Uinv^T), or y = P^T (Linv^T z_i) (3), into ybuf (ld bmax).
// grid = ceil(b / SOLVE_ROWS) CTAs; each stages the whole input block in
// shared memory (b x nrhs doubles) and produces SOLVE_ROWS rows.
template <typename T>
__global__ void __launch_bounds__(SOLVE_THREADS) k_solve_diag(BlrView<T> A, FactorWs<T> ws, int i, const T* z,
                                                              int64_t ldz, int nrhs, int which, T* ybuf) {
  extern __shared__ double xs[];          // b x nrhs input, then the slices' partial sums
  const int b = A.bs(i), ld = A.bmax;
  const int64_t o = A.off[i];
  const T* Mx = (which == 0 || which == 3) ? ws.Linv + (int64_t)i * ld * ld : ws.Uinv + (int64_t)i * ld * ld;
  const int* perm = ws.perm + (int64_t)i * ld;
  for (int e = threadIdx.x; e < b * nrhs; e += blockDim.x) {
    const int r = e % b, c = e / b;
    xs[e] = double(z[o + (which == 0 ? perm[r] : r) + (int64_t)c * ldz]);
  }
  __syncthreads();
  const int r0 = blockIdx.x * SOLVE_ROWS;
  const int nr = min(SOLVE_ROWS, b - r0);
  if (which <= 1) {
    // rows r0.. of M x: thread (rl, sl) sums the inner slice sl of row rl
    double* part = xs + (int64_t)b * nrhs;
    const int rl = threadIdx.x % SOLVE_ROWS, sl = threadIdx.x / SOLVE_ROWS;  // SOLVE_THREADS / SOLVE_ROWS slices
    const int nsl = SOLVE_THREADS / SOLVE_ROWS;
    const int tlen = (b + nsl - 1) / nsl;
    const int t0 = sl * tlen, t1 = min(b, t0 + tlen);
    double acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = 0.0;
    if (rl < nr) {
      const T* mrow = Mx + r0 + rl;
#pragma unroll 4
      for (int t = t0; t < t1; ++t) {
        const double mv = double(mrow[(int64_t)t * ld]);
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < nrhs) acc[c] += mv * xs[t + c * b];
      }
    }
    #pragma unroll
    for (int c = 0; c < 8; ++c) if (c < nrhs) part[(sl * SOLVE_ROWS + rl) * 8 + c] = acc[c];
    __syncthreads();
    for (int e = threadIdx.x; e < nr * nrhs; e += blockDim.x) {
      const int r = e % nr, c = e / nr;
      double s = 0.0;
      for (int q = 0; q < nsl; ++q) s += part[(q * SOLVE_ROWS + r) * 8 + c];
      ybuf[r0 + r + (int64_t)c * ld] = T(s);
    }
  } else {
    // rows r0.. of M^T x: a warp per output row reads column r of M
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int rl = wid; rl < nr; rl += nw) {
      const int r = r0 + rl;
      const T* mcol = Mx + (int64_t)r * ld;
      double acc[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[c] = 0.0;
#pragma unroll 4
      for (int t = lane; t < b; t += 32) {
        const double mv = double(mcol[t]);
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < nrhs) acc[c] += mv * xs[t + c * b];
      }
      #pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c >= nrhs) break;
        const double sum = warp_sum(acc[c]);
        if (lane == 0) ybuf[(which == 3 ? perm[r] : r) + (int64_t)c * ld] = T(sum);
      }
    }
  }
}

// z_j -= Blk y_i for every target j of step i, with the solved block y_i in
// ybuf, then z_i = y_i:
// mode 0: targets j > i using blocks (j, i)        [forward, L]
// mode 1: targets j < i using blocks (j, i)        [backward, U]
// mode 2: targets j > i using blocks (i, j)^T      [transpose forward, U^T]
// mode 3: targets j < i using blocks (i, j)^T      [transpose backward, L^T]
// One thread-block cluster of SC_CLUSTER CTAs per target j (grid =
// max(ntarget, 1) clusters; the first cluster also copies y_i into z_i).  For a low-rank block U S V^T the cluster's CTAs split the
// work three ways and exchange the pieces through distributed shared memory:
//   A: CTA q contracts columns [q cw, (q+1) cw) of the inner basis with y_i
//      (t1 = inner^T y, one warp per column);
//   B: after a cluster barrier every CTA gathers all of t1, then CTA q forms
//      rows [q cw, (q+1) cw) of t2 = S t1 (S^T t1 when transposing);
//   C: after a second barrier every CTA gathers all of t2 and updates its
//      row tile z_j(tile) -= outer(tile, :) t2.
// A third barrier keeps every CTA's shared memory alive until the gathers of
// the others are done.  A dense block is applied tile by tile in phase C.
// Every CTA reaches the three barriers.
constexpr int SC_CLUSTER = 8;
constexpr int SMEM_OPTIN_MAX = 227 * 1024;   // dynamic shared memory a CTA may opt into

// Rows of t2 per CTA at most (the stride of the phase-B partial sums).
FRANK_HD int solve_cl_rows(int kcap) { return (kcap + SC_CLUSTER - 1) / SC_CLUSTER; }

// Doubles of the partial-sum area: phase B (SOLVE_THREADS / 32 warps x
// solve_cl_rows x 8) and phase C (SOLVE_THREADS / 64 splits x 64 rows x 8).
FRANK_HD int64_t solve_cl_part(int kcap) {
  const int64_t b = (int64_t)(SOLVE_THREADS / 32) * solve_cl_rows(kcap) * 8, c = (int64_t)(SOLVE_THREADS / 64) * 64 * 8;
  return b > c ? b : c;
}

// dynamic shared memory: ys (bmax x nrhs), t1, t2 (kcap x nrhs each) and the
// partial sums
FRANK_HD size_t solve_scatter_cl_smem(int bmax, int kcap, int nrhs) {
  return ((size_t)bmax * nrhs + 2 * (size_t)kcap * nrhs + (size_t)solve_cl_part(kcap)) * sizeof(double);
}

template <typename T>
__global__ void __cluster_dims__(SC_CLUSTER, 1, 1) __launch_bounds__(SOLVE_THREADS)
    k_solve_scatter_cl(BlrView<T> A, int i, T* z, int64_t ldz, int nrhs, int mode, const T* ybuf, int ntarget) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ double csm[];
  const int ld = A.bmax;
  const int bi = A.bs(i);
  const int64_t oi = A.off[i];
  const int q = (int)cl.block_rank();
  const int t = blockIdx.x / SC_CLUSTER;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double* ys = csm;
  double* t1 = ys + (int64_t)A.bmax * nrhs;
  double* t2 = t1 + (int64_t)A.kcap * nrhs;
  double* part = t2 + (int64_t)A.kcap * nrhs;   // partial sums (solve_cl_part doubles)
  const int pstride = solve_cl_rows(A.kcap);
  // y_i -> z_i, one row tile per CTA of the first cluster
  if (t == 0) {
    const int tl = (bi + SC_CLUSTER - 1) / SC_CLUSTER, r0 = q * tl, r1 = min(bi, r0 + tl);
    for (int e = threadIdx.x; e < (r1 - r0) * nrhs; e += blockDim.x) {
      const int r = r0 + e % (r1 - r0), c = e / (r1 - r0);
      z[oi + r + (int64_t)c * ldz] = ybuf[r + (int64_t)c * ld];
    }
  }
  const bool active = t < ntarget;
  const bool tr = (mode >= 2);
  int j = 0, bj = 0, r = 0, bi_ = 0, bj_ = 0;
  bool lr = false;
  if (active) {
    j = (mode == 0 || mode == 2) ? i + 1 + t : t;
    bj = A.bs(j);
    bi_ = tr ? i : j;
    bj_ = tr ? j : i;
    lr = A.is_lr(bi_, bj_);
    r = lr ? A.rank[bi_ * A.nb + bj_] : 0;
  }
  const int cw = (r + SC_CLUSTER - 1) / SC_CLUSTER;   // columns of t1 / rows of t2 per CTA
  const int c0 = min(r, q * cw), c1 = min(r, c0 + cw);
  if (active) {
    for (int e = threadIdx.x; e < bi * nrhs; e += blockDim.x) {
      const int rr = e % bi, c = e / bi;
      ys[e] = double(ybuf[rr + (int64_t)c * ld]);
    }
  }
  __syncthreads();
  // A: t1(c0:c1, :) = inner(:, c0:c1)^T y
  const T* U = lr ? A.u(bi_, bj_) : nullptr;
  const T* S = lr ? A.s(bi_, bj_) : nullptr;
  const T* V = lr ? A.vt(bi_, bj_) : nullptr;
  const T* inner = tr ? U : V;
  const T* outer = tr ? V : U;
  if (lr) {
    for (int cc = c0 + wid; cc < c1; cc += nw) {
      const T* col = inner + (int64_t)cc * ld;
      double acc[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[c] = 0.0;
#pragma unroll 4
      for (int x = lane; x < bi; x += 32) {
        const double v = double(col[x]);
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < nrhs) acc[c] += v * ys[x + c * bi];
      }
      #pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c >= nrhs) break;
        const double sum = warp_sum(acc[c]);
        if (lane == 0) t1[cc + c * r] = sum;
      }
    }
  }
  cl.sync();
  // B: gather t1, then t2(c0:c1, :) = S(c0:c1, :) t1 (warps split the inner index)
  if (lr) {
    for (int qq = 0; qq < SC_CLUSTER; ++qq) {
      if (qq == q) continue;
      const int a0 = min(r, qq * cw), a1 = min(r, a0 + cw);
      const double* rt1 = cl.map_shared_rank(t1, qq);
      for (int e = threadIdx.x; e < (a1 - a0) * nrhs; e += blockDim.x) {
        const int c = a0 + e % (a1 - a0), h = e / (a1 - a0);
        t1[c + h * r] = rt1[c + h * r];
      }
    }
    __syncthreads();
    const int tw = (r + nw - 1) / nw, x0 = min(r, wid * tw), x1 = min(r, x0 + tw);
    for (int cb = c0; cb < c1; cb += 32) {
      const int c = cb + lane;
      double acc[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) acc[h] = 0.0;
      if (c < c1) {
#pragma unroll 4
        for (int x = x0; x < x1; ++x) {
          const double sv = tr ? double(S[x + (int64_t)c * A.kcap]) : double(S[c + (int64_t)x * A.kcap]);
#pragma unroll
          for (int h = 0; h < 8; ++h)
            if (h < nrhs) acc[h] += sv * t1[x + h * r];
        }
      }
      if (c < c1)
        #pragma unroll
        for (int h = 0; h < 8; ++h) if (h < nrhs) part[((int64_t)wid * pstride + (c - c0)) * 8 + h] = acc[h];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < (c1 - c0) * nrhs; e += blockDim.x) {
      const int cl_ = e % (c1 - c0), h = e / (c1 - c0);
      double sum = 0.0;
      for (int w = 0; w < nw; ++w) sum += part[((int64_t)w * pstride + cl_) * 8 + h];
      t2[c0 + cl_ + h * r] = sum;
    }
  }
  cl.sync();
  // C: gather t2, then the row tile of the target
  if (lr) {
    for (int qq = 0; qq < SC_CLUSTER; ++qq) {
      if (qq == q) continue;
      const int a0 = min(r, qq * cw), a1 = min(r, a0 + cw);
      const double* rt2 = cl.map_shared_rank(t2, qq);
      for (int e = threadIdx.x; e < (a1 - a0) * nrhs; e += blockDim.x) {
        const int c = a0 + e % (a1 - a0), h = e / (a1 - a0);
        t2[c + h * r] = rt2[c + h * r];
      }
    }
  }
  cl.sync();
  if (!active) return;
  const int64_t oj = A.off[j];
  const int tl = (bj + SC_CLUSTER - 1) / SC_CLUSTER, row0 = q * tl, row1 = min(bj, row0 + tl);
  if (lr) {
    // 64 rows x (SOLVE_THREADS / 64) splits of the inner index per pass
    const int ns = SOLVE_THREADS / 64, rl = threadIdx.x % 64, sl = threadIdx.x / 64;
    const int xw = (r + ns - 1) / ns, x0 = min(r, sl * xw), x1 = min(r, x0 + xw);
    for (int rb = row0; rb < row1; rb += 64) {
      const int rr = rb + rl;
      double acc[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) acc[h] = 0.0;
      if (rr < row1) {
#pragma unroll 4
        for (int x = x0; x < x1; ++x) {
          const double ov = double(outer[rr + (int64_t)x * ld]);
#pragma unroll
          for (int h = 0; h < 8; ++h)
            if (h < nrhs) acc[h] += ov * t2[x + h * r];
        }
      }
      __syncthreads();
      #pragma unroll
      for (int h = 0; h < 8; ++h) if (h < nrhs) part[((int64_t)sl * 64 + rl) * 8 + h] = acc[h];
      __syncthreads();
      for (int e = threadIdx.x; e < 64 * nrhs; e += blockDim.x) {
        const int rl2 = e % 64, h = e / 64, row = rb + rl2;
        if (row < row1) {
          double sum = 0.0;
          for (int w = 0; w < ns; ++w) sum += part[((int64_t)w * 64 + rl2) * 8 + h];
          z[oj + row + (int64_t)h * ldz] = T(double(z[oj + row + (int64_t)h * ldz]) - sum);
        }
      }
    }
  } else {
    const T* Dm = A.dense(bi_, bj_);
    if (!tr) {
      for (int rr = row0 + threadIdx.x; rr < row1; rr += blockDim.x) {
        double acc[8];
#pragma unroll
        for (int h = 0; h < 8; ++h) acc[h] = 0.0;
#pragma unroll 4
        for (int x = 0; x < bi; ++x) {
          const double dv = double(Dm[rr + (int64_t)x * ld]);
#pragma unroll
          for (int h = 0; h < 8; ++h)
            if (h < nrhs) acc[h] += dv * ys[x + h * bi];
        }
        #pragma unroll
        for (int h = 0; h < 8; ++h) if (h < nrhs) z[oj + rr + (int64_t)h * ldz] = T(double(z[oj + rr + (int64_t)h * ldz]) - acc[h]);
      }
    } else {
      for (int rr = row0 + wid; rr < row1; rr += nw) {
        double acc[8];
#pragma unroll
        for (int h = 0; h < 8; ++h) acc[h] = 0.0;
        for (int x = lane; x < bi; x += 32) {
          const double dv = double(Dm[x + (int64_t)rr * ld]);
#pragma unroll
          for (int h = 0; h < 8; ++h)
            if (h < nrhs) acc[h] += dv * ys[x + h * bi];
        }
        #pragma unroll
        for (int h = 0; h < 8; ++h) {
          if (h >= nrhs) break;
          const double sum = warp_sum(acc[h]);
          if (lane == 0) z[oj + rr + (int64_t)h * ldz] = T(double(z[oj + rr + (int64_t)h * ldz]) - sum);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// K6: FP64 H-matvec partials: part[(i*nb + j)] = A(i,j) x_j  (bmax x nrhs each)
// grid (nb, nb); then k_matvec_reduce sums over j in fixed order.
// ---------------------------------------------------------------------------
constexpr int MV_THREADS = 256;

// dynamic shared memory of k_matvec_blocks: x_j (bmax x nrhs), t1, t2 (kcap x nrhs)
FRANK_HD size_t matvec_smem(int bmax, int kcap, int nrhs) {
  return ((size_t)bmax * nrhs + 2 * (size_t)kcap * nrhs) * sizeof(double);
}

// Each element of the block (U, S, V or the dense block) is read once and
// applied to all nrhs columns of x_j, which is staged in shared memory.
__global__ void __launch_bounds__(MV_THREADS) k_matvec_blocks(BlrView<double> H, const double* x, int64_t ldx,
                                                              int nrhs, double* part, int transpose) {
  // part(i, j) = A(i, j) x_j, or A(j, i)^T x_j when transposing
  const int i = blockIdx.y, j = blockIdx.x;
  const int nb = H.nb, ld = H.bmax;
  const int bi = H.bs(i), bj = H.bs(j);
  const int64_t oj = H.off[j];
  const int gi = transpose ? j : i, gj = transpose ? i : j;   // stored block (gi, gj)
  double* out = part + (int64_t)(i * nb + j) * ld * nrhs;
  extern __shared__ double msm[];
  double* xs = msm;                                  // bj x nrhs
  double* t1 = xs + (int64_t)H.bmax * nrhs;          // r x nrhs
  double* t2 = t1 + (int64_t)H.kcap * nrhs;          // r x nrhs
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int e = threadIdx.x; e < bj * nrhs; e += blockDim.x) {
    const int t = e % bj, h = e / bj;
    xs[e] = x[oj + t + (int64_t)h * ldx];
  }
  __syncthreads();
  if (H.is_lr(gi, gj)) {
    const int r = H.rank[gi * nb + gj];
    const double* U = H.u(gi, gj);
    const double* S = H.s(gi, gj);
    const double* V = H.vt(gi, gj);
    const double* inner = transpose ? U : V;   // length bj (rows of x_j)
    const double* outer = transpose ? V : U;   // length bi
    for (int c = wid; c < r; c += nw) {
      const double* col = inner + (int64_t)c * ld;
      double acc[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) acc[h] = 0.0;
#pragma unroll 4
      for (int t = lane; t < bj; t += 32) {
        const double v = col[t];
#pragma unroll
        for (int h = 0; h < 8; ++h)
          if (h < nrhs) acc[h] += v * xs[t + h * bj];
      }
      #pragma unroll
      for (int h = 0; h < 8; ++h) {
        if (h >= nrhs) break;
        const double sum = warp_sum(acc[h]);
        if (lane == 0) t1[c + h * r] = sum;
      }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < r; c += blockDim.x) {
      double acc[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) acc[h] = 0.0;
#pragma unroll 4
      for (int t = 0; t < r; ++t) {
        const double sv = transpose ? S[t + (int64_t)c * H.kcap] : S[c + (int64_t)t * H.kcap];
#pragma unroll
        for (int h = 0; h < 8; ++h)
          if (h < nrhs) acc[h] += sv * t1[t + h * r];
      }
      #pragma unroll
      for (int h = 0; h < 8; ++h) if (h < nrhs) t2[c + h * r] = acc[h];
    }
    __syncthreads();
    for (int rr = threadIdx.x; rr < bi; rr += blockDim.x) {
      double acc[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) acc[h] = 0.0;
#pragma unroll 4
      for (int t = 0; t < r; ++t) {
        const double ov = outer[rr + (int64_t)t * ld];
#pragma unroll
        for (int h = 0; h < 8; ++h)
          if (h < nrhs) acc[h] += ov * t2[t + h * r];
      }
      #pragma unroll
      for (int h = 0; h < 8; ++h) if (h < nrhs) out[rr + (int64_t)h * ld] = acc[h];
    }
  } else {
    const double* Dm = H.dense(gi, gj);
    if (!transpose) {
      for (int rr = threadIdx.x; rr < bi; rr += blockDim.x) {
        double acc[8];
#pragma unroll
        for (int h = 0; h < 8; ++h) acc[h] = 0.0;
#pragma unroll 4
        for (int t = 0; t < bj; ++t) {
          const double dv = Dm[rr + (int64_t)t * ld];
#pragma unroll
          for (int h = 0; h < 8; ++h)
            if (h < nrhs) acc[h] += dv * xs[t + h * bj];
        }
        #pragma unroll
        for (int h = 0; h < 8; ++h) if (h < nrhs) out[rr + (int64_t)h * ld] = acc[h];
      }
    } else {
      for (int rr = wid; rr < bi; rr += nw) {
        double acc[8];
#pragma unroll
        for (int h = 0; h < 8; ++h) acc[h] = 0.0;
#pragma unroll 4
        for (int t = lane; t < bj; t += 32) {
          const double dv = Dm[t + (int64_t)rr * ld];
#pragma unroll
          for (int h = 0; h < 8; ++h)
            if (h < nrhs) acc[h] += dv * xs[t + h * bj];
        }
        #pragma unroll
        for (int h = 0; h < 8; ++h) {
          if (h >= nrhs) break;
          const double sum = warp_sum(acc[h]);
          if (lane == 0) out[rr + (int64_t)h * ld] = sum;
        }
      }
    }
  }
}

// y_i = sum_j part(i,j) (fixed order).  If b != null: y = b - A x (residual).
__global__ void k_matvec_reduce(BlrView<double> H, const double* part, int nrhs, const double* bvec, int64_t ldb,
                                double* y, int64_t ldy) {
  const int i = blockIdx.x;
  const int nb = H.nb, ld = H.bmax;
  const int bi = H.bs(i);
  const int64_t oi = H.off[i];
  for (int e = threadIdx.x; e < bi * nrhs; e += blockDim.x) {
    const int rr = e % bi, h = e / bi;
    double s = 0.0;
    for (int j = 0; j < nb; ++j) s += part[(int64_t)(i * nb + j) * ld * nrhs + rr + (int64_t)h * ld];
    if (bvec) s = bvec[oi + rr + (int64_t)h * ldb] - s;
    y[oi + rr + (int64_t)h * ldy] = s;
  }
}

// column 2-norms squared of an n x nrhs matrix: per-CTA partials part[blk*nrhs + h]
__global__ void k_colnorm2(const double* v, int64_t n, int64_t ldv, int nrhs, double* part) {
  __shared__ double red[32];
  for (int h = 0; h < nrhs; ++h) {
    double s = 0.0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
      const double a = v[r + h * ldv];
      s += a * a;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.x * nrhs + h] = s;
  }
}

template <typename TD, typename TS>
__global__ void k_cast_copy(const TS* src, int64_t lds, TD* dst, int64_t ldd, int64_t n, int nrhs) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % n, h = e / n;
    dst[r + h * ldd] = TD(src[r + h * lds]);
  }
}

// x += T(d)
// y0 = alpha * y + beta * y0 over n x nrhs (both ld n)
__global__ void k_axpby(double alpha, const double* y, double beta, double* y0, int64_t n, int nrhs) {
  const int64_t tot = n * nrhs;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x)
    y0[e] = alpha * y[e] + (beta == 0.0 ? 0.0 : beta * y0[e]);
}

template <typename TS>
__global__ void k_axpy_cast(const TS* d, int64_t ldd, double* x, int64_t ldx, int64_t n, int nrhs) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % n, h = e / n;
    x[r + h * ldx] += double(d[r + h * ldd]);
  }
}

// ---------------------------------------------------------------------------
// Adjoint contraction for the exponential kernel A_ij = exp(-r_ij/theta) +
// nugget*delta_ij: partial sums of sum_h sum_ij lambda_ih (dA_ij/dtheta) x_jh
// with dA/dtheta = exp(-r/theta) r / theta^2, evaluated on the fly (the
// kernel matrix is never formed).  64 x 64 tiles of point pairs per CTA,
// points and vectors staged in shared memory; one partial per CTA, summed on
// the host in a fixed order.
// ---------------------------------------------------------------------------
constexpr int DT_TILE = 64;

__global__ void __launch_bounds__(256) k_dtheta_contract(const double* x, int dim, int64_t n, double theta,
                                                          const double* lam, int64_t ldl, const double* xv,
                                                          int64_t ldx, int nrhs, double* partial) {
  __shared__ double pi[3][DT_TILE], pj[3][DT_TILE];
  __shared__ double li[8][DT_TILE], xj[8][DT_TILE];
  __shared__ double red[32];
  const int64_t i0 = (int64_t)blockIdx.y * DT_TILE, j0 = (int64_t)blockIdx.x * DT_TILE;
  for (int e = threadIdx.x; e < DT_TILE * dim; e += blockDim.x) {
    const int t = e % DT_TILE, d = e / DT_TILE;
    pi[d][t] = (i0 + t < n) ? x[d * n + i0 + t] : 0.0;
    pj[d][t] = (j0 + t < n) ? x[d * n + j0 + t] : 0.0;
  }
  for (int e = threadIdx.x; e < DT_TILE * nrhs; e += blockDim.x) {
    const int t = e % DT_TILE, h = e / DT_TILE;
    li[h][t] = (i0 + t < n) ? lam[i0 + t + h * ldl] : 0.0;
    xj[h][t] = (j0 + t < n) ? xv[j0 + t + h * ldx] : 0.0;
  }
  __syncthreads();
  double acc = 0.0;
  const double inv_t2 = 1.0 / (theta * theta);
  for (int e = threadIdx.x; e < DT_TILE * DT_TILE; e += blockDim.x) {
    const int a = e % DT_TILE, c = e / DT_TILE;
    if (i0 + a >= n || j0 + c >= n) continue;
    double r2 = 0.0;
    for (int d = 0; d < dim; ++d) { const double t = pi[d][a] - pj[d][c]; r2 += t * t; }
    const double r = sqrt(r2);
    const double da = exp(-r / theta) * r * inv_t2;
    double w = 0.0;
    for (int h = 0; h < nrhs; ++h) w += li[h][a] * xj[h][c];
    acc += da * w;
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = acc;
}

// ---------------------------------------------------------------------------
// Construction on the device (FP64): kernel evaluation and compression.
// ---------------------------------------------------------------------------
struct KernelDesc {
  int kind;
  int dim;
  const double* x;   // dim x n, axis-major
  int64_t n;
  double p0, p1;
};

FRANK_D double kernel_eval(const KernelDesc& K, int64_t gi, int64_t gj) {
  double r2 = 0.0;
  for (int d = 0; d < K.dim; ++d) {
    const double t = K.x[d * K.n + gi] - K.x[d * K.n + gj];
    r2 += t * t;
  }
  const double r = sqrt(r2);
  switch (K.kind) {
    case 0: return 1.0 / (r + 1e-3);                                   // functions.cpp:92-109
    case 1: return exp(-1.0 * r2) / (r + 1e-3);                        // functions.cpp:111-128
    case 2: return -log(r + 1e-3) + (gi == gj ? K.p0 : 0.0);
    default: return exp(-r / K.p0) + (gi == gj ? K.p1 : 0.0);
  }
}

// Dense blocks of A_H: one CTA per dense block (listed in blocks[]).
__global__ void k_build_dense(BlrView<double> H, KernelDesc K, const int* blocks, int nblocks) {
  for (int t = blockIdx.x; t < nblocks; t += gridDim.x) {
    const int blk = blocks[t];
    const int i = blk / H.nb, j = blk % H.nb;
    const int bi = H.bs(i), bj = H.bs(j);
    double* Dm = H.dense(i, j);
    for (int64_t e = threadIdx.x; e < (int64_t)bi * bj; e += blockDim.x) {
      const int r = e % bi, c = e / bi;
      Dm[r + (int64_t)c * H.bmax] = kernel_eval(K, H.off[i] + r, H.off[j] + c);
    }
  }
}

// Admissible blocks: evaluate, truncated column-pivoted QR to eps * ||A||_F
// (operations/LAPACK/geqp3.cpp:71-192, LAWN 176 norm down-dating), Q by
// applying the reflectors, R with columns permuted back, then RQ of R
// (via QR of the column-reversed R^T) so S is upper triangular and V has
// orthonormal rows (classes/low_rank.cpp:50-59).  One CTA per block, FP64
// scratch per CTA slot: A (b x b), Q (b x b), X (b x b), norms, pivots.
constexpr int BUILD_THREADS = 512;

__global__ void __launch_bounds__(BUILD_THREADS) k_build_lowrank(BlrView<double> H, KernelDesc K, const int* blocks,
                                                                 int nblocks, double eps, double* scratch,
                                                                 int64_t stride, int* err) {
  __shared__ double red[32];
  __shared__ int redi[32];
  const int ld = H.bmax;
  double* base = scratch + (int64_t)blockIdx.x * stride;
  double* Am = base;                               // b x b
  double* Qm = Am + (int64_t)ld * ld;              // b x b
  double* Xm = Qm + (int64_t)ld * ld;              // b x b
  double* cnorm = Xm + (int64_t)ld * ld;           // b
  double* partial = cnorm + ld;                    // b
  double* tau = partial + ld;                      // b
  double* tau2 = tau + ld;                         // b
  int* jpvt = reinterpret_cast<int*>(tau2 + ld);   // b
  int* jinv = jpvt + ld;                           // b
  const double dlamch_e = 1.1102230246251565e-16;  // LAPACK dlamch('e') = eps/2 (rounding)
  const double tol3z = sqrt(dlamch_e);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int t = blockIdx.x; t < nblocks; t += gridDim.x) {
    const int blk = blocks[t];
    const int i = blk / H.nb, j = blk % H.nb;
    const int m = H.bs(i), n = H.bs(j);
    const int mind = min(m, n);
    for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) {
      const int r = e % m, c = e / m;
      Am[r + (int64_t)c * m] = kernel_eval(K, H.off[i] + r, H.off[j] + c);
    }
    __syncthreads();
    double fro = 0.0;
    for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) fro += Am[e] * Am[e];
    fro = block_sum(fro, red);
    for (int c = wid; c < n; c += nw) {
      double s = 0.0;
      for (int r = lane; r < m; r += 32) s += Am[r + (int64_t)c * m] * Am[r + (int64_t)c * m];
      s = warp_sum(s);
      if (lane == 0) { cnorm[c] = sqrt(s); partial[c] = sqrt(s); jpvt[c] = c; }
    }
    __syncthreads();
    const double threshold = eps * sqrt(fro);
    double maxc;
    {
      double best = -1.0; int bi = -1;
      for (int c = threadIdx.x; c < n; c += blockDim.x) if (cnorm[c] > best) { best = cnorm[c]; bi = c; }
      block_argmax_abs(best < 0 ? 0.0 : best, bi, red, redi, &maxc);
    }
    int r = 0;
    if (maxc <= dlamch_e) {
      // zero block: Q = e_0, R = 0 (geqp3.cpp:97-102)
      for (int e = threadIdx.x; e < m; e += blockDim.x) H.u(i, j)[e] = (e == 0) ? 1.0 : 0.0;
      for (int e = threadIdx.x; e < n; e += blockDim.x) H.vt(i, j)[e] = (e == 0) ? 1.0 : 0.0;
      if (threadIdx.x == 0) { H.s(i, j)[0] = 0.0; H.rank[blk] = 1; }
      __syncthreads();
      continue;
    }
    while (r < mind && maxc > threshold) {
      // pivot: first max over cnorm[r..n)
      double best = -1.0; int bi = -1;
      for (int c = r + threadIdx.x; c < n; c += blockDim.x) if (cnorm[c] > best) { best = cnorm[c]; bi = c; }
      double dummy;
      const int kp = block_argmax_abs(best < 0 ? 0.0 : best, bi, red, redi, &dummy);
      if (kp != r) {
        for (int e = threadIdx.x; e < m; e += blockDim.x) {
          const double a = Am[e + (int64_t)r * m];
          Am[e + (int64_t)r * m] = Am[e + (int64_t)kp * m];
          Am[e + (int64_t)kp * m] = a;
        }
        if (threadIdx.x == 0) {
          double a = cnorm[r]; cnorm[r] = cnorm[kp]; cnorm[kp] = a;
          a = partial[r]; partial[r] = partial[kp]; partial[kp] = a;
          int q = jpvt[r]; jpvt[r] = jpvt[kp]; jpvt[kp] = q;
        }
      }
      __syncthreads();
      // reflector on column r, rows r..m-1 (dlarfg)
      double* col = Am + (int64_t)r * m;
      double s = 0.0;
      for (int e = r + 1 + threadIdx.x; e < m; e += blockDim.x) s += col[e] * col[e];
      const double xn2 = block_sum(s, red);
      const double alpha = col[r];
      double tt = 0.0, beta = alpha, scal = 0.0;
      if (xn2 > 0.0) {
        const double nrm = sqrt(alpha * alpha + xn2);
        beta = alpha >= 0.0 ? -nrm : nrm;
        tt = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
        for (int e = r + 1 + threadIdx.x; e < m; e += blockDim.x) col[e] *= scal;
      }
      __syncthreads();
      if (threadIdx.x == 0) { col[r] = beta; tau[r] = tt; }
      __syncthreads();
      if (r < mind - 1 && tt != 0.0) {
        for (int c = r + 1 + wid; c < n; c += nw) {
          double* cc = Am + (int64_t)c * m;
          double w = (lane == 0) ? cc[r] : 0.0;
          for (int e = r + 1 + lane; e < m; e += 32) w += col[e] * cc[e];
          w = warp_sum(w) * tt;
          if (lane == 0) cc[r] -= w;
          for (int e = r + 1 + lane; e < m; e += 32) cc[e] -= w * col[e];
        }
      }
      __syncthreads();
      // norm down-date (geqp3.cpp:137-159)
      for (int c = r + 1 + wid; c < n; c += nw) {
        if (cnorm[c] != 0.0) {
          double temp = fabs(Am[r + (int64_t)c * m] / cnorm[c]);
          temp = fmax(0.0, (1.0 - temp) * (1.0 + temp));
          const double ratio = cnorm[c] / partial[c];
          const double temp2 = temp * ratio * ratio;
          if (temp2 > tol3z) {
            if (lane == 0) cnorm[c] = cnorm[c] * sqrt(temp);
          } else {
            double s2 = 0.0;
            if (r < m - 1)
              for (int e = r + 1 + lane; e < m; e += 32) s2 += Am[e + (int64_t)c * m] * Am[e + (int64_t)c * m];
            s2 = warp_sum(s2);
            if (lane == 0) { cnorm[c] = (r < m - 1) ? sqrt(s2) : 0.0; partial[c] = cnorm[c]; }
          }
        }
        __syncwarp();
      }
      __syncthreads();
      ++r;
      best = -1.0; bi = -1;
      for (int c = r + threadIdx.x; c < n; c += blockDim.x) if (cnorm[c] > best) { best = cnorm[c]; bi = c; }
      block_argmax_abs(best < 0 ? 0.0 : best, bi, red, redi, &maxc);
      if (r >= n) maxc = 0.0;
    }
    if (r > H.kcap) { if (threadIdx.x == 0) atomicAdd(err + ERR_RANK_OVERFLOW, 1); }
    // Q (m x r) = H_0..H_{r-1} [I_r; 0]
    for (int64_t e = threadIdx.x; e < (int64_t)m * r; e += blockDim.x) {
      const int rr = e % m, c = e / m;
      Qm[rr + (int64_t)c * m] = (rr == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    cta_apply_q(m, r, Am, m, tau, r, Qm, (int64_t)m);
    // inverse pivot: R_perm[:, jpvt[c]] = R[:, c]; build X = (R_perm)^T reversed columns:
    // X (n x r): X[c, a] = R_perm[r-1-a, c]
    for (int c = threadIdx.x; c < n; c += blockDim.x) jinv[jpvt[c]] = c;
    __syncthreads();
    for (int64_t e = threadIdx.x; e < (int64_t)n * r; e += blockDim.x) {
      const int c = e % n, a = e / n;
      const int row = r - 1 - a;
      const int src = jinv[c];
      Xm[c + (int64_t)a * n] = (row <= src) ? Am[row + (int64_t)src * m] : 0.0;
    }
    __syncthreads();
    // QR of X (n x r): X = Qt Rt; S = J Rt^T J, Vt[:, a] = Qt[:, r-1-a]
    cta_householder_qr(n, r, Xm, n, tau2, red);
    const int rs = min(r, H.kcap);
    double* Sd = H.s(i, j);
    for (int64_t e = threadIdx.x; e < (int64_t)rs * rs; e += blockDim.x) {
      const int a = e % rs, c = e / rs;
      // S[a][c] = Rt[r-1-c][r-1-a] (upper triangular in (a, c))
      const int ra = r - 1 - c, ca = r - 1 - a;
      Sd[a + (int64_t)c * H.kcap] = (ra <= ca) ? Xm[ra + (int64_t)ca * n] : 0.0;
    }
    // explicit Qt (n x r) into Qm's second half? reuse Am (no longer needed)
    double* Qt = Am;
    for (int64_t e = threadIdx.x; e < (int64_t)n * r; e += blockDim.x) {
      const int rr = e % n, c = e / n;
      Qt[rr + (int64_t)c * n] = (rr == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    cta_apply_q(n, r, Xm, n, tau2, r, Qt, (int64_t)n);
    double* Ud = H.u(i, j);
    double* Vd = H.vt(i, j);
    for (int64_t e = threadIdx.x; e < (int64_t)m * rs; e += blockDim.x) {
      const int rr = e % m, c = e / m;
      Ud[rr + (int64_t)c * ld] = Qm[rr + (int64_t)c * m];
    }
    for (int64_t e = threadIdx.x; e < (int64_t)n * rs; e += blockDim.x) {
      const int rr = e % n, a = e / n;
      Vd[rr + (int64_t)a * ld] = Qt[rr + (int64_t)(r - 1 - a) * n];
    }
    if (threadIdx.x == 0) H.rank[blk] = rs;
    __syncthreads();
  }
}

// Fixed-rank compression of the admissible blocks by randomized SVD
// (classes/low_rank.cpp:40-48 -> operations/randomized/rsvd.cpp:17-29):
// Y = A Omega with the reference's Omega (uniform [0,1), std::mt19937 seeded
// 0, row-major n x p, the same matrix for every block of that width; passed
// in by the host), Q = qr(Y), B = Q^T A, thin SVD of B by one-sided Jacobi
// on B^T with the rotations accumulated in p appended rows, U = Q Ub, then
// truncation to `rank`.  One CTA per block, FP64 scratch slot per CTA:
// A (b x b), Y / Q (b x p), Bt (b + p) x p, small vectors.
__global__ void __launch_bounds__(BUILD_THREADS) k_build_lowrank_rsvd(BlrView<double> H, KernelDesc K,
                                                                      const int* blocks, int nblocks, int rank,
                                                                      int p, const double* omega_full,
                                                                      const double* omega_last, int64_t stride,
                                                                      double* scratch, int* err) {
  __shared__ double red[32];
  __shared__ double gsm[2 * 16 * 64];
  __shared__ int flag;
  const int ld = H.bmax;
  double* base = scratch + (int64_t)blockIdx.x * stride;
  double* Am = base;                               // m x n
  double* Ym = Am + (int64_t)ld * ld;              // m x p (QR in place)
  double* Qm = Ym + (int64_t)ld * p;               // m x p explicit Q
  double* Bt = Qm + (int64_t)ld * p;               // (n + p) x p
  double* tau = Bt + (int64_t)(ld + p) * p;        // p
  double* sig = tau + p;                           // p
  int* ord = reinterpret_cast<int*>(sig + p);      // p
  for (int t = blockIdx.x; t < nblocks; t += gridDim.x) {
    const int blk = blocks[t];
    const int i = blk / H.nb, j = blk % H.nb;
    const int m = H.bs(i), n = H.bs(j);
    const double* Om = (n == ld) ? omega_full : omega_last;   // n x p row-major
    for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) {
      const int r = e % m, c = e / m;
      Am[r + (int64_t)c * m] = kernel_eval(K, H.off[i] + r, H.off[j] + c);
    }
    __syncthreads();
    // Y = A Omega: Omega row-major n x p == column-major p x n, used transposed
    cta_gemm<double, BUILD_THREADS>(m, p, n, 1.0, Am, m, false, Om, p, true, 0.0, Ym, m, gsm);
    cta_householder_qr(m, p, Ym, m, tau, red);
    for (int64_t e = threadIdx.x; e < (int64_t)m * p; e += blockDim.x) {
      const int r = e % m, c = e / m;
      Qm[e] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    cta_apply_q(m, p, Ym, m, tau, p, Qm, (int64_t)m);
    // Bt (n x p) = (Q^T A)^T = A^T Q; identity appended below (p x p)
    cta_gemm<double, BUILD_THREADS>(n, p, m, 1.0, Am, m, true, Qm, m, false, 0.0, Bt, n + p, gsm);
    for (int e = threadIdx.x; e < p * p; e += blockDim.x) {
      const int r = e % p, c = e / p;
      Bt[(n + r) + (int64_t)c * (n + p)] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    const int sweeps = cta_jacobi_columns(n, p, Bt, n + p, 60, &flag, n + p);
    if (sweeps < 0 && threadIdx.x == 0) atomicAdd(err + ERR_JACOBI, 1);
    // Bt columns: W Sigma (top n rows), Z (bottom p rows); B = Z Sigma W^T
    for (int c = threadIdx.x >> 5; c < p; c += blockDim.x >> 5) {
      double sacc = 0.0;
      for (int r = threadIdx.x & 31; r < n; r += 32) sacc += Bt[r + (int64_t)c * (n + p)] * Bt[r + (int64_t)c * (n + p)];
      sacc = warp_sum(sacc);
      if ((threadIdx.x & 31) == 0) sig[c] = sqrt(sacc);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < p; c += blockDim.x) {
      const double v = sig[c];
      int pos = 0;
      for (int d = 0; d < p; ++d) pos += (sig[d] > v) || (sig[d] == v && d < c);
      ord[pos] = c;
    }
    __syncthreads();
    const int rk = min(rank, H.kcap);
    if (rank > H.kcap && threadIdx.x == 0) atomicAdd(err + ERR_RANK_OVERFLOW, 1);
    double* Ud = H.u(i, j);
    double* Vd = H.vt(i, j);
    double* Sd = H.s(i, j);
    // U = Q Z[:, ord] (m x rk); Vt = W[:, ord] (n x rk) normalised; S = diag
    for (int64_t e = threadIdx.x; e < (int64_t)m * rk; e += blockDim.x) {
      const int r = e % m, c = e / m;
      const int src = ord[c];
      double acc = 0.0;
      for (int t = 0; t < p; ++t) acc += Qm[r + (int64_t)t * m] * Bt[(n + t) + (int64_t)src * (n + p)];
      Ud[r + (int64_t)c * ld] = acc;
    }
    for (int64_t e = threadIdx.x; e < (int64_t)n * rk; e += blockDim.x) {
      const int r = e % n, c = e / n;
      const int src = ord[c];
      const double sv = sig[src];
      Vd[r + (int64_t)c * ld] = sv > 0.0 ? Bt[r + (int64_t)src * (n + p)] / sv : 0.0;
    }
    for (int64_t e = threadIdx.x; e < (int64_t)rk * rk; e += blockDim.x) {
      const int r = e % rk, c = e / rk;
      Sd[r + (int64_t)c * H.kcap] = (r == c) ? sig[ord[c]] : 0.0;
    }
    if (threadIdx.x == 0) H.rank[blk] = rk;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Batched factorization of independent systems: one launch per elimination
// step covers every system of a batch (grid.z = system).  Each CTA reads its
// system's views and parameters from a device table and leaves at once when
// its system has no step i or fewer tasks than its block index; the bodies
// are the single-system kernels' own.
// ---------------------------------------------------------------------------
template <typename T>
struct SysDev {
  BlrView<double> H;
  BlrView<T> W;
  FactorWs<T> ws;
  int* work;              // recompression task counters of the system ([nb])
  double* rscratch;       // reset-truncation scratch (k_truncate_lr)
  int64_t rstride;
  double core_scale, thr_trunc;
  int smax, core_method, proj_tol, split_p, core_smem, dupd_band, pretrunc, has_lr;
};

template <typename T>
__global__ void k_reset_b(const SysDev<T>* S) {
  const SysDev<T>& s = S[blockIdx.z];
  if ((int)blockIdx.x >= s.H.nb * s.H.nb) return;
  k_reset_impl<T>(s.H, s.W);
}

template <typename T>
__global__ void __launch_bounds__(TRUNC_THREADS) k_truncate_lr_b(const SysDev<T>* S) {
  const SysDev<T>& s = S[blockIdx.z];
  if (!s.pretrunc) return;
  k_truncate_lr_impl<T>(s.H, s.W, s.ws, s.thr_trunc, s.rscratch, s.rstride);
}

template <typename T>
__global__ void __launch_bounds__(GETRF_AUX_THREADS) k_getrf_load_b(const SysDev<T>* S, int i) {
  const SysDev<T>& s = S[blockIdx.z];
  if (i >= s.W.nb) return;
  k_getrf_load_impl<T>(s.W, s.ws, i);
}

template <typename T>
__global__ void __launch_bounds__(GETRF_THREADS) k_getrf_panel_b(const SysDev<T>* S, int i, int jb) {
  const SysDev<T>& s = S[blockIdx.z];
  if (i >= s.W.nb || jb >= s.W.bs(i)) return;
  k_getrf_panel_impl<T>(s.W, s.ws, i, jb);
}

template <typename T>
__global__ void __launch_bounds__(GETRF_AUX_THREADS) k_getrf_trail_b(const SysDev<T>* S, int i, int jb) {
  const SysDev<T>& s = S[blockIdx.z];
  if (i >= s.W.nb) return;
  const int b = s.W.bs(i);
  const int m2 = b - jb - min(32, b - jb);
  const int nt = (m2 + 63) / 64;
  if (m2 <= 0 || (int)blockIdx.x >= nt * nt) return;
  k_getrf_trail_impl<T>(s.W, s.ws, i, jb);
}

template <typename T>
__global__ void __launch_bounds__(GETRF_AUX_THREADS) k_getrf_store_b(const SysDev<T>* S, int i) {
  const SysDev<T>& s = S[blockIdx.z];
  if (i >= s.W.nb) return;
  k_getrf_store_impl<T>(s.W, s.ws, i);
}

template <typename T>
__global__ void __launch_bounds__(TRINV_THREADS) k_trinv_b(const SysDev<T>* S, int i, int cw) {
  const SysDev<T>& s = S[blockIdx.z];
  if (i >= s.W.nb || (int)blockIdx.x >= 2 * ((s.W.bs(i) + cw - 1) / cw)) return;
  k_trinv_impl<T>(s.W, s.ws, i, cw);
}

template <typename T>
__global__ void __launch_bounds__(PANEL_THREADS) k_panel_gather_b(const SysDev<T>* S, int i) {
  const SysDev<T>& s = S[blockIdx.z];
  if ((int)blockIdx.x >= s.W.nb - i - 1) return;
  k_panel_gather_impl<T>(s.W, s.ws, i);
}

template <typename T>
__global__ void __launch_bounds__(PANEL_THREADS) k_panel_mul_b(const SysDev<T>* S, int i) {
  const SysDev<T>& s = S[blockIdx.z];
  if ((int)blockIdx.x >= 2 * (s.W.nb - i - 1)) return;
  k_panel_mul_impl<T>(s.W, s.ws, i);
}

template <typename T>
__global__ void __launch_bounds__(PANEL_THREADS) k_panel_fin_b(const SysDev<T>* S, int i) {
  const SysDev<T>& s = S[blockIdx.z];
  if ((int)blockIdx.x >= 2 * (s.W.nb - i - 1)) return;
  k_panel_fin_impl<T>(s.W, s.ws, i);
}

template <typename T>
__global__ void __launch_bounds__(DUPD_THREADS) k_update_dense_b(const SysDev<T>* S, int i, int mode) {
  const SysDev<T>& s = S[blockIdx.z];
  if (i >= s.W.nb - 1) return;
  k_update_dense_impl<T>(s.W, s.ws, i, s.dupd_band, mode);
}

template <typename T>
__global__ void __launch_bounds__(RECOMP_THREADS) k_recompress_b(const SysDev<T>* S, int i) {
  const SysDev<T>& s = S[blockIdx.z];
  if (i >= s.W.nb - 1 || !s.has_lr) return;
  k_recompress_impl<T>(s.W, s.ws, i, s.smax, s.core_method, s.core_scale, 0, s.work + i, 0, nullptr, nullptr,
                       s.proj_tol, s.split_p, s.core_smem);
}

}  // namespace frank
