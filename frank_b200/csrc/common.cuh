// Device helpers shared by the BLR-LU kernels: reductions, a CTA-wide tiled
// GEMM on column-major operands, Householder QR / Q application, and a
// one-sided Jacobi SVD.  Every routine here is executed cooperatively by all
// threads of one thread block (CTA) and ends with a __syncthreads().
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#define FRANK_HD __host__ __device__ __forceinline__
#define FRANK_D __device__ __forceinline__

namespace frank {

// Error word layout (device int array of the plan).
enum ErrSlot {
  ERR_SINGULAR_STEP = 0,   // 1 + first block step whose getrf met a zero pivot
  ERR_RANK_OVERFLOW = 1,   // count of recompressions clamped at the capacity
  ERR_JACOBI = 2,          // count of core SVDs that hit the sweep limit
  ERR_BOUNDS = 3,          // count of index checks that failed (skipped access)
  ERR_MAX_RANK = 4,        // largest rank produced by a recompression
  ERR_RECOMP = 5,          // recompressions performed (low 31 bits)
  ERR_SLOTS = 8
};

// Algorithmic FLOP counters (device unsigned long long array of the plan),
// one per kernel class of the factorization.
enum FlopSlot { FLOP_GETRF = 0, FLOP_PANEL = 1, FLOP_DENSE = 2, FLOP_RECOMP = 3, FLOP_TRINV = 4, FLOP_SLOTS = 5 };

FRANK_D double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

FRANK_D float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the CTA; `red` is shared scratch of >= 32 doubles.  All threads
// receive the result.
FRANK_D double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = (threadIdx.x < (unsigned)nw) ? red[threadIdx.x] : 0.0;
  if (wid == 0) t = warp_sum(t);
  if (threadIdx.x == 0) red[0] = t;
  __syncthreads();
  double r = red[0];
  __syncthreads();
  return r;
}

// Arg-max of |v| over the CTA with ties broken toward the smallest index
// (LAPACK idamax semantics).  Returns the index; *absval gets the value.
FRANK_D int block_argmax_abs(double v, int idx, double* redv, int* redi, double* absval) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  double a = fabs(v);
  if (idx < 0) a = -1.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double oa = __shfl_xor_sync(0xffffffffu, a, o);
    int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    if (oa > a || (oa == a && oi >= 0 && (idx < 0 || oi < idx))) { a = oa; idx = oi; }
  }
  __syncthreads();
  if (lane == 0) { redv[wid] = a; redi[wid] = idx; }
  __syncthreads();
  if (wid == 0) {
    a = (lane < nw) ? redv[lane] : -1.0;
    idx = (lane < nw) ? redi[lane] : -1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double oa = __shfl_xor_sync(0xffffffffu, a, o);
      int oi = __shfl_xor_sync(0xffffffffu, idx, o);
      if (oa > a || (oa == a && oi >= 0 && (idx < 0 || oi < idx))) { a = oa; idx = oi; }
    }
    if (lane == 0) { redv[0] = a; redi[0] = idx; }
  }
  __syncthreads();
  int r = redi[0];
  *absval = redv[0];
  __syncthreads();
  return r;
}

// One-barrier variants of block_sum / block_argmax_abs for the pivoted QR's
// per-step reductions: each warp's partial goes to red, and after the barrier
// every thread combines the nw partials itself (same order everywhere, so all
// threads agree).  The caller must pass another block barrier before red is
// written again (the pivoted QR's steps do).
FRANK_D double block_sum1(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < nw; ++w) t += red[w];
  return t;
}

FRANK_D int block_argmax_abs1(double v, int idx, double* redv, int* redi, double* absval) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  double a = fabs(v);
  if (idx < 0) a = -1.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double oa = __shfl_xor_sync(0xffffffffu, a, o);
    int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    if (oa > a || (oa == a && oi >= 0 && (idx < 0 || oi < idx))) { a = oa; idx = oi; }
  }
  if (lane == 0) { redv[wid] = a; redi[wid] = idx; }
  __syncthreads();
  a = -1.0;
  idx = -1;
  for (int w = 0; w < nw; ++w) {
    const double oa = redv[w];
    const int oi = redi[w];
    if (oa > a || (oa == a && oi >= 0 && (idx < 0 || oi < idx))) { a = oa; idx = oi; }
  }
  *absval = a;
  return idx;
}

// ---------------------------------------------------------------------------
// CTA-wide GEMM: C(m x n) = alpha * op(A) * op(B) + beta * C, column-major.
// op(A) is m x k: A is (m x k, lda) when !ta, (k x m, lda) when ta.
// op(B) is k x n: B is (k x n, ldb) when !tb, (n x k, ldb) when tb.
// beta == 0 never reads C.  64x64 output tiles, k in steps of 16, operands
// staged through shared memory in the accumulate type.  `smem` must hold
// 2 * 16 * 64 TACC values.  Requires blockDim.x == NT (256 or 512).
// ---------------------------------------------------------------------------
template <typename TACC, int NT, typename TA, typename TB, typename TC>
FRANK_D void cta_gemm(int m, int n, int k, TACC alpha, const TA* __restrict__ A, int64_t lda, bool ta,
                      const TB* __restrict__ B, int64_t ldb, bool tb, TACC beta, TC* C, int64_t ldc,
                      TACC* smem) {
  constexpr int BM = 64, BN = 64, BK = 16;
  constexpr int TM = 4, TN = (NT == 256) ? 4 : 2;
  static_assert((BM / TM) * (BN / TN) == NT, "tile/threads mismatch");
  TACC* As = smem;            // [BK][BM]
  TACC* Bs = smem + BK * BM;  // [BK][BN]
  const int tid = threadIdx.x;
  const int tr = tid % (BM / TM);   // row group
  const int tc = tid / (BM / TM);   // col group
  if (m <= 0 || n <= 0) { __syncthreads(); return; }
  for (int r0 = 0; r0 < m; r0 += BM) {
    for (int c0 = 0; c0 < n; c0 += BN) {
      TACC acc[TM][TN];
#pragma unroll
      for (int a = 0; a < TM; ++a)
#pragma unroll
        for (int b = 0; b < TN; ++b) acc[a][b] = TACC(0);
      for (int k0 = 0; k0 < k; k0 += BK) {
        for (int idx = tid; idx < BM * BK; idx += NT) {
          int rr, kk;
          if (!ta) { rr = idx % BM; kk = idx / BM; } else { kk = idx % BK; rr = idx / BK; }
          const int gr = r0 + rr, gk = k0 + kk;
          TACC v = TACC(0);
          if (gr < m && gk < k) v = ta ? TACC(A[gk + (int64_t)gr * lda]) : TACC(A[gr + (int64_t)gk * lda]);
          As[kk * BM + rr] = v;
        }
        for (int idx = tid; idx < BN * BK; idx += NT) {
          int cc, kk;
          if (!tb) { kk = idx % BK; cc = idx / BK; } else { cc = idx % BN; kk = idx / BN; }
          const int gc = c0 + cc, gk = k0 + kk;
          TACC v = TACC(0);
          if (gc < n && gk < k) v = tb ? TACC(B[gc + (int64_t)gk * ldb]) : TACC(B[gk + (int64_t)gc * ldb]);
          Bs[kk * BN + cc] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
          TACC av[TM], bv[TN];
#pragma unroll
          for (int a = 0; a < TM; ++a) av[a] = As[kk * BM + tr + a * (BM / TM)];
#pragma unroll
          for (int b = 0; b < TN; ++b) bv[b] = Bs[kk * BN + tc + b * (BN / TN)];
#pragma unroll
          for (int a = 0; a < TM; ++a)
#pragma unroll
            for (int b = 0; b < TN; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
        }
        __syncthreads();
      }
#pragma unroll
      for (int a = 0; a < TM; ++a) {
        const int gr = r0 + tr + a * (BM / TM);
        if (gr >= m) continue;
#pragma unroll
        for (int b = 0; b < TN; ++b) {
          const int gc = c0 + tc + b * (BN / TN);
          if (gc >= n) continue;
          TC* p = C + gr + (int64_t)gc * ldc;
          TACC v = alpha * acc[a][b];
          if (beta != TACC(0)) v += beta * TACC(*p);
          *p = TC(v);
        }
      }
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Householder QR (LAPACK dgeqr2 / dlarfg conventions) of the column-major
// m x n matrix A (lda) in FP64, in place: R on and above the diagonal, the
// reflector vectors v (v_0 = 1 implicit) below, tau[min(m,n)].
// Warps take columns, lanes take rows.
// ---------------------------------------------------------------------------
FRANK_D void cta_householder_qr(int m, int n, double* A, int64_t lda, double* tau, double* red) {
  // Two barriers per column: the warp that updates column j+1 also leaves
  // that column's squared norm below its diagonal for step j+1 (red[30..31],
  // double-buffered; block_sum uses red[0 .. nw-1], so blockDim.x <= 960).
  const int kmin = m < n ? m : n;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (kmin <= 0) return;
  double* xn = red + 30;
  {
    double s = 0.0;
    for (int r = 1 + threadIdx.x; r < m; r += blockDim.x) s += A[r] * A[r];
    s = block_sum(s, red);
    if (threadIdx.x == 0) xn[0] = s;
    __syncthreads();
  }
  for (int j = 0; j < kmin; ++j) {
    double* col = A + (int64_t)j * lda;
    const double xnorm2 = xn[j & 1];
    const double alpha = col[j];
    double t = 0.0, beta = alpha, scal = 0.0;
    if (xnorm2 > 0.0) {
      const double nrm = sqrt(alpha * alpha + xnorm2);
      beta = alpha >= 0.0 ? -nrm : nrm;
      t = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
      for (int r = j + 1 + threadIdx.x; r < m; r += blockDim.x) col[r] *= scal;
    }
    __syncthreads();
    if (threadIdx.x == 0) { col[j] = beta; tau[j] = t; }
    // apply H = I - t v v^T to columns j+1..n-1 (v_j = 1 implicit; rows > j)
    for (int c = j + 1 + wid; c < n; c += nw) {
      double* cc = A + (int64_t)c * lda;
      if (t != 0.0) {
        double w = 0.0;
        if (lane == 0) w = cc[j];
        for (int r = j + 1 + lane; r < m; r += 32) w += col[r] * cc[r];
        w = warp_sum(w) * t;
        if (lane == 0) cc[j] -= w;
        for (int r = j + 1 + lane; r < m; r += 32) cc[r] -= w * col[r];
      }
      if (c == j + 1) {
        __syncwarp();
        double s2 = 0.0;
        for (int r = j + 2 + lane; r < m; r += 32) s2 += cc[r] * cc[r];
        s2 = warp_sum(s2);
        if (lane == 0) xn[(j + 1) & 1] = s2;
      }
    }
    __syncthreads();
  }
}

// X (m x r, ldx) := Q X where Q = H_0 H_1 ... H_{k-1} from cta_householder_qr
// (reflectors in V, m x k, ldv).  LAPACK dorm2r, left, no transpose.
template <typename TX>
FRANK_D void cta_apply_q(int m, int k, const double* V, int64_t ldv, const double* tau,
                         int r, TX* X, int64_t ldx) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j = k - 1; j >= 0; --j) {
    const double t = tau[j];
    if (t != 0.0) {
      const double* v = V + (int64_t)j * ldv;
      for (int c = wid; c < r; c += nw) {
        TX* xc = X + (int64_t)c * ldx;
        double w = 0.0;
        if (lane == 0) w = double(xc[j]);
        for (int i = j + 1 + lane; i < m; i += 32) w += v[i] * double(xc[i]);
        w = warp_sum(w) * t;
        if (lane == 0) xc[j] = TX(double(xc[j]) - w);
        for (int i = j + 1 + lane; i < m; i += 32) xc[i] = TX(double(xc[i]) - w * v[i]);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// One-sided (Hestenes) Jacobi on the columns of G (m x n, ldg), FP64, in
// place: on return the columns are mutually orthogonal, G = U * Sigma
// (unsorted).  Pairs are scheduled by the round-robin (circle) method so a
// round's pairs are disjoint; each warp rotates one pair at a time.
// Rotation: zeta = (beta - alpha) / (2 gamma), t = sign(zeta) /
// (|zeta| + sqrt(1 + zeta^2)), c = 1/sqrt(1+t^2), s = c t (Demmel & Veselic,
// "Jacobi's method is more accurate than QR", 1992).  Returns the number of
// sweeps, or -1 if max_sweeps was reached without convergence.
// ---------------------------------------------------------------------------
FRANK_D int cta_jacobi_columns(int m, int n, double* G, int64_t ldg, int max_sweeps, int* flag, int m_rot = -1) {
  // rotation angles from rows [0, m); rotations applied to rows [0, m_rot)
  // (m_rot > m accumulates the right singular vectors in appended rows)
  if (m_rot < m) m_rot = m;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int N2 = n + (n & 1);
  const double tol = (double)(m > 1 ? m : 1) * 2.220446049250313e-16;
  if (n < 2) { __syncthreads(); return 0; }
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    if (threadIdx.x == 0) *flag = 0;
    __syncthreads();
    for (int round = 0; round < N2 - 1; ++round) {
      for (int pr = wid; pr < N2 / 2; pr += nw) {
        int p, q;
        if (pr == 0) { p = N2 - 1; q = round; }
        else { p = (round + pr) % (N2 - 1); q = (round - pr + N2 - 1) % (N2 - 1); }
        if (p >= n || q >= n) continue;
        if (p > q) { int t = p; p = q; q = t; }
        double* gp = G + (int64_t)p * ldg;
        double* gq = G + (int64_t)q * ldg;
        double a = 0.0, b = 0.0, g = 0.0;
        for (int i = lane; i < m; i += 32) {
          const double x = gp[i], y = gq[i];
          a = fma(x, x, a); b = fma(y, y, b); g = fma(x, y, g);
        }
        a = warp_sum(a); b = warp_sum(b); g = warp_sum(g);
        if (a == 0.0 || b == 0.0) continue;
        if (fabs(g) <= tol * sqrt(a) * sqrt(b)) continue;
        const double zeta = (b - a) / (2.0 * g);
        const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t);
        const double s = c * t;
        for (int i = lane; i < m_rot; i += 32) {
          const double x = gp[i], y = gq[i];
          gp[i] = c * x - s * y;
          gq[i] = s * x + c * y;
        }
        if (lane == 0) *flag = 1;
      }
      __syncthreads();
    }
    const int rotated = *flag;
    __syncthreads();
    if (!rotated) return sweep + 1;
  }
  return -1;
}

}  // namespace frank

namespace frank {

// ---------------------------------------------------------------------------
// Blocked Householder QR in FP64 (LAPACK dgeqrf with dgeqr2 panels, dlarft
// forward/columnwise T factors and dlarfb trailing updates), column-major A
// (m x n, lda) in global memory.  Panels of QRB columns are factored in shared
// memory; the trailing matrix is updated as A -= V (T^T (V^T A)) by two
// CTA GEMMs.  On return A holds R and the reflectors, tau[min(m,n)], and the
// T factor of panel p at Tf + p*QRB*QRB (column-major, ld QRB).
// Shared memory: smP (m*QRB doubles), smT (QRB*QRB), gsm (cta_gemm tiles),
// red (32).  Global scratch W (QRB x n doubles).
// ---------------------------------------------------------------------------
constexpr int QRB = 32;

// After the call, p[0] of lane l holds the sum over the warp of p[l] (the 32
// sums of a warp's 32-vectors, one per lane, by recursive halving: 31
// exchanges instead of 32 butterfly reductions).
FRANK_D void warp_transpose_sum(double (&p)[32]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 16; k >= 1; k >>= 1) {
    const bool up = (lane & k) != 0;
#pragma unroll
    for (int i = 0; i < k; ++i) {
      const double send = up ? p[i] : p[i + k];
      const double keep = up ? p[i + k] : p[i];
      p[i] = keep + __shfl_xor_sync(0xffffffffu, send, k);
    }
  }
}

// W (jn x r, ld QRB) = V^T X over rows [0, kr): V (jn <= 32 columns, ldv) in
// shared memory, X (ldx) anywhere.  One warp per column of X, lanes down the
// rows with jn partial sums each, then warp_transpose_sum.  Ends with a
// block barrier.
template <typename TX>
FRANK_D void panel_vtx(int kr, int jn, const double* smV, int64_t ldv, const TX* X, int64_t ldx, int r, double* W) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // (column of X, half of V's columns) per warp: 16 partial sums per lane
  const int halves = jn > 16 ? 2 : 1;
  for (int t = wid; t < r * halves; t += nw) {
    const int c = t / halves, j0 = (t % halves) * 16;
    const int jm = min(16, jn - j0);
    const TX* xc = X + (int64_t)c * ldx;
    const double* vb = smV + (int64_t)j0 * ldv;
    double p[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) p[j] = 0.0;
    int row = lane;
    for (; row + 96 < kr; row += 128) {
      const double x0 = double(xc[row]), x1 = double(xc[row + 32]), x2 = double(xc[row + 64]),
                   x3 = double(xc[row + 96]);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (j < jm) {
          const double* v = vb + (int64_t)j * ldv + row;
          p[j] += v[0] * x0 + v[32] * x1 + v[64] * x2 + v[96] * x3;
        }
    }
    for (; row < kr; row += 32) {
      const double xv = double(xc[row]);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (j < jm) p[j] += vb[row + (int64_t)j * ldv] * xv;
    }
    // recursive halving over 16 values, then one butterfly level: lane l
    // (l < 16) ends with the sum of p[l]
#pragma unroll
    for (int k = 8; k >= 1; k >>= 1) {
      const bool up = (lane & k) != 0;
#pragma unroll
      for (int i = 0; i < k; ++i) {
        const double send = up ? p[i] : p[i + k];
        const double keep = up ? p[i + k] : p[i];
        p[i] = keep + __shfl_xor_sync(0xffffffffu, send, k);
      }
    }
    const double tot = p[0] + __shfl_xor_sync(0xffffffffu, p[0], 16);
    if (lane < jm) W[j0 + lane + (int64_t)c * QRB] = tot;
  }
  __syncthreads();
}

// X (rows [0, mr), r columns, ldx) -= V W with V (mr x jn, ldv) in shared
// memory and W (jn x r, ld QRB): one thread per row, the row of V in
// registers.  Ends with a block barrier.
FRANK_D void panel_x_minus_vw(int mr, int jn, const double* smV, int64_t ldv, const double* W, int r, double* X,
                              int64_t ldx) {
  for (int row = threadIdx.x; row < mr; row += blockDim.x) {
    double v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = (j < jn) ? smV[row + (int64_t)j * ldv] : 0.0;
    int c = 0;
    for (; c + 1 < r; c += 2) {
      const double* w0 = W + (int64_t)c * QRB;
      const double* w1 = w0 + QRB;
      double a0 = 0.0, a1 = 0.0;
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < jn) { a0 += v[j] * w0[j]; a1 += v[j] * w1[j]; }
      double* x0 = X + row + (int64_t)c * ldx;
      double* x1 = x0 + ldx;
      const double y0 = *x0, y1 = *x1;
      *x0 = y0 - a0;
      *x1 = y1 - a1;
    }
    if (c < r) {
      const double* w0 = W + (int64_t)c * QRB;
      double a0 = 0.0;
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < jn) a0 += v[j] * w0[j];
      X[row + (int64_t)c * ldx] -= a0;
    }
  }
  __syncthreads();
}

// Gram-based T factor of the panel V (mr x jn, unit lower trapezoid in smV).
FRANK_D void cta_larft(int mr, int jn, const double* smV, const double* tau, double* smT) {
  // G = V^T V (jn x jn, in smT), then T column by column (dlarft recurrence
  // T(0:j, j) = -tau_j T(0:j, 0:j) G(0:j, j)): lane i keeps row i of T in
  // registers, so the recurrence needs no barrier between columns.
  panel_vtx(mr, jn, smV, mr, smV, mr, jn, smT);
  if (threadIdx.x < 32) {
    const int i = threadIdx.x;
    double trow[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) trow[l] = 0.0;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if (j < jn) {
        double s = 0.0;
#pragma unroll
        for (int l = 0; l < 32; ++l)
          if (l < j && l >= i) s += trow[l] * smT[l + j * QRB];
        if (i < j) trow[j] = -tau[j] * s;
        else if (i == j) trow[j] = tau[j];
      }
    }
    __syncwarp();
#pragma unroll
    for (int l = 0; l < 32; ++l)
      if (i < QRB && l < QRB) smT[i + l * QRB] = (i < jn && l < jn && l >= i) ? trow[l] : 0.0;
  }
  __syncthreads();
}

// Load the panel's reflectors from A (rows j0.., cols j0..j0+jn) into smV as a
// clean unit-lower-trapezoidal matrix (mr x jn, ld mr).
FRANK_D void cta_load_v(int mr, int jn, const double* Ap, int64_t lda, double* smV) {
  for (int e = threadIdx.x; e < mr * jn; e += blockDim.x) {
    const int r = e % mr, c = e / mr;
    smV[e] = (r > c) ? Ap[r + (int64_t)c * lda] : (r == c ? 1.0 : 0.0);
  }
  __syncthreads();
}

#ifdef FRANK_PHASE_TIMING
__device__ unsigned long long g_sub_cycles[16];
#define SUB_BEGIN() long long _sb_t0 = clock64()
#define SUB_MARK(k)                                                                         \
  do {                                                                                      \
    __syncthreads();                                                                        \
    if (threadIdx.x == 0) {                                                                 \
      const long long _t = clock64();                                                      \
      atomicAdd(&g_sub_cycles[(k)], (unsigned long long)(_t - _sb_t0));                     \
      _sb_t0 = _t;                                                                          \
    }                                                                                       \
  } while (0)
#else
#define SUB_BEGIN() do {} while (0)
#define SUB_MARK(k) do {} while (0)
#endif

template <int NT>
FRANK_D void cta_qr_blocked(int m, int n, double* A, int64_t lda, double* tau, double* Tf, double* W,
                            double* smP, double* smT, double* gsm, double* red, int max_panels = 1 << 20,
                            int max_jn = QRB) {
  const int kmin = m < n ? m : n;
  SUB_BEGIN();
  for (int j0 = 0; j0 < kmin && j0 / QRB < max_panels; j0 += QRB) {
    const int jn = min(min(QRB, max_jn), kmin - j0);
    const int mr = m - j0;
    double* Ap = A + j0 + (int64_t)j0 * lda;
    for (int e = threadIdx.x; e < mr * jn; e += blockDim.x) {
      const int r = e % mr, c = e / mr;
      smP[e] = Ap[r + (int64_t)c * lda];
    }
    __syncthreads();
    SUB_MARK(0);
    cta_householder_qr(mr, jn, smP, mr, tau + j0, red);
    SUB_MARK(1);
    for (int e = threadIdx.x; e < mr * jn; e += blockDim.x) {
      const int r = e % mr, c = e / mr;
      Ap[r + (int64_t)c * lda] = smP[e];
      smP[e] = (r > c) ? smP[e] : (r == c ? 1.0 : 0.0);
    }
    __syncthreads();
    SUB_MARK(2);
    cta_larft(mr, jn, smP, tau + j0, smT);
    double* Tp = Tf + (int64_t)(j0 / QRB) * QRB * QRB;
    for (int e = threadIdx.x; e < QRB * QRB; e += blockDim.x) Tp[e] = smT[e];
    SUB_MARK(3);
    const int nc = n - j0 - jn;
    if (nc > 0) {
      double* At = A + j0 + (int64_t)(j0 + jn) * lda;
      // W = V^T At (jn x nc)
      panel_vtx(mr, jn, smP, mr, At, lda, nc, W);
      // W = T^T W (T upper triangular): column per thread
      for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        // unrolled over the panel width so that w stays in registers
        double w[QRB];
#pragma unroll
        for (int i = 0; i < QRB; ++i) w[i] = (i < jn) ? W[i + (int64_t)c * QRB] : 0.0;
#pragma unroll
        for (int i = QRB - 1; i >= 0; --i) {
          if (i < jn) {
            double s = 0.0;
#pragma unroll
            for (int l = 0; l <= i; ++l) s += smT[l + i * QRB] * w[l];
            W[i + (int64_t)c * QRB] = s;
          }
        }
      }
      __syncthreads();
      // At -= V W
      panel_x_minus_vw(mr, jn, smP, mr, W, nc, At, lda);
    }
    SUB_MARK(4);
  }
  __syncthreads();
}

// X (m x r, ldx, FP64) := Q X with Q from cta_qr_blocked (k = min(m, ncols)
// reflectors).  Panels applied last to first: X -= V (T (V^T X)).  Rows of X
// at or below nz are zero on entry (nz = m if unknown): the first panel
// applied then only contracts rows j0 .. nz-1 in V^T X.
template <int NT>
FRANK_D void cta_apply_q_blocked(int m, int k, const double* A, int64_t lda, const double* Tf, int r,
                                 double* X, int64_t ldx, double* W, double* smP, double* smT, double* gsm,
                                 int nz = -1) {
  if (k <= 0 || r <= 0) { __syncthreads(); return; }
  if (nz < 0 || nz > m) nz = m;
  const int np = (k + QRB - 1) / QRB;
  for (int p = np - 1; p >= 0; --p) {
    const int j0 = p * QRB;
    const int jn = min(QRB, k - j0);
    const int mr = m - j0;
    const int kr = min(mr, max(0, nz - j0));   // rows of X that can be nonzero
    nz = m;                                    // after this panel X is full
    if (kr == 0) continue;                     // V^T X = 0: the panel is the identity on X
    SUB_BEGIN();
    cta_load_v(mr, jn, A + j0 + (int64_t)j0 * lda, lda, smP);
    for (int e = threadIdx.x; e < QRB * QRB; e += blockDim.x) smT[e] = Tf[(int64_t)p * QRB * QRB + e];
    __syncthreads();
    SUB_MARK(5);
    double* Xp = X + j0;
    panel_vtx(kr, jn, smP, mr, Xp, ldx, r, W);
    SUB_MARK(6);
    for (int c = threadIdx.x; c < r; c += blockDim.x) {
      // unrolled over the panel width so that w stays in registers
      double w[QRB];
#pragma unroll
      for (int i = 0; i < QRB; ++i) w[i] = (i < jn) ? W[i + (int64_t)c * QRB] : 0.0;
#pragma unroll
      for (int i = 0; i < QRB; ++i) {
        if (i < jn) {
          double s = 0.0;
#pragma unroll
          for (int l = i; l < QRB; ++l) s += smT[i + l * QRB] * w[l];
          W[i + (int64_t)c * QRB] = s;
        }
      }
    }
    __syncthreads();
    SUB_MARK(7);
    panel_x_minus_vw(mr, jn, smP, mr, W, r, Xp, ldx);
    SUB_MARK(8);
  }
}

// T factors (dlarft, forward / columnwise) of the first k Householder
// reflectors stored below the diagonal of A (m rows, lda; tau), panel by panel
// of QRB columns into Tf + p * QRB * QRB -- the layout cta_apply_q_blocked
// reads -- for reflectors produced by a column-by-column factorization.
FRANK_D void cta_form_t(int m, int k, const double* A, int64_t lda, const double* tau, double* Tf, double* smP,
                        double* smT) {
  for (int j0 = 0; j0 < k; j0 += QRB) {
    const int jn = min(QRB, k - j0);
    const int mr = m - j0;
    cta_load_v(mr, jn, A + j0 + (int64_t)j0 * lda, lda, smP);
    cta_larft(mr, jn, smP, tau + j0, smT);
    double* Tp = Tf + (int64_t)(j0 / QRB) * QRB * QRB;
    for (int e = threadIdx.x; e < QRB * QRB; e += blockDim.x) Tp[e] = smT[e];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Truncated column-pivoted Householder QR (restating
// operations/LAPACK/geqp3.cpp:71-192: pivot = first column of largest
// down-dated norm, dlarfg reflector, LAWN 176 norm down-dating, stop when the
// largest remaining norm <= thr or after maxr steps).  In place on A (m x n,
// lda, FP64; shared or global memory).  Returns the rank r; jpvt[c] is the
// original column at pivoted position c.  cnorm/partial: n doubles each.
// ---------------------------------------------------------------------------
FRANK_D int cta_truncated_geqp3(int m, int n, double* A, int64_t lda, double thr, int maxr, double* tau,
                                double* cnorm, double* partial, int* jpvt, double* red, int* redi) {
  const double dlamch_e = 1.1102230246251565e-16;
  const double tol3z = sqrt(dlamch_e);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int mind = min(min(m, n), maxr);
  for (int c = wid; c < n; c += nw) {
    double s = 0.0;
    for (int r = lane; r < m; r += 32) s += A[r + (int64_t)c * lda] * A[r + (int64_t)c * lda];
    s = warp_sum(s);
    if (lane == 0) { cnorm[c] = sqrt(s); partial[c] = sqrt(s); jpvt[c] = c; }
  }
  __syncthreads();
  // the arg-max of the remaining column norms serves both the stopping test
  // and the next pivot (the norms do not change in between)
  double maxc;
  int kp_next;
  {
    double best = -1.0; int bi = -1;
    for (int c = threadIdx.x; c < n; c += blockDim.x) if (cnorm[c] > best) { best = cnorm[c]; bi = c; }
    kp_next = block_argmax_abs(best < 0 ? 0.0 : best, bi, red, redi, &maxc);
  }
  int r = 0;
  while (r < mind && maxc > thr) {
    double best = -1.0; int bi = -1;
    const int kp = kp_next;
    if (kp != r) {
      for (int e = threadIdx.x; e < m; e += blockDim.x) {
        const double a = A[e + (int64_t)r * lda];
        A[e + (int64_t)r * lda] = A[e + (int64_t)kp * lda];
        A[e + (int64_t)kp * lda] = a;
      }
      if (threadIdx.x == 0) {
        double a = cnorm[r]; cnorm[r] = cnorm[kp]; cnorm[kp] = a;
        a = partial[r]; partial[r] = partial[kp]; partial[kp] = a;
        int q = jpvt[r]; jpvt[r] = jpvt[kp]; jpvt[kp] = q;
      }
    }
    __syncthreads();
    double* col = A + (int64_t)r * lda;
    // every thread reads alpha before the reduction's barriers, so thread 0
    // may overwrite col[r] below without a barrier of its own
    const double alpha = col[r];
    double s = 0.0;
    for (int e = r + 1 + threadIdx.x; e < m; e += blockDim.x) s += col[e] * col[e];
    const double xn2 = block_sum1(s, red);
    double tt = 0.0, beta = alpha;
    if (xn2 > 0.0) {
      const double nrm = sqrt(alpha * alpha + xn2);
      beta = alpha >= 0.0 ? -nrm : nrm;
      tt = (beta - alpha) / beta;
      const double scal = 1.0 / (alpha - beta);
      for (int e = r + 1 + threadIdx.x; e < m; e += blockDim.x) col[e] *= scal;
    }
    // the scaling leaves col[r] alone: one barrier for both
    if (threadIdx.x == 0) { col[r] = beta; tau[r] = tt; }
    __syncthreads();
    if (r < min(m, n) - 1 && tt != 0.0) {
      // four columns per warp pass, so that each lane has four independent
      // load streams in flight (the trailing matrix is often in L2)
      for (int c0 = r + 1 + 4 * wid; c0 < n; c0 += 4 * nw) {
        const int nc = min(4, n - c0);
        double* p0 = A + (int64_t)c0 * lda;
        double* p1 = nc > 1 ? p0 + lda : p0;
        double* p2 = nc > 2 ? p0 + 2 * lda : p0;
        double* p3 = nc > 3 ? p0 + 3 * lda : p0;
        double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0;
        if (lane == 0) { w0 = p0[r]; w1 = p1[r]; w2 = p2[r]; w3 = p3[r]; }
        for (int e = r + 1 + lane; e < m; e += 32) {
          const double v = col[e];
          w0 = fma(v, p0[e], w0); w1 = fma(v, p1[e], w1); w2 = fma(v, p2[e], w2); w3 = fma(v, p3[e], w3);
        }
        w0 = warp_sum(w0) * tt; w1 = warp_sum(w1) * tt; w2 = warp_sum(w2) * tt; w3 = warp_sum(w3) * tt;
        if (lane == 0) {
          p0[r] -= w0;
          if (nc > 1) p1[r] -= w1;
          if (nc > 2) p2[r] -= w2;
          if (nc > 3) p3[r] -= w3;
        }
        for (int e = r + 1 + lane; e < m; e += 32) {
          const double v = col[e];
          p0[e] -= w0 * v;
          if (nc > 1) p1[e] -= w1 * v;
          if (nc > 2) p2[e] -= w2 * v;
          if (nc > 3) p3[e] -= w3 * v;
        }
      }
    }
    __syncthreads();
    // norm down-dating, one column per thread; a column whose down-dated norm
    // is unreliable is marked (-1) and recomputed by a warp below
    for (int c = r + 1 + threadIdx.x; c < n; c += blockDim.x) {
      if (cnorm[c] != 0.0) {
        double temp = fabs(A[r + (int64_t)c * lda] / cnorm[c]);
        temp = fmax(0.0, (1.0 - temp) * (1.0 + temp));
        const double ratio = cnorm[c] / partial[c];
        const double temp2 = temp * ratio * ratio;
        cnorm[c] = temp2 > tol3z ? cnorm[c] * sqrt(temp) : -1.0;
      }
    }
    __syncthreads();
    for (int c = r + 1 + wid; c < n; c += nw) {
      if (cnorm[c] < 0.0) {
        double s2 = 0.0;
        if (r < m - 1)
          for (int e = r + 1 + lane; e < m; e += 32) s2 += A[e + (int64_t)c * lda] * A[e + (int64_t)c * lda];
        s2 = warp_sum(s2);
        if (lane == 0) { cnorm[c] = (r < m - 1) ? sqrt(s2) : 0.0; partial[c] = cnorm[c]; }
      }
      __syncwarp();
    }
    __syncthreads();
    ++r;
    best = -1.0; bi = -1;
    for (int c = r + threadIdx.x; c < n; c += blockDim.x) if (cnorm[c] > best) { best = cnorm[c]; bi = c; }
    kp_next = block_argmax_abs1(best < 0 ? 0.0 : best, bi, red, redi, &maxc);
    if (r >= n) maxc = 0.0;
  }
  __syncthreads();
  return r;
}


// ---------------------------------------------------------------------------
// The same truncated column-pivoted QR (same pivots, same stopping rule and
// norm down-dating) blocked as LAPACK's dlaqps: QB pivot steps per panel, each
// step updating only its pivot column and pivot row from the panel's
// reflectors and an n x QB matrix F (F(:, k) = tau_k A^T v_k, corrected for
// the panel's earlier reflectors), the trailing matrix updated once per panel
// as A -= V F^T (a CTA GEMM).  A step reads the trailing matrix once instead
// of reading and writing it, which is what bounds a core too large for shared
// memory (it lives in L2).  A column whose down-dated norm is unreliable ends
// the panel; its norm is recomputed after the trailing update.  F: n x QB
// doubles (ld n), anywhere; red holds the panel's auxiliary vector between
// the reflector and the next pivot search.  Returns the rank r.
// ---------------------------------------------------------------------------
template <int NT>
FRANK_D int cta_truncated_geqp3_blocked(int m, int n, double* A, int64_t lda, double thr, int maxr, double* tau,
                                        double* cnorm, double* partial, int* jpvt, double* red, int* redi,
                                        double* F, double* gsm) {
  constexpr int QB = 32;
  const double dlamch_e = 1.1102230246251565e-16;
  const double tol3z = sqrt(dlamch_e);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int mind = min(min(m, n), maxr);
  for (int c = wid; c < n; c += nw) {
    double s = 0.0;
    for (int r = lane; r < m; r += 32) s += A[r + (int64_t)c * lda] * A[r + (int64_t)c * lda];
    s = warp_sum(s);
    if (lane == 0) { cnorm[c] = sqrt(s); partial[c] = sqrt(s); jpvt[c] = c; }
  }
  __syncthreads();
  double maxc;
  int kp_next;
  {
    double best = -1.0; int bi = -1;
    for (int c = threadIdx.x; c < n; c += blockDim.x) if (cnorm[c] > best) { best = cnorm[c]; bi = c; }
    kp_next = block_argmax_abs(best < 0 ? 0.0 : best, bi, red, redi, &maxc);
  }
  int r = 0;
  while (r < mind && maxc > thr) {
    const int j0 = r;
    const int kbmax = min(QB, mind - j0);
    int k = 0;
    bool recompute = false;
    while (k < kbmax && maxc > thr) {
      const int j = j0 + k;
      const int kp = kp_next;
      if (kp != j) {
        for (int e = threadIdx.x; e < m; e += blockDim.x) {
          const double a = A[e + (int64_t)j * lda];
          A[e + (int64_t)j * lda] = A[e + (int64_t)kp * lda];
          A[e + (int64_t)kp * lda] = a;
        }
        for (int t = threadIdx.x; t < k; t += blockDim.x) {
          const double a = F[j + (int64_t)t * n];
          F[j + (int64_t)t * n] = F[kp + (int64_t)t * n];
          F[kp + (int64_t)t * n] = a;
        }
        if (threadIdx.x == 0) {
          double a = cnorm[j]; cnorm[j] = cnorm[kp]; cnorm[kp] = a;
          a = partial[j]; partial[j] = partial[kp]; partial[kp] = a;
          int q = jpvt[j]; jpvt[j] = jpvt[kp]; jpvt[kp] = q;
        }
      }
      __syncthreads();
      double* col = A + (int64_t)j * lda;
      // pivot column, rows j.. : the panel's earlier reflectors (rows above j
      // were brought up to date by the earlier pivot-row updates)
      if (k > 0) {
        for (int e = j + threadIdx.x; e < m; e += blockDim.x) {
          double s = 0.0;
          for (int t = 0; t < k; ++t) s += A[e + (int64_t)(j0 + t) * lda] * F[j + (int64_t)t * n];
          col[e] -= s;
        }
        __syncthreads();
      }
      const double alpha = col[j];
      double s = 0.0;
      for (int e = j + 1 + threadIdx.x; e < m; e += blockDim.x) s += col[e] * col[e];
      const double xn2 = block_sum1(s, red);
      double tt = 0.0, beta = alpha;
      if (xn2 > 0.0) {
        const double nrm = sqrt(alpha * alpha + xn2);
        beta = alpha >= 0.0 ? -nrm : nrm;
        tt = (beta - alpha) / beta;
        const double scal = 1.0 / (alpha - beta);
        for (int e = j + 1 + threadIdx.x; e < m; e += blockDim.x) col[e] *= scal;
      }
      // the reflector's unit entry in place while F and the pivot row are formed
      if (threadIdx.x == 0) { col[j] = 1.0; tau[j] = tt; }
      __syncthreads();
      // F(c, k) = tt A(j:m, c)^T v for c > j (four columns per warp pass), 0 above
      for (int c0 = j + 1 + 4 * wid; c0 < n; c0 += 4 * nw) {
        const int nc = min(4, n - c0);
        const double* p0 = A + (int64_t)c0 * lda;
        const double* p1 = nc > 1 ? p0 + lda : p0;
        const double* p2 = nc > 2 ? p0 + 2 * lda : p0;
        const double* p3 = nc > 3 ? p0 + 3 * lda : p0;
        double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0;
        for (int e = j + lane; e < m; e += 32) {
          const double v = col[e];
          w0 = fma(v, p0[e], w0); w1 = fma(v, p1[e], w1); w2 = fma(v, p2[e], w2); w3 = fma(v, p3[e], w3);
        }
        w0 = warp_sum(w0); w1 = warp_sum(w1); w2 = warp_sum(w2); w3 = warp_sum(w3);
        if (lane == 0) {
          double* fk = F + (int64_t)k * n + c0;
          fk[0] = tt * w0;
          if (nc > 1) fk[1] = tt * w1;
          if (nc > 2) fk[2] = tt * w2;
          if (nc > 3) fk[3] = tt * w3;
        }
      }
      for (int c = threadIdx.x; c <= j && c < n; c += blockDim.x) F[c + (int64_t)k * n] = 0.0;
      // aux(t) = -tt A(j:m, j0+t)^T v for the panel's earlier reflectors
      for (int t = wid; t < k; t += nw) {
        const double* pt = A + (int64_t)(j0 + t) * lda;
        double w = 0.0;
        for (int e = j + lane; e < m; e += 32) w = fma(pt[e], col[e], w);
        w = warp_sum(w);
        if (lane == 0) red[t] = -tt * w;
      }
      __syncthreads();
      if (k > 0) {
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
          double a = 0.0;
          for (int t = 0; t < k; ++t) a += F[c + (int64_t)t * n] * red[t];
          F[c + (int64_t)k * n] += a;
        }
        __syncthreads();
      }
      // pivot row j: A(j, c) -= A(j, j0:j+1) F(c, 0:k+1)^T for c > j
      for (int c = j + 1 + threadIdx.x; c < n; c += blockDim.x) {
        double a = 0.0;
        for (int t = 0; t <= k; ++t) a += A[j + (int64_t)(j0 + t) * lda] * F[c + (int64_t)t * n];
        A[j + (int64_t)c * lda] -= a;
      }
      __syncthreads();
      if (threadIdx.x == 0) col[j] = beta;
      // norm down-dating from the updated pivot row; unreliable ones marked
      for (int c = j + 1 + threadIdx.x; c < n; c += blockDim.x) {
        if (cnorm[c] != 0.0) {
          double temp = fabs(A[j + (int64_t)c * lda] / cnorm[c]);
          temp = fmax(0.0, (1.0 - temp) * (1.0 + temp));
          const double ratio = cnorm[c] / partial[c];
          const double temp2 = temp * ratio * ratio;
          cnorm[c] = temp2 > tol3z ? cnorm[c] * sqrt(temp) : -1.0;
        }
      }
      __syncthreads();
      ++k;
      // next pivot; a marked column ends the panel (reported as an infinite norm)
      double best = -1.0; int bi = -1;
      for (int c = j + 1 + threadIdx.x; c < n; c += blockDim.x) {
        const double v = cnorm[c] < 0.0 ? INFINITY : cnorm[c];
        if (v > best) { best = v; bi = c; }
      }
      kp_next = block_argmax_abs1(best < 0 ? 0.0 : best, bi, red, redi, &maxc);
      if (j + 1 >= n) maxc = 0.0;
      if (isinf(maxc)) { recompute = true; break; }
    }
    r = j0 + k;
    // trailing matrix: A(r:m, r:n) -= A(r:m, j0:r) F(r:n, 0:k)^T
    if (k > 0 && r < m && r < n)
      cta_gemm<double, NT>(m - r, n - r, k, -1.0, A + r + (int64_t)j0 * lda, lda, false, F + r, n, true, 1.0,
                           A + r + (int64_t)r * lda, lda, gsm);
    if (recompute) {
      for (int c = r + wid; c < n; c += nw) {
        if (cnorm[c] < 0.0) {
          double s2 = 0.0;
          for (int e = r + lane; e < m; e += 32) s2 += A[e + (int64_t)c * lda] * A[e + (int64_t)c * lda];
          s2 = warp_sum(s2);
          if (lane == 0) { cnorm[c] = r < m ? sqrt(s2) : 0.0; partial[c] = cnorm[c]; }
        }
      }
      __syncthreads();
      double best = -1.0; int bi = -1;
      for (int c = r + threadIdx.x; c < n; c += blockDim.x) if (cnorm[c] > best) { best = cnorm[c]; bi = c; }
      kp_next = block_argmax_abs(best < 0 ? 0.0 : best, bi, red, redi, &maxc);
      if (r >= n) maxc = 0.0;
    }
    if (k == 0) break;
  }
  __syncthreads();
  return r;
}


// ---------------------------------------------------------------------------
// Truncated column-pivoted QR with randomized block pivoting (Martinsson,
// Quintana-Orti, Heavner, van de Geijn, "Householder QR factorization with
// randomization for column pivoting (HQRRP)", SIAM J. Sci. Comput. 39, 2017):
// per panel of QRB columns, a sketch Y = Omega A_trail (QRB + 8 rows, Omega
// uniform in [-1, 1) from a counter-based hash) picks the panel's pivots by a
// pivoted QR of Y, the chosen columns move to the panel, and an unpivoted
// blocked Householder step factors the panel and updates the trailing matrix
// with two CTA GEMMs -- instead of one pivot search and one pass over the
// trailing matrix per column.  The stopping rule is the unblocked one,
// evaluated exactly: after each panel the norms of every remaining column at
// every step t of the panel follow from the updated rows (the later
// reflectors act orthogonally below row t), and the rank is the first step
// whose remaining columns are all at most thr.  Same outputs as
// cta_truncated_geqp3 (R and reflectors in A, tau, jpvt); the pivots are a
// randomized choice, so ranks can differ from the column-by-column search by
// a few.  Scratch ws (global): 40 (m + n) + 40 + 33 n + 8 n + QRB^2 doubles
// (rqrcp_scratch); smP / smT / gsm as cta_qr_blocked.  Returns the rank.
// ---------------------------------------------------------------------------
FRANK_HD int64_t rqrcp_scratch(int m, int n) {
  return 40 * ((int64_t)m + n) + 40 + 33 * (int64_t)n + 8 * (int64_t)n + 32 * 32 + 64;
}

FRANK_D double rqrcp_omega(uint64_t k) {
  k += 0x9E3779B97F4A7C15ull;
  k = (k ^ (k >> 30)) * 0xBF58476D1CE4E5B9ull;
  k = (k ^ (k >> 27)) * 0x94D049BB133111EBull;
  k ^= k >> 31;
  return (double)(k >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

template <int NT>
FRANK_D int cta_rand_qrcp(int m, int n, double* A, int64_t lda, double thr, int maxr, double* tau, int* jpvt,
                          double* ws, double* smP, double* smT, double* gsm, double* red, int* redi) {
  constexpr int SBMAX = QRB + 8;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int mind = min(min(m, n), maxr);
  double* Om = ws;                                   // SBMAX x m
  double* Y = Om + (int64_t)SBMAX * m;               // SBMAX x n
  double* tau_s = Y + (int64_t)SBMAX * n;            // SBMAX
  double* cn_s = tau_s + SBMAX;                      // n
  double* pn_s = cn_s + n;                           // n
  double* nrm2 = pn_s + n;                           // n
  double* Wt = nrm2 + n;                             // QRB x n
  double* Tf = Wt + (int64_t)QRB * n;                // QRB x QRB
  int* jp_s = reinterpret_cast<int*>(Tf + QRB * QRB);   // n
  int* pos = jp_s + n;                               // n
  int* inv = pos + n;                                // n
  int* swp = inv + n;                                // QRB
  for (int c = threadIdx.x; c < n; c += blockDim.x) jpvt[c] = c;
  // the unblocked rule's first test: every column at most thr
  double best = 0.0;
  for (int c = wid; c < n; c += nw) {
    double s2 = 0.0;
    for (int e = lane; e < m; e += 32) s2 += A[e + (int64_t)c * lda] * A[e + (int64_t)c * lda];
    s2 = warp_sum(s2);
    best = fmax(best, s2);
  }
  if (lane == 0) red[wid] = best;
  __syncthreads();
  best = 0.0;
  for (int w = 0; w < nw; ++w) best = fmax(best, red[w]);
  __syncthreads();
  if (mind == 0 || sqrt(best) <= thr) return 0;
  int r = 0;
  int panel = 0;
  while (r < mind) {
    const int b = min(QRB, mind - r);
    const int mr = m - r, nr = n - r;
    const int sb = min(b + 8, mr);
    // 1. sketch of the trailing matrix
    for (int64_t e = threadIdx.x; e < (int64_t)sb * mr; e += blockDim.x)
      Om[e] = rqrcp_omega(((uint64_t)panel << 40) ^ (uint64_t)e);
    __syncthreads();
    cta_gemm<double, NT>(sb, nr, mr, 1.0, Om, sb, false, A + r + (int64_t)r * lda, lda, false, 0.0, Y, sb, gsm);
    // 2. the panel's pivots: b steps of the pivoted QR of the sketch
    cta_truncated_geqp3(sb, nr, Y, sb, -1.0, b, tau_s, cn_s, pn_s, jp_s, red, redi);
    // 3. swaps that bring the chosen columns to r .. r+b-1, then applied row-parallel
    if (threadIdx.x == 0) {
      for (int c = 0; c < nr; ++c) { pos[c] = c; inv[c] = c; }
      for (int t = 0; t < b; ++t) {
        const int want = jp_s[t], cur = pos[want], o = inv[t];
        swp[t] = cur;
        inv[t] = want; inv[cur] = o; pos[want] = t; pos[o] = cur;
        const int q = jpvt[r + t]; jpvt[r + t] = jpvt[r + cur]; jpvt[r + cur] = q;
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < m; e += blockDim.x)
      for (int t = 0; t < b; ++t) {
        const int cur = swp[t];
        if (cur != t) {
          double* a0 = A + e + (int64_t)(r + t) * lda;
          double* a1 = A + e + (int64_t)(r + cur) * lda;
          const double v = *a0; *a0 = *a1; *a1 = v;
        }
      }
    __syncthreads();
    // 4. unpivoted Householder panel and its trailing update
    cta_qr_blocked<NT>(mr, nr, A + r + (int64_t)r * lda, lda, tau + r, Tf, Wt, smP, smT, gsm, red, 1, b);
    // 5. exact norms of the remaining columns at every step t of the panel:
    //    panel column j (t <= j < b): sum_{i=t..j} R(r+i, r+j)^2; trailing
    //    column c: ||A(r+b:, c)||^2 + sum_{i=t..b-1} A(r+i, c)^2
    for (int c = r + b + wid; c < n; c += nw) {
      double s2 = 0.0;
      for (int e = r + b + lane; e < m; e += 32) s2 += A[e + (int64_t)c * lda] * A[e + (int64_t)c * lda];
      s2 = warp_sum(s2);
      if (lane == 0) nrm2[c] = s2;
    }
    __syncthreads();
    // maxima over columns per step t, as the bits of non-negative doubles
    // (ordered like unsigned integers) in gsm
    unsigned long long* mx = reinterpret_cast<unsigned long long*>(gsm);
    for (int t = threadIdx.x; t <= QRB; t += blockDim.x) mx[t] = 0ull;
    __syncthreads();
    for (int c0 = r + b; c0 < n; c0 += blockDim.x) {
      const int c = c0 + threadIdx.x;
      const bool on = c < n;
      double s2 = on ? nrm2[c] : 0.0;
      double v = s2;
      for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
      if (lane == 0) atomicMax(mx + b, (unsigned long long)__double_as_longlong(v));
      for (int t = b - 1; t >= 0; --t) {
        if (on) {
          const double a = A[r + t + (int64_t)c * lda];
          s2 += a * a;
        }
        v = s2;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) atomicMax(mx + t, (unsigned long long)__double_as_longlong(v));
      }
    }
    for (int j = threadIdx.x; j < b; j += blockDim.x) {
      double s2 = 0.0;
      for (int t = j; t >= 0; --t) {
        const double a = A[r + t + (int64_t)(r + j) * lda];
        s2 += a * a;
        atomicMax(mx + t, (unsigned long long)__double_as_longlong(s2));
      }
    }
    __syncthreads();
    // every thread reads the same maxima: the first step whose remaining
    // columns are all at most thr (b: none in this panel)
    int stop = -1;
    for (int t = 0; t <= b; ++t)
      if (sqrt(__longlong_as_double((long long)mx[t])) <= thr) { stop = t; break; }
    __syncthreads();
    if (stop >= 0) return r + stop;
    r += b;
    ++panel;
  }
  __syncthreads();
  return r;
}

}  // namespace frank

namespace frank {

// ---------------------------------------------------------------------------
// Pivoted Cholesky (LAPACK dpstf2 order: pivot = largest remaining diagonal of
// the Schur complement, stop when it drops to tol_rel * the largest initial
// diagonal or after maxr steps) of the symmetric positive semi-definite n x n
// matrix A (full storage, column-major, lda; FP64; shared or global memory),
// in place with explicit symmetric row/column swaps.  On return rows 0..r-1
// of A hold R (upper trapezoid, columns in pivoted order) with
// A(piv, piv) ~= R^T R, piv[c] = original index of pivoted column c.
// Returns r.
// ---------------------------------------------------------------------------
FRANK_D int cta_pivoted_cholesky(int n, double* A, int64_t lda, int* piv, double tol_rel, int maxr, double* red,
                                 int* redi) {
  for (int c = threadIdx.x; c < n; c += blockDim.x) piv[c] = c;
  double dmax0;
  {
    double best = -1.0; int bi = -1;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      const double d = A[t + (int64_t)t * lda];
      if (d > best) { best = d; bi = t; }
    }
    block_argmax_abs(best < 0 ? 0.0 : best, bi, red, redi, &dmax0);
  }
  const double stop = tol_rel * dmax0;
  const int rmax = min(n, maxr);
  int j = 0;
  for (; j < rmax; ++j) {
    double best = -1.0; int bi = -1;
    for (int t = j + threadIdx.x; t < n; t += blockDim.x) {
      const double d = A[t + (int64_t)t * lda];
      if (d > best) { best = d; bi = t; }
    }
    double dmax;
    const int p = block_argmax_abs(best < 0 ? 0.0 : best, bi, red, redi, &dmax);
    if (!(dmax > stop) || dmax <= 0.0) break;
    if (p != j) {
      // swap columns j, p (all rows), then rows j, p (all columns)
      for (int r = threadIdx.x; r < n; r += blockDim.x) {
        const double a = A[r + (int64_t)j * lda];
        A[r + (int64_t)j * lda] = A[r + (int64_t)p * lda];
        A[r + (int64_t)p * lda] = a;
      }
      __syncthreads();
      for (int c = threadIdx.x; c < n; c += blockDim.x) {
        const double a = A[j + (int64_t)c * lda];
        A[j + (int64_t)c * lda] = A[p + (int64_t)c * lda];
        A[p + (int64_t)c * lda] = a;
      }
      if (threadIdx.x == 0) { const int q = piv[j]; piv[j] = piv[p]; piv[p] = q; }
      __syncthreads();
    }
    const double rjj = sqrt(A[j + (int64_t)j * lda]);
    __syncthreads();
    for (int c = j + 1 + threadIdx.x; c < n; c += blockDim.x) A[j + (int64_t)c * lda] /= rjj;
    if (threadIdx.x == 0) A[j + (int64_t)j * lda] = rjj;
    __syncthreads();
    // trailing Schur complement: A[t, c] -= R[j, t] R[j, c] for t, c > j
    const int nt = n - j - 1;
    for (int e = threadIdx.x; e < nt * nt; e += blockDim.x) {
      const int t = j + 1 + e % nt, c = j + 1 + e / nt;
      A[t + (int64_t)c * lda] -= A[j + (int64_t)t * lda] * A[j + (int64_t)c * lda];
    }
    __syncthreads();
  }
  __syncthreads();
  return j;
}

// X (r x nc, ldx) := R11^{-1} X with R11 the leading r x r upper triangle of R
// (ldr); one thread per column, back substitution.
FRANK_D void cta_upper_solve(int r, const double* R, int64_t ldr, int nc, double* X, int64_t ldx) {
  for (int c = threadIdx.x; c < nc; c += blockDim.x) {
    double* x = X + (int64_t)c * ldx;
    for (int i = r - 1; i >= 0; --i) {
      double s = x[i];
      for (int t = i + 1; t < r; ++t) s -= R[i + (int64_t)t * ldr] * x[t];
      x[i] = s / R[i + (int64_t)i * ldr];
    }
  }
  __syncthreads();
}

}  // namespace frank

namespace frank {

// ---------------------------------------------------------------------------
// Warp-level small dense factorizations (one warp, __syncwarp only).  Used on
// matrices of a few dozen rows / columns held in shared memory, where a
// block-wide barrier per column step would dominate.
// ---------------------------------------------------------------------------
FRANK_D void warp_argmax(double& v, int& idx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    if (ov > v || (ov == v && oi >= 0 && (idx < 0 || oi < idx))) { v = ov; idx = oi; }
  }
}

// Pivoted Cholesky of the symmetric PSD n x n A (full storage, lda), in place
// (same contract as cta_pivoted_cholesky).
FRANK_D int warp_pivoted_cholesky(int n, double* A, int64_t lda, int* piv, double tol_rel, int maxr) {
  const int lane = threadIdx.x & 31;
  for (int c = lane; c < n; c += 32) piv[c] = c;
  double d0 = -1.0; int i0 = -1;
  for (int t = lane; t < n; t += 32) { const double d = A[t + (int64_t)t * lda]; if (d > d0) { d0 = d; i0 = t; } }
  warp_argmax(d0, i0);
  const double stop = tol_rel * d0;
  const int rmax = min(n, maxr);
  int j = 0;
  for (; j < rmax; ++j) {
    double dm = -1.0; int p = -1;
    for (int t = j + lane; t < n; t += 32) { const double d = A[t + (int64_t)t * lda]; if (d > dm) { dm = d; p = t; } }
    warp_argmax(dm, p);
    if (!(dm > stop) || dm <= 0.0) break;
    if (p != j) {
      for (int r = lane; r < n; r += 32) {
        const double a = A[r + (int64_t)j * lda]; A[r + (int64_t)j * lda] = A[r + (int64_t)p * lda]; A[r + (int64_t)p * lda] = a;
      }
      __syncwarp();
      for (int c = lane; c < n; c += 32) {
        const double a = A[j + (int64_t)c * lda]; A[j + (int64_t)c * lda] = A[p + (int64_t)c * lda]; A[p + (int64_t)c * lda] = a;
      }
      if (lane == 0) { const int q = piv[j]; piv[j] = piv[p]; piv[p] = q; }
      __syncwarp();
    }
    const double rjj = sqrt(A[j + (int64_t)j * lda]);
    __syncwarp();
    for (int c = j + 1 + lane; c < n; c += 32) A[j + (int64_t)c * lda] /= rjj;
    if (lane == 0) A[j + (int64_t)j * lda] = rjj;
    __syncwarp();
    // trailing Schur complement, lanes over columns c (each lane updates its column)
    for (int c = j + 1 + lane; c < n; c += 32) {
      const double rc = A[j + (int64_t)c * lda];
      for (int t = j + 1; t < n; ++t) A[t + (int64_t)c * lda] -= A[j + (int64_t)t * lda] * rc;
    }
    __syncwarp();
  }
  __syncwarp();
  return j;
}

// Householder reflector of x (length m, stride 1) in place (dlarfg); returns tau.
FRANK_D double warp_larfg(int m, double* x) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int e = 1 + lane; e < m; e += 32) s += x[e] * x[e];
  s = warp_sum(s);
  const double alpha = x[0];
  double t = 0.0;
  if (s > 0.0) {
    const double nrm = sqrt(alpha * alpha + s);
    const double beta = alpha >= 0.0 ? -nrm : nrm;
    t = (beta - alpha) / beta;
    const double scal = 1.0 / (alpha - beta);
    for (int e = 1 + lane; e < m; e += 32) x[e] *= scal;
    __syncwarp();
    if (lane == 0) x[0] = beta;
  }
  __syncwarp();
  return t;
}

// apply H = I - t v v^T (v in column vcol, v_0 = 1 implicit, rows j..m-1) to
// column c of A (rows j..m-1)
FRANK_D void warp_apply_reflector(int j, int m, const double* v, double t, double* a) {
  const int lane = threadIdx.x & 31;
  double w = (lane == 0) ? a[j] : 0.0;
  for (int e = j + 1 + lane; e < m; e += 32) w += v[e] * a[e];
  w = warp_sum(w) * t;
  if (lane == 0) a[j] -= w;
  for (int e = j + 1 + lane; e < m; e += 32) a[e] -= w * v[e];
  __syncwarp();
}

FRANK_D void warp_householder_qr(int m, int n, double* A, int64_t lda, double* tau) {
  const int lane = threadIdx.x & 31;
  const int kmin = min(m, n);
  for (int j = 0; j < kmin; ++j) {
    double* col = A + (int64_t)j * lda;
    const double t = warp_larfg(m - j, col + j);
    if (lane == 0) tau[j] = t;
    if (t != 0.0)
      for (int c = j + 1; c < n; ++c) warp_apply_reflector(j, m, col, t, A + (int64_t)c * lda);
  }
  __syncwarp();
}

// X (m x r) := Q X, Q = H_0 ... H_{k-1} from warp_householder_qr / geqp3.
FRANK_D void warp_apply_q(int m, int k, const double* V, int64_t ldv, const double* tau, int r, double* X,
                          int64_t ldx) {
  for (int j = k - 1; j >= 0; --j) {
    const double t = tau[j];
    if (t == 0.0) continue;
    for (int c = 0; c < r; ++c) warp_apply_reflector(j, m, V + (int64_t)j * ldv, t, X + (int64_t)c * ldx);
  }
}

// Truncated column-pivoted QR (same contract as cta_truncated_geqp3).
FRANK_D int warp_truncated_geqp3(int m, int n, double* A, int64_t lda, double thr, int maxr, double* tau,
                                 double* cnorm, double* partial, int* jpvt) {
  const double dlamch_e = 1.1102230246251565e-16;
  const double tol3z = sqrt(dlamch_e);
  const int lane = threadIdx.x & 31;
  const int mind = min(min(m, n), maxr);
  for (int c = 0; c < n; ++c) {
    double s = 0.0;
    for (int r = lane; r < m; r += 32) s += A[r + (int64_t)c * lda] * A[r + (int64_t)c * lda];
    s = warp_sum(s);
    if (lane == 0) { cnorm[c] = sqrt(s); partial[c] = sqrt(s); jpvt[c] = c; }
  }
  __syncwarp();
  double maxc = -1.0; int mi = -1;
  for (int c = lane; c < n; c += 32) if (cnorm[c] > maxc) { maxc = cnorm[c]; mi = c; }
  warp_argmax(maxc, mi);
  int r = 0;
  while (r < mind && maxc > thr) {
    double best = -1.0; int kp = -1;
    for (int c = r + lane; c < n; c += 32) if (cnorm[c] > best) { best = cnorm[c]; kp = c; }
    warp_argmax(best, kp);
    if (kp != r) {
      for (int e = lane; e < m; e += 32) {
        const double a = A[e + (int64_t)r * lda]; A[e + (int64_t)r * lda] = A[e + (int64_t)kp * lda]; A[e + (int64_t)kp * lda] = a;
      }
      if (lane == 0) {
        double a = cnorm[r]; cnorm[r] = cnorm[kp]; cnorm[kp] = a;
        a = partial[r]; partial[r] = partial[kp]; partial[kp] = a;
        const int q = jpvt[r]; jpvt[r] = jpvt[kp]; jpvt[kp] = q;
      }
      __syncwarp();
    }
    double* col = A + (int64_t)r * lda;
    double tt;
    if (r < m - 1) tt = warp_larfg(m - r, col + r);
    else tt = 0.0;
    if (lane == 0) tau[r] = tt;
    __syncwarp();
    if (r < min(m, n) - 1 && tt != 0.0)
      for (int c = r + 1; c < n; ++c) warp_apply_reflector(r, m, col, tt, A + (int64_t)c * lda);
    // norm down-date (LAWN 176), lanes over columns
    for (int c = r + 1 + lane; c < n; c += 32) {
      if (cnorm[c] != 0.0) {
        double temp = fabs(A[r + (int64_t)c * lda] / cnorm[c]);
        temp = fmax(0.0, (1.0 - temp) * (1.0 + temp));
        const double ratio = cnorm[c] / partial[c];
        if (temp * ratio * ratio > tol3z) {
          cnorm[c] = cnorm[c] * sqrt(temp);
        } else {
          double s2 = 0.0;
          for (int e = r + 1; e < m; ++e) s2 += A[e + (int64_t)c * lda] * A[e + (int64_t)c * lda];
          cnorm[c] = (r < m - 1) ? sqrt(s2) : 0.0;
          partial[c] = cnorm[c];
        }
      }
    }
    __syncwarp();
    ++r;
    maxc = -1.0; mi = -1;
    for (int c = r + lane; c < n; c += 32) if (cnorm[c] > maxc) { maxc = cnorm[c]; mi = c; }
    warp_argmax(maxc, mi);
    if (r >= n) maxc = 0.0;
  }
  __syncwarp();
  return r;
}

// X (r x nc) := R11^{-1} X, R11 upper r x r; lanes over columns.
FRANK_D void warp_upper_solve(int r, const double* R, int64_t ldr, int nc, double* X, int64_t ldx) {
  const int lane = threadIdx.x & 31;
  for (int c = lane; c < nc; c += 32) {
    double* x = X + (int64_t)c * ldx;
    for (int i = r - 1; i >= 0; --i) {
      double s = x[i];
      for (int t = i + 1; t < r; ++t) s -= R[i + (int64_t)t * ldr] * x[t];
      x[i] = s / R[i + (int64_t)i * ldr];
    }
  }
  __syncwarp();
}

// C (m x n, ldc, FP64) = alpha * A^T B with A (k x m), B (k x n) column-major
// and k long (the rows of the bases): one warp per output, lanes over k.
// Coalesced reads of columns of A and B; one block barrier at the end.
template <typename TA, typename TB>
FRANK_D void cta_gemm_tn_dot(int m, int n, int k, double alpha, const TA* A, int64_t lda, const TB* B, int64_t ldb,
                             double* C, int64_t ldc) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int e = wid; e < m * n; e += nw) {
    const int a = e % m, c = e / m;
    const TA* pa = A + (int64_t)a * lda;
    const TB* pb = B + (int64_t)c * ldb;
    double s = 0.0;
    for (int t = lane; t < k; t += 32) s += double(pa[t]) * double(pb[t]);
    s = warp_sum(s);
    if (lane == 0) C[a + (int64_t)c * ldc] = alpha * s;
  }
  __syncthreads();
}

// C (m x n, ldc) = A (m x k, lda) X (k x n, ldx, FP64) [+ C if accumulate],
// m long (the rows of the bases), k and n small: threads over rows, each
// thread keeps up to 8 outputs in registers per pass over X's columns.
template <typename TA, typename TC>
FRANK_D void cta_gemm_tall(int m, int n, int k, const TA* A, int64_t lda, const double* X, int64_t ldx, TC* C,
                           int64_t ldc, bool accumulate, double alpha = 1.0) {
  for (int c0 = 0; c0 < n; c0 += 8) {
    const int nc = min(8, n - c0);
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      double acc[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[c] = 0.0;
      for (int t = 0; t < k; ++t) {
        const double av = double(A[r + (int64_t)t * lda]);
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < nc) acc[c] += av * X[t + (int64_t)(c0 + c) * ldx];
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c >= nc) break;
        TC* pc = C + r + (int64_t)(c0 + c) * ldc;
        *pc = TC(accumulate ? double(*pc) + alpha * acc[c] : alpha * acc[c]);
      }
    }
  }
  __syncthreads();
}

// Project the columns of Y (m x p, ldy) out of the span of Q (m x k, ldq,
// orthonormal columns), twice (classical Gram-Schmidt with one
// re-orthogonalisation): Z (k x p, ldz) = Q^T Y_0, Y = (I - Q Q^T)^2 Y_0,
// Y_0 = Q Z + Y.  Z2 (k x p, ld k) is scratch.  Skinny shapes use the warp /
// row kernels, larger ones the tiled CTA GEMM.
template <int NT>
FRANK_D void cta_project_out(int m, int k, int p, const double* Q, int64_t ldq, double* Y, int64_t ldy, double* Z,
                             int64_t ldz, double* Z2, double* gsm) {
  for (int pass = 0; pass < 2; ++pass) {
    double* Zp = pass ? Z2 : Z;
    const int64_t ldp = pass ? k : ldz;
    if ((int64_t)k * p <= 1024) cta_gemm_tn_dot(k, p, m, 1.0, Q, ldq, Y, ldy, Zp, ldp);
    else cta_gemm<double, NT>(k, p, m, 1.0, Q, ldq, true, Y, ldy, false, 0.0, Zp, ldp, gsm);
    if (p <= 16) cta_gemm_tall(m, p, k, Q, ldq, Zp, ldp, Y, ldy, true, -1.0);
    else cta_gemm<double, NT>(m, p, k, -1.0, Q, ldq, false, Zp, ldp, false, 1.0, Y, ldy, gsm);
  }
  for (int64_t e = threadIdx.x; e < (int64_t)k * p; e += blockDim.x) {
    const int r = e % k, c = e / k;
    Z[r + (int64_t)c * ldz] += Z2[e];
  }
  __syncthreads();
}

}  // namespace frank
