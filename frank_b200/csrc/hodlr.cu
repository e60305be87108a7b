// Multi-level H-LU on the device: FRANK's recursive getrf_omm(Hierarchical)
// (operations/LAPACK/getrf.cpp:45-65) for a Hierarchical matrix with a binary
// cluster tree and weak admissibility -- Hierarchical(kernel, params, n, n,
// rank, nleaf, admis = 0, 2, 2) (classes/hierarchical.cpp:49-109,
// matrix_initializer.cpp:51-58 position-based: every off-diagonal child is
// LowRank, every diagonal child recurses until it is a dense leaf), fixed
// rank k.
//
// Layout in HBM (FP64, column-major), levels l = 1 .. L, n = b 2^L:
//   leaves      D[p]        b x b, p = 0 .. 2^L - 1 (A_H: D0; factor: D,
//                            packed pivoted LU after getrf)
//   LowRank     (l, c)      c = 0 .. 2^l - 1: rows of cluster c of level l,
//                            columns of its sibling c ^ 1, size s_l = n >> l:
//                            U (s_l x k), S (k x k), V (k x s_l, ld k); all
//                            blocks of a level are one contiguous slab, so a
//                            level's blocks are one strided batch
//   per leaf    Linv, Uinv, Uinv^T (b x b), pivots.
//
// getrf(node) = getrf(left); U_up <- L_left^{-1} P U_up and V_low <- V_low
// U_left^{-1} (two substitution walks in one launch); the Schur update
// -L_low U_up = LowRank(U_low, S', V_up), S' = -(S_low V_low)(U_up S_up)
// (gemm.cpp:374-393), added into the right child by splitting it over the
// child's blocks (addition.cpp:62-66): dense leaves += (U S') V, LowRank
// blocks += by the batched LowRank addition of ops.cu (fast_rounded_addition,
// the reference's default for fixed rank, addition.cpp:133-203, or
// rounded_addition), one launch per level and parity; then getrf(right).
// The shapes are static (fixed rank), so the whole factorization is one
// stream of launches, captured once into a CUDA graph and replayed.
//
// Pivoting: the leaves take dgetrf's partial pivoting with the interchanges
// applied (P A = L U with P = blockdiag(P_p)); the L blocks keep their rows
// in natural order and each substitution applies P_p to its running
// right-hand side when it reaches leaf p, which is the same thing.  The
// reference discards the pivots (getrf.cpp:67-84); the two agree whenever
// dgetrf does not swap rows.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <cooperative_groups.h>

// The BLR engine's kernels (leaf LU, explicit inverses, kernel evaluation)
// are compiled into this translation unit under a private name, so that none
// of their symbols collides with the engine's own copy in api.cu.
#define frank frank_blr_private
namespace {
#include "blr_kernels.cuh"
namespace blr = frank_blr_private;
}  // namespace
#undef frank

#include "../../include/frank_b200.h"
#include "ops_tasks.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace frank {
int set_error(int code, const std::string& msg);
namespace ops {
int64_t qr_ws(int m, int n);
int64_t svd_scratch(int m, int n);
int64_t lr_add_ws(int m, int n, int ka, int kb);
void launch_gemm(cudaStream_t s, int m, int n, int k, int count, double alpha, const double* a, int64_t lda,
                 int64_t sa, bool ta, const double* b, int64_t ldb, int64_t sb, bool tb, double beta, double* c,
                 int64_t ldc, int64_t sc);
void launch_qr(cudaStream_t s, int m, int n, int count, const double* a, int64_t lda, int64_t sa, double* q,
               int64_t ldq, int64_t sq, double* r, int64_t ldr, int64_t sr, double* scratch, int64_t ws);
void launch_svd(cudaStream_t s, int m, int n, int count, const double* a, int64_t lda, int64_t sa, double* u,
                int64_t ldu, int64_t su, double* sv, int64_t ss, double* vt, int64_t ldvt, int64_t svt,
                double* scratch, int64_t ws, int* err);
int lr_add_shm_bytes(int ka, int kb);
int lr_add_prepare(int bytes);
void launch_lr_add_tasks(cudaStream_t s, int count, const LrAddTask* tasks, int kmax, int fast, double* scratch,
                         int* err, int shm_bytes);
}  // namespace ops
}  // namespace frank

namespace {
namespace hk {

using blr::KernelDesc;
using blr::kernel_eval;

constexpr int HMAX_RANK = 64;   // k <= 64: two rank rows per lane in the walks
constexpr int HMAX_LEAF = 512;  // b <= 512
constexpr int WT = 256;         // threads of the update / matvec kernels
constexpr int WWT = 1024;       // threads of a substitution walk (many loads in flight per SM)
constexpr int WCW = 4;          // right-hand-side columns per walking CTA
// dynamic shared memory of a walk: r, per-warp partials, t1, t2
constexpr int WALK_SMEM = (WCW * HMAX_LEAF + (WWT / 32) * WCW * HMAX_RANK + 2 * WCW * HMAX_RANK) * 8;
constexpr int KG_P = 72;        // rsvd sample width the construction product holds (k + 5 <= 69)

enum { HERR_JACOBI = 8, HERR_RANK = 9, HERR_SLOTS = 16 };

// Device view of one H-matrix's blocks (working copy or A_H).
struct HView {
  int64_t n;
  int b, L, k;
  const double* D;
  const double* U;
  const double* S;
  const double* V;
  FRANK_D int64_t s(int l) const { return n >> l; }
  FRANK_D const double* u(int l, int c) const { return U + (int64_t)(l - 1) * n * k + (int64_t)c * s(l) * k; }
  FRANK_D const double* v(int l, int c) const { return V + (int64_t)(l - 1) * n * k + (int64_t)c * s(l) * k; }
  FRANK_D const double* sm(int l, int c) const { return S + ((int64_t)(1 << l) - 2 + c) * k * k; }
};

struct LeafFactors {
  const double* Linv;   // [P][b*b] unit lower inverse
  const double* Uinv;   // [P][b*b] upper inverse
  const double* UinvT;  // [P][b*b] transpose of Uinv (lower)
  const int* perm;      // [P][b] (P_p r)[i] = r[perm[i]]
};

// One substitution walk over the leaves of node (l0, c0) on ncols columns of
// B (element (i, c) at B[i rs + c cs], i relative to the node's first row).
//   mode 0: B <- L^{-1} P B  (forward; leaf p: x = Linv_p P_p r, then the
//           lower block of every ancestor whose left child ends at p:
//           B_right -= U (S (V B_left)))
//   mode 1: B <- U^{-T} B    (forward on U^T; leaf: x = Uinv_p^T r, then the
//           upper block: B_right -= V^T (S^T (U^T B_left)))
//   mode 2: B <- U^{-1} B    (backward; leaf: x = Uinv_p r, then the upper
//           block of every ancestor whose right child starts at p:
//           B_left -= U (S (V B_right)))
// Each CTA owns WCW columns and walks the leaves in order on its own; the
// columns are independent, so no CTA waits for another.
struct Walk {
  int mode, l0, c0, ncols;
  double* B;
  int64_t rs, cs;
};

FRANK_D void walk_body(const HView& h, const LeafFactors& f, const Walk& J) {
  extern __shared__ double wsm[];
  double(*r)[HMAX_LEAF] = reinterpret_cast<double(*)[HMAX_LEAF]>(wsm);
  double(*part)[WCW][HMAX_RANK] = reinterpret_cast<double(*)[WCW][HMAX_RANK]>(wsm + WCW * HMAX_LEAF);
  double(*t1)[HMAX_RANK] =
      reinterpret_cast<double(*)[HMAX_RANK]>(wsm + WCW * HMAX_LEAF + (WWT / 32) * WCW * HMAX_RANK);
  double(*t2)[HMAX_RANK] = t1 + WCW;
  const int col0 = blockIdx.x * WCW;
  if (col0 >= J.ncols) return;
  const int nc = min(WCW, J.ncols - col0);
  const int b = h.b, k = h.k, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int hl = h.L - J.l0;
  const int np = 1 << hl;
  const int p0 = J.c0 << hl;
  const int64_t row0 = (int64_t)p0 * b;
  double* B = J.B + (int64_t)col0 * J.cs;
  const int64_t rs = J.rs, cs = J.cs;
  for (int step = 0; step < np; ++step) {
    const int p = J.mode == 2 ? p0 + np - 1 - step : p0 + step;
    const int64_t pr = (int64_t)p * b - row0;
    // leaf solve
    const int* perm = f.perm + (int64_t)p * b;
    for (int e = tid; e < WCW * b; e += WWT) {
      const int c = e / b, i = e % b;
      const int src = J.mode == 0 ? perm[i] : i;
      r[c][i] = c < nc ? B[(pr + src) * rs + c * cs] : 0.0;
    }
    __syncthreads();
    const double* Op = (J.mode == 0 ? f.Linv : (J.mode == 1 ? f.UinvT : f.Uinv)) + (int64_t)p * b * b;
    for (int i = tid; i < b; i += WWT) {
      double acc[WCW];
#pragma unroll
      for (int c = 0; c < WCW; ++c) acc[c] = 0.0;
      if (J.mode == 2) {
#pragma unroll 8
        for (int j = i; j < b; ++j) {
          const double a = Op[i + (int64_t)j * b];
#pragma unroll
          for (int c = 0; c < WCW; ++c) acc[c] += a * r[c][j];
        }
      } else {
        // Linv is unit lower (diagonal not read); Uinv^T is lower with its diagonal
        const int jend = J.mode == 0 ? i : i + 1;
#pragma unroll 8
        for (int j = 0; j < jend; ++j) {
          const double a = Op[i + (int64_t)j * b];
#pragma unroll
          for (int c = 0; c < WCW; ++c) acc[c] += a * r[c][j];
        }
        if (J.mode == 0) {
#pragma unroll
          for (int c = 0; c < WCW; ++c) acc[c] += r[c][i];
        }
      }
      for (int c = 0; c < nc; ++c) B[(pr + i) * rs + c * cs] = acc[c];
    }
    __syncthreads();
    // updates of the ancestors' off-diagonal blocks that this leaf completes
    for (int hh = 1; hh <= hl; ++hh) {
      const int a = p >> hh, half = 1 << (hh - 1), first = a << hh;
      const bool fire = J.mode == 2 ? (p == first + half) : (p == first + half - 1);
      if (!fire) continue;
      const int lv = h.L - hh + 1;
      const int64_t sl = h.s(lv);
      const int blk = J.mode == 0 ? 2 * a + 1 : 2 * a;
      const double* Ub = h.u(lv, blk);
      const double* Sb = h.sm(lv, blk);
      const double* Vb = h.v(lv, blk);
      const int64_t src = (int64_t)(J.mode == 2 ? first + half : first) * b - row0;
      const int64_t dst = (int64_t)(J.mode == 2 ? first : first + half) * b - row0;
      // t1 (k x nc) = V B_src (modes 0, 2) or U^T B_src (mode 1)
      if (J.mode != 1) {
        double acc[2][WCW];
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
          for (int c = 0; c < WCW; ++c) acc[q][c] = 0.0;
        for (int64_t i = wid; i < sl; i += WWT / 32) {
          double xv[WCW];
#pragma unroll
          for (int c = 0; c < WCW; ++c) xv[c] = c < nc ? B[(src + i) * rs + c * cs] : 0.0;
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int rr = lane + 32 * q;
            if (rr < k) {
              const double vv = Vb[rr + i * k];
#pragma unroll
              for (int c = 0; c < WCW; ++c) acc[q][c] += vv * xv[c];
            }
          }
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int rr = lane + 32 * q;
          if (rr < k)
#pragma unroll
            for (int c = 0; c < WCW; ++c) part[wid][c][rr] = acc[q][c];
        }
      } else {
        for (int rr = wid; rr < k; rr += WWT / 32) {
          double acc[WCW];
#pragma unroll
          for (int c = 0; c < WCW; ++c) acc[c] = 0.0;
          for (int64_t i = lane; i < sl; i += 32) {
            const double uv = Ub[i + rr * sl];
#pragma unroll
            for (int c = 0; c < WCW; ++c) acc[c] += uv * (c < nc ? B[(src + i) * rs + c * cs] : 0.0);
          }
#pragma unroll
          for (int c = 0; c < WCW; ++c) {
            const double v = blr::warp_sum(acc[c]);
            if (lane == 0) {
              part[0][c][rr] = v;
              for (int w = 1; w < WWT / 32; ++w) part[w][c][rr] = 0.0;
            }
          }
        }
      }
      __syncthreads();
      for (int e = tid; e < WCW * k; e += WWT) {
        const int c = e / k, rr = e % k;
        double v = 0.0;
        for (int w = 0; w < WWT / 32; ++w) v += part[w][c][rr];
        t1[c][rr] = v;
      }
      __syncthreads();
      // t2 = S t1 (modes 0, 2) or S^T t1 (mode 1)
      for (int e = tid; e < WCW * k; e += WWT) {
        const int c = e / k, rr = e % k;
        double v = 0.0;
        for (int q = 0; q < k; ++q) v += (J.mode == 1 ? Sb[q + (int64_t)rr * k] : Sb[rr + (int64_t)q * k]) * t1[c][q];
        t2[c][rr] = v;
      }
      __syncthreads();
      // B_dst -= U t2 (modes 0, 2) or V^T t2 (mode 1)
      for (int64_t i = tid; i < sl; i += WWT) {
        double acc[WCW];
#pragma unroll
        for (int c = 0; c < WCW; ++c) acc[c] = 0.0;
        for (int q = 0; q < k; ++q) {
          const double a = J.mode == 1 ? Vb[q + i * k] : Ub[i + (int64_t)q * sl];
#pragma unroll
          for (int c = 0; c < WCW; ++c) acc[c] += a * t2[c][q];
        }
        for (int c = 0; c < nc; ++c) B[(dst + i) * rs + c * cs] -= acc[c];
      }
      __syncthreads();
    }
  }
}

__global__ void __launch_bounds__(WWT) k_h_walk(HView h, LeafFactors f, Walk j0, Walk j1) {
  walk_body(h, f, blockIdx.y == 0 ? j0 : j1);
}

// S' = -(S_low (V_low U_up) S_up) (k x k) for the Schur update of a node:
// V_low (k x s, ld k), U_up (s x k, ld s).  Each CTA reduces a range of s
// into its partial; the last CTA to finish (counter) sums the partials in
// CTA order and forms S'.  `counter` returns to 0.
__global__ void __launch_bounds__(WT) k_h_core(int64_t s, int k, const double* Vl, const double* Uu, const double* Sl,
                                               const double* Su, double* partial, double* Sp, int* counter) {
  // tiles of V_low and U_up during the reduction, X = V_low U_up after it
  __shared__ double sm[2 * 32 * (HMAX_RANK + 1)];
  __shared__ int last;
  double(*tv)[HMAX_RANK + 1] = reinterpret_cast<double(*)[HMAX_RANK + 1]>(sm);
  double(*tu)[HMAX_RANK + 1] = reinterpret_cast<double(*)[HMAX_RANK + 1]>(sm + 32 * (HMAX_RANK + 1));
  double* X = sm;
  const int tid = threadIdx.x;
  const int64_t chunk = (s + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * chunk, i1 = min(s, i0 + chunk);
  const int kk = k * k;
  double acc[HMAX_RANK * HMAX_RANK / WT];
#pragma unroll
  for (int q = 0; q < HMAX_RANK * HMAX_RANK / WT; ++q) acc[q] = 0.0;
  for (int64_t t0 = i0; t0 < i1; t0 += 32) {
    const int tn = (int)min((int64_t)32, i1 - t0);
    for (int e = tid; e < 32 * k; e += WT) {
      const int t = e / k, rr = e % k;
      tv[t][rr] = t < tn ? Vl[rr + (t0 + t) * k] : 0.0;
    }
    for (int e = tid; e < 32 * k; e += WT) {
      const int rr = e / 32, t = e % 32;
      tu[t][rr] = t < tn ? Uu[(t0 + t) + (int64_t)rr * s] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < HMAX_RANK * HMAX_RANK / WT; ++q) {
      const int e = tid + q * WT;
      if (e < kk) {
        const int rr = e % k, cc = e / k;
        double v = 0.0;
        for (int t = 0; t < 32; ++t) v += tv[t][rr] * tu[t][cc];
        acc[q] += v;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < HMAX_RANK * HMAX_RANK / WT; ++q) {
    const int e = tid + q * WT;
    if (e < kk) partial[(int64_t)blockIdx.x * kk + e] = acc[q];
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) last = atomicAdd(counter, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int e = tid; e < kk; e += WT) {
    double v = 0.0;
    for (int g = 0; g < (int)gridDim.x; ++g) v += partial[(int64_t)g * kk + e];
    X[e] = v;                                     // X = V_low U_up (col-major k x k)
  }
  __syncthreads();
  double* Y = partial;                            // Y = S_low X, over the partials (all read above)
  for (int e = tid; e < kk; e += WT) {
    const int rr = e % k, cc = e / k;
    double v = 0.0;
    for (int q = 0; q < k; ++q) v += Sl[rr + q * k] * X[q + cc * k];
    Y[e] = v;
  }
  __syncthreads();
  for (int e = tid; e < kk; e += WT) {            // S' = -(Y S_up)
    const int rr = e % k, cc = e / k;
    double v = 0.0;
    for (int q = 0; q < k; ++q) v += Y[rr + q * k] * Su[q + cc * k];
    Sp[e] = -v;
  }
  if (tid == 0) *counter = 0;
}

// Uinv^T of one leaf (b x b), for the transposed substitution.
__global__ void k_h_transpose(int b, const double* A, double* At) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)b * b;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = e % b, j = e / b;
    At[j + (int64_t)i * b] = A[e];
  }
}

// Dense leaves of A_H: D[p] = K(rows of p, cols of p).
__global__ void k_h_build_leaves(KernelDesc K, int b, int P, double* D) {
  const int64_t tot = (int64_t)P * b * b;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = e / ((int64_t)b * b);
    const int r = (int)(e % b), c = (int)((e / b) % b);
    D[e] = kernel_eval(K, p * b + r, p * b + c);
  }
}

// Z (s x p) = K(R, C) W for every block c of a level (blockIdx.y): R the
// rows of cluster c, C the rows of its sibling (swap = 0), or the two
// exchanged (swap = 1, the transposed product K(C, R) of an off-diagonal
// block, used for Q^T A).  The kernel is evaluated tile by tile, never
// stored.  W, Z: ld s, block stride s p.
__global__ void __launch_bounds__(WT) k_h_kgemm(KernelDesc K, int64_t s, int p, int swap, const double* W,
                                                double* Z) {
  __shared__ double Ks[64][33];
  __shared__ double Ws[32][KG_P];
  const int c = blockIdx.y;
  const int64_t R0 = (int64_t)(swap ? (c ^ 1) : c) * s, C0 = (int64_t)(swap ? c : (c ^ 1)) * s;
  const double* Wc = W + (int64_t)c * s * p;
  double* Zc = Z + (int64_t)c * s * p;
  const int64_t r0 = (int64_t)blockIdx.x * 64;
  const int tid = threadIdx.x, row = tid & 63, g = tid >> 6;
  const int rn = (int)min((int64_t)64, s - r0);
  double acc[KG_P / 4];
#pragma unroll
  for (int u = 0; u < KG_P / 4; ++u) acc[u] = 0.0;
  for (int64_t t0 = 0; t0 < s; t0 += 32) {
    const int tn = (int)min((int64_t)32, s - t0);
    for (int e = tid; e < 64 * 32; e += WT) {
      const int i = e % 64, t = e / 64;
      Ks[i][t] = (i < rn && t < tn) ? kernel_eval(K, R0 + r0 + i, C0 + t0 + t) : 0.0;
    }
    for (int e = tid; e < 32 * p; e += WT) {
      const int t = e % 32, j = e / 32;
      Ws[t][j] = t < tn ? Wc[(t0 + t) + (int64_t)j * s] : 0.0;
    }
    __syncthreads();
    for (int t = 0; t < 32; ++t) {
      const double kv = Ks[row][t];
#pragma unroll
      for (int u = 0; u < KG_P / 4; ++u) {
        const int j = g + 4 * u;
        if (j < p) acc[u] += kv * Ws[t][j];
      }
    }
    __syncthreads();
  }
  if (row < rn) {
#pragma unroll
    for (int u = 0; u < KG_P / 4; ++u) {
      const int j = g + 4 * u;
      if (j < p) Zc[(r0 + row) + (int64_t)j * s] = acc[u];
    }
  }
}

// Omega of every block of a level (s x p row-major, the reference's fill
// order) to the column-major W the product reads.
__global__ void k_h_omega(int64_t s, int p, int nblk, const double* om, double* W) {
  const int64_t tot = (int64_t)nblk * s * p;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % s, j = (e / s) % p;
    W[e] = om[i * p + j];
  }
}

// After the SVD Z = K(C, R) Q = U2 diag(sv) Vt2 (Q^T A = Vt2^T diag(sv)
// U2^T): V (k x s, ld k) = U2(:, :k)^T and S = diag(sv(:k)) of every block
// of a level.
__global__ void k_h_finish_v(int64_t s, int p, int k, int nblk, const double* U2, const double* sv, double* V,
                             double* S) {
  const int64_t totv = (int64_t)nblk * s * k;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < totv; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / (s * k), rem = e % (s * k);
    const int64_t rr = rem % k, i = rem / k;
    V[e] = U2[c * s * p + i + rr * s];
  }
  const int64_t tots = (int64_t)nblk * k * k;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tots; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / ((int64_t)k * k), rem = e % ((int64_t)k * k);
    const int rr = (int)(rem % k), cc = (int)(rem / k);
    S[e] = rr == cc ? sv[c * p + rr] : 0.0;
  }
}

constexpr int MV_CHUNK = 1024;

// Level-parallel solve.  With W_X = M_right(U_low) and Z_X = U_left^{-1} U_up
// precomputed per node X (M = the permuted forward substitution of a
// subtree), L^{-1} P b and U^{-1} y are: every leaf at once, then for each
// level from the bottom up, every node at once: x_right -= W_X S_low V_low
// x_left (forward), x_left -= Z_X S_up V_up x_right (backward).
//
// Leaves: x_p <- Linv_p P_p x_p (mode 0) or Uinv_p x_p (mode 2); grid: leaves x
// column groups of WCW.
__global__ void __launch_bounds__(WT) k_h_leaf_apply(int b, int mode, LeafFactors f, double* x, int64_t ldx,
                                                     int nrhs) {
  __shared__ double r[WCW][HMAX_LEAF];
  const int p = blockIdx.x, c0 = blockIdx.y * WCW;
  const int nc = min(WCW, nrhs - c0);
  const int* perm = f.perm + (int64_t)p * b;
  double* xp = x + (int64_t)p * b + (int64_t)c0 * ldx;
  for (int e = threadIdx.x; e < WCW * b; e += WT) {
    const int c = e / b, i = e % b;
    r[c][i] = c < nc ? xp[(mode == 0 ? perm[i] : i) + c * ldx] : 0.0;
  }
  __syncthreads();
  const double* Op = (mode == 0 ? f.Linv : f.Uinv) + (int64_t)p * b * b;
  for (int i = threadIdx.x; i < b; i += WT) {
    double acc[WCW];
#pragma unroll
    for (int c = 0; c < WCW; ++c) acc[c] = mode == 0 ? r[c][i] : 0.0;
    const int j0 = mode == 0 ? 0 : i, j1 = mode == 0 ? i : b;
#pragma unroll 8
    for (int j = j0; j < j1; ++j) {
      const double a = Op[i + (int64_t)j * b];
#pragma unroll
      for (int c = 0; c < WCW; ++c) acc[c] += a * r[c][j];
    }
    for (int c = 0; c < nc; ++c) xp[i + c * ldx] = acc[c];
  }
}

// Partials T[node][chunk] (k x nrhs) = V_c(:, chunk) x(cols of c, chunk) for
// the blocks c = 2 node + parity of level l (grid: chunks x nodes).
__global__ void __launch_bounds__(WT) k_h_sv_t(HView h, int l, int parity, const double* x, int64_t ldx, int nrhs,
                                               double* part) {
  __shared__ double red[WT / 32][HMAX_RANK];
  const int node = blockIdx.y, c = 2 * node + parity, k = h.k;
  const int64_t sl = h.s(l);
  const int nch = (int)((sl + MV_CHUNK - 1) / MV_CHUNK);
  const int64_t i0 = (int64_t)blockIdx.x * MV_CHUNK, i1 = min(sl, i0 + MV_CHUNK);
  const double* Vb = h.v(l, c);
  const int64_t col0 = (int64_t)(c ^ 1) * sl;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int q = 0; q < nrhs; ++q) {
    double acc[2] = {0.0, 0.0};
    for (int64_t i = i0 + wid; i < i1; i += WT / 32) {
      const double xv = x[col0 + i + q * ldx];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int rr = lane + 32 * t;
        if (rr < k) acc[t] += Vb[rr + i * k] * xv;
      }
    }
#pragma unroll
    for (int t = 0; t < 2; ++t)
      if (lane + 32 * t < k) red[wid][lane + 32 * t] = acc[t];
    __syncthreads();
    for (int rr = threadIdx.x; rr < k; rr += WT) {
      double v = 0.0;
      for (int w = 0; w < WT / 32; ++w) v += red[w][rr];
      part[(((int64_t)node * nch + blockIdx.x) * nrhs + q) * k + rr] = v;
    }
    __syncthreads();
  }
}

// x(rows of c) -= WZ_c S_c sum_chunks T[node][chunk], c = 2 node + parity
// (grid: row tiles x nodes); hw.U addresses the W / Z slab, hw.S the factor's S.
__global__ void __launch_bounds__(WT) k_h_sv_u(HView hw, int l, int parity, int nrhs, const double* part, double* x,
                                               int64_t ldx) {
  __shared__ double t1[HMAX_RANK];
  __shared__ double t2[HMAX_RANK];
  const int node = blockIdx.y, c = 2 * node + parity, k = hw.k;
  const int64_t sl = hw.s(l);
  const int nch = (int)((sl + MV_CHUNK - 1) / MV_CHUNK);
  const double* Wb = hw.u(l, c);
  const double* Sb = hw.sm(l, c);
  const int64_t row0 = (int64_t)c * sl;
  const int64_t i = (int64_t)blockIdx.x * WT + threadIdx.x;
  for (int q = 0; q < nrhs; ++q) {
    for (int rr = threadIdx.x; rr < k; rr += WT) {
      double v = 0.0;
      for (int g = 0; g < nch; ++g) v += part[(((int64_t)node * nch + g) * nrhs + q) * k + rr];
      t1[rr] = v;
    }
    __syncthreads();
    for (int rr = threadIdx.x; rr < k; rr += WT) {
      double v = 0.0;
      for (int t = 0; t < k; ++t) v += Sb[rr + t * k] * t1[t];
      t2[rr] = v;
    }
    __syncthreads();
    if (i < sl) {
      double v = 0.0;
      for (int t = 0; t < k; ++t) v += Wb[i + (int64_t)t * sl] * t2[t];
      x[row0 + i + q * ldx] -= v;
    }
    __syncthreads();
  }
}

// y_p = D_p x_p for every leaf (grid: leaves), nrhs columns.
__global__ void __launch_bounds__(WT) k_h_mv_leaf(int b, const double* D, const double* x, int64_t ldx, double* y,
                                                  int64_t ldy, int nrhs) {
  __shared__ double xs[HMAX_LEAF];
  const int p = blockIdx.x;
  const double* Dp = D + (int64_t)p * b * b;
  for (int c = 0; c < nrhs; ++c) {
    for (int i = threadIdx.x; i < b; i += WT) xs[i] = x[(int64_t)p * b + i + c * ldx];
    __syncthreads();
    for (int i = threadIdx.x; i < b; i += WT) {
      double v = 0.0;
      for (int j = 0; j < b; ++j) v += Dp[i + (int64_t)j * b] * xs[j];
      y[(int64_t)p * b + i + c * ldy] = v;
    }
    __syncthreads();
  }
}

// Partials T[c][chunk] (k x nrhs) = V_c(:, chunk) x(cols of c, chunk) of one
// level (grid: chunks x blocks).
__global__ void __launch_bounds__(WT) k_h_mv_t(HView h, int l, const double* x, int64_t ldx, int nrhs,
                                               double* part) {
  __shared__ double red[WT / 32][HMAX_RANK];
  const int c = blockIdx.y, k = h.k;
  const int64_t sl = h.s(l);
  const int nch = (int)((sl + MV_CHUNK - 1) / MV_CHUNK);
  const int64_t i0 = (int64_t)blockIdx.x * MV_CHUNK, i1 = min(sl, i0 + MV_CHUNK);
  const double* Vb = h.v(l, c);
  const int64_t col0 = (int64_t)(c ^ 1) * sl;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int q = 0; q < nrhs; ++q) {
    double acc[2] = {0.0, 0.0};
    for (int64_t i = i0 + wid; i < i1; i += WT / 32) {
      const double xv = x[col0 + i + q * ldx];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int rr = lane + 32 * t;
        if (rr < k) acc[t] += Vb[rr + i * k] * xv;
      }
    }
#pragma unroll
    for (int t = 0; t < 2; ++t)
      if (lane + 32 * t < k) red[wid][lane + 32 * t] = acc[t];
    __syncthreads();
    for (int rr = threadIdx.x; rr < k; rr += WT) {
      double v = 0.0;
      for (int w = 0; w < WT / 32; ++w) v += red[w][rr];
      part[(((int64_t)c * nch + blockIdx.x) * nrhs + q) * k + rr] = v;
    }
    __syncthreads();
  }
}

// y(rows of c) += U_c S_c sum_chunks T[c][chunk] (grid: row tiles x blocks).
__global__ void __launch_bounds__(WT) k_h_mv_u(HView h, int l, int nrhs, const double* part, double* y, int64_t ldy) {
  __shared__ double t1[HMAX_RANK];
  __shared__ double t2[HMAX_RANK];
  const int c = blockIdx.y, k = h.k;
  const int64_t sl = h.s(l);
  const int nch = (int)((sl + MV_CHUNK - 1) / MV_CHUNK);
  const double* Ub = h.u(l, c);
  const double* Sb = h.sm(l, c);
  const int64_t row0 = (int64_t)c * sl;
  const int64_t i = (int64_t)blockIdx.x * WT + threadIdx.x;
  for (int q = 0; q < nrhs; ++q) {
    for (int rr = threadIdx.x; rr < k; rr += WT) {
      double v = 0.0;
      for (int g = 0; g < nch; ++g) v += part[(((int64_t)c * nch + g) * nrhs + q) * k + rr];
      t1[rr] = v;
    }
    __syncthreads();
    for (int rr = threadIdx.x; rr < k; rr += WT) {
      double v = 0.0;
      for (int t = 0; t < k; ++t) v += Sb[rr + t * k] * t1[t];
      t2[rr] = v;
    }
    __syncthreads();
    if (i < sl) {
      double v = 0.0;
      for (int t = 0; t < k; ++t) v += Ub[i + (int64_t)t * sl] * t2[t];
      y[row0 + i + q * ldy] += v;
    }
    __syncthreads();
  }
}

// r = b - y (in y), column sums of squares of r and b into nrm[2 c], nrm[2 c + 1]
// (one CTA per column, fixed reduction order).
__global__ void __launch_bounds__(WT) k_h_residual(int64_t n, const double* bb, int64_t ldb, double* y, int64_t ldy,
                                                   double* nrm) {
  __shared__ double red[2][WT / 32];
  const int c = blockIdx.x;
  double sr = 0.0, sb = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += WT) {
    const double bv = bb[i + c * ldb];
    const double rv = bv - y[i + c * ldy];
    y[i + c * ldy] = rv;
    sr += rv * rv;
    sb += bv * bv;
  }
  sr = blr::warp_sum(sr);
  sb = blr::warp_sum(sb);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = sr;
    red[1][threadIdx.x >> 5] = sb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, d = 0.0;
    for (int w = 0; w < WT / 32; ++w) { a += red[0][w]; d += red[1][w]; }
    nrm[2 * c] = a;
    nrm[2 * c + 1] = d;
  }
}

// x += d
__global__ void k_h_axpy(int64_t n, int nrhs, const double* d, int64_t ldd, double* x, int64_t ldx) {
  const int64_t tot = n * nrhs;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % n, c = e / n;
    x[i + c * ldx] += d[i + c * ldd];
  }
}

}  // namespace hk
}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

struct frank_hodlr {
  int64_t n = 0;
  int b = 0, L = 0, k = 0, P = 0;
  int fast = 1;                     // fast_rounded_addition (1) or rounded_addition (0)
  int sm_count = 148;
  cudaStream_t s = nullptr;         // capture stream
  double *D0 = nullptr, *U0 = nullptr, *S0 = nullptr, *V0 = nullptr;
  double *D = nullptr, *U = nullptr, *S = nullptr, *V = nullptr;
  double *Linv = nullptr, *Uinv = nullptr, *UinvT = nullptr;
  int *perm = nullptr, *ipiv = nullptr;
  double* getrf_scratch = nullptr;
  int* geom = nullptr;              // leaf BlrView geometry: off {0, b}, dslot {0}, lslot {-1}
  unsigned long long* flops = nullptr;
  int* err = nullptr;
  int* kfill = nullptr;             // [L + 1][P] ranks, all k (one row per level's stream)
  int* counter = nullptr;
  double* Sp = nullptr;             // S' of every internal node's update ([2^L - 1][k x k])
  double* core_part = nullptr;      // [CORE_GRID][k*k]
  double* Wu = nullptr;             // U_low S' (n/2 x k)
  double* lr_scratch = nullptr;     // addition scratch, one region per level
  int64_t lr_cap = 0;
  std::vector<int64_t> lr_base;     // [L + 1] start of level j's region
  std::vector<cudaStream_t> ls;     // [L + 1] one stream per level for the LowRank additions
  std::vector<cudaEvent_t> lev;     // [L + 1] last addition enqueued on level j's stream
  cudaEvent_t ev_fork = nullptr, ev_core = nullptr;
  double* WZ = nullptr;             // per node: W (lower block's slot) and Z (upper block's slot), U-shaped
  cudaStream_t ps = nullptr;        // their walks, beside the factorization
  cudaEvent_t ev_pre = nullptr, ev_ps = nullptr;
  ::frank::ops::LrAddTask* tasks_d = nullptr;   // every update's additions, in launch order
  std::vector<::frank::ops::LrAddTask> tasks_h;
  int64_t ntasks_cap = 0;
  int lr_shm = 0;
  double* mv_part = nullptr;
  int64_t mv_part_cap = 0;
  double* work = nullptr;           // refinement: residual / correction (n x nrhs)
  int64_t work_cap = 0;
  double* nrm = nullptr;            // 2 x nrhs
  cudaGraphExec_t gexec = nullptr;
  bool have_A = false, factored = false;
  int64_t launches = 0;
  float factor_ms = 0.f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};

namespace {

constexpr int CORE_GRID = 64;

#define H_TRY(expr)                                                                                         \
  do {                                                                                                      \
    cudaError_t _e = (expr);                                                                                \
    if (_e != cudaSuccess)                                                                                  \
      return ::frank::set_error(FRANK_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));        \
  } while (0)

int hfail(int code, const std::string& msg) { return ::frank::set_error(code, msg); }

int64_t s_of(const frank_hodlr* h, int l) { return h->n >> l; }
int64_t u_off(const frank_hodlr* h, int l, int c) { return (int64_t)(l - 1) * h->n * h->k + (int64_t)c * s_of(h, l) * h->k; }
int64_t s_off(const frank_hodlr* h, int l, int c) { return ((int64_t)(1 << l) - 2 + c) * h->k * h->k; }
int64_t nblocks_s(const frank_hodlr* h) { return ((int64_t)1 << (h->L + 1)) - 2; }

hk::HView view(const frank_hodlr* h, bool factor) {
  hk::HView v;
  v.n = h->n;
  v.b = h->b;
  v.L = h->L;
  v.k = h->k;
  v.D = factor ? h->D : h->D0;
  v.U = factor ? h->U : h->U0;
  v.S = factor ? h->S : h->S0;
  v.V = factor ? h->V : h->V0;
  return v;
}

hk::LeafFactors leaf_factors(const frank_hodlr* h) {
  return hk::LeafFactors{h->Linv, h->Uinv, h->UinvT, h->perm};
}

// leaf p as a one-block BlrView for the BLR engine's leaf LU and inverse kernels
void leaf_view(const frank_hodlr* h, int p, blr::BlrView<double>& A, blr::FactorWs<double>& ws) {
  A.nb = 1;
  A.bmax = h->b;
  A.kcap = 0;
  A.off = h->geom;
  A.dslot = h->geom + 2;
  A.lslot = h->geom + 3;
  A.rank = nullptr;
  A.D = h->D + (int64_t)p * h->b * h->b;
  A.U = A.S = A.Vt = nullptr;
  std::memset(&ws, 0, sizeof(ws));
  ws.perm = h->perm + (int64_t)p * h->b;
  ws.ipiv = h->ipiv + (int64_t)p * h->b;
  ws.Linv = h->Linv + (int64_t)p * h->b * h->b;
  ws.Uinv = h->Uinv + (int64_t)p * h->b * h->b;
  ws.getrf_scratch = h->getrf_scratch;
  ws.err = h->err;
  ws.flops = h->flops;
}

void enqueue_leaf(frank_hodlr* h, int p, cudaStream_t s) {
  blr::BlrView<double> A;
  blr::FactorWs<double> ws;
  leaf_view(h, p, A, ws);
  const int b = h->b;
  blr::k_getrf_load<double><<<64, blr::GETRF_AUX_THREADS, 0, s>>>(A, ws, 0);
  ++h->launches;
  for (int jb = 0; jb < b; jb += 32) {
    blr::k_getrf_panel<double><<<1, blr::GETRF_THREADS, 0, s>>>(A, ws, 0, jb);
    ++h->launches;
    const int m2 = b - jb - std::min(32, b - jb);
    if (m2 > 0) {
      const int nt = (m2 + 63) / 64;
      blr::k_getrf_trail<double><<<nt * nt, blr::GETRF_AUX_THREADS, 0, s>>>(A, ws, 0, jb);
      ++h->launches;
    }
  }
  blr::k_getrf_store<double><<<64, blr::GETRF_AUX_THREADS, 0, s>>>(A, ws, 0);
  const int cw = blr::trinv_width(b);
  const int nblk = (b + cw - 1) / cw;
  blr::k_trinv<double><<<2 * nblk, blr::TRINV_THREADS, (size_t)b * cw * sizeof(double), s>>>(A, ws, 0, cw);
  hk::k_h_transpose<<<64, 256, 0, s>>>(b, ws.Uinv, h->UinvT + (int64_t)p * b * b);
  h->launches += 3;
}

// LowRank(U_x, S'_node, V_x) (n_node x n_node, U_x ld s(lr), V_x ld k) added
// into node (lr, cr) of the working copy: the dense leaves on stream s, the
// LowRank blocks of each level j on that level's stream (after the node's
// core, event ev_core), so that the additions into blocks needed late (the
// large ones near the top of the node) run beside the factorization of the
// node's first children.
void enqueue_update(frank_hodlr* h, int lr, int cr, const double* Ux, const double* Vx, const double* Sp,
                    cudaStream_t s) {
  const int k = h->k, b = h->b;
  const int64_t sn = s_of(h, lr);
  // Wu = U_x S'
  ::frank::ops::launch_gemm(s, (int)sn, k, k, 1, 1.0, Ux, sn, 0, false, Sp, k, 0, false, 0.0, h->Wu, sn, 0);
  // dense leaves of the node: D_p += Wu(rows of p) V_x(:, cols of p)
  const int nleaf = 1 << (h->L - lr);
  const int pf = cr << (h->L - lr);
  ::frank::ops::launch_gemm(s, b, b, k, nleaf, 1.0, h->Wu, sn, b, false, Vx, k, (int64_t)b * k, false, 1.0,
                            h->D + (int64_t)pf * b * b, b, (int64_t)b * b);
  h->launches += 2;
  // LowRank blocks of the node, one launch per level from the task table
  for (int j = lr + 1; j <= h->L; ++j) {
    const int64_t sj = s_of(h, j);
    const int cbase = cr << (j - lr);
    const int64_t t0 = (int64_t)h->tasks_h.size();
    int64_t off = 0;
    int idx = 0;
    for (int c = cbase; c < cbase + (1 << (j - lr)); ++c, ++idx) {
      ::frank::ops::LrAddTask t;
      t.ua = h->U + u_off(h, j, c);
      t.sa = h->S + s_off(h, j, c);
      t.va = h->V + u_off(h, j, c);
      t.ub = Ux + (int64_t)(c - cbase) * sj;                    // rows of cluster c within the node
      t.sb = Sp;
      t.vb = Vx + (int64_t)((c ^ 1) - cbase) * sj * k;          // columns of its sibling
      t.ldua = sj; t.ldsa = k; t.ldva = k; t.ldub = sn; t.ldsb = k; t.ldvb = k;
      t.scratch_off = h->lr_base[j] + off;
      t.ka = h->kfill + (int64_t)j * h->P + idx;
      t.kb = t.ka;
      t.m = t.n = (int)sj;
      h->tasks_h.push_back(t);
      off += ::frank::ops::lr_add_ws((int)sj, (int)sj, k, k);
    }
    cudaStream_t sj_stream = h->ls[j];
    cudaStreamWaitEvent(sj_stream, h->ev_core, 0);
    ::frank::ops::launch_lr_add_tasks(sj_stream, idx, h->tasks_d + t0, k, h->fast, h->lr_scratch,
                                      h->err + hk::HERR_JACOBI, h->lr_shm);
    cudaEventRecord(h->lev[j], sj_stream);
    ++h->launches;
  }
}

// WZ(l, c) <- the substitution (mode 0: L with pivots, 2: U) of cluster
// (l, c)'s subtree applied to the U factor of block (l, c), on stream ps after
// everything enqueued so far on s.
void enqueue_precompute(frank_hodlr* h, int l, int c, int mode, cudaStream_t s) {
  const int k = h->k;
  const int64_t sl = s_of(h, l);
  cudaEventRecord(h->ev_pre, s);
  cudaStreamWaitEvent(h->ps, h->ev_pre, 0);
  cudaMemcpyAsync(h->WZ + u_off(h, l, c), h->U + u_off(h, l, c), sizeof(double) * sl * k, cudaMemcpyDeviceToDevice,
                  h->ps);
  hk::Walk j0{mode, l, c, k, h->WZ + u_off(h, l, c), 1, sl}, none{0, 0, 0, 0, nullptr, 1, 1};
  hk::k_h_walk<<<dim3((k + hk::WCW - 1) / hk::WCW, 1), hk::WWT, hk::WALK_SMEM, h->ps>>>(view(h, true),
                                                                                       leaf_factors(h), j0, none);
  ++h->launches;
}

void enqueue_node(frank_hodlr* h, int l, int c, cudaStream_t s) {
  if (l == h->L) {
    enqueue_leaf(h, c, s);
    return;
  }
  const int k = h->k;
  enqueue_node(h, l + 1, 2 * c, s);
  const int up = 2 * c, lo = 2 * c + 1;
  const int64_t sc = s_of(h, l + 1);
  // the node's own off-diagonal blocks: every addition into them enqueued so far
  cudaStreamWaitEvent(s, h->lev[l + 1], 0);
  // U_up <- L_left^{-1} P U_up (trsm.cpp:106-115 -> 117-125 -> leaves);
  // V_low <- V_low U_left^{-1}
  hk::Walk j0{0, l + 1, 2 * c, k, h->U + u_off(h, l + 1, up), 1, sc};
  hk::Walk j1{1, l + 1, 2 * c, k, h->V + u_off(h, l + 1, lo), k, 1};
  hk::k_h_walk<<<dim3((k + hk::WCW - 1) / hk::WCW, 2), hk::WWT, hk::WALK_SMEM, s>>>(view(h, true), leaf_factors(h),
                                                                                   j0, j1);
  // for the level-parallel solve, beside the factorization: Z = U_left^{-1} U_up
  enqueue_precompute(h, l + 1, up, 2, s);
  // S' = -(S_low V_low)(U_up S_up), one k x k slot per internal node
  double* Sp = h->Sp + ((int64_t)(1 << l) - 1 + c) * k * k;
  const int grid = (int)std::min<int64_t>(CORE_GRID, (sc + 511) / 512);
  hk::k_h_core<<<grid, hk::WT, 0, s>>>(sc, k, h->V + u_off(h, l + 1, lo), h->U + u_off(h, l + 1, up),
                                       h->S + s_off(h, l + 1, lo), h->S + s_off(h, l + 1, up), h->core_part, Sp,
                                       h->counter);
  cudaEventRecord(h->ev_core, s);
  h->launches += 2;
  enqueue_update(h, l + 1, lo, h->U + u_off(h, l + 1, lo), h->V + u_off(h, l + 1, up), Sp, s);
  enqueue_node(h, l + 1, 2 * c + 1, s);
  // W = M_right(U_low), once the right child is factored
  enqueue_precompute(h, l + 1, lo, 0, s);
}

int enqueue_factor(frank_hodlr* h, cudaStream_t s) {
  const int64_t nk = (int64_t)h->L * h->n * h->k;
  H_TRY(cudaMemcpyAsync(h->D, h->D0, sizeof(double) * (size_t)h->P * h->b * h->b, cudaMemcpyDeviceToDevice, s));
  H_TRY(cudaMemcpyAsync(h->U, h->U0, sizeof(double) * (size_t)nk, cudaMemcpyDeviceToDevice, s));
  H_TRY(cudaMemcpyAsync(h->V, h->V0, sizeof(double) * (size_t)nk, cudaMemcpyDeviceToDevice, s));
  H_TRY(cudaMemcpyAsync(h->S, h->S0, sizeof(double) * (size_t)nblocks_s(h) * h->k * h->k, cudaMemcpyDeviceToDevice, s));
  H_TRY(cudaMemsetAsync(h->err, 0, sizeof(int) * hk::HERR_SLOTS, s));
  h->launches = 0;
  h->tasks_h.clear();
  H_TRY(cudaEventRecord(h->ev_fork, s));
  H_TRY(cudaStreamWaitEvent(h->ps, h->ev_fork, 0));
  for (int j = 1; j <= h->L; ++j) {
    H_TRY(cudaStreamWaitEvent(h->ls[j], h->ev_fork, 0));
    H_TRY(cudaEventRecord(h->lev[j], h->ls[j]));
  }
  enqueue_node(h, 0, 0, s);
  for (int j = 1; j <= h->L; ++j) {
    H_TRY(cudaEventRecord(h->lev[j], h->ls[j]));
    H_TRY(cudaStreamWaitEvent(s, h->lev[j], 0));
  }
  H_TRY(cudaEventRecord(h->ev_ps, h->ps));
  H_TRY(cudaStreamWaitEvent(s, h->ev_ps, 0));
  H_TRY(cudaGetLastError());
  return FRANK_OK;
}

int check_errors(frank_hodlr* h, cudaStream_t s) {
  int e[hk::HERR_SLOTS];
  H_TRY(cudaMemcpyAsync(e, h->err, sizeof(e), cudaMemcpyDeviceToHost, s));
  H_TRY(cudaStreamSynchronize(s));
  if (e[blr::ERR_SINGULAR_STEP]) return hfail(FRANK_ERR_SINGULAR, "a leaf getrf met a zero pivot");
  if (e[hk::HERR_JACOBI]) return hfail(FRANK_ERR_NOT_CONVERGED, "one-sided Jacobi reached its sweep limit");
  if (e[hk::HERR_RANK]) return hfail(FRANK_ERR_RANK_OVERFLOW, "a recompressed rank exceeded the fixed rank");
  return FRANK_OK;
}

void free_plan(frank_hodlr* h) {
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  for (void* p : {(void*)h->D0, (void*)h->U0, (void*)h->S0, (void*)h->V0, (void*)h->D, (void*)h->U, (void*)h->S,
                  (void*)h->V, (void*)h->Linv, (void*)h->Uinv, (void*)h->UinvT, (void*)h->perm, (void*)h->ipiv,
                  (void*)h->getrf_scratch, (void*)h->geom, (void*)h->flops, (void*)h->err, (void*)h->kfill,
                  (void*)h->counter, (void*)h->Sp, (void*)h->core_part, (void*)h->Wu, (void*)h->lr_scratch,
                  (void*)h->mv_part, (void*)h->work, (void*)h->nrm, (void*)h->tasks_d})
    if (p) cudaFree(p);
  if (h->e0) cudaEventDestroy(h->e0);
  if (h->e1) cudaEventDestroy(h->e1);
  for (cudaStream_t x : h->ls) if (x) cudaStreamDestroy(x);
  for (cudaEvent_t x : h->lev) if (x) cudaEventDestroy(x);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_core) cudaEventDestroy(h->ev_core);
  if (h->ev_pre) cudaEventDestroy(h->ev_pre);
  if (h->ev_ps) cudaEventDestroy(h->ev_ps);
  if (h->ps) cudaStreamDestroy(h->ps);
  if (h->WZ) cudaFree(h->WZ);
  if (h->s) cudaStreamDestroy(h->s);
  delete h;
}

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
  return cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * std::max<size_t>(count, 1));
}

int check_block(const frank_hodlr* h, int l, int c) {
  if (!h) return hfail(FRANK_ERR_INVALID, "null H-matrix");
  if (l < 1 || l > h->L || c < 0 || c >= (1 << l)) return hfail(FRANK_ERR_INVALID, "no such LowRank block");
  return FRANK_OK;
}

int ensure_mv(frank_hodlr* h, int nrhs) {
  // the partials of one level at a time: 2^l blocks x chunks x nrhs x k
  int64_t need = 0;
  for (int l = 1; l <= h->L; ++l)
    need = std::max(need, ((int64_t)1 << l) * ((s_of(h, l) + hk::MV_CHUNK - 1) / hk::MV_CHUNK) * nrhs * h->k);
  if (need > h->mv_part_cap) {
    if (h->mv_part) cudaFree(h->mv_part);
    h->mv_part = nullptr;
    H_TRY(dalloc(&h->mv_part, (size_t)need));
    h->mv_part_cap = need;
  }
  return FRANK_OK;
}

// y = A_H x (FP64), stream-ordered.
int enqueue_matvec(frank_hodlr* h, const double* x, int64_t ldx, double* y, int64_t ldy, int nrhs, cudaStream_t s) {
  int rc = ensure_mv(h, nrhs);
  if (rc) return rc;
  const hk::HView v = view(h, false);
  hk::k_h_mv_leaf<<<h->P, hk::WT, 0, s>>>(h->b, h->D0, x, ldx, y, ldy, nrhs);
  for (int l = 1; l <= h->L; ++l) {
    const int64_t sl = s_of(h, l);
    const int nch = (int)((sl + hk::MV_CHUNK - 1) / hk::MV_CHUNK);
    hk::k_h_mv_t<<<dim3(nch, 1 << l), hk::WT, 0, s>>>(v, l, x, ldx, nrhs, h->mv_part);
    hk::k_h_mv_u<<<dim3((unsigned)((sl + hk::WT - 1) / hk::WT), 1 << l), hk::WT, 0, s>>>(v, l, nrhs, h->mv_part, y,
                                                                                          ldy);
  }
  H_TRY(cudaGetLastError());
  return FRANK_OK;
}

// passes: 1 = forward (L with the pivots), 2 = backward (U), 3 = both.
int enqueue_solve(frank_hodlr* h, double* d_b, int64_t ldb, int nrhs, cudaStream_t s, int passes = 3) {
  int rc = ensure_mv(h, nrhs);
  if (rc) return rc;
  const hk::HView v = view(h, true);
  hk::HView vw = v;
  vw.U = h->WZ;
  const hk::LeafFactors f = leaf_factors(h);
  const dim3 gleaf(h->P, (nrhs + hk::WCW - 1) / hk::WCW);
  for (int pass = 0; pass < 2; ++pass) {
    if (!(passes & (1 << pass))) continue;
    // forward: leaves with L and pivots, then lower blocks (odd); backward:
    // leaves with U, then upper blocks (even)
    hk::k_h_leaf_apply<<<gleaf, hk::WT, 0, s>>>(h->b, pass == 0 ? 0 : 2, f, d_b, ldb, nrhs);
    const int parity = pass == 0 ? 1 : 0;
    for (int l = h->L; l >= 1; --l) {
      const int64_t sl = s_of(h, l);
      const int nch = (int)((sl + hk::MV_CHUNK - 1) / hk::MV_CHUNK);
      const int nodes = 1 << (l - 1);
      hk::k_h_sv_t<<<dim3(nch, nodes), hk::WT, 0, s>>>(v, l, parity, d_b, ldb, nrhs, h->mv_part);
      hk::k_h_sv_u<<<dim3((unsigned)((sl + hk::WT - 1) / hk::WT), nodes), hk::WT, 0, s>>>(vw, l, parity, nrhs,
                                                                                           h->mv_part, d_b, ldb);
    }
  }
  H_TRY(cudaGetLastError());
  return FRANK_OK;
}

}  // namespace

extern "C" {

int frank_hodlr_create(int64_t n, int leaf, int rank, frank_hodlr** out) {
  if (!out) return hfail(FRANK_ERR_INVALID, "null output pointer");
  *out = nullptr;
  if (leaf < 8 || leaf > hk::HMAX_LEAF || n < 2 * (int64_t)leaf || n % leaf)
    return hfail(FRANK_ERR_INVALID, "H-matrix: need 8 <= leaf <= 512 and n a multiple of leaf, n >= 2 leaf");
  int64_t P = n / leaf;
  int L = 0;
  while (((int64_t)1 << L) < P) ++L;
  if (((int64_t)1 << L) != P || L > 20)
    return hfail(FRANK_ERR_UNSUPPORTED, "H-matrix: n / leaf must be a power of two (binary cluster tree)");
  if (rank < 1 || rank > hk::HMAX_RANK || rank > leaf)
    return hfail(FRANK_ERR_INVALID, "H-matrix: need 1 <= rank <= min(64, leaf)");
  frank_hodlr* h = new frank_hodlr();
  h->n = n;
  h->b = leaf;
  h->L = L;
  h->k = rank;
  h->P = (int)P;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, dev);
  const int64_t nk = (int64_t)L * n * rank, sk = nblocks_s(h) * rank * rank, dd = P * leaf * leaf;
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  A(dalloc(&h->D0, dd)); A(dalloc(&h->D, dd));
  A(dalloc(&h->U0, nk)); A(dalloc(&h->U, nk)); A(dalloc(&h->V0, nk)); A(dalloc(&h->V, nk));
  A(dalloc(&h->S0, sk)); A(dalloc(&h->S, sk));
  A(dalloc(&h->Linv, dd)); A(dalloc(&h->Uinv, dd)); A(dalloc(&h->UinvT, dd));
  A(dalloc(&h->perm, P * leaf)); A(dalloc(&h->ipiv, P * leaf));
  A(dalloc(&h->getrf_scratch, (size_t)leaf * leaf + 32 * leaf));
  A(dalloc(&h->geom, 4)); A(dalloc(&h->flops, blr::FLOP_SLOTS)); A(dalloc(&h->err, hk::HERR_SLOTS));
  A(dalloc(&h->kfill, (size_t)(L + 1) * P)); A(dalloc(&h->counter, 1));
  A(dalloc(&h->Sp, (size_t)P * rank * rank)); A(dalloc(&h->core_part, (size_t)CORE_GRID * rank * rank));
  A(dalloc(&h->Wu, (size_t)(n / 2) * rank));
  // LowRank additions: per level j a scratch region for its largest launch
  // (2^(j-1) blocks of order n >> j, the update of the root's right child),
  // and the task table of all updates
  int64_t cap = 0, ntask = 0;
  h->lr_base.assign(L + 2, 0);
  for (int j = 1; j <= L; ++j) {
    h->lr_base[j] = cap;
    if (j >= 2) cap += ((int64_t)1 << (j - 1)) * ::frank::ops::lr_add_ws((int)(n >> j), (int)(n >> j), rank, rank);
  }
  for (int lr = 1; lr <= L; ++lr) ntask += ((int64_t)1 << (lr - 1)) * (((int64_t)1 << (L - lr + 1)) - 2);
  if (cap > 0) A(dalloc(&h->lr_scratch, (size_t)cap));
  h->lr_cap = cap;
  h->ntasks_cap = ntask;
  A(cudaMalloc(reinterpret_cast<void**>(&h->tasks_d), sizeof(::frank::ops::LrAddTask) * std::max<int64_t>(ntask, 1)));
  h->ls.assign(L + 1, nullptr);
  h->lev.assign(L + 1, nullptr);
  for (int j = 0; j <= L; ++j) {
    A(cudaStreamCreateWithFlags(&h->ls[j], cudaStreamNonBlocking));
    A(cudaEventCreateWithFlags(&h->lev[j], cudaEventDisableTiming));
  }
  A(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
  A(cudaEventCreateWithFlags(&h->ev_core, cudaEventDisableTiming));
  A(cudaEventCreateWithFlags(&h->ev_pre, cudaEventDisableTiming));
  A(cudaEventCreateWithFlags(&h->ev_ps, cudaEventDisableTiming));
  A(cudaStreamCreateWithFlags(&h->ps, cudaStreamNonBlocking));
  A(dalloc(&h->WZ, (size_t)nk));
  h->lr_shm = ::frank::ops::lr_add_shm_bytes(rank, rank);
  A(cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking));
  A(cudaEventCreate(&h->e0));
  A(cudaEventCreate(&h->e1));
  if (e != cudaSuccess) {
    free_plan(h);
    return hfail(FRANK_ERR_CUDA, std::string("H-matrix allocation: ") + cudaGetErrorString(e));
  }
  const int geom[4] = {0, leaf, 0, -1};
  std::vector<int> kf((size_t)(L + 1) * P, rank);
  A(cudaMemcpy(h->geom, geom, sizeof(geom), cudaMemcpyHostToDevice));
  A(cudaMemcpy(h->kfill, kf.data(), sizeof(int) * kf.size(), cudaMemcpyHostToDevice));
  A(cudaMemset(h->counter, 0, sizeof(int)));
  A(cudaMemset(h->flops, 0, sizeof(unsigned long long) * blr::FLOP_SLOTS));
  A(cudaMemset(h->D0, 0, sizeof(double) * dd));
  A(cudaMemset(h->U0, 0, sizeof(double) * nk));
  A(cudaMemset(h->V0, 0, sizeof(double) * nk));
  A(cudaMemset(h->S0, 0, sizeof(double) * sk));
  A(cudaFuncSetAttribute(blr::k_trinv<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, blr::TRINV_SMEM_MAX));
  A(cudaFuncSetAttribute(hk::k_h_walk, cudaFuncAttributeMaxDynamicSharedMemorySize, hk::WALK_SMEM));
  if (e == cudaSuccess && h->lr_shm > 0 && ::frank::ops::lr_add_prepare(h->lr_shm) != FRANK_OK) h->lr_shm = 0;
  if (e != cudaSuccess) {
    free_plan(h);
    return hfail(FRANK_ERR_CUDA, std::string("H-matrix set-up: ") + cudaGetErrorString(e));
  }
  *out = h;
  return FRANK_OK;
}

int frank_hodlr_destroy(frank_hodlr* h) {
  if (h) {
    cudaDeviceSynchronize();
    free_plan(h);
  }
  return FRANK_OK;
}

int frank_hodlr_shape(const frank_hodlr* h, int64_t* n, int* leaf, int* rank, int* levels) {
  if (!h) return hfail(FRANK_ERR_INVALID, "null H-matrix");
  if (n) *n = h->n;
  if (leaf) *leaf = h->b;
  if (rank) *rank = h->k;
  if (levels) *levels = h->L;
  return FRANK_OK;
}

int frank_hodlr_set_lra(frank_hodlr* h, const char* name) {
  if (!h || !name) return hfail(FRANK_ERR_INVALID, "null argument");
  const std::string s(name);
  int fast;
  if (s == "fast_rounded_addition" || s.empty()) fast = 1;
  else if (s == "rounded_addition") fast = 0;
  else return hfail(FRANK_ERR_UNSUPPORTED, "H-matrix: LowRank addition must be fast_rounded_addition or rounded_addition");
  if (fast != h->fast && h->gexec) {
    cudaGraphExecDestroy(h->gexec);
    h->gexec = nullptr;
  }
  h->fast = fast;
  h->factored = false;
  return FRANK_OK;
}

int frank_hodlr_set_dense(frank_hodlr* h, int leaf, const double* a, int64_t ld) {
  if (!h || !a) return hfail(FRANK_ERR_INVALID, "null argument");
  if (leaf < 0 || leaf >= h->P || ld < h->b) return hfail(FRANK_ERR_INVALID, "bad leaf or leading dimension");
  H_TRY(cudaMemcpy2D(h->D0 + (int64_t)leaf * h->b * h->b, sizeof(double) * h->b, a, sizeof(double) * ld,
                     sizeof(double) * h->b, h->b, cudaMemcpyHostToDevice));
  h->have_A = true;
  h->factored = false;
  return FRANK_OK;
}

int frank_hodlr_set_lowrank(frank_hodlr* h, int level, int index, const double* u, const double* s,
                            const double* v) {
  int rc = check_block(h, level, index);
  if (rc) return rc;
  if (!u || !s || !v) return hfail(FRANK_ERR_INVALID, "null argument");
  const int64_t sl = s_of(h, level), k = h->k;
  H_TRY(cudaMemcpy(h->U0 + u_off(h, level, index), u, sizeof(double) * sl * k, cudaMemcpyHostToDevice));
  H_TRY(cudaMemcpy(h->V0 + u_off(h, level, index), v, sizeof(double) * sl * k, cudaMemcpyHostToDevice));
  H_TRY(cudaMemcpy(h->S0 + s_off(h, level, index), s, sizeof(double) * k * k, cudaMemcpyHostToDevice));
  h->have_A = true;
  h->factored = false;
  return FRANK_OK;
}

int frank_hodlr_get_dense(const frank_hodlr* h, int which, int leaf, double* a, int64_t ld) {
  if (!h || !a) return hfail(FRANK_ERR_INVALID, "null argument");
  if (leaf < 0 || leaf >= h->P || ld < h->b) return hfail(FRANK_ERR_INVALID, "bad leaf or leading dimension");
  const double* src = (which ? h->D : h->D0) + (int64_t)leaf * h->b * h->b;
  H_TRY(cudaMemcpy2D(a, sizeof(double) * ld, src, sizeof(double) * h->b, sizeof(double) * h->b, h->b,
                     cudaMemcpyDeviceToHost));
  return FRANK_OK;
}

int frank_hodlr_get_lowrank(const frank_hodlr* h, int which, int level, int index, double* u, double* s, double* v) {
  int rc = check_block(h, level, index);
  if (rc) return rc;
  const int64_t sl = s_of(h, level), k = h->k;
  if (u) H_TRY(cudaMemcpy(u, (which ? h->U : h->U0) + u_off(h, level, index), sizeof(double) * sl * k,
                          cudaMemcpyDeviceToHost));
  if (v) H_TRY(cudaMemcpy(v, (which ? h->V : h->V0) + u_off(h, level, index), sizeof(double) * sl * k,
                          cudaMemcpyDeviceToHost));
  if (s) H_TRY(cudaMemcpy(s, (which ? h->S : h->S0) + s_off(h, level, index), sizeof(double) * k * k,
                          cudaMemcpyDeviceToHost));
  return FRANK_OK;
}

int frank_hodlr_get_pivots(const frank_hodlr* h, int leaf, int* ipiv) {
  if (!h || !ipiv) return hfail(FRANK_ERR_INVALID, "null argument");
  if (leaf < 0 || leaf >= h->P) return hfail(FRANK_ERR_INVALID, "bad leaf");
  if (!h->factored) return hfail(FRANK_ERR_STATE, "getrf has not run");
  H_TRY(cudaMemcpy(ipiv, h->ipiv + (int64_t)leaf * h->b, sizeof(int) * h->b, cudaMemcpyDeviceToHost));
  return FRANK_OK;
}

int frank_hodlr_build_kernel(frank_hodlr* h, int kernel, const double* points, int dim, const double* kparams,
                             void* stream) {
  if (!h || !points) return hfail(FRANK_ERR_INVALID, "null argument");
  if (kernel < 0 || kernel > 3 || dim < 1 || dim > 3) return hfail(FRANK_ERR_INVALID, "bad kernel or dimension");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t n = h->n;
  const int k = h->k;
  double* dx = nullptr;
  H_TRY(dalloc(&dx, (size_t)dim * n));
  H_TRY(cudaMemcpy(dx, points, sizeof(double) * dim * n, cudaMemcpyHostToDevice));
  hk::KernelDesc K;
  K.kind = kernel;
  K.dim = dim;
  K.x = dx;
  K.n = n;
  K.p0 = kparams ? kparams[0] : 0.0;
  K.p1 = kparams ? kparams[1] : 0.0;
  hk::k_h_build_leaves<<<4 * h->sm_count, 256, 0, s>>>(K, h->b, h->P, h->D0);
  // LowRank(Dense, rank) on every off-diagonal block, level by level:
  // rsvd (rsvd.cpp:17-29) with sample min(k + 5, s) and the reference's
  // Omega (random_uniform, std::mt19937 seeded 0, functions.cpp:52-66);
  // the block is never stored: Y = A Omega and Z = A^T Q evaluate it tile by tile.
  int rc = FRANK_OK;
  double *W = nullptr, *Y = nullptr, *Q = nullptr, *R = nullptr, *Z = nullptr, *U2 = nullptr, *sv = nullptr,
         *Vt2 = nullptr, *Ur = nullptr, *om = nullptr, *sc = nullptr;
  int* errd = h->err;
  const int64_t pmax = std::min<int64_t>(k + 5, h->b);
  const size_t slab = (size_t)n * pmax;   // one level: 2^l blocks of s_l x p
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  int64_t ws_max = 0;
  for (int l = 1; l <= h->L; ++l) {
    const int64_t sl = s_of(h, l);
    const int p = (int)std::min<int64_t>(k + 5, sl);
    ws_max = std::max(ws_max, std::max(::frank::ops::qr_ws((int)sl, p), ::frank::ops::svd_scratch(p, p)) << l);
  }
  A(dalloc(&W, slab)); A(dalloc(&Y, slab)); A(dalloc(&Q, slab)); A(dalloc(&Z, slab)); A(dalloc(&U2, slab));
  A(dalloc(&R, (size_t)pmax * pmax << h->L)); A(dalloc(&Vt2, (size_t)pmax * pmax << h->L));
  A(dalloc(&Ur, (size_t)pmax * pmax << h->L));
  A(dalloc(&sv, (size_t)pmax << h->L)); A(dalloc(&om, (size_t)(n / 2) * pmax)); A(dalloc(&sc, (size_t)ws_max));
  A(cudaMemsetAsync(errd, 0, sizeof(int) * hk::HERR_SLOTS, s));
  for (int l = 1; l <= h->L && e == cudaSuccess; ++l) {
    const int64_t sl = s_of(h, l);
    const int p = (int)std::min<int64_t>(k + 5, sl);
    const int nb = 1 << l;
    std::vector<double> omh((size_t)sl * p);
    {
      std::mt19937 gen;
      gen.seed(0);
      std::uniform_real_distribution<double> dist(0.0, 1.0);
      for (auto& x : omh) x = dist(gen);
    }
    A(cudaMemcpyAsync(om, omh.data(), sizeof(double) * omh.size(), cudaMemcpyHostToDevice, s));
    hk::k_h_omega<<<4 * h->sm_count, 256, 0, s>>>(sl, p, nb, om, W);
    hk::k_h_kgemm<<<dim3((unsigned)((sl + 63) / 64), nb), hk::WT, 0, s>>>(K, sl, p, 0, W, Y);
    ::frank::ops::launch_qr(s, (int)sl, p, nb, Y, sl, sl * p, Q, sl, sl * p, R, p, (int64_t)p * p, sc,
                            ::frank::ops::qr_ws((int)sl, p));
    hk::k_h_kgemm<<<dim3((unsigned)((sl + 63) / 64), nb), hk::WT, 0, s>>>(K, sl, p, 1, Q, Z);
    // Z = A^T Q = Qz Rz, Rz = Ur diag(sv) Vt2: the SVD of the small Rz only
    // (Q^T A = Vt2^T diag(sv) (Qz Ur)^T)
    ::frank::ops::launch_qr(s, (int)sl, p, nb, Z, sl, sl * p, U2, sl, sl * p, R, p, (int64_t)p * p, sc,
                            ::frank::ops::qr_ws((int)sl, p));
    ::frank::ops::launch_svd(s, p, p, nb, R, p, (int64_t)p * p, Ur, p, (int64_t)p * p, sv, p, Vt2, p,
                             (int64_t)p * p, sc, ::frank::ops::svd_scratch(p, p), errd + hk::HERR_JACOBI);
    ::frank::ops::launch_gemm(s, (int)sl, p, p, nb, 1.0, U2, sl, sl * p, false, Ur, p, (int64_t)p * p, false, 0.0, Z,
                              sl, sl * p);
    // U = Q Vt2(:k, :)^T, V = (Qz Ur)(:, :k)^T, S = diag(sv(:k))
    ::frank::ops::launch_gemm(s, (int)sl, k, p, nb, 1.0, Q, sl, sl * p, false, Vt2, p, (int64_t)p * p, true, 0.0,
                              h->U0 + u_off(h, l, 0), sl, sl * k);
    hk::k_h_finish_v<<<4 * h->sm_count, 256, 0, s>>>(sl, p, k, nb, Z, sv, h->V0 + u_off(h, l, 0),
                                                     h->S0 + s_off(h, l, 0));
    A(cudaGetLastError());
    A(cudaStreamSynchronize(s));
  }
  A(cudaStreamSynchronize(s));
  for (void* ptr : {(void*)W, (void*)Y, (void*)Q, (void*)R, (void*)Z, (void*)U2, (void*)sv, (void*)Vt2, (void*)Ur,
                    (void*)om, (void*)sc, (void*)dx})
    if (ptr) cudaFree(ptr);
  if (e != cudaSuccess) return hfail(FRANK_ERR_CUDA, std::string("H-matrix construction: ") + cudaGetErrorString(e));
  int eh[hk::HERR_SLOTS];
  H_TRY(cudaMemcpy(eh, errd, sizeof(eh), cudaMemcpyDeviceToHost));
  if (eh[hk::HERR_JACOBI]) rc = hfail(FRANK_ERR_NOT_CONVERGED, "one-sided Jacobi reached its sweep limit");
  h->have_A = true;
  h->factored = false;
  return rc;
}

int frank_hodlr_getrf(frank_hodlr* h, void* stream) {
  if (!h) return hfail(FRANK_ERR_INVALID, "null H-matrix");
  if (!h->have_A) return hfail(FRANK_ERR_STATE, "H-matrix has no blocks");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!h->gexec) {
    H_TRY(cudaStreamSynchronize(s));
    H_TRY(cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_factor(h, h->s);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(h->s, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ce != cudaSuccess) return hfail(FRANK_ERR_CUDA, std::string("H-LU capture: ") + cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&h->gexec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return hfail(FRANK_ERR_CUDA, std::string("H-LU graph: ") + cudaGetErrorString(ie));
    if ((int64_t)h->tasks_h.size() > h->ntasks_cap) return hfail(FRANK_ERR_INVALID, "H-LU: task table overflow");
    if (!h->tasks_h.empty())
      H_TRY(cudaMemcpy(h->tasks_d, h->tasks_h.data(), sizeof(::frank::ops::LrAddTask) * h->tasks_h.size(),
                       cudaMemcpyHostToDevice));
  }
  H_TRY(cudaEventRecord(h->e0, s));
  H_TRY(cudaGraphLaunch(h->gexec, s));
  H_TRY(cudaEventRecord(h->e1, s));
  int rc = check_errors(h, s);
  H_TRY(cudaEventElapsedTime(&h->factor_ms, h->e0, h->e1));
  h->factored = rc == FRANK_OK;
  return rc;
}

int frank_hodlr_solve_device(frank_hodlr* h, double* d_b, int64_t ldb, int nrhs, void* stream) {
  if (!h || !d_b) return hfail(FRANK_ERR_INVALID, "null argument");
  if (nrhs < 1 || ldb < h->n) return hfail(FRANK_ERR_INVALID, "bad right-hand sides");
  if (!h->factored) return hfail(FRANK_ERR_STATE, "solve before getrf");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = enqueue_solve(h, d_b, ldb, nrhs, s);
  if (rc) return rc;
  H_TRY(cudaStreamSynchronize(s));
  return FRANK_OK;
}

int frank_hodlr_trsm_device(frank_hodlr* h, int uplo, double* d_b, int64_t ldb, int nrhs, void* stream) {
  if (!h || !d_b) return hfail(FRANK_ERR_INVALID, "null argument");
  if (nrhs < 1 || ldb < h->n || (uplo != FRANK_LOWER && uplo != FRANK_UPPER))
    return hfail(FRANK_ERR_INVALID, "bad right-hand sides or triangle");
  if (!h->factored) return hfail(FRANK_ERR_STATE, "trsm before getrf");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = enqueue_solve(h, d_b, ldb, nrhs, s, uplo == FRANK_LOWER ? 1 : 2);
  if (rc) return rc;
  H_TRY(cudaStreamSynchronize(s));
  return FRANK_OK;
}

int frank_hodlr_matvec_device(frank_hodlr* h, const double* d_x, int64_t ldx, double* d_y, int64_t ldy, int nrhs,
                              void* stream) {
  if (!h || !d_x || !d_y) return hfail(FRANK_ERR_INVALID, "null argument");
  if (nrhs < 1 || ldx < h->n || ldy < h->n) return hfail(FRANK_ERR_INVALID, "bad vectors");
  if (!h->have_A) return hfail(FRANK_ERR_STATE, "H-matrix has no blocks");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = enqueue_matvec(h, d_x, ldx, d_y, ldy, nrhs, s);
  if (rc) return rc;
  H_TRY(cudaStreamSynchronize(s));
  return FRANK_OK;
}

int frank_hodlr_refine_device(frank_hodlr* h, const double* d_b, int64_t ldb, double* d_x, int64_t ldx, int nrhs,
                              double tol, int max_iter, int* iters, double* relres, void* stream) {
  if (!h || !d_b || !d_x) return hfail(FRANK_ERR_INVALID, "null argument");
  if (nrhs < 1 || ldb < h->n || ldx < h->n || max_iter < 0) return hfail(FRANK_ERR_INVALID, "bad arguments");
  if (!h->factored) return hfail(FRANK_ERR_STATE, "refine before getrf");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t need = h->n * nrhs;
  if (need > h->work_cap) {
    if (h->work) cudaFree(h->work);
    if (h->nrm) cudaFree(h->nrm);
    h->work = nullptr;
    h->nrm = nullptr;
    H_TRY(dalloc(&h->work, (size_t)need));
    H_TRY(dalloc(&h->nrm, 2 * (size_t)nrhs));
    h->work_cap = need;
  }
  // x0 = (LU)^{-1} b, then x += (LU)^{-1} (b - A_H x) until every column's
  // relative residual is below tol
  H_TRY(cudaMemcpy2DAsync(d_x, sizeof(double) * ldx, d_b, sizeof(double) * ldb, sizeof(double) * h->n, nrhs,
                          cudaMemcpyDeviceToDevice, s));
  int rc = enqueue_solve(h, d_x, ldx, nrhs, s);
  if (rc) return rc;
  std::vector<double> nr(2 * (size_t)nrhs);
  double worst = 0.0;
  int it = 0;
  for (;; ++it) {
    rc = enqueue_matvec(h, d_x, ldx, h->work, h->n, nrhs, s);
    if (rc) return rc;
    hk::k_h_residual<<<nrhs, hk::WT, 0, s>>>(h->n, d_b, ldb, h->work, h->n, h->nrm);
    H_TRY(cudaMemcpyAsync(nr.data(), h->nrm, sizeof(double) * nr.size(), cudaMemcpyDeviceToHost, s));
    H_TRY(cudaStreamSynchronize(s));
    worst = 0.0;
    for (int c = 0; c < nrhs; ++c) worst = std::max(worst, std::sqrt(nr[2 * c] / std::max(nr[2 * c + 1], 1e-300)));
    if (worst <= tol || it >= max_iter) break;
    rc = enqueue_solve(h, h->work, h->n, nrhs, s);
    if (rc) return rc;
    hk::k_h_axpy<<<2 * h->sm_count, 256, 0, s>>>(h->n, nrhs, h->work, h->n, d_x, ldx);
  }
  H_TRY(cudaGetLastError());
  if (iters) *iters = it;
  if (relres) *relres = worst;
  return worst <= tol ? FRANK_OK : hfail(FRANK_ERR_NOT_CONVERGED, "H-LU refinement did not reach the tolerance");
}

int frank_hodlr_stats(const frank_hodlr* h, int64_t* launches, double* factor_ms) {
  if (!h) return hfail(FRANK_ERR_INVALID, "null H-matrix");
  if (launches) *launches = h->launches;
  if (factor_ms) *factor_ms = h->factor_ms;
  return FRANK_OK;
}

}  // extern "C"
