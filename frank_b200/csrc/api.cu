// Host side of the BLR-LU engine: plan allocation, the per-step driver of the
// factorization (captured once into a CUDA graph and replayed), block
// substitution, the FP64 H-matvec, iterative refinement and the C ABI
// declared in include/frank_b200.h.
#include "blr_kernels.cuh"
#include "../../include/frank_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <random>
#include <tuple>
#include <string>
#include <vector>

using namespace frank;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define CUDA_TRY(expr)                                                                      \
  do {                                                                                      \
    cudaError_t _e = (expr);                                                                \
    if (_e != cudaSuccess)                                                                  \
      return fail(FRANK_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));      \
  } while (0)

template <typename P>
cudaError_t dalloc(P** p, size_t count) {
  *p = nullptr;
  if (count == 0) return cudaSuccess;
  return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(P));
}

// Device allocation owned by a scope: freed on every return path.
template <typename P>
struct DevBuf {
  P* ptr = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { if (ptr) cudaFree(ptr); }
  cudaError_t alloc(size_t count) { return dalloc(&ptr, count); }
  P* get() const { return ptr; }
};

}  // namespace

namespace frank {
// Error text for the per-operation entry points (ops.cu).
int set_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace frank

struct frank_blr {
  int64_t n = 0;
  int nb = 0, bmax = 0, kcap = 0, precision = 0, fixed_rank = 0;
  double eps = 0.0, admis = 0.0;
  int device = 0, sm_count = 0;
  std::vector<int> off_h, dslot_h, lslot_h;
  int ndense = 0, nlr = 0;
  bool dense_offdiag = false;
  // device geometry
  int *d_off = nullptr, *d_dslot = nullptr, *d_lslot = nullptr;
  int *d_rankH = nullptr, *d_rankW = nullptr;
  // A_H (FP64)
  double *Hd = nullptr, *Hu = nullptr, *Hs = nullptr, *Hv = nullptr;
  // working copy (T)
  void *Wd = nullptr, *Wu = nullptr, *Ws = nullptr, *Wv = nullptr;
  // factor workspace
  int *perm = nullptr, *ipiv = nullptr, *err = nullptr, *work = nullptr;
  void *Linv = nullptr, *Uinv = nullptr, *WL = nullptr, *WU = nullptr;
  double *getrf_scratch = nullptr, *dscratch = nullptr, *rscratch = nullptr;
  double* rsplit = nullptr;     // scratch slots of split recompression targets
  double* host_io = nullptr;    // device copies of b and x for frank_blr_refine
  size_t host_io_cap = 0;
  int* split_done = nullptr;    // [nb][SPLIT_MAX] side counters
  int nsplit = 0;               // split slots allocated
  int64_t dstride = 0, rstride = 0;
  int grid_dense = 0, grid_recomp = 0, smax = 0;
  int core_method = CORE_RRQR;   // core of tolerance plans
  int core_fixed = CORE_FAST;    // core of fixed-rank plans (FRANK_LRA unset: fast_rounded_addition)
  bool proj_tol = true;          // tolerance plans: projected bases (QR of the update's remainder only)
  bool orth_pending = false;     // caller-given low-rank blocks not yet given orthonormal bases
  // launch parameters the autotuner chooses (frank_blr_autotune)
  int dupd_band = DUPD_BAND;     // rows per dense-update task
  int split_p = SPLIT_P;         // split band-1 targets above this operand rank (0: never)
  int core_smem = RECOMP_REGION; // recompression cores up to this many doubles stay in shared memory
  double core_scale = 0.1;
  int grid_gram = 0;
  double gram_tol = 1e-12;
  bool gram = false;
  // solve / matvec temporaries (nrhs <= 8 per pass)
  void* z = nullptr;         // n x 8 (T)
  void* stmp = nullptr;      // bmax x 8 (T)
  void* sctmp = nullptr;     // nb x bmax x 8 (T)
  double* part = nullptr;    // nb*nb x bmax x 8
  double* vtmp = nullptr;    // n x 8 x 3 (residual, correction, rhs copy)
  double* nrm = nullptr;     // norm partials
  double* nrm_h = nullptr;   // pinned host mirror
  int nrm_blocks = 0;
  // state
  bool factored = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t graph_stream = nullptr;
  int64_t launches = 0;        // kernels in the factorization graph
  int64_t solve_launches = 0;  // kernels issued by solve / matvec / refine since the last getrf
  int err_h[ERR_SLOTS] = {0};
  unsigned long long* flops = nullptr;
  unsigned long long flops_h[FLOP_SLOTS] = {0};
  // timing events recorded inside the captured graph: [step][class][begin,end]
  std::vector<cudaEvent_t> ev;
  double class_ms[FLOP_SLOTS] = {0};
  bool timed = false;  // timing events recorded in the captured graph (opt-in:
                       // event-record nodes serialise the graph's branches)
  bool want_timing = false;
  // captured solves (graph of cast / diagonal / scatter launches), keyed by
  // buffer, leading dimension, RHS count and direction
  struct SolveGraph {
    cudaGraphExec_t exec = nullptr;
    const void* ptr = nullptr;
    int64_t ld = 0;
    int nrhs = 0;
    bool transpose = false;
    int part = 0;
    int64_t kernels = 0;
  };
  std::vector<SolveGraph> solve_graphs;
  cudaStream_t cap_stream = nullptr;   // private stream the solves are captured on
  int solve_chunk = 8;                 // RHS per solve pass (bounded by the scatter's shared memory)
  // lookahead: second capture stream and its dependency events
  cudaStream_t aux = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> getrf_done, dense_done, panel_done, next_done;
};

namespace {

template <typename T>
BlrView<T> work_view(frank_blr* p) {
  BlrView<T> v;
  v.nb = p->nb; v.bmax = p->bmax; v.kcap = p->kcap;
  v.off = p->d_off; v.dslot = p->d_dslot; v.lslot = p->d_lslot; v.rank = p->d_rankW;
  v.D = static_cast<T*>(p->Wd); v.U = static_cast<T*>(p->Wu);
  v.S = static_cast<T*>(p->Ws); v.Vt = static_cast<T*>(p->Wv);
  return v;
}

BlrView<double> h_view(const frank_blr* p) {
  BlrView<double> v;
  v.nb = p->nb; v.bmax = p->bmax; v.kcap = p->kcap;
  v.off = p->d_off; v.dslot = p->d_dslot; v.lslot = p->d_lslot; v.rank = p->d_rankH;
  v.D = p->Hd; v.U = p->Hu; v.S = p->Hs; v.Vt = p->Hv;
  return v;
}

template <typename T>
FactorWs<T> factor_ws(frank_blr* p) {
  FactorWs<T> w;
  w.perm = p->perm; w.ipiv = p->ipiv;
  w.Linv = static_cast<T*>(p->Linv); w.Uinv = static_cast<T*>(p->Uinv);
  w.WL = static_cast<T*>(p->WL); w.WU = static_cast<T*>(p->WU);
  w.getrf_scratch = p->getrf_scratch;
  w.dscratch = p->dscratch; w.dscratch_stride = p->dstride;
  w.rscratch = p->rscratch; w.rscratch_stride = p->rstride;
  w.err = p->err; w.work = p->work; w.flops = p->flops; w.fixed_rank = p->fixed_rank; w.eps = p->eps;
  return w;
}

size_t tsize(const frank_blr* p) { return p->precision == FRANK_PREC_FP64 ? sizeof(double) : sizeof(float); }

int check_block(const frank_blr* p, int i, int j) {
  if (!p) return fail(FRANK_ERR_INVALID, "null plan");
  if (i < 0 || j < 0 || i >= p->nb || j >= p->nb) return fail(FRANK_ERR_INVALID, "block index out of range");
  return FRANK_OK;
}

// Enqueue all launches of one factorization on stream s.
// The Gram-based recompression serves the mixed path with the RRQR core at a
// tolerance (fixed-rank plans and the SVD core use the Householder kernel).
bool use_gram(const frank_blr* p) {
  return p->precision == FRANK_PREC_MIXED && p->fixed_rank == 0 && p->core_method == CORE_RRQR && p->gram;
}

// Mixed plans with the RRQR core truncate the working copy to the factor
// tolerance at reset (needs a recompression scratch slot of 4 k^2 + 8 k).
bool pretruncate(const frank_blr* p) {
  return p->precision == FRANK_PREC_MIXED && p->fixed_rank == 0 && p->core_method == CORE_RRQR && p->nlr > 0 &&
         p->rstride >= 4 * (int64_t)p->kcap * p->kcap + 8 * (int64_t)p->kcap;
}

// timing events per step: one pair per operation class, plus one for the
// update of the next diagonal block (counted with the dense class)
constexpr int EV_DENSE_NEXT = FLOP_SLOTS, EV_SLOTS = FLOP_SLOTS + 1;
cudaEvent_t& ev_at(frank_blr* p, int step, int cls, int end) { return p->ev[((size_t)step * EV_SLOTS + cls) * 2 + end]; }

// Split recompression targets (two CTAs per large band-1 target) on plans
// with the full recompression grid (not the reduced grids of batched plans).
bool split_on(const frank_blr* p) { return p->nb > 2 && p->grid_recomp >= p->sm_count - 1; }

// Per-CTA scratch of the update / recompression kernels, sized by the grids.
int ensure_scratch(frank_blr* p) {
  if (!p->dscratch) CUDA_TRY(dalloc(&p->dscratch, (size_t)p->grid_dense * p->dstride));
  if (p->nlr > 0 && split_on(p) && !p->rsplit) {
    // one slot per band-1 task of the first step (at most SPLIT_MAX); the
    // split is an optimisation, so without the memory the plan runs without it
    p->nsplit = std::min(SPLIT_MAX, 2 * (p->nb - 2));
    if (dalloc(&p->rsplit, (size_t)p->nsplit * p->rstride) != cudaSuccess ||
        dalloc(&p->split_done, (size_t)p->nb * SPLIT_MAX) != cudaSuccess) {
      cudaGetLastError();
      if (p->rsplit) cudaFree(p->rsplit);
      if (p->split_done) cudaFree(p->split_done);
      p->rsplit = nullptr;
      p->split_done = nullptr;
      p->nsplit = 0;
    }
  }
  if (p->nlr > 0 && !p->rscratch)
    CUDA_TRY(dalloc(&p->rscratch, (size_t)std::max(p->grid_recomp, p->precision == FRANK_PREC_MIXED ? p->grid_gram : 0) *
                                      p->rstride));
  return FRANK_OK;
}

// Orthonormal bases for the caller's low-rank blocks of A_H (once after
// frank_blr_set_lowrank calls, before the next factorization).
int orthonormalize_inputs(frank_blr* p, cudaStream_t s) {
  if (!p->orth_pending || p->nlr == 0) { p->orth_pending = false; return FRANK_OK; }
  int rc = ensure_scratch(p);
  if (rc) return rc;
  const int64_t need = 2 * ((int64_t)p->bmax + p->kcap) * p->kcap + 3 * (int64_t)p->kcap * p->kcap + 2 * p->kcap;
  if (need > p->rstride) return fail(FRANK_ERR_INVALID, "orthonormalisation scratch");
  k_orthonormalize_lr<<<p->grid_recomp, ORTH_THREADS, 0, s>>>(h_view(p), p->rscratch, p->rstride);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(s));
  p->orth_pending = false;
  return FRANK_OK;
}

// One factorization on stream s.  After step i's panels, a second stream
// (p->aux) updates the diagonal block (i+1, i+1), runs the leaf getrf of
// step i+1 and the explicit inverses of its factors, and then updates the
// step's other dense targets, all overlapping step i's recompressions on s
// (lookahead of depth one); the main stream waits for the dense updates and
// the inverses before the next panels.  The recompression grid leaves one SM
// free for the second stream.
template <typename T>
int enqueue_factor(frank_blr* p, cudaStream_t s, bool timing = true) {
  p->timed = timing;
  BlrView<double> H = h_view(p);
  BlrView<T> W = work_view<T>(p);
  FactorWs<T> ws = factor_ws<T>(p);
  cudaStream_t s2 = p->aux;
  int64_t launches = 0;
  k_reset<T><<<p->nb * p->nb, 256, 0, s>>>(H, W);
  ++launches;
  CUDA_TRY(cudaMemsetAsync(p->err, 0, ERR_SLOTS * sizeof(int), s));
  CUDA_TRY(cudaMemsetAsync(p->flops, 0, FLOP_SLOTS * sizeof(unsigned long long), s));
  CUDA_TRY(cudaMemsetAsync(p->work, 0, 2 * p->nb * sizeof(int), s));
  if (p->split_done) CUDA_TRY(cudaMemsetAsync(p->split_done, 0, (size_t)p->nb * SPLIT_MAX * sizeof(int), s));
  CUDA_TRY(cudaEventRecord(p->fork, s));
  CUDA_TRY(cudaStreamWaitEvent(s2, p->fork, 0));
  if (pretruncate(p)) {
    // mixed plans: the factor's tolerance is looser than A_H's, so the working
    // copy's low-rank blocks are truncated to it before the first step (beside
    // the first leaf getrf, which reads only the dense diagonal block)
    k_truncate_lr<T><<<std::max(p->grid_recomp, p->grid_gram), TRUNC_THREADS, 0, s>>>(
        H, W, ws, p->core_scale * p->eps, p->rscratch, p->rstride);
    ++launches;
  }
  // explicit inverses of a step's diagonal factors, all column blocks in
  // parallel; on the second stream right after the leaf getrf, except in a
  // replay with timing events (there on the main stream, serialised)
  auto trinv_on = [&](int step, cudaStream_t st) -> int {
    const int cw = trinv_width(p->bmax);
    const int nblk = (int)((p->off_h[step + 1] - p->off_h[step] + cw - 1) / cw);
    if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, step, FLOP_TRINV, 0), st, cudaEventRecordExternal));
    k_trinv<T><<<2 * nblk, TRINV_THREADS, (size_t)p->bmax * cw * sizeof(double), st>>>(W, ws, step, cw);
    if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, step, FLOP_TRINV, 1), st, cudaEventRecordExternal));
    ++launches;
    return FRANK_OK;
  };
  auto getrf_on_aux = [&](int step) -> int {
    if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, step, FLOP_GETRF, 0), s2, cudaEventRecordExternal));
    {
      // leaf LU as load / (panel, tiled trailing update) x panels / store
      const int b = p->off_h[step + 1] - p->off_h[step];
      k_getrf_load<T><<<64, GETRF_AUX_THREADS, 0, s2>>>(W, ws, step);
      for (int jb = 0; jb < b; jb += 32) {
        k_getrf_panel<T><<<1, GETRF_THREADS, 0, s2>>>(W, ws, step, jb);
        const int m2 = b - jb - std::min(32, b - jb);
        if (m2 > 0) {
          const int nt = (m2 + 63) / 64;
          k_getrf_trail<T><<<nt * nt, GETRF_AUX_THREADS, 0, s2>>>(W, ws, step, jb);
          ++launches;
        }
        ++launches;
      }
      k_getrf_store<T><<<64, GETRF_AUX_THREADS, 0, s2>>>(W, ws, step);
      launches += 1;
    }
    if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, step, FLOP_GETRF, 1), s2, cudaEventRecordExternal));
    if (!timing) {
      const int rc2 = trinv_on(step, s2);
      if (rc2) return rc2;
    }
    CUDA_TRY(cudaEventRecord(p->getrf_done[step], s2));
    return FRANK_OK;
  };
  int rc = getrf_on_aux(0);
  if (rc) return rc;
  ++launches;   // the getrf load kernel
  for (int i = 0; i < p->nb; ++i) {
    CUDA_TRY(cudaStreamWaitEvent(s, p->getrf_done[i], 0));
    if (timing && (rc = trinv_on(i, s))) return rc;
    const int m = p->nb - i - 1;
    if (m == 0) break;
    if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, i, FLOP_PANEL, 0), s, cudaEventRecordExternal));
    {
      const int rt = (p->bmax + PANEL_TILE - 1) / PANEL_TILE;
      k_panel_gather<T><<<dim3(m, rt), PANEL_THREADS, 0, s>>>(W, ws, i);
      k_panel_mul<T><<<dim3(2 * m, rt), PANEL_THREADS, 0, s>>>(W, ws, i);
      k_panel_fin<T><<<dim3(2 * m, rt), PANEL_THREADS, 0, s>>>(W, ws, i);
      launches += 2;
    }
    if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, i, FLOP_PANEL, 1), s, cudaEventRecordExternal));
    ++launches;
    const int mm = m * m;
    // Dense targets on the second stream, concurrently with the
    // recompressions (the two write disjoint blocks and read the same
    // panels): the next diagonal block first, its leaf getrf, then the other
    // dense targets.  The next panel overwrites WL / WU, so the main stream
    // waits for all of it after the recompressions.
    // A replay with timing events keeps the dense updates on the main stream
    // (serialised), so that their events time the kernels and not their
    // overlap with the recompressions.
    cudaStream_t sd = timing ? s : s2;
    CUDA_TRY(cudaEventRecord(p->panel_done[i], s));
    if (sd != s) CUDA_TRY(cudaStreamWaitEvent(sd, p->panel_done[i], 0));
    {
      const int band = std::min(p->dupd_band, p->bmax);
      const int nbands = (p->bmax + band - 1) / band;
      if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, i, EV_DENSE_NEXT, 0), sd, cudaEventRecordExternal));
      // one task per band; its CTA index picks a scratch slot (grid_dense of them)
      k_update_dense<T><<<std::min(nbands, p->grid_dense), DUPD_THREADS, 0, sd>>>(W, ws, i, p->dupd_band, DUPD_NEXT);
      if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, i, EV_DENSE_NEXT, 1), sd, cudaEventRecordExternal));
      ++launches;
      if (sd == s) {
        CUDA_TRY(cudaEventRecord(p->next_done[i], s));
        CUDA_TRY(cudaStreamWaitEvent(s2, p->next_done[i], 0));
      }
      if ((rc = getrf_on_aux(i + 1))) return rc;
      ++launches;   // the getrf load kernel
      if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, i, FLOP_DENSE, 0), sd, cudaEventRecordExternal));
      if (m > 1) {
        k_update_dense<T><<<(int)std::min<int64_t>((int64_t)mm * nbands, p->grid_dense), DUPD_THREADS, 0, sd>>>(
            W, ws, i, p->dupd_band, DUPD_REST);
        ++launches;
      }
      if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, i, FLOP_DENSE, 1), sd, cudaEventRecordExternal));
      CUDA_TRY(cudaEventRecord(p->dense_done[i], sd));
    }
    if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, i, FLOP_RECOMP, 0), s, cudaEventRecordExternal));
    if (p->nlr > 0) {
      if (use_gram(p)) {
        // mixed path: Gram-based recompression of every low-rank x low-rank
        // update; the Householder kernel takes any target with a dense operand
        k_recompress_gram<T><<<std::min(mm, p->grid_gram), GRAM_THREADS, GRAM_SMEM_BYTES, s>>>(
            W, ws, i, p->smax, p->core_scale, p->gram_tol, p->work + i);
        ++launches;
        if (p->dense_offdiag) {
          k_recompress<T><<<std::min(mm, p->grid_recomp), RECOMP_THREADS, RECOMP_SMEM_BYTES, s>>>(
              W, ws, i, p->smax, p->core_method, p->core_scale, 1, p->work + p->nb + i, 0, nullptr, nullptr, 0, 0,
              p->core_smem);
          ++launches;
        }
      } else {
        k_recompress<T><<<std::min(mm, p->grid_recomp), RECOMP_THREADS, RECOMP_SMEM_BYTES, s>>>(
            W, ws, i, p->smax, p->fixed_rank > 0 ? p->core_fixed : p->core_method, p->core_scale, 0, p->work + i,
            p->rsplit ? p->nsplit : 0, p->rsplit, p->split_done ? p->split_done + (size_t)i * SPLIT_MAX : nullptr,
            p->proj_tol ? 1 : 0, p->split_p, p->core_smem);
        ++launches;
      }
    }
    if (timing) CUDA_TRY(cudaEventRecordWithFlags(ev_at(p, i, FLOP_RECOMP, 1), s, cudaEventRecordExternal));
    CUDA_TRY(cudaStreamWaitEvent(s, p->dense_done[i], 0));
  }
  CUDA_TRY(cudaStreamWaitEvent(s, p->getrf_done[p->nb - 1], 0));
  CUDA_TRY(cudaGetLastError());
  p->launches = launches;
  return FRANK_OK;
}

// Per-class device time of the last factorization from the graph's events.
int collect_times(frank_blr* p) {
  for (int c = 0; c < FLOP_SLOTS; ++c) p->class_ms[c] = 0.0;
  if (!p->timed) return FRANK_OK;
  for (int i = 0; i < p->nb; ++i)
    for (int c = 0; c < EV_SLOTS; ++c) {
      if (i == p->nb - 1 && c != FLOP_GETRF && c != FLOP_TRINV) continue;
      float ms = 0.f;
      cudaError_t e = cudaEventElapsedTime(&ms, ev_at(p, i, c, 0), ev_at(p, i, c, 1));
      if (e != cudaSuccess) return fail(FRANK_ERR_CUDA, std::string("event timing: ") + cudaGetErrorString(e));
      p->class_ms[c == EV_DENSE_NEXT ? FLOP_DENSE : c] += ms;
    }
  return FRANK_OK;
}

// Status, counters and timings of a factorization that has completed.
int finish_factor(frank_blr* p) {
  CUDA_TRY(cudaMemcpy(p->err_h, p->err, ERR_SLOTS * sizeof(int), cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(p->flops_h, p->flops, FLOP_SLOTS * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  p->factored = true;
  p->solve_launches = 0;
  {
    int rc = collect_times(p);
    if (rc) return rc;
  }
  if (p->err_h[ERR_SINGULAR_STEP] != 0) {
    char buf[128];
    snprintf(buf, sizeof buf, "zero pivot in the leaf getrf of diagonal block %d", p->err_h[ERR_SINGULAR_STEP] - 1);
    return fail(FRANK_ERR_SINGULAR, buf);
  }
  if (p->err_h[ERR_BOUNDS] != 0) return fail(FRANK_ERR_INVALID, "stacked rank exceeded the recompression scratch");
  if (p->err_h[ERR_RANK_OVERFLOW] != 0) return fail(FRANK_ERR_RANK_OVERFLOW, "a recompressed rank exceeded max_rank and was clamped");
  return FRANK_OK;
}

template <typename T>
int run_factor(frank_blr* p, cudaStream_t s) {
  {
    int rc0 = orthonormalize_inputs(p, s);
    if (rc0) return rc0;
  }
  if (!p->graph_exec) {
    // Capture the whole step sequence once; kernel arguments are fixed
    // device pointers, ranks are read from device tables at run time.
    int rc0 = ensure_scratch(p);
    if (rc0) return rc0;
    CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_factor<T>(p, s, p->want_timing);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc != FRANK_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return fail(FRANK_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    p->graph = g;
    CUDA_TRY(cudaGraphInstantiate(&p->graph_exec, g, 0));
  }
  CUDA_TRY(cudaGraphLaunch(p->graph_exec, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return finish_factor(p);
}

// ---- solve --------------------------------------------------------------

// part: 0 both sweeps, 1 the forward sweep only (L), 2 the backward sweep only (U).
template <typename T>
int enqueue_solve(frank_blr* p, T* z, int64_t ldz, int nrhs, bool transpose, cudaStream_t s, int part = 0) {
  BlrView<T> W = work_view<T>(p);
  FactorWs<T> ws = factor_ws<T>(p);
  T* ybuf = static_cast<T*>(p->stmp);
  const int nb = p->nb;
  const int gd = (p->bmax + SOLVE_ROWS - 1) / SOLVE_ROWS;
  const size_t shd = ((size_t)p->bmax * nrhs + (size_t)(SOLVE_THREADS / SOLVE_ROWS) * SOLVE_ROWS * 8) * sizeof(double);
  const size_t shs = solve_scatter_cl_smem(p->bmax, p->kcap, nrhs);
  auto step = [&](int i, int dmode, int smode, int ntarget) {
    k_solve_diag<T><<<gd, SOLVE_THREADS, shd, s>>>(W, ws, i, z, ldz, nrhs, dmode, ybuf);
    k_solve_scatter_cl<T><<<std::max(ntarget, 1) * SC_CLUSTER, SOLVE_THREADS, shs, s>>>(W, i, z, ldz, nrhs, smode,
                                                                                       ybuf, ntarget);
  };
  if (!transpose) {
    if (part != 2) for (int i = 0; i < nb; ++i) step(i, 0, 0, nb - i - 1);
    if (part != 1) for (int i = nb - 1; i >= 0; --i) step(i, 1, 1, i);
  } else {
    for (int i = 0; i < nb; ++i) step(i, 2, 2, nb - i - 1);
    for (int i = nb - 1; i >= 0; --i) step(i, 3, 3, i);
  }
  CUDA_TRY(cudaGetLastError());
  return FRANK_OK;
}

int grid_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 4096); }

// Enqueue the launches of one solve of d_b (double, n x nrhs, in place): the
// FP64 plan solves in place, the mixed plan casts to its FP32 vector, solves
// and casts back.
int enqueue_solve_all(frank_blr* p, double* d_b, int64_t ldb, int nrhs, bool transpose, cudaStream_t s,
                      int part = 0) {
  for (int c0 = 0; c0 < nrhs; c0 += p->solve_chunk) {
    const int nr = std::min(p->solve_chunk, nrhs - c0);
    double* b = d_b + c0 * ldb;
    if (p->precision == FRANK_PREC_FP64) {
      int rc = enqueue_solve<double>(p, b, ldb, nr, transpose, s, part);
      if (rc) return rc;
    } else {
      float* z = static_cast<float*>(p->z);
      k_cast_copy<float, double><<<grid_for(p->n * nr), 256, 0, s>>>(b, ldb, z, p->n, p->n, nr);
      int rc = enqueue_solve<float>(p, z, p->n, nr, transpose, s, part);
      if (rc) return rc;
      k_cast_copy<double, float><<<grid_for(p->n * nr), 256, 0, s>>>(z, p->n, b, ldb, p->n, nr);
    }
  }
  CUDA_TRY(cudaGetLastError());
  return FRANK_OK;
}

void drop_solve_graphs(frank_blr* p) {
  for (auto& g : p->solve_graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  p->solve_graphs.clear();
}

// d_b (double, n x nrhs) -> solve in T -> back into d_b.  The 2 nb launches
// per pass are captured once per (buffer, ld, nrhs, direction) on the plan's
// private capture stream and replayed as one graph launch on `s`.
int solve_device_impl(frank_blr* p, double* d_b, int64_t ldb, int nrhs, bool transpose, cudaStream_t s,
                      int part = 0) {
  if (!p->factored) return fail(FRANK_ERR_STATE, "solve before getrf");
  frank_blr::SolveGraph* hit = nullptr;
  for (auto& g : p->solve_graphs)
    if (g.ptr == d_b && g.ld == ldb && g.nrhs == nrhs && g.transpose == transpose && g.part == part) hit = &g;
  if (!hit) {
    if (!p->cap_stream) CUDA_TRY(cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking));
    if (p->solve_graphs.size() >= 4) drop_solve_graphs(p);
    CUDA_TRY(cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_solve_all(p, d_b, ldb, nrhs, transpose, p->cap_stream, part);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(p->cap_stream, &g);
    if (rc != FRANK_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return fail(FRANK_ERR_CUDA, std::string("solve capture: ") + cudaGetErrorString(e));
    frank_blr::SolveGraph sg;
    size_t nodes = 0;
    cudaGraphGetNodes(g, nullptr, &nodes);
    e = cudaGraphInstantiate(&sg.exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(FRANK_ERR_CUDA, std::string("solve graph: ") + cudaGetErrorString(e));
    sg.ptr = d_b; sg.ld = ldb; sg.nrhs = nrhs; sg.transpose = transpose; sg.part = part; sg.kernels = (int64_t)nodes;
    p->solve_graphs.push_back(sg);
    hit = &p->solve_graphs.back();
  }
  p->solve_launches += hit->kernels;
  CUDA_TRY(cudaGraphLaunch(hit->exec, s));
  return FRANK_OK;
}

int matvec_device_impl(frank_blr* p, const double* x, int64_t ldx, double* y, int64_t ldy, int nrhs,
                       const double* bres, int64_t ldb, cudaStream_t s, bool transpose = false) {
  BlrView<double> H = h_view(p);
  for (int c0 = 0; c0 < nrhs; c0 += 8) {
    const int nr = std::min(8, nrhs - c0);
    const size_t shm = matvec_smem(p->bmax, p->kcap, nr);
    p->solve_launches += 2;
    k_matvec_blocks<<<dim3(p->nb, p->nb), MV_THREADS, shm, s>>>(H, x + c0 * ldx, ldx, nr, p->part, transpose ? 1 : 0);
    k_matvec_reduce<<<p->nb, 256, 0, s>>>(H, p->part, nr, bres ? bres + c0 * ldb : nullptr, ldb, y + c0 * ldy, ldy);
  }
  CUDA_TRY(cudaGetLastError());
  return FRANK_OK;
}

// max_j ||v_j|| / ||w_j|| with host reduction of per-CTA partials.
int colnorms(frank_blr* p, const double* v, int64_t ldv, int nrhs, std::vector<double>& out, cudaStream_t s) {
  out.assign(nrhs, 0.0);
  for (int c0 = 0; c0 < nrhs; c0 += 8) {
    const int nr = std::min(8, nrhs - c0);
    ++p->solve_launches;
    k_colnorm2<<<p->nrm_blocks, 256, 0, s>>>(v + c0 * ldv, p->n, ldv, nr, p->nrm);
    CUDA_TRY(cudaMemcpyAsync(p->nrm_h, p->nrm, sizeof(double) * p->nrm_blocks * nr, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    for (int b = 0; b < p->nrm_blocks; ++b)
      for (int h = 0; h < nr; ++h) out[c0 + h] += p->nrm_h[b * nr + h];
  }
  for (auto& v2 : out) v2 = std::sqrt(v2);
  return FRANK_OK;
}

// Column norms in two halves for batched use: enqueue (kernel + async copy
// to the plan's pinned mirror), then read after the stream has synchronised.
int colnorms_enqueue(frank_blr* p, const double* v, int64_t ldv, int nrhs, cudaStream_t s) {
  ++p->solve_launches;
  k_colnorm2<<<p->nrm_blocks, 256, 0, s>>>(v, p->n, ldv, nrhs, p->nrm);
  CUDA_TRY(cudaMemcpyAsync(p->nrm_h, p->nrm, sizeof(double) * p->nrm_blocks * nrhs, cudaMemcpyDeviceToHost, s));
  return FRANK_OK;
}

void colnorms_read(const frank_blr* p, int nrhs, std::vector<double>& out) {
  out.assign(nrhs, 0.0);
  for (int b = 0; b < p->nrm_blocks; ++b)
    for (int h = 0; h < nrhs; ++h) out[h] += p->nrm_h[b * nrhs + h];
  for (auto& v2 : out) v2 = std::sqrt(v2);
}

int refine_device_impl(frank_blr* p, const double* b, int64_t ldb, double* x, int64_t ldx, int nrhs, double tol,
                       int maxit, int* iters, double* resid, cudaStream_t s, bool transpose = false) {
  if (!p->factored) return fail(FRANK_ERR_STATE, "refine before getrf");
  if (nrhs > 8) return fail(FRANK_ERR_UNSUPPORTED, "refine takes at most 8 right-hand sides per call");
  int rc;
  std::vector<double> bn, rn;
  if ((rc = colnorms(p, b, ldb, nrhs, bn, s))) return rc;
  // every solve acts on the plan's residual / correction buffer r, so one
  // captured solve graph serves the whole refinement
  double* r = p->vtmp;  // n x nrhs residual / correction
  // x0 = (LU)^{-1} b
  CUDA_TRY(cudaMemcpy2DAsync(r, p->n * sizeof(double), b, ldb * sizeof(double), p->n * sizeof(double), nrhs,
                             cudaMemcpyDeviceToDevice, s));
  if ((rc = solve_device_impl(p, r, p->n, nrhs, transpose, s))) return rc;
  CUDA_TRY(cudaMemcpy2DAsync(x, ldx * sizeof(double), r, p->n * sizeof(double), p->n * sizeof(double), nrhs,
                             cudaMemcpyDeviceToDevice, s));
  int it = 0;
  double res = 0.0;
  for (;;) {
    if ((rc = matvec_device_impl(p, x, ldx, r, p->n, nrhs, b, ldb, s, transpose))) return rc;
    if ((rc = colnorms(p, r, p->n, nrhs, rn, s))) return rc;
    res = 0.0;
    for (int h = 0; h < nrhs; ++h) res = std::max(res, rn[h] / (bn[h] > 0.0 ? bn[h] : 1.0));
    if (res <= tol || it >= maxit) break;
    if ((rc = solve_device_impl(p, r, p->n, nrhs, transpose, s))) return rc;
    ++p->solve_launches;
    k_axpy_cast<double><<<grid_for(p->n * nrhs), 256, 0, s>>>(r, p->n, x, ldx, p->n, nrhs);
    ++it;
  }
  CUDA_TRY(cudaStreamSynchronize(s));
  if (iters) *iters = it;
  if (resid) *resid = res;
  if (res > tol) return fail(FRANK_ERR_NOT_CONVERGED, "refinement reached maxit before the tolerance");
  return FRANK_OK;
}

void free_plan(frank_blr* p) {
  if (!p) return;
  if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  void* ptrs[] = {p->d_off, p->d_dslot, p->d_lslot, p->d_rankH, p->d_rankW, p->Hd, p->Hu, p->Hs, p->Hv,
                  p->Wd, p->Wu, p->Ws, p->Wv, p->perm, p->ipiv, p->err, p->work, p->Linv, p->Uinv, p->WL, p->WU,
                  p->getrf_scratch, p->dscratch, p->rscratch, p->z, p->stmp, p->sctmp, p->part, p->vtmp, p->nrm,
                  p->rsplit, p->split_done, p->host_io};
  for (void* q : ptrs) if (q) cudaFree(q);
  if (p->flops) cudaFree(p->flops);
  for (cudaEvent_t e : p->ev) if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : p->getrf_done) if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : p->dense_done) if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : p->panel_done) if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : p->next_done) if (e) cudaEventDestroy(e);
  if (p->fork) cudaEventDestroy(p->fork);
  if (p->aux) cudaStreamDestroy(p->aux);
  if (p->graph_stream) cudaStreamDestroy(p->graph_stream);
  drop_solve_graphs(p);
  if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
  if (p->nrm_h) cudaFreeHost(p->nrm_h);
  delete p;
}

}  // namespace

namespace {
template <typename T>
void to_double(const std::vector<char>& raw, std::vector<double>& out, size_t count) {
  out.resize(count);
  const T* t = reinterpret_cast<const T*>(raw.data());
  for (size_t e = 0; e < count; ++e) out[e] = double(t[e]);
}

int fetch(const frank_blr* p, int which, const void* src, size_t count, std::vector<double>& out) {
  const size_t es = which ? tsize(p) : sizeof(double);
  std::vector<char> raw(count * es);
  cudaError_t e = cudaMemcpy(raw.data(), src, raw.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(FRANK_ERR_CUDA, cudaGetErrorString(e));
  if (es == sizeof(double)) to_double<double>(raw, out, count);
  else to_double<float>(raw, out, count);
  return FRANK_OK;
}
}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* frank_last_error(void) { return g_last_error.c_str(); }

int frank_device_info(char* name, int name_len, int* sm_count, int* cc_major, int* cc_minor) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
  if (name && name_len > 0) { strncpy(name, prop.name, name_len - 1); name[name_len - 1] = 0; }
  if (sm_count) *sm_count = prop.multiProcessorCount;
  if (cc_major) *cc_major = prop.major;
  if (cc_minor) *cc_minor = prop.minor;
  return FRANK_OK;
}

namespace {
// Block (i, j) of a geometry-based plan is admissible when admis^2 diam^2 <
// dist^2 for the bounding boxes of its row and column points, each padded by
// 0.5 (classes/initialization_helpers/matrix_initializer.cpp:51-91).
bool geometry_admissible(const double* x, int dim, int64_t n, int64_t r0, int64_t rn, int64_t c0, int64_t cn,
                         double admis) {
  const double off = 0.5;
  double len_r = 0.0, len_c = 0.0, dist = 0.0;
  for (int d = 0; d < dim; ++d) {
    const double* ax = x + (int64_t)d * n;
    const double rmin = *std::min_element(ax + r0, ax + r0 + rn) - off, rmax = *std::max_element(ax + r0, ax + r0 + rn) + off;
    const double cmin = *std::min_element(ax + c0, ax + c0 + cn) - off, cmax = *std::max_element(ax + c0, ax + c0 + cn) + off;
    len_r = std::max(len_r, rmax - rmin);
    len_c = std::max(len_c, cmax - cmin);
    const double dc = std::fabs((rmin + (rmax - rmin) / 2.0) - (cmin + (cmax - cmin) / 2.0));
    dist += dc * dc;
  }
  const double diam = std::max(len_r, len_c);
  return admis * admis * diam * diam < dist;
}

int create_impl(const frank_blr_desc* d, const double* points, int dim, frank_blr** out);
}  // namespace

int frank_blr_create(const frank_blr_desc* d, frank_blr** out) { return create_impl(d, nullptr, 0, out); }

int frank_blr_create_geometric(const frank_blr_desc* d, const double* points, int dim, frank_blr** out) {
  if (!points || dim < 1 || dim > 3) return fail(FRANK_ERR_INVALID, "geometry-based admissibility needs points, dim 1..3");
  return create_impl(d, points, dim, out);
}

}  // extern "C"

namespace {
int create_impl(const frank_blr_desc* d, const double* points, int dim, frank_blr** out) {
  if (!d || !out) return fail(FRANK_ERR_INVALID, "null descriptor");
  *out = nullptr;
  if (d->n <= 0 || d->nb <= 0 || d->nb > d->n) return fail(FRANK_ERR_INVALID, "need 0 < nb <= n");
  if (d->precision != FRANK_PREC_FP64 && d->precision != FRANK_PREC_MIXED)
    return fail(FRANK_ERR_INVALID, "unknown precision");
  if (d->fixed_rank < 0 || d->eps < 0.0 || (d->fixed_rank == 0 && d->eps <= 0.0))
    return fail(FRANK_ERR_INVALID, "need fixed_rank > 0 or eps > 0");
  frank_blr* p = new frank_blr();
  p->n = d->n; p->nb = d->nb; p->precision = d->precision; p->fixed_rank = d->fixed_rank;
  p->eps = d->eps; p->admis = d->admis;
  // IndexRange::split (index_range.cpp:15-24)
  const int64_t child = (d->n + d->nb - 1) / d->nb;
  p->off_h.resize(d->nb + 1);
  for (int i = 0; i < d->nb; ++i) p->off_h[i] = (int)(child * i);
  p->off_h[d->nb] = (int)d->n;
  for (int i = 0; i < d->nb; ++i)
    if (p->off_h[i + 1] - p->off_h[i] <= 0) { delete p; return fail(FRANK_ERR_INVALID, "empty block from the split"); }
  p->bmax = (int)child;
  if (p->bmax > 1024) { delete p; return fail(FRANK_ERR_UNSUPPORTED, "block size above 1024"); }
  // the recompression's Householder panels (bmax x 32 doubles plus their T
  // factor) live in shared memory
  if ((int64_t)p->bmax * QRB + QRB * QRB > RECOMP_REGION) {
    delete p;
    return fail(FRANK_ERR_UNSUPPORTED, "block size above " + std::to_string((RECOMP_REGION - QRB * QRB) / QRB) +
                                           " (recompression panels in shared memory)");
  }
  p->kcap = d->max_rank > 0 ? std::min(d->max_rank, p->bmax) : p->bmax;
  if (p->fixed_rank > p->kcap) p->kcap = std::min(p->fixed_rank, p->bmax);
  const int nb = d->nb;
  p->dslot_h.assign(nb * nb, -1);
  p->lslot_h.assign(nb * nb, -1);
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      const int bi = p->off_h[i + 1] - p->off_h[i], bj = p->off_h[j + 1] - p->off_h[j];
      const bool adm = (i != j) && bi > 1 && bj > 1 &&
                       (points ? geometry_admissible(points, dim, d->n, p->off_h[i], bi, p->off_h[j], bj, d->admis)
                               : std::abs(i - j) > (int)d->admis);
      if (adm) p->lslot_h[i * nb + j] = p->nlr++;
      else { p->dslot_h[i * nb + j] = p->ndense++; if (i != j) p->dense_offdiag = true; }
    }
  cudaDeviceProp prop;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) { delete p; return fail(FRANK_ERR_CUDA, std::string("device: ") + cudaGetErrorString(e)); }
  p->device = dev;
  p->sm_count = prop.multiProcessorCount;
  const size_t ts = tsize(p);
  const int64_t bm = p->bmax, kc = p->kcap;
  p->smax = (int)(kc + (p->dense_offdiag ? bm : kc));
  const RecompLayout L = recomp_layout(p->bmax, p->smax);
  const GramLayout LG = gram_layout(p->bmax, p->smax);
  p->rstride = std::max(L.total, LG.total);
  p->dstride = 2 * bm * bm;
  p->grid_recomp = std::max(1, std::min(nb * nb, p->sm_count - 1));
  p->grid_gram = std::max(1, std::min(nb * nb, 2 * (p->sm_count - 1)));
  p->grid_dense = std::max(1, std::min(nb * nb, 2 * p->sm_count));
  p->nrm_blocks = 256;
#define ALLOC(ptr, cnt)                                                                   \
  do {                                                                                    \
    cudaError_t _e = dalloc(&(ptr), (cnt));                                               \
    if (_e != cudaSuccess) {                                                              \
      free_plan(p);                                                                       \
      return fail(FRANK_ERR_CUDA, std::string("cudaMalloc " #ptr ": ") + cudaGetErrorString(_e)); \
    }                                                                                     \
  } while (0)
  ALLOC(p->d_off, nb + 1);
  ALLOC(p->d_dslot, nb * nb);
  ALLOC(p->d_lslot, nb * nb);
  ALLOC(p->d_rankH, nb * nb);
  ALLOC(p->d_rankW, nb * nb);
  ALLOC(p->Hd, p->ndense * bm * bm);
  ALLOC(p->Hu, p->nlr * bm * kc);
  ALLOC(p->Hs, p->nlr * kc * kc);
  ALLOC(p->Hv, p->nlr * bm * kc);
  char* t;
  ALLOC(t, p->ndense * bm * bm * ts); p->Wd = t;
  ALLOC(t, p->nlr * bm * kc * ts); p->Wu = t;
  ALLOC(t, p->nlr * kc * kc * ts); p->Ws = t;
  ALLOC(t, p->nlr * bm * kc * ts); p->Wv = t;
  ALLOC(p->perm, nb * bm);
  ALLOC(p->ipiv, nb * bm);
  ALLOC(p->err, ERR_SLOTS);
  ALLOC(p->work, 2 * nb);
  ALLOC(p->flops, FLOP_SLOTS);
  ALLOC(t, nb * bm * bm * ts); p->Linv = t;
  ALLOC(t, nb * bm * bm * ts); p->Uinv = t;
  ALLOC(t, nb * bm * bm * ts); p->WL = t;
  ALLOC(t, nb * bm * bm * ts); p->WU = t;
  ALLOC(p->getrf_scratch, bm * bm + 32 * bm);
  // dscratch / rscratch are allocated at the first factorization (ensure_scratch),
  // so frank_blr_set_grid can size them for batched use first.
  ALLOC(t, p->n * 8 * ts); p->z = t;
  ALLOC(t, bm * 8 * ts); p->stmp = t;
  ALLOC(t, (int64_t)nb * bm * 8 * ts); p->sctmp = t;
  ALLOC(p->part, (int64_t)nb * nb * bm * 8);
  ALLOC(p->vtmp, p->n * 8 * 3);
  ALLOC(p->nrm, p->nrm_blocks * 8);
#undef ALLOC
  if (cudaMallocHost(reinterpret_cast<void**>(&p->nrm_h), sizeof(double) * p->nrm_blocks * 8) != cudaSuccess) {
    free_plan(p);
    return fail(FRANK_ERR_CUDA, "cudaMallocHost");
  }
  p->ev.assign((size_t)nb * EV_SLOTS * 2, nullptr);
  for (auto& e : p->ev)
    if (cudaEventCreate(&e) != cudaSuccess) { free_plan(p); return fail(FRANK_ERR_CUDA, "cudaEventCreate"); }
  p->getrf_done.assign(nb, nullptr);
  p->dense_done.assign(nb, nullptr);
  p->panel_done.assign(nb, nullptr);
  p->next_done.assign(nb, nullptr);
  for (auto* v : {&p->getrf_done, &p->dense_done, &p->panel_done, &p->next_done})
    for (auto& e : *v)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
        free_plan(p);
        return fail(FRANK_ERR_CUDA, "cudaEventCreate");
      }
  if (cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&p->aux, cudaStreamNonBlocking) != cudaSuccess) {
    free_plan(p);
    return fail(FRANK_ERR_CUDA, "lookahead stream");
  }
  std::vector<int> zeros(nb * nb, 0);
  if (cudaMemcpy(p->d_off, p->off_h.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p->d_dslot, p->dslot_h.data(), sizeof(int) * nb * nb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p->d_lslot, p->lslot_h.data(), sizeof(int) * nb * nb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p->d_rankH, zeros.data(), sizeof(int) * nb * nb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p->d_rankW, zeros.data(), sizeof(int) * nb * nb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(p->Hd, 0, sizeof(double) * p->ndense * bm * bm) != cudaSuccess) {
    free_plan(p);
    return fail(FRANK_ERR_CUDA, "plan upload");
  }
  // dynamic shared memory of the solve / matvec kernels (8 RHS per pass)
  const int shm = (int)matvec_smem((int)bm, (int)kc, 8);
  const int shd = (int)((bm * 8 + (SOLVE_THREADS / SOLVE_ROWS) * SOLVE_ROWS * 8) * sizeof(double));
  // RHS per solve pass: the most whose scatter shared memory fits a CTA
  p->solve_chunk = 8;
  while (p->solve_chunk > 1 && solve_scatter_cl_smem((int)bm, (int)kc, p->solve_chunk) > (size_t)SMEM_OPTIN_MAX)
    p->solve_chunk /= 2;
  const int shs = (int)solve_scatter_cl_smem((int)bm, (int)kc, p->solve_chunk);
  cudaFuncSetAttribute(k_matvec_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, shm);
  cudaFuncSetAttribute(k_solve_scatter_cl<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, shs);
  cudaFuncSetAttribute(k_solve_scatter_cl<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, shs);
  cudaFuncSetAttribute(k_solve_diag<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, shd);
  cudaFuncSetAttribute(k_solve_diag<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, shd);
  cudaFuncSetAttribute(k_trinv<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, TRINV_SMEM_MAX);
  cudaFuncSetAttribute(k_trinv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, TRINV_SMEM_MAX);
  cudaFuncSetAttribute(k_recompress<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, RECOMP_SMEM_BYTES);
  cudaFuncSetAttribute(k_recompress<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, RECOMP_SMEM_BYTES);
  cudaFuncSetAttribute(k_recompress_b<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, RECOMP_SMEM_BYTES);
  cudaFuncSetAttribute(k_recompress_b<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, RECOMP_SMEM_BYTES);
  cudaFuncSetAttribute(k_trinv_b<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, TRINV_SMEM_MAX);
  cudaFuncSetAttribute(k_trinv_b<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, TRINV_SMEM_MAX);
  cudaFuncSetAttribute(k_recompress_gram<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, GRAM_SMEM_BYTES);
  cudaFuncSetAttribute(k_recompress_gram<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, GRAM_SMEM_BYTES);
  *out = p;
  return FRANK_OK;
}
}  // namespace

extern "C" {

int frank_blr_destroy(frank_blr* p) {
  if (!p) return FRANK_OK;
  cudaDeviceSynchronize();
  free_plan(p);
  return FRANK_OK;
}

int frank_blr_offsets(const frank_blr* p, int64_t* offsets) {
  if (!p || !offsets) return fail(FRANK_ERR_INVALID, "null argument");
  for (int i = 0; i <= p->nb; ++i) offsets[i] = p->off_h[i];
  return FRANK_OK;
}

int frank_blr_set_dense(frank_blr* p, int i, int j, const double* a, int64_t ld, int rowmajor) {
  int rc = check_block(p, i, j);
  if (rc) return rc;
  if (!a) return fail(FRANK_ERR_INVALID, "null data");
  const int s = p->dslot_h[i * p->nb + j];
  if (s < 0) return fail(FRANK_ERR_INVALID, "block is low rank under the plan's admissibility");
  const int bi = p->off_h[i + 1] - p->off_h[i], bj = p->off_h[j + 1] - p->off_h[j];
  if (ld < (rowmajor ? bj : bi)) return fail(FRANK_ERR_INVALID, "leading dimension too small");
  std::vector<double> h((size_t)p->bmax * p->bmax, 0.0);
  for (int c = 0; c < bj; ++c)
    for (int r = 0; r < bi; ++r) h[r + (size_t)c * p->bmax] = rowmajor ? a[(size_t)r * ld + c] : a[r + (size_t)c * ld];
  CUDA_TRY(cudaMemcpy(p->Hd + (size_t)s * p->bmax * p->bmax, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  p->factored = false;
  return FRANK_OK;
}

int frank_blr_set_lowrank(frank_blr* p, int i, int j, int rank, const double* U, int64_t ldu, const double* S,
                          int64_t lds, const double* V, int64_t ldv, int rowmajor) {
  int rc = check_block(p, i, j);
  if (rc) return rc;
  const int s = p->lslot_h[i * p->nb + j];
  if (s < 0) return fail(FRANK_ERR_INVALID, "block is dense under the plan's admissibility");
  if (rank <= 0 || rank > p->kcap) return fail(FRANK_ERR_RANK_OVERFLOW, "rank outside [1, max_rank]");
  if (!U || !S || !V) return fail(FRANK_ERR_INVALID, "null data");
  const int bi = p->off_h[i + 1] - p->off_h[i], bj = p->off_h[j + 1] - p->off_h[j];
  const int64_t bm = p->bmax, kc = p->kcap;
  std::vector<double> hu(bm * kc, 0.0), hs(kc * kc, 0.0), hv(bm * kc, 0.0);
  for (int c = 0; c < rank; ++c)
    for (int r = 0; r < bi; ++r) hu[r + c * bm] = rowmajor ? U[(size_t)r * ldu + c] : U[r + (size_t)c * ldu];
  for (int c = 0; c < rank; ++c)
    for (int r = 0; r < rank; ++r) hs[r + c * kc] = rowmajor ? S[(size_t)r * lds + c] : S[r + (size_t)c * lds];
  // V is rank x bj; stored transposed: Vt[col + a*bm] = V(a, col)
  for (int a = 0; a < rank; ++a)
    for (int c = 0; c < bj; ++c) hv[c + a * bm] = rowmajor ? V[(size_t)a * ldv + c] : V[a + (size_t)c * ldv];
  CUDA_TRY(cudaMemcpy(p->Hu + s * bm * kc, hu.data(), hu.size() * sizeof(double), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(p->Hs + s * kc * kc, hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(p->Hv + s * bm * kc, hv.data(), hv.size() * sizeof(double), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(p->d_rankH + i * p->nb + j, &rank, sizeof(int), cudaMemcpyHostToDevice));
  p->factored = false;
  p->orth_pending = true;
  return FRANK_OK;
}

int frank_blr_build_kernel(frank_blr* p, int kernel, const double* points, int dim, const double* kparams,
                           double eps, void* stream) {
  if (!p || !points) return fail(FRANK_ERR_INVALID, "null argument");
  if (kernel < 0 || kernel > 3 || dim < 1 || dim > 3) return fail(FRANK_ERR_INVALID, "bad kernel or dim");
  if (eps <= 0.0 && p->fixed_rank <= 0)
    return fail(FRANK_ERR_UNSUPPORTED, "on-device construction needs eps > 0 or a fixed-rank plan");
  if (kernel == FRANK_KERNEL_EXP && !(kparams && kparams[0] > 0.0))
    return fail(FRANK_ERR_INVALID, "exp kernel needs theta > 0");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // construction temporaries: freed on every return path
  DevBuf<double> dx, d_of, d_ol, scratch;
  DevBuf<int> d_dl, d_ll;
  CUDA_TRY(dx.alloc((size_t)dim * p->n));
  CUDA_TRY(cudaMemcpy(dx.get(), points, sizeof(double) * dim * p->n, cudaMemcpyHostToDevice));
  KernelDesc K;
  K.kind = kernel; K.dim = dim; K.x = dx.get(); K.n = p->n;
  K.p0 = kparams ? kparams[0] : 0.0;
  K.p1 = kparams ? kparams[1] : 0.0;
  std::vector<int> dl, ll;
  for (int b = 0; b < p->nb * p->nb; ++b) {
    if (p->dslot_h[b] >= 0) dl.push_back(b);
    else ll.push_back(b);
  }
  CUDA_TRY(d_dl.alloc(dl.size()));
  CUDA_TRY(d_ll.alloc(ll.size()));
  if (!dl.empty()) CUDA_TRY(cudaMemcpy(d_dl.get(), dl.data(), sizeof(int) * dl.size(), cudaMemcpyHostToDevice));
  if (!ll.empty()) CUDA_TRY(cudaMemcpy(d_ll.get(), ll.data(), sizeof(int) * ll.size(), cudaMemcpyHostToDevice));
  BlrView<double> H = h_view(p);
  if (!dl.empty()) k_build_dense<<<(int)std::min<size_t>(dl.size(), 4096), 256, 0, s>>>(H, K, d_dl.get(), (int)dl.size());
  int rc = FRANK_OK;
  if (!ll.empty() && eps <= 0.0) {
    // fixed rank: LowRank(Dense, rank) -> rsvd with sample min(rank + 5, m, n)
    // and the reference's Omega (random_uniform, functions.cpp:52-66)
    const int64_t bm = p->bmax;
    const int last = p->off_h[p->nb] - p->off_h[p->nb - 1];
    const int psamp = std::min<int>(p->fixed_rank + 5, std::min<int>(bm, last));
    if (p->fixed_rank + 5 > last && last != bm)
      return fail(FRANK_ERR_UNSUPPORTED, "fixed-rank construction with a short last block below rank + 5");
    auto omega = [&](int ncols) {
      std::mt19937 gen;
      gen.seed(0);
      std::uniform_real_distribution<double> dist(0.0, 1.0);
      std::vector<double> om((size_t)ncols * psamp);
      for (auto& v : om) v = dist(gen);
      return om;
    };
    const std::vector<double> of = omega((int)bm), ol = omega(last);
    CUDA_TRY(d_of.alloc(of.size()));
    CUDA_TRY(d_ol.alloc(ol.size()));
    CUDA_TRY(cudaMemcpy(d_of.get(), of.data(), sizeof(double) * of.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_ol.get(), ol.data(), sizeof(double) * ol.size(), cudaMemcpyHostToDevice));
    const int64_t stride = bm * bm + 2 * bm * psamp + (bm + psamp) * psamp + 4 * psamp + 64;
    const int grid = (int)std::min<size_t>(ll.size(), (size_t)2 * p->sm_count);
    CUDA_TRY(scratch.alloc((size_t)stride * grid));
    CUDA_TRY(cudaMemsetAsync(p->err, 0, ERR_SLOTS * sizeof(int), s));
    k_build_lowrank_rsvd<<<grid, BUILD_THREADS, 0, s>>>(H, K, d_ll.get(), (int)ll.size(), p->fixed_rank, psamp,
                                                        d_of.get(), d_ol.get(), stride, scratch.get(), p->err);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s));
    CUDA_TRY(cudaMemcpy(p->err_h, p->err, ERR_SLOTS * sizeof(int), cudaMemcpyDeviceToHost));
    if (p->err_h[ERR_RANK_OVERFLOW]) rc = fail(FRANK_ERR_RANK_OVERFLOW, "the fixed rank exceeds max_rank");
  } else if (!ll.empty()) {
    const int64_t bm = p->bmax;
    const int64_t stride = 3 * bm * bm + 6 * bm;
    const int grid = (int)std::min<size_t>(ll.size(), (size_t)2 * p->sm_count);
    CUDA_TRY(scratch.alloc((size_t)stride * grid));
    CUDA_TRY(cudaMemsetAsync(p->err, 0, ERR_SLOTS * sizeof(int), s));
    k_build_lowrank<<<grid, BUILD_THREADS, 0, s>>>(H, K, d_ll.get(), (int)ll.size(), eps, scratch.get(), stride, p->err);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s));
    CUDA_TRY(cudaMemcpy(p->err_h, p->err, ERR_SLOTS * sizeof(int), cudaMemcpyDeviceToHost));
    if (p->err_h[ERR_RANK_OVERFLOW]) rc = fail(FRANK_ERR_RANK_OVERFLOW, "a compressed block exceeded max_rank and was truncated");
  }
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(s));
  p->factored = false;
  return rc;
}

int frank_blr_block_info(const frank_blr* p, int which, int i, int j, int* type, int* rank) {
  int rc = check_block(p, i, j);
  if (rc) return rc;
  const bool lr = p->lslot_h[i * p->nb + j] >= 0;
  if (type) *type = lr ? FRANK_BLOCK_LOWRANK : FRANK_BLOCK_DENSE;
  if (rank) {
    *rank = 0;
    if (lr) CUDA_TRY(cudaMemcpy(rank, (which ? p->d_rankW : p->d_rankH) + i * p->nb + j, sizeof(int), cudaMemcpyDeviceToHost));
  }
  return FRANK_OK;
}


int frank_blr_get_dense(const frank_blr* p, int which, int i, int j, double* a, int64_t ld, int rowmajor) {
  int rc = check_block(p, i, j);
  if (rc) return rc;
  const int s = p->dslot_h[i * p->nb + j];
  if (s < 0) return fail(FRANK_ERR_INVALID, "block is low rank");
  const int bi = p->off_h[i + 1] - p->off_h[i], bj = p->off_h[j + 1] - p->off_h[j];
  const size_t cnt = (size_t)p->bmax * p->bmax;
  const char* base = which ? static_cast<const char*>(p->Wd) + s * cnt * tsize(p)
                           : reinterpret_cast<const char*>(p->Hd + s * cnt);
  std::vector<double> h;
  if ((rc = fetch(p, which, base, cnt, h))) return rc;
  for (int c = 0; c < bj; ++c)
    for (int r = 0; r < bi; ++r) {
      const double v = h[r + (size_t)c * p->bmax];
      if (rowmajor) a[(size_t)r * ld + c] = v; else a[r + (size_t)c * ld] = v;
    }
  return FRANK_OK;
}

int frank_blr_get_lowrank(const frank_blr* p, int which, int i, int j, double* U, int64_t ldu, double* S,
                          int64_t lds, double* V, int64_t ldv, int rowmajor) {
  int rc = check_block(p, i, j);
  if (rc) return rc;
  const int s = p->lslot_h[i * p->nb + j];
  if (s < 0) return fail(FRANK_ERR_INVALID, "block is dense");
  int rank = 0;
  CUDA_TRY(cudaMemcpy(&rank, (which ? p->d_rankW : p->d_rankH) + i * p->nb + j, sizeof(int), cudaMemcpyDeviceToHost));
  const int bi = p->off_h[i + 1] - p->off_h[i], bj = p->off_h[j + 1] - p->off_h[j];
  const size_t bm = p->bmax, kc = p->kcap;
  const size_t es = which ? tsize(p) : sizeof(double);
  const char* bu = which ? static_cast<const char*>(p->Wu) : reinterpret_cast<const char*>(p->Hu);
  const char* bs = which ? static_cast<const char*>(p->Ws) : reinterpret_cast<const char*>(p->Hs);
  const char* bv = which ? static_cast<const char*>(p->Wv) : reinterpret_cast<const char*>(p->Hv);
  std::vector<double> hu, hs, hv;
  if ((rc = fetch(p, which, bu + s * bm * kc * es, bm * kc, hu))) return rc;
  if ((rc = fetch(p, which, bs + s * kc * kc * es, kc * kc, hs))) return rc;
  if ((rc = fetch(p, which, bv + s * bm * kc * es, bm * kc, hv))) return rc;
  for (int c = 0; c < rank; ++c)
    for (int r = 0; r < bi; ++r) {
      const double v = hu[r + c * bm];
      if (rowmajor) U[(size_t)r * ldu + c] = v; else U[r + (size_t)c * ldu] = v;
    }
  for (int c = 0; c < rank; ++c)
    for (int r = 0; r < rank; ++r) {
      const double v = hs[r + c * kc];
      if (rowmajor) S[(size_t)r * lds + c] = v; else S[r + (size_t)c * lds] = v;
    }
  for (int a = 0; a < rank; ++a)
    for (int c = 0; c < bj; ++c) {
      const double v = hv[c + a * bm];
      if (rowmajor) V[(size_t)a * ldv + c] = v; else V[a + (size_t)c * ldv] = v;
    }
  return FRANK_OK;
}

int frank_blr_get_pivots(const frank_blr* p, int i, int* ipiv) {
  int rc = check_block(p, i, i);
  if (rc) return rc;
  if (!p->factored) return fail(FRANK_ERR_STATE, "pivots before getrf");
  const int b = p->off_h[i + 1] - p->off_h[i];
  CUDA_TRY(cudaMemcpy(ipiv, p->ipiv + (size_t)i * p->bmax, sizeof(int) * b, cudaMemcpyDeviceToHost));
  for (int r = 0; r < b; ++r) ipiv[r] += 1;
  return FRANK_OK;
}

int frank_blr_set_lra(frank_blr* p, const char* name, double core_scale) {
  if (!p || !name) return fail(FRANK_ERR_INVALID, "null argument");
  const std::string n(name);
  // addition.cpp:191-203: "rounded_addition" selects it for every plan;
  // "fast_rounded_addition" (the reference's default) falls back to
  // rounded_addition on tolerance plans (addition.cpp:138-143); the engine's
  // RRQR cores are selected by name; "naive" is refused (its ranks grow
  // without bound, a plan's rank capacity is fixed)
  bool proj = false;
  if (n == "naive" || n == "naive_addition")
    return fail(FRANK_ERR_UNSUPPORTED, "naive addition needs unbounded ranks; a plan has a fixed rank capacity "
                                       "(frank_lowrank_add_batched supports it)");
  if (n == "rounded_addition") { p->core_method = CORE_SVD; p->core_fixed = CORE_SVD; p->gram = false; }
  else if (n == "fast_rounded_addition") { p->core_method = CORE_SVD; p->core_fixed = CORE_FAST; p->gram = false; }
  else if (n == "rounded_addition_rrqr") { p->core_method = CORE_RRQR; p->core_fixed = CORE_SVD; p->gram = false; }
  else if (n == "rounded_addition_rrqr_proj") {
    p->core_method = CORE_RRQR; p->core_fixed = CORE_FAST; p->gram = false; proj = true;
  }
  else if (n == "rounded_addition_rrqr_gram") { p->core_method = CORE_RRQR; p->core_fixed = CORE_SVD; p->gram = true; }
  else return fail(FRANK_ERR_UNSUPPORTED, "unknown FRANK_LRA value: " + n);
  p->proj_tol = proj;
  p->core_scale = core_scale > 0.0 ? core_scale : 0.1;
  if (p->graph_exec) { cudaGraphExecDestroy(p->graph_exec); p->graph_exec = nullptr; }
  if (p->graph) { cudaGraphDestroy(p->graph); p->graph = nullptr; }
  p->factored = false;
  return FRANK_OK;
}

int frank_blr_getrf(frank_blr* p, void* stream) {
  if (!p) return fail(FRANK_ERR_INVALID, "null plan");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!s) {
    if (!p->graph_stream) CUDA_TRY(cudaStreamCreateWithFlags(&p->graph_stream, cudaStreamNonBlocking));
    s = p->graph_stream;
  }
  p->factored = false;
  return p->precision == FRANK_PREC_FP64 ? run_factor<double>(p, s) : run_factor<float>(p, s);
}

int frank_blr_solve_device(frank_blr* p, double* d_b, int64_t ldb, int nrhs, void* stream) {
  if (!p || !d_b || nrhs < 1 || ldb < p->n) return fail(FRANK_ERR_INVALID, "bad solve arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = solve_device_impl(p, d_b, ldb, nrhs, false, s);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(s));
  return FRANK_OK;
}

int frank_blr_solve_transpose_device(frank_blr* p, double* d_b, int64_t ldb, int nrhs, void* stream) {
  if (!p || !d_b || nrhs < 1 || ldb < p->n) return fail(FRANK_ERR_INVALID, "bad solve arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = solve_device_impl(p, d_b, ldb, nrhs, true, s);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(s));
  return FRANK_OK;
}

// Device copies for the host-buffer entry points (b, x or y): kept by the
// plan and grown on demand, so that repeated calls do not allocate.  Returns
// two n x nrhs regions.
namespace {
int host_io(frank_blr* p, int nrhs, double** a, double** b) {
  const size_t need = (size_t)p->n * nrhs;
  if (need > p->host_io_cap) {
    if (p->host_io) cudaFree(p->host_io);
    p->host_io = nullptr;
    p->host_io_cap = 0;
    CUDA_TRY(cudaMalloc(&p->host_io, 2 * need * sizeof(double)));
    p->host_io_cap = need;
  }
  *a = p->host_io;
  *b = p->host_io + need;
  return FRANK_OK;
}
}  // namespace

int frank_blr_solve(frank_blr* p, double* b, int64_t ldb, int nrhs, void* stream) {
  if (!p || !b || nrhs < 1 || ldb < p->n) return fail(FRANK_ERR_INVALID, "bad solve arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *d = nullptr, *unused = nullptr;
  {
    const int rc0 = host_io(p, nrhs, &d, &unused);
    if (rc0) return rc0;
  }
  CUDA_TRY(cudaMemcpy2DAsync(d, p->n * sizeof(double), b, ldb * sizeof(double), p->n * sizeof(double), nrhs,
                             cudaMemcpyHostToDevice, s));
  int rc = solve_device_impl(p, d, p->n, nrhs, false, s);
  if (rc == FRANK_OK) {
    cudaError_t e = cudaMemcpy2DAsync(b, ldb * sizeof(double), d, p->n * sizeof(double), p->n * sizeof(double), nrhs,
                                      cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(FRANK_ERR_CUDA, cudaGetErrorString(e));
  }
  return rc;
}

int frank_blr_trsm(frank_blr* p, int uplo, double* b, int64_t ldb, int nrhs, void* stream) {
  if (!p || !b || nrhs < 1 || ldb < p->n || (uplo != FRANK_LOWER && uplo != FRANK_UPPER))
    return fail(FRANK_ERR_INVALID, "bad trsm arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *d = nullptr, *unused = nullptr;
  {
    const int rc0 = host_io(p, nrhs, &d, &unused);
    if (rc0) return rc0;
  }
  CUDA_TRY(cudaMemcpy2DAsync(d, p->n * sizeof(double), b, ldb * sizeof(double), p->n * sizeof(double), nrhs,
                             cudaMemcpyHostToDevice, s));
  int rc = solve_device_impl(p, d, p->n, nrhs, false, s, uplo == FRANK_LOWER ? 1 : 2);
  if (rc == FRANK_OK) {
    cudaError_t e = cudaMemcpy2DAsync(b, ldb * sizeof(double), d, p->n * sizeof(double), p->n * sizeof(double), nrhs,
                                      cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(FRANK_ERR_CUDA, cudaGetErrorString(e));
  }
  return rc;
}

int frank_blr_gemv(frank_blr* p, double alpha, const double* x, int64_t ldx, double beta, double* y, int64_t ldy,
                   int nrhs, void* stream) {
  if (!p || !x || !y || nrhs < 1 || ldx < p->n || ldy < p->n) return fail(FRANK_ERR_INVALID, "bad gemv arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *dx = nullptr, *dy = nullptr;
  {
    const int rc0 = host_io(p, nrhs, &dx, &dy);
    if (rc0) return rc0;
  }
  CUDA_TRY(cudaMemcpy2DAsync(dx, p->n * sizeof(double), x, ldx * sizeof(double), p->n * sizeof(double), nrhs,
                             cudaMemcpyHostToDevice, s));
  double* dy0 = p->vtmp;     // beta * y needs the old y on the device
  CUDA_TRY(cudaMemcpy2DAsync(dy0, p->n * sizeof(double), y, ldy * sizeof(double), p->n * sizeof(double), nrhs,
                             cudaMemcpyHostToDevice, s));
  int rc = matvec_device_impl(p, dx, p->n, dy, p->n, nrhs, nullptr, 0, s);
  if (rc == FRANK_OK) {
    ++p->solve_launches;
    k_axpby<<<grid_for(p->n * nrhs), 256, 0, s>>>(alpha, dy, beta, dy0, p->n, nrhs);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(y, ldy * sizeof(double), dy0, p->n * sizeof(double), p->n * sizeof(double), nrhs,
                            cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(FRANK_ERR_CUDA, cudaGetErrorString(e));
  }
  return rc;
}

int frank_blr_matvec_device(frank_blr* p, const double* d_x, int64_t ldx, double* d_y, int64_t ldy, int nrhs,
                            void* stream) {
  if (!p || !d_x || !d_y || nrhs < 1 || ldx < p->n || ldy < p->n) return fail(FRANK_ERR_INVALID, "bad matvec arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = matvec_device_impl(p, d_x, ldx, d_y, ldy, nrhs, nullptr, 0, s);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(s));
  return FRANK_OK;
}

int frank_blr_matvec(frank_blr* p, const double* x, int64_t ldx, double* y, int64_t ldy, int nrhs, void* stream) {
  if (!p || !x || !y || nrhs < 1 || ldx < p->n || ldy < p->n) return fail(FRANK_ERR_INVALID, "bad matvec arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *dx = nullptr, *dy = nullptr;
  {
    const int rc0 = host_io(p, nrhs, &dx, &dy);
    if (rc0) return rc0;
  }
  CUDA_TRY(cudaMemcpy2DAsync(dx, p->n * sizeof(double), x, ldx * sizeof(double), p->n * sizeof(double), nrhs,
                             cudaMemcpyHostToDevice, s));
  int rc = matvec_device_impl(p, dx, p->n, dy, p->n, nrhs, nullptr, 0, s);
  if (rc == FRANK_OK) {
    cudaError_t e = cudaMemcpy2DAsync(y, ldy * sizeof(double), dy, p->n * sizeof(double), p->n * sizeof(double), nrhs,
                                      cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(FRANK_ERR_CUDA, cudaGetErrorString(e));
  }
  return rc;
}

int frank_blr_refine_device(frank_blr* p, const double* d_b, int64_t ldb, double* d_x, int64_t ldx, int nrhs,
                            double tol, int maxit, int* iters, double* resid, void* stream) {
  if (!p || !d_b || !d_x || nrhs < 1 || ldb < p->n || ldx < p->n || maxit < 0)
    return fail(FRANK_ERR_INVALID, "bad refine arguments");
  return refine_device_impl(p, d_b, ldb, d_x, ldx, nrhs, tol, maxit, iters, resid, static_cast<cudaStream_t>(stream));
}

int frank_blr_refine(frank_blr* p, const double* b, int64_t ldb, double* x, int64_t ldx, int nrhs, double tol,
                     int maxit, int* iters, double* resid, void* stream) {
  if (!p || !b || !x || nrhs < 1 || ldb < p->n || ldx < p->n || maxit < 0)
    return fail(FRANK_ERR_INVALID, "bad refine arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *db = nullptr, *dx = nullptr;
  {
    const int rc0 = host_io(p, nrhs, &db, &dx);
    if (rc0) return rc0;
  }
  CUDA_TRY(cudaMemcpy2DAsync(db, p->n * sizeof(double), b, ldb * sizeof(double), p->n * sizeof(double), nrhs,
                             cudaMemcpyHostToDevice, s));
  int rc = refine_device_impl(p, db, p->n, dx, p->n, nrhs, tol, maxit, iters, resid, s);
  if (rc == FRANK_OK || rc == FRANK_ERR_NOT_CONVERGED) {
    cudaError_t e = cudaMemcpy2DAsync(x, ldx * sizeof(double), dx, p->n * sizeof(double), p->n * sizeof(double), nrhs,
                                      cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(FRANK_ERR_CUDA, cudaGetErrorString(e));
  }
  return rc;
}

int frank_blr_write_json(const frank_blr* p, int which, const char* path) {
  if (!p || !path || (which != 0 && which != 1)) return fail(FRANK_ERR_INVALID, "bad write_json arguments");
  if (which == 1 && (!p->factored || p->precision != FRANK_PREC_FP64))
    return fail(FRANK_ERR_UNSUPPORTED, "write_json of the factor needs a factored FP64 plan");
  const int nb = p->nb, bm = p->bmax, kc = p->kcap;
  const double* D = which ? static_cast<const double*>(p->Wd) : p->Hd;
  const double* U = which ? static_cast<const double*>(p->Wu) : p->Hu;
  const double* S = which ? static_cast<const double*>(p->Ws) : p->Hs;
  const double* V = which ? static_cast<const double*>(p->Wv) : p->Hv;
  const int* rk = which ? p->d_rankW : p->d_rankH;
  std::vector<int> ranks((size_t)nb * nb);
  CUDA_TRY(cudaMemcpy(ranks.data(), rk, sizeof(int) * ranks.size(), cudaMemcpyDeviceToHost));
  // scratch: U / Vt factors of an SVD (bm x bm each), singular values, the
  // small core products (kc x kc each)
  DevBuf<double> su, ss, sv, qa, ra, qb, rb, t1, t2;
  CUDA_TRY(su.alloc((size_t)bm * bm));
  CUDA_TRY(ss.alloc((size_t)bm));
  CUDA_TRY(sv.alloc((size_t)bm * bm));
  CUDA_TRY(qa.alloc((size_t)bm * kc));
  CUDA_TRY(ra.alloc((size_t)kc * kc));
  CUDA_TRY(qb.alloc((size_t)bm * kc));
  CUDA_TRY(rb.alloc((size_t)kc * kc));
  CUDA_TRY(t1.alloc((size_t)kc * kc));
  CUDA_TRY(t2.alloc((size_t)kc * kc));
  std::string out;
  char buf[64];
  auto num = [&](double v) { snprintf(buf, sizeof buf, "%.17g", v); out += buf; };
  const int64_t n = p->n;
  out += "{\"abs_pos\":[0,0],\"children\":[";
  for (int i = 0; i < nb; ++i) {
    out += i ? ",[" : "[";
    for (int j = 0; j < nb; ++j) {
      const int bi = p->off_h[i + 1] - p->off_h[i], bj = p->off_h[j + 1] - p->off_h[j], k = std::min(bi, bj);
      std::vector<double> sval(k, 0.0);
      const int ls = p->lslot_h[i * nb + j];
      int rc = FRANK_OK;
      const int r = ls >= 0 ? ranks[i * nb + j] : 0;
      if (ls < 0) {
        rc = frank_svd_batched(bi, bj, 1, D + (size_t)p->dslot_h[i * nb + j] * bm * bm, bm, 0, su.get(), bi, 0,
                               ss.get(), 0, sv.get(), k, 0, nullptr);
        if (rc == FRANK_OK) CUDA_TRY(cudaMemcpy(sval.data(), ss.get(), sizeof(double) * k, cudaMemcpyDeviceToHost));
      } else if (r > 0) {
        // singular values of U S V from its core R_u S R_v^T (QR of both bases)
        const double* u = U + (size_t)ls * bm * kc;
        const double* vt = V + (size_t)ls * bm * kc;
        const double* sm = S + (size_t)ls * kc * kc;
        rc = frank_qr_batched(bi, r, 1, u, bm, 0, qa.get(), bi, 0, ra.get(), r, 0, nullptr);
        if (rc == FRANK_OK) rc = frank_qr_batched(bj, r, 1, vt, bm, 0, qb.get(), bj, 0, rb.get(), r, 0, nullptr);
        if (rc == FRANK_OK)
          rc = frank_gemm_batched(r, r, r, 1, 1.0, ra.get(), r, 0, 0, sm, kc, 0, 0, 0.0, t1.get(), r, 0, nullptr);
        if (rc == FRANK_OK)
          rc = frank_gemm_batched(r, r, r, 1, 1.0, t1.get(), r, 0, 0, rb.get(), r, 0, 1, 0.0, t2.get(), r, 0, nullptr);
        if (rc == FRANK_OK)
          rc = frank_svd_batched(r, r, 1, t2.get(), r, 0, su.get(), r, 0, ss.get(), 0, sv.get(), r, 0, nullptr);
        if (rc == FRANK_OK) CUDA_TRY(cudaMemcpy(sval.data(), ss.get(), sizeof(double) * r, cudaMemcpyDeviceToHost));
      }
      if (rc != FRANK_OK) return rc;
      out += j ? ",{" : "{";
      snprintf(buf, sizeof buf, "\"abs_pos\":[%d,%d],\"dim\":[%d,%d],\"level\":1,", i, j, bi, bj);
      out += buf;
      if (ls >= 0) {
        snprintf(buf, sizeof buf, "\"rank\":%d,", r);
        out += buf;
      }
      out += "\"svalues\":[";
      for (int c = 0; c < k; ++c) {
        if (c) out += ",";
        num(sval[c]);
      }
      out += ls >= 0 ? "],\"type\":\"LowRank\"}" : "],\"type\":\"Dense\"}";
    }
    out += "]";
  }
  snprintf(buf, sizeof buf, "],\"dim\":[%lld,%lld],\"level\":0,\"type\":\"Hierarchical\"}", (long long)n, (long long)n);
  out += buf;
  FILE* f = fopen(path, "w");
  if (!f) return fail(FRANK_ERR_INVALID, std::string("cannot write ") + path);
  const size_t w = fwrite(out.data(), 1, out.size(), f);
  fclose(f);
  if (w != out.size()) return fail(FRANK_ERR_INVALID, std::string("short write to ") + path);
  return FRANK_OK;
}

namespace {

// Chosen launch parameters per workload shape, for the life of the process.
struct TuneKey {
  int64_t n;
  int nb, precision, fixed_rank, core_method, lra_fixed;
  double eps;
  bool operator<(const TuneKey& o) const {
    return std::tie(n, nb, precision, fixed_rank, core_method, lra_fixed, eps) <
           std::tie(o.n, o.nb, o.precision, o.fixed_rank, o.core_method, o.lra_fixed, o.eps);
  }
};
struct TuneVal {
  int band, split, proj, core_smem;
  double ms;
};
std::map<TuneKey, TuneVal> g_tuned;
std::mutex g_tune_mutex;

void drop_graph(frank_blr* p) {
  if (p->graph_exec) { cudaGraphExecDestroy(p->graph_exec); p->graph_exec = nullptr; }
  if (p->graph) { cudaGraphDestroy(p->graph); p->graph = nullptr; }
  p->factored = false;
}

// Device time (ms) of one factorization with the plan's current parameters:
// one launch to capture, then the faster of two timed replays.
int time_factor(frank_blr* p, cudaStream_t s, double* ms) {
  drop_graph(p);
  int rc = frank_blr_getrf(p, s);
  if (rc != FRANK_OK && rc != FRANK_ERR_RANK_OVERFLOW) return rc;
  cudaEvent_t a = nullptr, b = nullptr;
  CUDA_TRY(cudaEventCreate(&a));
  CUDA_TRY(cudaEventCreate(&b));
  double best = 1e300;
  for (int k = 0; k < 2 && rc == FRANK_OK; ++k) {
    cudaEventRecord(a, s);
    rc = frank_blr_getrf(p, s);
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    best = std::min(best, (double)t);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = best;
  return rc == FRANK_ERR_RANK_OVERFLOW ? FRANK_OK : rc;
}

}  // namespace

int frank_blr_autotune(frank_blr* p, int force, void* stream) {
  if (!p) return fail(FRANK_ERR_INVALID, "null plan");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!s) {
    if (!p->graph_stream) CUDA_TRY(cudaStreamCreateWithFlags(&p->graph_stream, cudaStreamNonBlocking));
    s = p->graph_stream;
  }
  const TuneKey key{p->n, p->nb, p->precision, p->fixed_rank, p->core_method, p->core_fixed, p->eps};
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tuned.find(key);
    if (!force && it != g_tuned.end()) {
      p->dupd_band = it->second.band;
      p->split_p = it->second.split;
      p->proj_tol = it->second.proj != 0;
      p->core_smem = it->second.core_smem;
      drop_graph(p);
      return FRANK_OK;
    }
  }
  // coordinate descent over the launch parameters, one at a time, each
  // candidate timed on the plan's own factorization
  double best = 0.0;
  int rc = time_factor(p, s, &best);
  if (rc) return rc;
  auto try_values = [&](int* field, std::initializer_list<int> vals) -> int {
    const int keep = *field;
    int chosen = keep;
    for (int v : vals) {
      if (v == keep) continue;
      *field = v;
      double t = 0.0;
      const int r = time_factor(p, s, &t);
      if (r) { *field = keep; return r; }
      if (t < best) { best = t; chosen = v; }
    }
    *field = chosen;
    return FRANK_OK;
  };
  if ((rc = try_values(&p->dupd_band, {64, 128, 256}))) return rc;
  if (p->nlr > 0 && split_on(p) && p->rsplit) {
    if ((rc = try_values(&p->split_p, {0, 16, 32, 48, 64, 96}))) return rc;
  }
  if (p->nlr > 0 && p->fixed_rank == 0 && p->core_method == CORE_RRQR && !p->gram) {
    int proj = p->proj_tol ? 1 : 0;
    const int keep = proj;
    p->proj_tol = !keep;
    double t = 0.0;
    if ((rc = time_factor(p, s, &t))) { p->proj_tol = keep; return rc; }
    if (t < best) { best = t; proj = !keep; }
    p->proj_tol = proj != 0;
  }
  // largest recompression core kept in shared memory: larger ones take the
  // blocked / randomized paths in L2 (randomized pivoting for the RRQR core)
  if (p->nlr > 0 && (rc = try_values(&p->core_smem, {RECOMP_REGION, 16384, 6144}))) return rc;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tuned[key] = TuneVal{p->dupd_band, p->split_p, p->proj_tol ? 1 : 0, p->core_smem, best};
  }
  drop_graph(p);
  return FRANK_OK;
}

int frank_blr_set_tuning(frank_blr* p, int band_rows, int split_rank, int projected) {
  if (!p || band_rows < 16 || split_rank < 0) return fail(FRANK_ERR_INVALID, "bad tuning values");
  p->dupd_band = band_rows;
  p->split_p = split_rank;
  p->proj_tol = projected != 0;
  drop_graph(p);
  return FRANK_OK;
}

int frank_blr_tuning(const frank_blr* p, int* band_rows, int* split_rank, int* projected) {
  if (!p) return fail(FRANK_ERR_INVALID, "null plan");
  if (band_rows) *band_rows = p->dupd_band;
  if (split_rank) *split_rank = p->split_p;
  if (projected) *projected = p->proj_tol ? 1 : 0;
  return FRANK_OK;
}

int frank_blr_core_smem(const frank_blr* p, int* doubles) {
  if (!p || !doubles) return fail(FRANK_ERR_INVALID, "null argument");
  *doubles = p->core_smem;
  return FRANK_OK;
}

int frank_blr_set_core_smem(frank_blr* p, int doubles) {
  if (!p || doubles < 1) return fail(FRANK_ERR_INVALID, "bad core size");
  p->core_smem = doubles;
  drop_graph(p);
  return FRANK_OK;
}

int frank_blr_kernel_times(const frank_blr* p, double* ms, double* flops) {
  if (!p) return fail(FRANK_ERR_INVALID, "null plan");
  // four reported classes; the inverse kernel's time belongs to class 0
  for (int c = 0; c < FLOP_TRINV; ++c) {
    if (ms) ms[c] = p->class_ms[c] + (c == FLOP_GETRF ? p->class_ms[FLOP_TRINV] : 0.0);
    if (flops) flops[c] = (double)p->flops_h[c];
  }
  return FRANK_OK;
}

int frank_blr_stats(const frank_blr* p, int64_t* launches, int64_t* recompressions, int64_t* max_rank_seen,
                    int64_t* rank_overflows) {
  if (!p) return fail(FRANK_ERR_INVALID, "null plan");
  if (launches) *launches = p->launches + p->solve_launches;
  if (recompressions) *recompressions = p->err_h[ERR_RECOMP];
  if (max_rank_seen) *max_rank_seen = p->err_h[ERR_MAX_RANK];
  if (rank_overflows) *rank_overflows = p->err_h[ERR_RANK_OVERFLOW];
  return FRANK_OK;
}

}  // extern "C"

extern "C" int frank_blr_matvec_transpose_device(frank_blr* p, const double* d_x, int64_t ldx, double* d_y,
                                                 int64_t ldy, int nrhs, void* stream) {
  if (!p || !d_x || !d_y || nrhs < 1 || ldx < p->n || ldy < p->n) return fail(FRANK_ERR_INVALID, "bad matvec arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = matvec_device_impl(p, d_x, ldx, d_y, ldy, nrhs, nullptr, 0, s, true);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(s));
  return FRANK_OK;
}

extern "C" int frank_blr_refine_transpose_device(frank_blr* p, const double* d_b, int64_t ldb, double* d_x,
                                                 int64_t ldx, int nrhs, double tol, int maxit, int* iters,
                                                 double* resid, void* stream) {
  if (!p || !d_b || !d_x || nrhs < 1 || ldb < p->n || ldx < p->n || maxit < 0)
    return fail(FRANK_ERR_INVALID, "bad refine arguments");
  return refine_device_impl(p, d_b, ldb, d_x, ldx, nrhs, tol, maxit, iters, resid, static_cast<cudaStream_t>(stream),
                            true);
}

extern "C" int frank_kernel_dtheta_contract(int kernel, const double* d_points, int dim, int64_t n,
                                            const double* kparams, const double* d_lambda, int64_t ldl,
                                            const double* d_x, int64_t ldx, int nrhs, double* out, void* stream) {
  if (kernel != FRANK_KERNEL_EXP) return fail(FRANK_ERR_UNSUPPORTED, "dA/dtheta is defined for the exp kernel only");
  if (!d_points || !kparams || !d_lambda || !d_x || !out || dim < 1 || dim > 3 || n < 1 || nrhs < 1 || nrhs > 8 ||
      ldl < n || ldx < n || !(kparams[0] > 0.0))
    return fail(FRANK_ERR_INVALID, "bad dtheta contraction arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t tiles = (n + DT_TILE - 1) / DT_TILE;
  if (tiles > 65535) return fail(FRANK_ERR_UNSUPPORTED, "too many points for the contraction grid");
  // per-tile partials from the stream-ordered pool (no device-wide
  // synchronisation, reused across calls by the pool)
  double* part = nullptr;
  CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&part), sizeof(double) * tiles * tiles, s));
  k_dtheta_contract<<<dim3((unsigned)tiles, (unsigned)tiles), 256, 0, s>>>(d_points, dim, n, kparams[0], d_lambda, ldl,
                                                                          d_x, ldx, nrhs, part);
  cudaError_t e = cudaGetLastError();
  std::vector<double> h((size_t)tiles * tiles);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s);
  cudaError_t ef = cudaFreeAsync(part, s);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(FRANK_ERR_CUDA, cudaGetErrorString(e));
  double acc = 0.0;
  for (double v : h) acc += v;
  *out = acc;
  return FRANK_OK;
}

// ===========================================================================
// Batches of independent systems (the batched uneven-systems workload):
// every plan's factorization is one branch of a single captured graph, so
// systems of different sizes run concurrently and the whole batch is one
// graph launch; the batched refinement synchronises the host once per
// iteration for all systems.
// ===========================================================================
struct frank_batch {
  std::vector<frank_blr*> plans;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> streams;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // one launch per elimination step over all systems (when they share the
  // block size and launch grids): the device table of the systems and the
  // step events of the two streams
  bool stepwise = false;
  void* d_sys = nullptr;
  cudaStream_t aux = nullptr;
  std::vector<cudaEvent_t> ev_getrf, ev_panel, ev_dense;
};

namespace {
void free_batch(frank_batch* B) {
  if (!B) return;
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  if (B->d_sys) cudaFree(B->d_sys);
  if (B->aux) cudaStreamDestroy(B->aux);
  for (auto* v : {&B->ev_getrf, &B->ev_panel, &B->ev_dense})
    for (auto e : *v) if (e) cudaEventDestroy(e);
  for (auto e : B->join) if (e) cudaEventDestroy(e);
  if (B->fork) cudaEventDestroy(B->fork);
  for (auto st : B->streams) if (st) cudaStreamDestroy(st);
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
}
}  // namespace

extern "C" int frank_blr_set_timing(frank_blr* p, int on) {
  if (!p) return fail(FRANK_ERR_INVALID, "null plan");
  if (p->want_timing != (on != 0)) {
    p->want_timing = on != 0;
    if (p->graph_exec) { cudaGraphExecDestroy(p->graph_exec); p->graph_exec = nullptr; }
    if (p->graph) { cudaGraphDestroy(p->graph); p->graph = nullptr; }
  }
  return FRANK_OK;
}

extern "C" int frank_blr_set_grid(frank_blr* p, int ctas) {
  if (!p || ctas < 1) return fail(FRANK_ERR_INVALID, "bad grid");
  cudaDeviceSynchronize();
  const int nb = p->nb;
  p->grid_recomp = std::max(1, std::min({nb * nb, p->sm_count - 1, ctas}));
  p->grid_gram = std::max(1, std::min({nb * nb, 2 * (p->sm_count - 1), 2 * ctas}));
  p->grid_dense = std::max(1, std::min({nb * nb, 2 * p->sm_count, ctas}));
  if (p->rscratch) { cudaFree(p->rscratch); p->rscratch = nullptr; }
  if (p->dscratch) { cudaFree(p->dscratch); p->dscratch = nullptr; }
  if (p->rsplit) { cudaFree(p->rsplit); p->rsplit = nullptr; }
  if (p->split_done) { cudaFree(p->split_done); p->split_done = nullptr; }
  if (p->graph_exec) { cudaGraphExecDestroy(p->graph_exec); p->graph_exec = nullptr; }
  if (p->graph) { cudaGraphDestroy(p->graph); p->graph = nullptr; }
  p->factored = false;
  return FRANK_OK;
}

extern "C" int frank_batch_create(frank_blr* const* plans, int count, frank_batch** out) {
  if (!plans || count < 1 || !out) return fail(FRANK_ERR_INVALID, "bad batch arguments");
  for (int k = 0; k < count; ++k) {
    if (!plans[k]) return fail(FRANK_ERR_INVALID, "null plan in batch");
    if (plans[k]->precision != plans[0]->precision) return fail(FRANK_ERR_UNSUPPORTED, "mixed precisions in one batch");
  }
  frank_batch* B = new frank_batch();
  B->plans.assign(plans, plans + count);
  B->streams.assign(count, nullptr);
  B->join.assign(count, nullptr);
  bool ok = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming) == cudaSuccess;
  for (int k = 0; ok && k < count; ++k)
    ok = cudaStreamCreateWithFlags(&B->streams[k], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&B->join[k], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) { free_batch(B); return fail(FRANK_ERR_CUDA, "batch streams"); }
  *out = B;
  return FRANK_OK;
}

extern "C" int frank_batch_destroy(frank_batch* B) {
  cudaDeviceSynchronize();
  free_batch(B);
  return FRANK_OK;
}

namespace {
// A batch factors step by step (one launch per elimination step over all
// systems) when its plans share the block size (every block full), the
// launch grids and the dense-update band, and use the Householder
// recompression; otherwise each system is its own branch of one graph.
bool batch_stepwise_ok(const frank_batch* B) {
  const frank_blr* q = B->plans[0];
  for (const frank_blr* p : B->plans) {
    if (p->bmax != q->bmax || p->n != (int64_t)p->nb * p->bmax || use_gram(p) || p->grid_recomp != q->grid_recomp ||
        p->grid_dense != q->grid_dense || p->grid_gram != q->grid_gram || p->dupd_band != q->dupd_band)
      return false;
  }
  return true;
}

// The step-by-step schedule of enqueue_factor over all systems of a batch:
// the same two streams and events, each launch with grid.z = systems.
// Device table of the systems, step events and the second stream (before
// the capture: allocations and copies are not captured).
template <typename T>
int prepare_stepwise(frank_batch* B) {
  const int K = (int)B->plans.size();
  int max_nb = 0;
  // systems in decreasing order of their number of steps: the systems that
  // still have a step i are then a prefix of the table, and each launch covers
  // only them (grid.z), the largest first in the block scheduling order
  std::vector<int> order(K);
  for (int k = 0; k < K; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return B->plans[a]->nb > B->plans[c]->nb; });
  std::vector<SysDev<T>> sys(K);
  for (int k = 0; k < K; ++k) {
    frank_blr* p = B->plans[order[k]];
    max_nb = std::max(max_nb, p->nb);
    SysDev<T>& d = sys[k];
    d.H = h_view(p);
    d.W = work_view<T>(p);
    d.ws = factor_ws<T>(p);
    d.work = p->work;
    d.rscratch = p->rscratch;
    d.rstride = p->rstride;
    d.core_scale = p->core_scale;
    d.thr_trunc = p->core_scale * p->eps;
    d.smax = p->smax;
    d.core_method = p->fixed_rank > 0 ? p->core_fixed : p->core_method;
    d.proj_tol = p->proj_tol ? 1 : 0;
    d.split_p = p->split_p;
    d.core_smem = p->core_smem;
    d.dupd_band = p->dupd_band;
    d.pretrunc = pretruncate(p) ? 1 : 0;
    d.has_lr = p->nlr > 0 ? 1 : 0;
  }
  if (!B->d_sys) CUDA_TRY(cudaMalloc(&B->d_sys, sizeof(SysDev<T>) * K));
  CUDA_TRY(cudaMemcpy(B->d_sys, sys.data(), sizeof(SysDev<T>) * K, cudaMemcpyHostToDevice));
  if ((int)B->ev_getrf.size() < max_nb) {
    for (auto* v : {&B->ev_getrf, &B->ev_panel, &B->ev_dense}) {
      const size_t old = v->size();
      v->resize(max_nb, nullptr);
      for (size_t e = old; e < v->size(); ++e)
        CUDA_TRY(cudaEventCreateWithFlags(&(*v)[e], cudaEventDisableTiming));
    }
  }
  if (!B->aux) CUDA_TRY(cudaStreamCreateWithFlags(&B->aux, cudaStreamNonBlocking));
  return FRANK_OK;
}

template <typename T>
int enqueue_factor_stepwise(frank_batch* B, cudaStream_t s) {
  const int K = (int)B->plans.size();
  frank_blr* q = B->plans[0];
  int max_nb = 0;
  bool any_trunc = false;
  for (frank_blr* p : B->plans) {
    max_nb = std::max(max_nb, p->nb);
    any_trunc = any_trunc || pretruncate(p);
  }
  const SysDev<T>* S = static_cast<const SysDev<T>*>(B->d_sys);
  // systems with a step i: a prefix of the table (ordered by decreasing nb)
  std::vector<int> nbs;
  for (frank_blr* p : B->plans) nbs.push_back(p->nb);
  auto active = [&](int i) {
    int c = 0;
    for (int v : nbs) c += v > i;
    return std::max(c, 1);
  };
  cudaStream_t s2 = B->aux;
  const int b = q->bmax;
  const int cw = trinv_width(b);
  const int rt = (b + PANEL_TILE - 1) / PANEL_TILE;
  const int band = std::min(q->dupd_band, b);
  const int nbands = (b + band - 1) / band;
  k_reset_b<T><<<dim3(max_nb * max_nb, 1, K), 256, 0, s>>>(S);
  for (frank_blr* p : B->plans) {
    CUDA_TRY(cudaMemsetAsync(p->err, 0, ERR_SLOTS * sizeof(int), s));
    CUDA_TRY(cudaMemsetAsync(p->flops, 0, FLOP_SLOTS * sizeof(unsigned long long), s));
    CUDA_TRY(cudaMemsetAsync(p->work, 0, 2 * p->nb * sizeof(int), s));
  }
  CUDA_TRY(cudaEventRecord(B->fork, s));
  CUDA_TRY(cudaStreamWaitEvent(s2, B->fork, 0));
  if (any_trunc)
    k_truncate_lr_b<T><<<dim3(std::max(q->grid_recomp, q->grid_gram), 1, K), TRUNC_THREADS, 0, s>>>(S);
  auto getrf_step = [&](int step) -> int {
    const int Kz = active(step);
    k_getrf_load_b<T><<<dim3(64, 1, Kz), GETRF_AUX_THREADS, 0, s2>>>(S, step);
    for (int jb = 0; jb < b; jb += 32) {
      k_getrf_panel_b<T><<<dim3(1, 1, Kz), GETRF_THREADS, 0, s2>>>(S, step, jb);
      const int m2 = b - jb - std::min(32, b - jb);
      if (m2 > 0) {
        const int nt = (m2 + 63) / 64;
        k_getrf_trail_b<T><<<dim3(nt * nt, 1, Kz), GETRF_AUX_THREADS, 0, s2>>>(S, step, jb);
      }
    }
    k_getrf_store_b<T><<<dim3(64, 1, Kz), GETRF_AUX_THREADS, 0, s2>>>(S, step);
    k_trinv_b<T><<<dim3(2 * ((b + cw - 1) / cw), 1, Kz), TRINV_THREADS, (size_t)b * cw * sizeof(double), s2>>>(
        S, step, cw);
    CUDA_TRY(cudaEventRecord(B->ev_getrf[step], s2));
    return FRANK_OK;
  };
  int rc = getrf_step(0);
  if (rc) return rc;
  for (int i = 0; i < max_nb; ++i) {
    CUDA_TRY(cudaStreamWaitEvent(s, B->ev_getrf[i], 0));
    const int m = max_nb - i - 1;
    if (m == 0) break;
    const int Kz = active(i + 1);   // systems with targets at step i (nb > i + 1)
    k_panel_gather_b<T><<<dim3(m, rt, Kz), PANEL_THREADS, 0, s>>>(S, i);
    k_panel_mul_b<T><<<dim3(2 * m, rt, Kz), PANEL_THREADS, 0, s>>>(S, i);
    k_panel_fin_b<T><<<dim3(2 * m, rt, Kz), PANEL_THREADS, 0, s>>>(S, i);
    CUDA_TRY(cudaEventRecord(B->ev_panel[i], s));
    CUDA_TRY(cudaStreamWaitEvent(s2, B->ev_panel[i], 0));
    k_update_dense_b<T><<<dim3(std::min(nbands, q->grid_dense), 1, Kz), DUPD_THREADS, 0, s2>>>(S, i, DUPD_NEXT);
    if ((rc = getrf_step(i + 1))) return rc;
    if (m > 1)
      k_update_dense_b<T><<<dim3((int)std::min<int64_t>((int64_t)m * m * nbands, q->grid_dense), 1, Kz), DUPD_THREADS,
                            0, s2>>>(S, i, DUPD_REST);
    CUDA_TRY(cudaEventRecord(B->ev_dense[i], s2));
    k_recompress_b<T><<<dim3(std::min(m * m, q->grid_recomp), 1, Kz), RECOMP_THREADS, RECOMP_SMEM_BYTES, s>>>(S, i);
    CUDA_TRY(cudaStreamWaitEvent(s, B->ev_dense[i], 0));
  }
  CUDA_TRY(cudaStreamWaitEvent(s, B->ev_getrf[max_nb - 1], 0));
  CUDA_TRY(cudaGetLastError());
  for (frank_blr* p : B->plans) { p->timed = false; p->launches = 0; }
  return FRANK_OK;
}

template <typename T>
int batch_capture(frank_batch* B) {
  cudaStream_t s = B->stream;
  for (frank_blr* p : B->plans) {
    int rc0 = ensure_scratch(p);
    if (rc0) return rc0;
  }
  B->stepwise = batch_stepwise_ok(B);
  if (B->stepwise) {
    int rc0 = prepare_stepwise<T>(B);
    if (rc0) return rc0;
    CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_factor_stepwise<T>(B, s);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc != FRANK_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return fail(FRANK_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(e));
    B->graph = g;
    CUDA_TRY(cudaGraphInstantiate(&B->exec, g, 0));
    return FRANK_OK;
  }
  CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = FRANK_OK;
  cudaError_t e = cudaEventRecord(B->fork, s);
  for (size_t k = 0; rc == FRANK_OK && e == cudaSuccess && k < B->plans.size(); ++k) {
    e = cudaStreamWaitEvent(B->streams[k], B->fork, 0);
    if (e == cudaSuccess) rc = enqueue_factor<T>(B->plans[k], B->streams[k], false);
    if (rc == FRANK_OK && e == cudaSuccess) e = cudaEventRecord(B->join[k], B->streams[k]);
    if (rc == FRANK_OK && e == cudaSuccess) e = cudaStreamWaitEvent(s, B->join[k], 0);
  }
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(s, &g);
  if (rc != FRANK_OK) { if (g) cudaGraphDestroy(g); return rc; }
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(FRANK_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  B->graph = g;
  CUDA_TRY(cudaGraphInstantiate(&B->exec, g, 0));
  return FRANK_OK;
}
}  // namespace

extern "C" int frank_batch_getrf(frank_batch* B, void* stream) {
  if (!B) return fail(FRANK_ERR_INVALID, "null batch");
  (void)stream;
  for (frank_blr* p : B->plans) {
    int rc = orthonormalize_inputs(p, B->stream);
    if (rc) return rc;
  }
  if (!B->exec) {
    int rc = B->plans[0]->precision == FRANK_PREC_FP64 ? batch_capture<double>(B) : batch_capture<float>(B);
    if (rc) return rc;
  }
  CUDA_TRY(cudaGraphLaunch(B->exec, B->stream));
  CUDA_TRY(cudaStreamSynchronize(B->stream));
  int first = FRANK_OK;
  for (frank_blr* p : B->plans) {
    int rc = finish_factor(p);
    if (rc && first == FRANK_OK) first = rc;
  }
  return first;
}

extern "C" int frank_batch_refine_device(frank_batch* B, const double* const* d_b, int64_t ldb, double* const* d_x,
                                         int64_t ldx, int nrhs, double tol, int maxit, int* iters, double* resid) {
  if (!B || !d_b || !d_x || nrhs < 1 || nrhs > 8 || maxit < 0) return fail(FRANK_ERR_INVALID, "bad batch refine arguments");
  const int K = (int)B->plans.size();
  for (int k = 0; k < K; ++k) {
    frank_blr* p = B->plans[k];
    if (!p->factored) return fail(FRANK_ERR_STATE, "batch refine before getrf");
    if (ldb < p->n || ldx < p->n) return fail(FRANK_ERR_INVALID, "leading dimension below a system's order");
  }
  std::vector<std::vector<double>> bn(K);
  std::vector<int> it(K, 0), done(K, 0);
  std::vector<double> res(K, 0.0);
  int rc;
  for (int k = 0; k < K; ++k) if ((rc = colnorms_enqueue(B->plans[k], d_b[k], ldb, nrhs, B->streams[k]))) return rc;
  for (int k = 0; k < K; ++k) {
    CUDA_TRY(cudaStreamSynchronize(B->streams[k]));
    colnorms_read(B->plans[k], nrhs, bn[k]);
  }
  for (int k = 0; k < K; ++k) {
    frank_blr* p = B->plans[k];
    CUDA_TRY(cudaMemcpy2DAsync(d_x[k], ldx * sizeof(double), d_b[k], ldb * sizeof(double), p->n * sizeof(double), nrhs,
                               cudaMemcpyDeviceToDevice, B->streams[k]));
    if ((rc = solve_device_impl(p, d_x[k], ldx, nrhs, false, B->streams[k]))) return rc;
  }
  for (;;) {
    int active = 0;
    for (int k = 0; k < K; ++k) {
      if (done[k]) continue;
      frank_blr* p = B->plans[k];
      if ((rc = matvec_device_impl(p, d_x[k], ldx, p->vtmp, p->n, nrhs, d_b[k], ldb, B->streams[k]))) return rc;
      if ((rc = colnorms_enqueue(p, p->vtmp, p->n, nrhs, B->streams[k]))) return rc;
      ++active;
    }
    if (!active) break;
    for (int k = 0; k < K; ++k) {
      if (done[k]) continue;
      frank_blr* p = B->plans[k];
      CUDA_TRY(cudaStreamSynchronize(B->streams[k]));
      std::vector<double> rn;
      colnorms_read(p, nrhs, rn);
      double r = 0.0;
      for (int h = 0; h < nrhs; ++h) r = std::max(r, rn[h] / (bn[k][h] > 0.0 ? bn[k][h] : 1.0));
      res[k] = r;
      if (r <= tol || it[k] >= maxit) { done[k] = 1; continue; }
      if ((rc = solve_device_impl(p, p->vtmp, p->n, nrhs, false, B->streams[k]))) return rc;
      ++p->solve_launches;
      k_axpy_cast<double><<<grid_for(p->n * nrhs), 256, 0, B->streams[k]>>>(p->vtmp, p->n, d_x[k], ldx, p->n, nrhs);
      ++it[k];
    }
  }
  for (int k = 0; k < K; ++k) CUDA_TRY(cudaStreamSynchronize(B->streams[k]));
  int status = FRANK_OK;
  for (int k = 0; k < K; ++k) {
    if (iters) iters[k] = it[k];
    if (resid) resid[k] = res[k];
    if (res[k] > tol) status = FRANK_ERR_NOT_CONVERGED;
  }
  if (status) return fail(status, "a system of the batch reached maxit before the tolerance");
  return FRANK_OK;
}

#ifdef FRANK_PHASE_TIMING
// Read and clear the recompression phase counters (timing builds only).
extern "C" int frank_debug_getrf_cycles(unsigned long long* c8) {
  CUDA_TRY(cudaMemcpyFromSymbol(c8, g_getrf_cycles, sizeof(unsigned long long) * 8));
  unsigned long long z[8] = {0};
  CUDA_TRY(cudaMemcpyToSymbol(g_getrf_cycles, z, sizeof(z)));
  return FRANK_OK;
}

extern "C" int frank_debug_sub_cycles(unsigned long long* c16) {
  CUDA_TRY(cudaMemcpyFromSymbol(c16, g_sub_cycles, sizeof(unsigned long long) * 16));
  unsigned long long z[16] = {0};
  CUDA_TRY(cudaMemcpyToSymbol(g_sub_cycles, z, sizeof(z)));
  return FRANK_OK;
}

extern "C" int frank_debug_tlog(long long* out, unsigned long long* n) {
  CUDA_TRY(cudaMemcpyFromSymbol(n, g_tlog_n, sizeof(unsigned long long)));
  const unsigned long long k = *n < 200000 ? *n : 200000;
  if (out) CUDA_TRY(cudaMemcpyFromSymbol(out, g_tlog, sizeof(long long) * 6 * k));
  unsigned long long z = 0;
  CUDA_TRY(cudaMemcpyToSymbol(g_tlog_n, &z, sizeof(z)));
  return FRANK_OK;
}

extern "C" int frank_debug_phase_cycles(unsigned long long* cycles24, unsigned long long* count3) {
  CUDA_TRY(cudaMemcpyFromSymbol(cycles24, g_phase_cycles, sizeof(unsigned long long) * 24));
  CUDA_TRY(cudaMemcpyFromSymbol(count3, g_phase_count, sizeof(unsigned long long) * 3));
  unsigned long long z[24] = {0};
  CUDA_TRY(cudaMemcpyToSymbol(g_phase_cycles, z, sizeof(z)));
  CUDA_TRY(cudaMemcpyToSymbol(g_phase_count, z, sizeof(unsigned long long) * 3));
  return FRANK_OK;
}
#endif

// ===========================================================================
// Allocation-free dense getrf (frank_getrf_dense_noalloc).
//
// For callers that cannot call cudaMalloc (inside an allocator callback, on an
// out-of-memory recovery path, under a pool that forbids growth).  All device
// scratch comes from the file-scope array below: the block copy D, the FP64
// work matrix of k_getrf, two reserved inverse-sized slots, the pivot
// and permutation vectors, and the small geometry / status words.  Nothing in
// this section changes the plan-based paths above.
// ===========================================================================
namespace {

constexpr int NOALLOC_N = FRANK_NOALLOC_MAX_N;
constexpr size_t NA_MAT = (size_t)NOALLOC_N * NOALLOC_N * sizeof(double);  // 512 KB
constexpr size_t NA_D = 0;
constexpr size_t NA_W = NA_D + NA_MAT;
constexpr size_t NA_LINV = NA_W + NA_MAT + (size_t)32 * NOALLOC_N * sizeof(double);  // k_getrf work + panel
constexpr size_t NA_UINV = NA_LINV + NA_MAT;
constexpr size_t NA_PERM = NA_UINV + NA_MAT;
constexpr size_t NA_IPIV = NA_PERM + NOALLOC_N * sizeof(int);
constexpr size_t NA_GEOM = NA_IPIV + NOALLOC_N * sizeof(int);            // off[2], dslot, lslot, rank
constexpr size_t NA_ERR = NA_GEOM + 8 * sizeof(int);                    // ERR_SLOTS ints
constexpr size_t NA_FLOPS = NA_ERR + ERR_SLOTS * sizeof(int);           // FLOP_SLOTS ull
constexpr size_t NA_BYTES = NA_FLOPS + FLOP_SLOTS * sizeof(unsigned long long);

// The scratch: fixed size, resident on every GPU that loads the library.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// Geometry of a one-block plan, pivots back to 1-based; device code names the
// array directly.
__global__ void k_noalloc_prepare(int n) {
  int* g = reinterpret_cast<int*>(g_noalloc_scratch + NA_GEOM);
  g[0] = 0; g[1] = n;   // off[0..1]
  g[2] = 0;             // dslot[0]
  g[3] = -1;            // lslot[0]
  g[4] = 0;             // rank[0]
  int* e = reinterpret_cast<int*>(g_noalloc_scratch + NA_ERR);
  for (int k = 0; k < ERR_SLOTS; ++k) e[k] = 0;
  unsigned long long* f = reinterpret_cast<unsigned long long*>(g_noalloc_scratch + NA_FLOPS);
  for (int k = 0; k < FLOP_SLOTS; ++k) f[k] = 0ull;
}

__global__ void k_noalloc_pivots(int n, int* out) {
  const int* ip = reinterpret_cast<const int*>(g_noalloc_scratch + NA_IPIV);
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) out[r] = ip[r] + 1;
}

// Device address of the scratch, looked up once per device context (the
// host-side name of a __device__ array is not a device address).  The entry
// is keyed by the driver's unique id of the current context, so a context
// created after cudaDeviceReset (where the module, and with it the array, is
// loaded afresh) triggers a new lookup instead of reusing a stale address.
constexpr int NA_MAX_DEVICES = 64;
struct NoallocEntry {
  unsigned char* addr = nullptr;
  unsigned long long ctx_id = 0;
};
NoallocEntry g_noalloc_addr[NA_MAX_DEVICES];
std::mutex g_noalloc_mutex;

// Unique id of the calling thread's current context (cuCtxGetCurrent +
// cuCtxGetId, reached through the runtime's driver entry-point query so the
// library does not link libcuda); 0 when the driver does not provide it.
unsigned long long current_context_id() {
  using GetCurrentFn = int (*)(void**);
  using GetIdFn = int (*)(void*, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetIdFn>(f);
    cudaGetLastError();
  });
  if (!get_current || !get_id) return 0;
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

int noalloc_setup(int dev, unsigned char** out) {
  if (dev < 0 || dev >= NA_MAX_DEVICES) return fail(FRANK_ERR_UNSUPPORTED, "device index beyond the set-up table");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  // A thread that has not used the runtime yet has no current context (id 0):
  // the lookup below makes the device's primary context current, and the id
  // is read again after it.
  const unsigned long long ctx = current_context_id();
  NoallocEntry& slot = g_noalloc_addr[dev];
  if (!slot.addr || ctx == 0 || slot.ctx_id != ctx) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
      return fail(FRANK_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
    // Under lazy module loading a kernel is loaded at its first launch, which
    // may allocate device memory; load the three kernels of this entry point
    // here, at set-up, so later calls load nothing.
    cudaFuncAttributes fa;
    CUDA_TRY(cudaFuncGetAttributes(&fa, k_noalloc_prepare));
    CUDA_TRY(cudaFuncGetAttributes(&fa, k_getrf<double>));
    CUDA_TRY(cudaFuncGetAttributes(&fa, k_noalloc_pivots));
    slot.addr = static_cast<unsigned char*>(ptr);
    slot.ctx_id = current_context_id();
  }
  *out = slot.addr;
  return FRANK_OK;
}

}  // namespace

extern "C" int frank_getrf_dense_noalloc(const double* d_a, int64_t lda, int n, double* d_lu, int64_t ldlu,
                                         int* d_ipiv, void* stream) {
  if (n < 1 || n > NOALLOC_N) {
    char buf[160];
    snprintf(buf, sizeof buf, "frank_getrf_dense_noalloc: n = %d outside 1..%d (the size of its fixed scratch)", n,
             NOALLOC_N);
    return fail(FRANK_ERR_UNSUPPORTED, buf);
  }
  if (!d_a || !d_lu || !d_ipiv || lda < n || ldlu < n) return fail(FRANK_ERR_INVALID, "bad noalloc getrf arguments");
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  unsigned char* base = nullptr;
  int rc = noalloc_setup(dev, &base);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int* geom = reinterpret_cast<int*>(base + NA_GEOM);
  BlrView<double> A;
  A.nb = 1; A.bmax = n; A.kcap = 0;
  A.off = geom; A.dslot = geom + 2; A.lslot = geom + 3; A.rank = geom + 4;
  A.D = reinterpret_cast<double*>(base + NA_D);
  A.U = A.S = A.Vt = nullptr;
  FactorWs<double> ws{};
  ws.perm = reinterpret_cast<int*>(base + NA_PERM);
  ws.ipiv = reinterpret_cast<int*>(base + NA_IPIV);
  ws.Linv = reinterpret_cast<double*>(base + NA_LINV);
  ws.Uinv = reinterpret_cast<double*>(base + NA_UINV);
  ws.getrf_scratch = reinterpret_cast<double*>(base + NA_W);
  ws.err = reinterpret_cast<int*>(base + NA_ERR);
  ws.flops = reinterpret_cast<unsigned long long*>(base + NA_FLOPS);
  k_noalloc_prepare<<<1, 1, 0, s>>>(n);
  CUDA_TRY(cudaMemcpy2DAsync(A.D, n * sizeof(double), d_a, lda * sizeof(double), n * sizeof(double), n,
                             cudaMemcpyDeviceToDevice, s));
  k_getrf<double><<<1, GETRF_THREADS, 0, s>>>(A, ws, 0);
  CUDA_TRY(cudaMemcpy2DAsync(d_lu, ldlu * sizeof(double), A.D, n * sizeof(double), n * sizeof(double), n,
                             cudaMemcpyDeviceToDevice, s));
  k_noalloc_pivots<<<1, 256, 0, s>>>(n, d_ipiv);
  CUDA_TRY(cudaGetLastError());
  int err_words[ERR_SLOTS];
  CUDA_TRY(cudaMemcpyAsync(err_words, ws.err, sizeof(err_words), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (err_words[ERR_SINGULAR_STEP] != 0) return fail(FRANK_ERR_SINGULAR, "zero pivot in the dense block");
  return FRANK_OK;
}

