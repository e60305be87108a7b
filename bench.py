"""Benchmark: BLR-LU factor + solve time to a 1e-10 residual, mixed vs plain FP64.

Workload (the headline configuration): Laplace-3D kernel 1/(r + 1e-3) on
N = 32768 uniform points in the unit cube (std::mt19937_64 seed 2, drawn
axis-major), Morton ordered (morton_index.cpp rule), BLR with 64 x 64 blocks
of 512, weak admissibility, A_H compressed on the device to eps = 1e-8, 4
right-hand sides b ~ N(0, 1) (std::mt19937_64 seed 3, column by column),
target max_j ||b_j - A_H x_j|| / ||b_j|| <= 1e-10.

One step = getrf (the FP32 factor at tolerance 3e-3 for "mixed", the FP64
factor at 1e-8 for "fp64") + iterative refinement against the FP64 A_H to
1e-10.  `value` is the mixed arm's time per step (seconds, device time by CUDA
events, max over ranks), with the FP64 arm reported beside it.  Inputs
(A_H: GBs) are larger than L2 and the working copy is reset from A_H at the
start of every getrf.

`--impl reference` times the reference itself (FRANK's C++ sources compiled
into oracle/_ref, on scipy's OpenBLAS with all host cores) on a bounded
sample of the same workload: the leading 8 x 8 blocks (N = 4096) of the same
point set, eps 1e-8, FRANK_LRA=rounded_addition, factor + solve.  The time is
reported as measured, not scaled; our engine's time on the same sample is
the key "sample" of our line.

Multi-GPU: replicas only -- each rank factors and solves its own system
(weak scaling), timings are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BLR-LU factor+solve time to 1e-10 residual: mixed vs plain FP64, 1 B200"
CFG = dict(n=32768, nb=64, dim=3, eps=1e-8, mixed_eps=3e-3, nrhs=4, tol=1e-10, kernel="laplace",
           point_seed=2, rhs_seed=3, morton_level=10)


class MT19937_64:
    """std::mt19937_64 seeded with `gen.seed(s)` (Matsumoto-Nishimura 64-bit
    Mersenne Twister: n = 312, m = 156, init multiplier 6364136223846793005),
    with libstdc++'s uniform_real_distribution<double>(0, 1) (one 64-bit draw
    per variate: double(g) / 2^64, clamped below 1) and
    normal_distribution<double>(0, 1) (Marsaglia polar method, the second
    variate of each accepted pair returned by the next call).  Pinned against
    g++ output in tests/golden/libstdcxx_mt19937_seed0.txt."""

    N, M = 312, 156
    A = 0xB5026F5AA96619E9
    UM, LM = 0xFFFFFFFF80000000, 0x7FFFFFFF

    def __init__(self, seed):
        import numpy as np
        mt = [seed & 0xFFFFFFFFFFFFFFFF]
        for i in range(1, self.N):
            mt.append((6364136223846793005 * (mt[-1] ^ (mt[-1] >> 62)) + i) & 0xFFFFFFFFFFFFFFFF)
        self.mt = np.array(mt, dtype=np.uint64)
        self.pos = self.N
        self.pending = np.empty(0, dtype=np.uint64)   # drawn but not consumed
        self.saved = None                               # cached second normal variate

    def _twist(self):
        import numpy as np
        mt, A, UM, LM = self.mt, np.uint64(self.A), np.uint64(self.UM), np.uint64(self.LM)
        one = np.uint64(1)
        y = (mt[0:156] & UM) | (mt[1:157] & LM)
        mt[0:156] = mt[156:312] ^ (y >> one) ^ ((y & one) * A)
        y = (mt[156:311] & UM) | (mt[157:312] & LM)
        mt[156:311] = mt[0:155] ^ (y >> one) ^ ((y & one) * A)
        y = (mt[311] & UM) | (mt[0] & LM)
        mt[311] = mt[155] ^ (y >> one) ^ ((y & one) * A)
        self.pos = 0

    def raw(self, count):
        import numpy as np
        out = np.empty(count, dtype=np.uint64)
        k = min(count, len(self.pending))
        out[:k] = self.pending[:k]
        self.pending = self.pending[k:]
        while k < count:
            if self.pos >= self.N:
                self._twist()
            take = min(count - k, self.N - self.pos)
            x = self.mt[self.pos:self.pos + take].copy()
            x ^= (x >> np.uint64(29)) & np.uint64(0x5555555555555555)
            x ^= (x << np.uint64(17)) & np.uint64(0x71D67FFFEDA60000)
            x ^= (x << np.uint64(37)) & np.uint64(0xFFF7EEE000000000)
            x ^= x >> np.uint64(43)
            out[k:k + take] = x
            self.pos += take
            k += take
        return out

    def uniform(self, count):
        import numpy as np
        return self._canonical(self.raw(count))

    @staticmethod
    def _canonical(r):
        import numpy as np
        u = r.astype(np.float64) / 18446744073709551616.0
        u[u >= 1.0] = np.nextafter(1.0, 0.0)
        return u

    def normal(self, count):
        import numpy as np
        out = []
        if count > 0 and self.saved is not None:
            out.append(self.saved)
            self.saved = None
        while len(out) < count:
            pairs = int((count - len(out)) * 0.7) + 16
            r = self.raw(2 * pairs)
            u = self._canonical(r)
            x, y = 2.0 * u[0::2] - 1.0, 2.0 * u[1::2] - 1.0
            r2 = x * x + y * y
            acc = np.nonzero(~((r2 > 1.0) | (r2 == 0.0)))[0]
            use = acc[: (count - len(out) + 1) // 2]
            if len(use) == 0:
                continue
            last = int(use[-1])
            self.pending = np.concatenate([r[2 * (last + 1):], self.pending])   # draws not consumed
            mult = np.sqrt(-2.0 * np.log(r2[use]) / r2[use])
            pv = np.empty(2 * len(use))
            pv[0::2] = y[use] * mult
            pv[1::2] = x[use] * mult
            out.extend(pv.tolist())
        if len(out) > count:
            self.saved = out[count]
        return np.array(out[:count])


def make_points(n, dim, seed, level):
    """n points uniform in [0, 1)^dim from std::mt19937_64 seeded `seed`,
    drawn axis-major (all x, then all y, ...; the reference's params[d][i]
    layout, functions.h:34-38), then Morton ordered
    (operations/misc/morton_index.cpp:36-98): the bounding box padded by 0.5,
    `level` bits interleaved per axis, stable sort by box number."""
    import numpy as np
    x = MT19937_64(seed).uniform(dim * n).reshape(dim, n)
    bmin = x.min(axis=1) - 0.5
    bsize = float((x.max(axis=1) - x.min(axis=1)).max()) + 1.0
    ix = (((x - bmin[:, None]) / bsize) * (1 << level)).astype(np.int64)
    code = np.zeros(n, dtype=np.int64)
    for lev in range(level):
        for d in range(dim):
            code += (ix[d] & 1) << (dim * lev + d)
            ix[d] >>= 1
    return x[:, np.argsort(code, kind="stable")].copy()


def make_rhs(n, nrhs, seed):
    """n x nrhs right-hand sides b ~ N(0, 1) from std::mt19937_64 seeded
    `seed`, column by column (Fortran order)."""
    import numpy as np
    return np.asfortranarray(MT19937_64(seed).normal(n * nrhs).reshape(nrhs, n).T)


class Clocks:
    """nvidia-smi samples during the timed region (read-only query)."""

    def __init__(self, gpu):
        self.f = tempfile.NamedTemporaryFile(prefix="clk", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.f.name):
            parts = [t.strip() for t in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1])); mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(values, world, device="cpu"):
    """Element-wise max over the ranks of a list of per-step times (the
    replicas-only multi-GPU reduction: no data-path collective, only this)."""
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.cpu().tolist()


def fp64_gemm_peak(torch):
    """Measured cuBLAS FP64 GEMM throughput (TFLOP/s), the FP64 roofline denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(); torch.matmul(a, b); e.record(); e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def fp32_gemm_peak(torch):
    """Measured cuBLAS FP32 GEMM throughput (TFLOP/s, TF32 off): the roofline
    denominator of the mixed plan's FP32 classes."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(3):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(); torch.matmul(a, b); e.record(); e.synchronize()
            best = min(best, s.elapsed_time(e) / 1e3)
        del a, b
        return 2.0 * n ** 3 / best / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def hbm_peak():
    """Measured copy bandwidth (GB/s) of MEASURED_PEAKS.json, else the
    pool's earlier measurement."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def plan_bytes(M, which, elem):
    """Bytes of the blocks of A_H (which 0) or of the factor (1): dense blocks
    b_i b_j, low-rank blocks U, S, V at their ranks; `elem` bytes per value."""
    nb = M.nb
    tot = 0
    for i in range(nb):
        for j in range(nb):
            bi, bj = M.block_size(i), M.block_size(j)
            if M.is_lowrank(i, j):
                r = M.rank(i, j, which)
                tot += (bi * r + r * r + bj * r) * elem
            elif which == 0 or i != j:
                tot += bi * bj * elem
    if which == 1:
        tot += sum(2 * M.block_size(i) ** 2 * elem for i in range(nb))   # explicit inverses of the diagonal factors
    return tot


def run_ours(args, rank, world):
    import numpy as np
    import torch
    import torch.distributed as dist
    from frank_b200 import BLRMatrix

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    c = CFG
    x = make_points(c["n"], c["dim"], c["point_seed"] + rank, c["morton_level"])
    b_host = make_rhs(c["n"], c["nrhs"], c["rhs_seed"] + rank)
    b_dev = torch.from_numpy(b_host.T.copy()).to("cuda")          # (nrhs, n) row-major == column-major n x nrhs
    x_dev = torch.zeros_like(b_dev)
    stream = torch.cuda.current_stream().cuda_stream

    arms = {}
    # mixed: FP32 factor at the loose tolerance; fp64: FP64 factor at the
    # workload's tolerance; fp64_at_mixed_eps (control): FP64 factor at the
    # mixed arm's tolerance, so the precision gain is seen apart from the
    # tolerance gain.  All three refine in FP64 to the same residual.
    for arm, prec, feps in (("mixed", "mixed", c["mixed_eps"]), ("fp64", "fp64", c["eps"]),
                            ("fp64_at_mixed_eps", "fp64", c["mixed_eps"])):
        M = BLRMatrix(c["n"], c["nb"], eps=feps, precision=prec)
        M.build_kernel(c["kernel"], x, c["eps"])
        # launch parameters by the plan's own autotuner (a few timed
        # factorizations, before the warm-up); the FP64 arm at 1e-8 keeps the
        # defaults, its factorizations being too long to tune within minutes
        tuning = M.autotune(stream=stream) if arm != "fp64" else M.tuning()
        torch.cuda.synchronize()

        def step():
            M.getrf(stream=stream)
            it, res = M.refine_device(b_dev.data_ptr(), x_dev.data_ptr(), c["nrhs"], tol=c["tol"], maxit=60,
                                      stream=stream)
            return it, res

        for _ in range(args.warmup):
            step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clk = Clocks(dev) if (rank == 0 and arm == "mixed") else None
        times, its, ress, kt = [], [], [], []
        for _ in range(args.steps):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            it, res = step()
            e.record()
            e.synchronize()
            times.append(s.elapsed_time(e) / 1e3)
            its.append(it); ress.append(res)
        torch.cuda.synchronize()
        clocks = clk.stop() if clk else None
        # per-kernel-class device times: one more factorization with CUDA
        # events recorded around every launch inside the graph (the event
        # nodes serialise the lookahead branch, so this replay is separate)
        M.set_timing(True)
        M.getrf(stream=stream)
        M.getrf(stream=stream)
        kt.append(M.kernel_times())
        M.set_timing(False)
        if world > 1:
            dist.barrier()
        # end to end through the host-buffer API (H2D of b and D2H of x inside);
        # one untimed call first, like the device-timed loop's warm-up (the
        # timing toggle above dropped the captured graph)
        M.getrf()
        M.refine(b_host, tol=c["tol"], maxit=60)
        e2e = []
        for _ in range(max(1, min(args.steps, 3)) if arm != "fp64_at_mixed_eps" else 0):
            t0 = time.perf_counter()
            M.getrf()
            xs, it_h, res_h = M.refine(b_host, tol=c["tol"], maxit=60)
            e2e.append(time.perf_counter() - t0)
        st = M.stats()
        # one solve and one FP64 H-matvec, timed alone (the HBM-bound classes)
        z = b_dev.clone()
        y = torch.zeros_like(b_dev)

        def ev(f, reps=3):
            ts_ = []
            for _ in range(reps):
                torch.cuda.synchronize()
                s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s_.record(); f(); e_.record(); e_.synchronize()
                ts_.append(s_.elapsed_time(e_))
            return statistics.median(ts_)
        solve_ms = ev(lambda: M.solve_device(z.data_ptr(), c["nrhs"], stream=stream))
        matvec_ms = ev(lambda: M.matvec_device(b_dev.data_ptr(), y.data_ptr(), c["nrhs"], stream=stream))
        elem = 8 if prec == "fp64" else 4
        ranks = [M.rank(i, j, 1) for i in range(c["nb"]) for j in range(c["nb"]) if i != j]
        arms[arm] = dict(times=times, its=its, res=ress, kt=kt, e2e=e2e, clocks=clocks, stats=st, tuning=tuning,
                         mean_rank=float(np.mean(ranks)), max_rank=int(max(ranks)), prec=prec, factor_eps=feps,
                         solve_ms=solve_ms, matvec_ms=matvec_ms, solve_bytes=plan_bytes(M, 1, elem),
                         matvec_bytes=plan_bytes(M, 0, 8))
        M.close()
        torch.cuda.synchronize()

    sample_ours = run_ours_sample(stream, 3)
    peaks = dict(fp64=fp64_gemm_peak(torch), fp32=fp32_gemm_peak(torch))
    # max over ranks of the per-step times
    for arm in arms:
        arms[arm]["times"] = max_over_ranks(arms[arm]["times"], world, "cuda")
        if arms[arm]["e2e"]:
            arms[arm]["e2e"] = max_over_ranks(arms[arm]["e2e"], world, "cuda")
    return arms, peaks, sample_ours


def kernel_roofline(arm, peaks, hbm):
    """Per kernel class: achieved against its bound.  Compute classes: the
    reference's algorithmic FLOPs (in-kernel counters, LAWN 41 counts) over
    the class's device time, against the measured FP64 or FP32 GEMM peak
    (the arithmetic the class runs in: the leaf LU and the recompression's
    QR / core are FP64 in both plans, panels and dense updates follow the
    plan).  HBM classes: the bytes of the blocks one solve / matvec reads
    over its time, against the measured copy bandwidth."""
    kt = arm["kt"][-1]
    work = "fp64" if arm["prec"] == "fp64" else "fp32"
    out = {}
    for cls, pipe in (("getrf", "fp64"), ("panel", work), ("dense_update", work), ("recompress", "fp64")):
        ms, fl = kt[cls]["ms"], kt[cls]["flops"]
        ach = fl / (ms / 1e3) / 1e12 if ms > 0 else 0.0
        out[cls] = {"ms": ms, "achieved": ach, "unit": "TFLOP/s", "peak": peaks[pipe], "frac": ach / peaks[pipe],
                    "bound": "compute (%s, SIMT)" % pipe}
    for cls, key in (("solve", "solve"), ("matvec", "matvec")):
        ms, by = arm[key + "_ms"], arm[key + "_bytes"]
        ach = by / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        out[cls] = {"ms": ms, "achieved": ach, "unit": "GB/s", "peak": hbm, "frac": ach / hbm, "bound": "hbm",
                    "bytes": by}
    return out


# The bounded sample of the workload that the CPU reference runs: the leading
# 8 x 8 blocks of 512 (N = 4096) of the same point set and the first 4096 rows
# of the same right-hand-side stream, eps 1e-8, FRANK_LRA=rounded_addition.
SAMPLE = dict(n=4096, nb=8)
SAMPLE_DESC = ("leading 8x8 blocks of 512 (N=4096) of the workload's point set, eps 1e-8, 4 RHS, "
               "FRANK_LRA=rounded_addition")


def sample_inputs():
    c = CFG
    x = make_points(c["n"], c["dim"], c["point_seed"], c["morton_level"])[:, :SAMPLE["n"]].copy()
    b = make_rhs(SAMPLE["n"], c["nrhs"], c["rhs_seed"])
    return x, b


def run_reference_sample(steps, warmup, threads):
    """The reference itself (FRANK's C++ compiled into oracle/_ref, on scipy's
    OpenBLAS with `threads` threads) on the sample: A_H built once, then
    warmup + steps factorizations of fresh copies of it, each followed by
    the two block substitutions; returns the per-step getrf + solve times
    (its own std::chrono timings, examples/h_lu.cpp:40-48) and its output."""
    exe = os.path.join(ROOT, "oracle", "_ref", "frank_ref")
    if not os.path.exists(exe):
        raise SystemExit("oracle/_ref/frank_ref is missing: build it with python oracle/build_ref.py")
    x, b = sample_inputs()
    with tempfile.TemporaryDirectory() as wd:
        px, pb = os.path.join(wd, "pts.bin"), os.path.join(wd, "rhs.bin")
        x.tofile(px)
        b.T.copy().tofile(pb)
        out = subprocess.check_output([exe, "--n", str(SAMPLE["n"]), "--nb", str(SAMPLE["nb"]), "--eps", "1e-8",
                                       "--lra", "rounded_addition", "--points", px, "--dim", "3", "--rhs", pb,
                                       "--nrhs", str(CFG["nrhs"]), "--residual", "--threads", str(threads),
                                       "--repeat", str(warmup + steps)], text=True)
    info = json.loads(out.strip().splitlines()[-1])
    t = [g + s for g, s in zip(info["getrf_s"], info["solve_s"])][warmup:]
    return t, info


def bench_reference(args, rank, world):
    """--impl reference: rank 0 runs the reference's own factor + solve on the
    bounded sample (unscaled; the full N=32768 workload takes tens of minutes
    of host time), other ranks exit without work."""
    if rank != 0:
        return
    cores = os.cpu_count()
    t, info = run_reference_sample(max(1, args.steps), args.warmup, cores)
    val = statistics.median(t)
    desc = "FRANK (its C++ sources, scipy OpenBLAS, %d threads) factor+solve of the %s; measured, not scaled" % (
        cores, SAMPLE_DESC)
    line = {"metric": METRIC, "value": val, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": val * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "blr-lu laplace3d sample N=4096 b=512 eps=1e-8 4rhs (leading 8x8 blocks of the "
                                   "N=32768 workload)", "parallelism": "host threads"},
            "impl": "reference",
            "cpu_baseline": {"value": val, "unit": "s", "cores": cores, "kind": "reference", "sample": desc},
            "reference_residual": info.get("residual"),
            "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours_sample(stream, steps):
    """Our engine on the same sample: FP64 plan with the reference's
    rounded_addition at eps 1e-8 (getrf + solve, the reference's sequence), and
    the mixed plan (factor at the bench's mixed tolerance + refinement to 1e-10)."""
    import numpy as np
    import torch
    from frank_b200 import BLRMatrix
    x, b = sample_inputs()
    n, nb = SAMPLE["n"], SAMPLE["nb"]
    bd = torch.from_numpy(b.T.copy()).to("cuda")
    out = {}
    for arm, feps, prec, lra in (("fp64_getrf_solve", 1e-8, "fp64", "rounded_addition"),
                                 ("mixed_to_1e-10", CFG["mixed_eps"], "mixed", None)):
        M = BLRMatrix(n, nb, eps=feps, precision=prec)
        M.build_kernel("laplace", x, 1e-8)
        if lra:
            M.set_lra(lra)
        xd = torch.zeros_like(bd)
        ts = []
        for k in range(2 + steps):
            torch.cuda.synchronize()
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record()
            M.getrf(stream=stream)
            if prec == "fp64":
                xd.copy_(bd)
                M.solve_device(xd.data_ptr(), CFG["nrhs"], stream=stream)
            else:
                M.refine_device(bd.data_ptr(), xd.data_ptr(), CFG["nrhs"], tol=CFG["tol"], maxit=60, stream=stream)
            e_.record()
            e_.synchronize()
            if k >= 2:
                ts.append(s_.elapsed_time(e_) / 1e3)
        out[arm] = statistics.median(ts)
        M.close()
    return out


# DRAM traffic of k_recompress per algorithmic FLOP, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum over all 15 recompression
# launches of `--profile-case n8192`, the mixed factor at the headline's
# tolerance: 1.616e9 bytes for 4.695e10 FLOPs; the workload is too large to
# capture whole).  The roofline's `traffic` scales it to the mean headline
# launch by the FLOPs that launch performs
# (profiles/k_recompress_blr_laplace3d_n8192.md).
RECOMP_BYTES_PER_FLOP = 1.616e9 / 4.695e10


def profile_case(name):
    """Small single-GPU cases for ncu captures (`--profile-case`): build the
    plan, run the factorization, print the per-class kernel times.
      n8192:       Laplace-3D N=8192 (the headline point stream), 16 x 16
                   blocks of 512, A_H eps 1e-8, mixed factor at the
                   headline's tolerance (the recompression profile case);
      n8192-solve: the same plan, then one 4-RHS solve and one H-matvec
                   (the solve / matvec profile case);
      headline:    the benchmark's workload (N=32768, 64 x 64 blocks of 512),
                   one mixed factorization and one refinement to 1e-10, no
                   timing events (the launch list of one step)."""
    import torch
    from frank_b200 import BLRMatrix
    if name not in ("n8192", "n8192-solve", "headline"):
        raise SystemExit("unknown profile case " + name)
    if name == "headline":
        x = make_points(CFG["n"], CFG["dim"], CFG["point_seed"], CFG["morton_level"])
        M = BLRMatrix(CFG["n"], CFG["nb"], eps=CFG["mixed_eps"], precision="mixed")
        M.build_kernel("laplace", x, CFG["eps"])
        b = torch.from_numpy(make_rhs(CFG["n"], CFG["nrhs"], CFG["rhs_seed"]).T.copy()).cuda()
        xd = torch.zeros_like(b)
        M.getrf()
        it, res = M.refine_device(b.data_ptr(), xd.data_ptr(), CFG["nrhs"], tol=CFG["tol"], maxit=60)
        torch.cuda.synchronize()
        print(json.dumps({"refine_iters": it, "residual": res, "stats": M.stats()}))
        M.close()
        return
    x = make_points(8192, 3, CFG["point_seed"], CFG["morton_level"])
    M = BLRMatrix(8192, 16, eps=CFG["mixed_eps"], precision="mixed")
    M.build_kernel("laplace", x, CFG["eps"])
    M.set_timing(True)
    M.getrf()
    if name == "n8192-solve":
        b = torch.from_numpy(make_rhs(8192, CFG["nrhs"], CFG["rhs_seed"]).T.copy()).cuda()
        y = torch.zeros_like(b)
        M.solve_device(b.data_ptr(), CFG["nrhs"])
        M.matvec_device(b.data_ptr(), y.data_ptr(), CFG["nrhs"])
    torch.cuda.synchronize()
    print(json.dumps(M.kernel_times()))
    M.close()


def workload_batched(args):
    """256 independent systems, N drawn uniformly from {1024, 2048, 4096, 8192}
    (numpy seed 4), 2-D points (seed 5 + s), Morton ordered, kernel
    -log(r + 1e-3) + N I, blocks of 256, A_H at eps 1e-6, FP32 factor at 1e-4,
    FP64 refinement of one RHS (seed 3) to 1e-10; all factorizations in one
    captured graph.  Prints one JSON line."""
    import numpy as np
    import torch
    from frank_b200 import BLRMatrix
    from frank_b200.batch import BLRBatch
    rng = np.random.default_rng(4)
    count = args.systems
    sizes = rng.choice([1024, 2048, 4096, 8192], size=count)
    nmax = int(sizes.max())
    plans, t0 = [], time.perf_counter()
    for s_, n in enumerate(sizes):
        x = make_points(int(n), 2, 5 + s_, 15)
        M = BLRMatrix(int(n), int(n) // 256, eps=1e-4, precision="mixed", max_rank=96)
        M.build_kernel("neglog", x, 1e-6, params=(float(n),))
        plans.append(M)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t0
    batch = BLRBatch(plans, grid=args.batch_grid)
    rb = np.random.default_rng(3)
    B = torch.zeros((count, nmax), dtype=torch.float64, device="cuda")
    for k, n in enumerate(sizes):
        B[k, :n] = torch.tensor(rb.standard_normal(int(n)))
    X = torch.zeros_like(B)
    bp = [B[k].data_ptr() for k in range(count)]
    xp = [X[k].data_ptr() for k in range(count)]
    for _ in range(args.warmup):
        batch.getrf(); batch.refine_device(bp, xp, nmax, 1, tol=1e-10)
    times, tg = [], []
    for _ in range(args.steps):
        torch.cuda.synchronize(); t0 = time.perf_counter()
        batch.getrf()
        torch.cuda.synchronize(); t1 = time.perf_counter()
        its, res = batch.refine_device(bp, xp, nmax, 1, tol=1e-10)
        torch.cuda.synchronize(); times.append(time.perf_counter() - t0); tg.append(t1 - t0)
    t = statistics.median(times)
    ranks = [p.rank(i, j, 1) for p in plans[:8] for i in range(p.nb) for j in range(p.nb) if i != j]
    print(json.dumps({"workload": "batched: 256 systems N in {1024..8192}, -log kernel + N I, b=256, eps 1e-6",
                      "value": t, "unit": "s", "systems_per_s": count / t, "systems": count,
                      "total_unknowns": int(sizes.sum()), "max_iters": int(max(its)), "max_residual": max(res),
                      "getrf_s": statistics.median(tg), "refine_s": t - statistics.median(tg),
                      "mean_rank_first8": float(np.mean(ranks)), "build_s": t_build,
                      "steps": args.steps, "warmup": args.warmup}), flush=True)


def workload_adjoint(args):
    """Exponential kernel exp(-r/0.2) + 1e-2 I on N = 16384 2-D points (seed 6),
    blocks of 512, eps 1e-9: loss 0.5 ||A(theta)^{-1} b||^2 with gradients in b
    and theta through the hand-written adjoint; checked against a dense FP64
    gradient (cuSOLVER through torch, as the reference check only)."""
    import numpy as np
    import torch
    from frank_b200.adjoint import solve_exp
    n, theta, nugget = 16384, 0.2, 1e-2
    rng = np.random.default_rng(6)
    pts = torch.tensor(make_points(n, 2, 6, 15))
    b0 = rng.standard_normal(n)
    out = {}
    for prec, feps in (("mixed", 1e-4), ("fp64", 1e-9)):
        times = []
        for _ in range(args.warmup + args.steps):
            bt = torch.tensor(b0, device="cuda", requires_grad=True)
            th = torch.tensor(theta, dtype=torch.float64, device="cuda", requires_grad=True)
            torch.cuda.synchronize(); t0 = time.perf_counter()
            x = solve_exp(bt, th, pts, n // 512, eps=1e-9, nugget=nugget, precision=prec, factor_eps=feps, tol=1e-12)
            loss = 0.5 * (x * x).sum()
            loss.backward()
            torch.cuda.synchronize(); times.append(time.perf_counter() - t0)
        out[prec] = dict(t=statistics.median(times[args.warmup:]), gb=bt.grad.detach().clone(), gth=th.grad.item())
    # dense FP64 reference gradient
    P = pts.cuda()
    d = torch.cdist(P.t(), P.t())
    A = torch.exp(-d / theta) + nugget * torch.eye(n, dtype=torch.float64, device="cuda")
    bd = torch.tensor(b0, device="cuda")
    xd = torch.linalg.solve(A, bd)
    lam = torch.linalg.solve(A.t(), xd)
    gth = -(lam @ ((torch.exp(-d / theta) * d / theta ** 2) @ xd)).item()
    del A, d
    line = {"workload": "adjoint: exp(-r/0.2)+1e-2 I, N=16384 2-D, b=512, eps 1e-9, loss 0.5||A^-1 b||^2",
            "unit": "s", "steps": args.steps, "warmup": args.warmup, "dense_grad_theta": gth}
    for prec in out:
        gb = out[prec]["gb"]
        line[prec] = {"value": out[prec]["t"], "grad_theta": out[prec]["gth"],
                      "grad_theta_rel_err": abs(out[prec]["gth"] - gth) / abs(gth),
                      "grad_b_rel_err": ((gb - lam).norm() / lam.norm()).item()}
    print(json.dumps(line), flush=True)


def run_hlu(n, steps, warmup):
    """Multi-level H-LU: Laplace-3D 1/(r+1e-3) on N = n Morton-ordered
    unit-cube points (seed 7), binary cluster tree with weak admissibility,
    leaves of 256, every off-diagonal block rank 32 (rsvd), FP64 factor, FP64
    refinement of 8 RHS (seed 8) against A_H to 1e-10.  A step is getrf +
    refine (wall clock around synchronised calls; the getrf's device time from
    CUDA events beside it); construction is timed apart.  Returns a dict."""
    import torch
    from frank_b200 import HMatrix
    leaf, rank, nrhs = 256, 32, 8
    pts = make_points(n, 3, 7, 10)
    M = HMatrix(n, leaf, rank)
    torch.cuda.synchronize(); t0 = time.perf_counter()
    M.build_kernel("laplace", pts)
    torch.cuda.synchronize(); t_build = time.perf_counter() - t0
    # column-major n x nrhs: the transpose of a contiguous nrhs x n tensor
    b = torch.tensor(MT19937_64(8).normal(n * nrhs).reshape(nrhs, n), device="cuda").t()
    X = torch.zeros((nrhs, n), dtype=torch.float64, device="cuda").t()
    its = res = None
    for _ in range(warmup):
        M.getrf(); M.refine_device(b.data_ptr(), X.data_ptr(), nrhs, tol=1e-10, maxit=50)
    times, tf = [], []
    for _ in range(steps):
        torch.cuda.synchronize(); t0 = time.perf_counter()
        M.getrf()
        torch.cuda.synchronize(); t1 = time.perf_counter()
        its, res = M.refine_device(b.data_ptr(), X.data_ptr(), nrhs, tol=1e-10, maxit=50)
        torch.cuda.synchronize(); times.append(time.perf_counter() - t0); tf.append(t1 - t0)
    # achieved residual, recomputed from the solution
    Y = torch.zeros_like(X)
    M.matvec_device(X.data_ptr(), Y.data_ptr(), nrhs)
    rel = ((b - Y).norm(dim=0) / b.norm(dim=0)).max().item()
    st = M.stats()
    out = {"workload": "hlu: laplace3d N=%d leaf=256 rank=32 weak admissibility, FP64, 8 rhs, tol 1e-10" % n,
           "metric": "time to 1e-10 (getrf + refine)", "value": statistics.median(times), "unit": "s",
           "getrf_s": statistics.median(tf), "getrf_device_ms": st["factor_ms"],
           "refine_s": statistics.median(times) - statistics.median(tf), "iterations": its,
           "residual": res, "residual_recomputed": rel, "launches_per_getrf": st["launches"],
           "levels": M.levels, "build_s": t_build, "steps": steps, "warmup": warmup}
    M.close()
    return out


def workload_hlu(args):
    """The multi-level H-LU workload (run_hlu) at --hlu-n; prints one JSON line."""
    print(json.dumps(run_hlu(args.hlu_n, args.steps, args.warmup)), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile-case", default=None, help="run a small ncu case instead of the benchmark")
    ap.add_argument("--workload", default="headline", choices=["headline", "batched", "adjoint", "hlu"],
                    help="headline (the bench line); batched / adjoint / hlu print their own JSON line")
    ap.add_argument("--hlu-n", type=int, default=131072, help="hlu workload: matrix order")
    ap.add_argument("--systems", type=int, default=256)
    ap.add_argument("--batch-grid", type=int, default=16,
                    help="batched workload: CTAs per system of the persistent kernels")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-hlu", action="store_true", help="leave out the multi-level H-LU key of the bench line")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case)
        return
    if args.workload == "batched":
        workload_batched(args)
        return
    if args.workload == "adjoint":
        workload_adjoint(args)
        return
    if args.workload == "hlu":
        workload_hlu(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            bench_reference(args, rank, world)
            return
        arms, peaks, sample_ours = run_ours(args, rank, world)
        peak64 = peaks["fp64"]
        hbm, hbm_src = hbm_peak()
        if rank != 0:
            return
        mx, fp, ctl = arms["mixed"], arms["fp64"], arms["fp64_at_mixed_eps"]
        t_mixed = statistics.median(mx["times"])
        t_fp64 = statistics.median(fp["times"])
        t_ctl = statistics.median(ctl["times"])
        kt = mx["kt"][-1]
        rec = kt["recompress"]
        achieved = rec["flops"] / (rec["ms"] / 1e3) / 1e12 if rec["ms"] > 0 else 0.0
        nrhs, n = CFG["nrhs"], CFG["n"]
        line = {
            "metric": METRIC, "value": t_mixed, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_mixed * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "blr-lu laplace3d N=32768 b=512 eps=1e-8 4rhs tol=1e-10",
                       "n": n, "block": n // CFG["nb"], "nrhs": nrhs, "mixed_factor_eps": CFG["mixed_eps"],
                       "parallelism": "replicas" if world > 1 else "single", "l2": "inputs larger than L2"},
            "fp64": {"value": t_fp64, "unit": "s", "iters": fp["its"][-1], "residual": fp["res"][-1],
                     "mean_rank": fp["mean_rank"], "max_rank": fp["max_rank"], "kernel_ms": fp["kt"][-1]},
            "mixed": {"iters": mx["its"][-1], "residual": mx["res"][-1], "mean_rank": mx["mean_rank"],
                      "max_rank": mx["max_rank"], "kernel_ms": kt, "tuning": mx["tuning"]},
            "fp64_at_mixed_eps": {"value": t_ctl, "unit": "s", "factor_eps": CFG["mixed_eps"],
                                  "iters": ctl["its"][-1], "residual": ctl["res"][-1], "mean_rank": ctl["mean_rank"],
                                  "max_rank": ctl["max_rank"], "kernel_ms": ctl["kt"][-1], "tuning": ctl["tuning"]},
            "speedup_mixed_vs_fp64": t_fp64 / t_mixed,
            "speedup_precision_only": t_ctl / t_mixed,
            "kernel_roofline": {a: kernel_roofline(arms[a], peaks, hbm) for a in ("mixed", "fp64")},
            "peaks": {"fp64_tflops": peaks["fp64"], "fp32_tflops": peaks["fp32"], "hbm_gbs": hbm,
                      "source": "cuBLAS DGEMM / SGEMM (TF32 off) 8192^3 measured in this run; HBM " + hbm_src},
            "e2e": {"value": statistics.median(mx["e2e"]), "unit": "s", "fp64_value": statistics.median(fp["e2e"]),
                    "h2d_bytes_per_step": n * nrhs * 8, "d2h_bytes_per_step": n * nrhs * 8},
            "roofline": {"kernel": "k_recompress (mixed factor)", "bound": "compute (fp64, SIMT)",
                         "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                         "frac": achieved / peak64 if peak64 else None,
                         "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run (FP64 is not in "
                                        "MEASURED_PEAKS.json)",
                         "traffic": RECOMP_BYTES_PER_FLOP * rec["flops"] / (CFG["nb"] - 1),
                         "traffic_note": "bytes per launch: DRAM bytes per FLOP of the N=8192 capture x the mean "
                                         "launch's FLOPs"},
            "gpu_launches": mx["stats"]["launches"],
            "clocks": mx["clocks"],
        }
        line["sample"] = dict(workload=SAMPLE_DESC, unit="s", **sample_ours)
        if world == 1 and not args.no_hlu:
            # the multi-level H-LU configuration beside the headline (its own timing)
            try:
                line["hlu"] = run_hlu(131072, args.steps, max(args.warmup, 3))
            except Exception as exc:  # reported, never silently dropped
                line["hlu"] = {"error": str(exc)}
        if not args.no_cpu_baseline:
            cores = os.cpu_count()
            t, info = run_reference_sample(3, 1, cores)
            line["cpu_baseline"] = {
                "value": statistics.median(t), "unit": "s", "cores": cores, "kind": "reference",
                "sample": "FRANK (its C++ sources, scipy OpenBLAS, %d threads) factor+solve of the %s; measured, "
                          "not scaled (our engine on the same sample: key 'sample')" % (cores, SAMPLE_DESC)}
        print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
