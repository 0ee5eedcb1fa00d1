"""Benchmark driver: batched factor-and-solve throughput on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

Prints ONE JSON line on rank 0.  A "step" is one pass of the hot path over one batch of
synthetic input already resident in HBM (value); "e2e" repeats it through the public C ABI
with the inputs copied from pinned host memory and the solutions read back every step
(batches of 64 MiB of inputs or more are streamed in 8 slices over 2 streams, so that
copies overlap kernels).

Workloads (synthetic inputs with the shapes and value distributions of the reference
configurations; no dataset is involved):
  dsgesv_n256 (default) the mixed-precision solver rocsolver_dsgesv_strided_batched (FP32 LU +
              FP64 iterative refinement, FP64 fallback) on the inputs of gesv_n256; value =
              its solves/s, with the plain FP64 getrf+getrs timed on the same inputs in the
              same run ("plain_fp64") and the backward error of every member checked.
  gesv_n256   n=256, batch 2048, nrhs 1, A = U diag(s) V' with cond log-uniform in
              [1e1, 1e6], b ~ U[-1,1]; dgetrf_strided_batched + dgetrs_strided_batched
              (plain FP64).  Metric: solves/s.
  getrf_n32   n=32, lda 32, batch 1000, nrhs 1, U[-1,1] from seed 0: dgetrf + dgetrs.
  potrf_n64   n=64, batch 20000, nrhs 4, A = G G' + n I: dpotrf + dpotrs.
  vbatched_4096  4096 members, n ~ U[8, 512], nrhs ~ U[1, 16], A ~ U[-1,1] + 0.1 n I:
              rocsolver_dgesv_vbatched captured once in a CUDA graph and replayed; reported
              next to the same members solved by per-size launches (dgetrf_batched +
              dgetrs_batched per distinct n, "per_size_launches").
  adjoint_n128   n=128, batch 8192, nrhs 8, FP64, A ~ U[-1,1] + 4 I factored once outside
              the timing, G ~ N(0,1): rocsolver_dgetrs_adjoint_strided_batched (gB, gA).
  adjoint_n128_fp32  the same in FP32 (rocsolver_sgetrs_adjoint_strided_batched).
  zgesv_n64   complex double, n=64, batch 8192, nrhs 1, real and imaginary parts of A and b
              ~ U[-1,1]: rocsolver_zgesv_strided_batched.
  getri_n64   n=64, batch 16384, A ~ U[-1,1] + 4 I factored once outside the timing:
              rocsolver_dgetri_strided_batched (inverse in place).
Inputs are larger than L2 (126 MB) for gesv_n256 and potrf_n64; getrf_n32 (8 MB) rotates
through 24 distinct copies of the batch so each step reads cold data.

Multi-GPU: the batch members are independent, so every rank runs its own full batch
(weak scaling, no collective on the data path); the time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


WORKLOADS = ("dsgesv_n256", "gesv_n256", "getrf_n32", "potrf_n64", "vbatched_4096",
             "adjoint_n128", "adjoint_n128_fp32", "zgesv_n64", "getri_n64")
EXTRA_WORKLOADS = ("vbatched_4096", "adjoint_n128", "adjoint_n128_fp32")
WIDE_WORKLOADS = ("zgesv_n64", "getri_n64")  # the complex and inverse entry points
# the workloads measured beside the headline in the default run (C1, C2, C4, C5, and the
# complex solve and the inverse)
NESTED = ("getrf_n32", "potrf_n64", "vbatched_4096", "adjoint_n128", "adjoint_n128_fp32",
          "zgesv_n64", "getri_n64")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="all", choices=["all"] + list(WORKLOADS),
                   help="all (default): the dsgesv_n256 headline line, with every other "
                        "workload measured in the same run under its \"configs\" key")
    p.add_argument("--cpu-seconds", type=float, default=12.0,
                   help="target CPU time of the bounded CPU-baseline sample (all cores)")
    p.add_argument("--cpu-seconds-extra", type=float, default=3.0,
                   help="the same for each workload nested under \"configs\"")
    return p.parse_args()


# ----------------------------------------------------------------------------- ranks
def max_over_ranks(torch, pg, value, device):
    """The largest value over all ranks (every rank's device time is reduced so that the
    reported time is the slowest rank's); value itself without a process group."""
    if pg is None:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------- peaks
def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "bf16_tflops": d.get("bf16_tflops", 1590.0),
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- inputs
def make_cond_matrices(torch, n, bc, seed, device, lo=1.0, hi=6.0):
    """A = U diag(s) V' with U, V from QR of Gaussians and s log-spaced from 1 to 1/kappa,
    log10(kappa) ~ U[lo, hi] per member.  Generated on the device in chunks."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    A = torch.empty(bc, n, n, dtype=torch.float64, device=device)
    chunk = 256
    for c0 in range(0, bc, chunk):
        c1 = min(bc, c0 + chunk)
        m = c1 - c0
        U, _ = torch.linalg.qr(torch.randn(m, n, n, generator=g, device=device,
                                           dtype=torch.float64))
        V, _ = torch.linalg.qr(torch.randn(m, n, n, generator=g, device=device,
                                           dtype=torch.float64))
        lk = lo + (hi - lo) * torch.rand(m, 1, generator=g, device=device, dtype=torch.float64)
        t = torch.linspace(0, 1, n, device=device, dtype=torch.float64)[None, :]
        s = torch.pow(10.0, -lk * t)
        A[c0:c1] = (U * s[:, None, :]) @ V.transpose(1, 2)
    return A


def colmajor(torch, A):
    """(bc, m, n) row-major torch tensor -> contiguous buffer whose member b is the
    column-major m x n matrix (lda = m)."""
    return A.transpose(1, 2).contiguous()


# ----------------------------------------------------------------------------- workloads
class Workload:
    pass


def build_workload(name, torch, rs, dev, handle):
    w = Workload()
    w.name = name
    if name in ("gesv_n256", "dsgesv_n256"):
        n, bc, nrhs = 256, 2048, 1
        A = make_cond_matrices(torch, n, bc, seed=2, device=dev)
        g = torch.Generator(device=dev)
        g.manual_seed(3)
        B = torch.rand(bc, n, nrhs, generator=g, device=dev, dtype=torch.float64) * 2 - 1
        w.A0 = colmajor(torch, A)            # pristine copy, column-major members
        w.B0 = colmajor(torch, B)
        w.Arow = A                           # for residual checks
        w.Brow = B
        w.n, w.bc, w.nrhs = n, bc, nrhs
        w.metric = "batched solves/s at FP64 backward err <=1e-13 (plain FP64 getrf+getrs)"
        w.unit = "solves/s"
        w.dtype = "f64"
        w.config = {"workload": "plain dgetrf+dgetrs strided_batched, n=256, batch=2048, nrhs=1, "
                               "cond log-uniform [1e1,1e6]", "n": n, "batch": bc, "nrhs": nrhs,
                    "l2": "inputs 1 GiB > L2 (126 MB); A restored from a pristine copy between "
                          "steps outside the timed events"}
        w.flops_per_unit = 2.0 * n ** 3 / 3 + 2.0 * n * n * nrhs
        w.bytes_per_unit_getrf = 2 * n * n * 8 + 4 * n + 4
        w.dominant = "getrf_cta_kernel<double, 256, 1, 32>"
        # DRAM bytes (read + write) per member of the dominant kernel: 1432.9 MB per 512
        # members from `ncu --set full --clock-control none -c 1 -k regex:getrf_cta
        # python -m rocsolver_b200.demo --case getrf --n 256 --batch 512 --reps 2`
        w.traffic_per_unit = 1432930560 / 512
        w.limiter = "latency: the per-column pivot chain (FP64 compute fraction beside it)"
        w.launches_per_step = 2
        if name == "dsgesv_n256":
            w.metric = ("batched solves/s at FP64 backward err <=1e-13: mixed+IR vs plain FP64 LU")
            w.config["workload"] = ("dsgesv_strided_batched (FP32 LU + FP64 IR, <=10 iters, FP64 "
                                    "fallback) vs plain dgetrf+dgetrs, n=256, batch=2048, nrhs=1, "
                                    "cond log-uniform [1e1,1e6]")
            w.dominant = ("getrf_cta_kernel<float, 128, 2, 32, TF32> (FP32 LU with split-TF32 "
                          "tensor-core trailing updates inside dsgesv)")
            # 714.1 MB per 512 members from `ncu --set full --clock-control none -c 1
            # -k regex:getrf_cta python -m rocsolver_b200.demo --case dsgesv --n 256
            # --batch 512 --reps 1`
            w.traffic_per_unit = 714073856 / 512
            w.limiter = "latency: the per-column pivot chain (TF32 tensor fraction beside it)"
            w.launches_per_step = 6
    elif name == "getrf_n32":
        n, bc, nrhs = 32, 1000, 1
        rng = np.random.default_rng(0)
        A = torch.from_numpy(rng.uniform(-1, 1, (bc, n, n))).to(dev)
        B = torch.from_numpy(rng.uniform(-1, 1, (bc, n, nrhs))).to(dev)
        w.A0 = colmajor(torch, A)
        w.B0 = colmajor(torch, B)
        w.Arow, w.Brow = A, B
        w.n, w.bc, w.nrhs = n, bc, nrhs
        w.metric = "batched solves/s (plain FP64 getrf+getrs, n=32)"
        w.unit = "solves/s"
        w.dtype = "f64"
        w.rotate = 24
        w.config = {"workload": "plain dgetrf+dgetrs strided_batched, n=32, lda=32, batch=1000, "
                               "nrhs=1, U[-1,1] seed 0", "n": n, "batch": bc, "nrhs": nrhs,
                    "l2": "24 distinct copies of the 8 MB batch rotated (192 MB > L2)"}
        w.flops_per_unit = 2.0 * n ** 3 / 3 + 2.0 * n * n * nrhs
        w.bytes_per_unit_getrf = 2 * n * n * 8 + 4 * n + 4
        w.dominant = "getrf_warp_kernel<double, 32>"
        # one ncu capture of the 8 MB batch (`ncu --set full --clock-control none -c 1
        # -k regex:getrf_warp python -m rocsolver_b200.demo --case getrf --n 32 --batch 1000
        # --reps 2`) reads 8.3 MB per 1000 members; the bench rotates 24 copies so that its
        # traffic is the algorithmic figure
        w.traffic_per_unit = 8269824 / 1000
        w.limiter = "latency: one serial 32-column chain per matrix"
        w.launches_per_step = 2
    elif name == "potrf_n64":
        n, bc, nrhs = 64, 20000, 4
        g = torch.Generator(device=dev)
        g.manual_seed(1)
        G = torch.randn(bc, n, n, generator=g, device=dev, dtype=torch.float64)
        A = G @ G.transpose(1, 2) + n * torch.eye(n, device=dev, dtype=torch.float64)
        del G
        B = torch.randn(bc, n, nrhs, generator=g, device=dev, dtype=torch.float64)
        w.A0 = colmajor(torch, A)
        w.B0 = colmajor(torch, B)
        w.Arow, w.Brow = A, B
        w.n, w.bc, w.nrhs = n, bc, nrhs
        w.metric = "batched SPD solves/s (FP64 potrf+potrs, n=64)"
        w.unit = "solves/s"
        w.dtype = "f64"
        w.config = {"workload": "dpotrf+dpotrs strided_batched lower, n=64, batch=20000, nrhs=4, "
                               "A = G G' + n I", "n": n, "batch": bc, "nrhs": nrhs,
                    "l2": "inputs 655 MB > L2; A restored between steps outside the timed events"}
        w.flops_per_unit = n ** 3 / 3.0 + n * n / 2.0 + n / 6.0 + 2.0 * n * n * nrhs
        w.bytes_per_unit_getrf = 2 * (n * (n + 1) // 2) * 8 + 4  # triangle read+write + info
        w.dominant = "potrf_reg_kernel<double, 64>"
        # 105.6 MB per 4000 members from `ncu --set full --clock-control none -c 1
        # -k regex:potrf_reg python -m rocsolver_b200.demo --case potrf --n 64 --batch 4000
        # --reps 2`
        w.traffic_per_unit = 105635840 / 4000
        w.limiter = "latency: one barrier per column"
        w.launches_per_step = 2
    else:
        raise ValueError(name)
    return w


def run_ours(w, torch, rs, dev, handle, steps, warmup):
    n, bc, nrhs = w.n, w.bc, w.nrhs
    rot = getattr(w, "rotate", 1)
    As = [w.A0.clone() for _ in range(rot)]
    Bs = [w.B0.clone() for _ in range(rot)]
    ipiv = torch.zeros(bc * n, dtype=torch.int32, device=dev)
    info = torch.zeros(bc, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    h = handle.value

    def launch(A, B):
        if w.name == "potrf_n64":
            st = rs.call("rocsolver_dpotrf_strided_batched", h, rs.FILL_LOWER, n, rs.ptr(A), n,
                         n * n, rs.ptr(info), bc)
            rs.check(st, "potrf")
            st = rs.call("rocsolver_dpotrs_strided_batched", h, rs.FILL_LOWER, n, nrhs, rs.ptr(A),
                         n, n * n, rs.ptr(B), n, n * nrhs, bc)
            rs.check(st, "potrs")
        else:
            st = rs.call("rocsolver_dgetrf_strided_batched", h, n, n, rs.ptr(A), n, n * n,
                         rs.ptr(ipiv), n, rs.ptr(info), bc)
            rs.check(st, "getrf")
            st = rs.call("rocsolver_dgetrs_strided_batched", h, rs.OP_N, n, nrhs, rs.ptr(A), n,
                         n * n, rs.ptr(ipiv), n, rs.ptr(B), n, n * nrhs, bc)
            rs.check(st, "getrs")

    def restore(i):
        As[i].copy_(w.A0)
        Bs[i].copy_(w.B0)

    for i in range(warmup):
        restore(i % rot)
        launch(As[i % rot], Bs[i % rot])
    torch.cuda.synchronize()
    for i in range(rot):
        restore(i)
    torch.cuda.synchronize()
    # timed region: per-step event pairs on the launching stream; the restore copies
    # (needed because the factorisation is in place) sit between the pairs
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    kev = []
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    time.sleep(0.3)
    for i in range(steps):
        j = i % rot
        if rot == 1 or (i > 0 and j == 0):
            for r in range(rot):
                restore(r)
        ev[i][0].record(stream)
        launch(As[j], Bs[j])
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    # kernel-only timing of the dominant factorisation kernel (same stream)
    fev = []
    for i in range(min(steps, 10)):
        restore(0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        if w.name == "potrf_n64":
            rs.check(rs.call("rocsolver_dpotrf_strided_batched", h, rs.FILL_LOWER, n,
                             rs.ptr(As[0]), n, n * n, rs.ptr(info), bc), "potrf")
        else:
            rs.check(rs.call("rocsolver_dgetrf_strided_batched", h, n, n, rs.ptr(As[0]), n,
                             n * n, rs.ptr(ipiv), n, rs.ptr(info), bc), "getrf")
        b.record(stream)
        fev.append((a, b))
    torch.cuda.synchronize()
    fact_ms = statistics.median([a.elapsed_time(b) for a, b in fev])
    # correctness of the last timed step: backward error per member, on the device
    restore(0)
    launch(As[0], Bs[0])
    X = Bs[0].view(bc, nrhs, n).transpose(1, 2)
    R = torch.bmm(w.Arow, X) - w.Brow
    num = R.abs().sum(2).amax(1)
    den = w.Arow.abs().sum(2).amax(1) * X.abs().sum(2).amax(1) + w.Brow.abs().sum(2).amax(1)
    berr = (num / den)
    info_h = info.cpu().numpy()
    return {"step_ms": step_ms, "fact_ms": fact_ms, "clocks": clocks,
            "berr_max": float(berr.max()), "berr_frac_1e13": float((berr <= 1e-13).double().mean()),
            "info_nonzero": int((info_h != 0).sum())}


def run_mixed(w, torch, rs, dev, handle, steps, warmup):
    """dsgesv on the same inputs: per-step event pairs around the API call (A and B are
    not modified by a converged solve; A is restored between steps anyway, outside the
    events, in case a member fell back to FP64)."""
    n, bc, nrhs = w.n, w.bc, w.nrhs
    A = w.A0.clone()
    B = w.B0.clone()
    X = torch.empty_like(B)
    ipiv = torch.zeros(bc * n, dtype=torch.int32, device=dev)
    info = torch.zeros(bc, dtype=torch.int32, device=dev)
    it = torch.zeros(bc, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    h = handle.value

    def call():
        rs.check(rs.call("rocsolver_dsgesv_strided_batched", h, n, nrhs, rs.ptr(A), n, n * n,
                         rs.ptr(ipiv), n, rs.ptr(B), n, n * nrhs, rs.ptr(X), n, n * nrhs,
                         rs.ptr(it), rs.ptr(info), bc), "dsgesv")

    for _ in range(warmup):
        A.copy_(w.A0)
        call()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    time.sleep(0.3)
    for i in range(steps):
        A.copy_(w.A0)
        ev[i][0].record(stream)
        call()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    # FP32 LU kernel alone (the same kernel dsgesv launches, through its entry point), for
    # the roofline
    A32 = w.A0.float()
    fev = []
    for _ in range(min(steps, 10)):
        Ac = A32.clone()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rs.check(rs.call("rocsolver_sgetrf_tf32_strided_batched", h, n, n, rs.ptr(Ac), n,
                         n * n, rs.ptr(ipiv), n, rs.ptr(info), bc), "sgetrf_tf32")
        b.record(stream)
        fev.append((a, b))
    torch.cuda.synchronize()
    fact_ms = statistics.median([a.elapsed_time(b) for a, b in fev])
    # accuracy of the last timed call: every member's backward error
    A.copy_(w.A0)
    call()
    Xr = X.view(bc, nrhs, n).transpose(1, 2)
    R = torch.bmm(w.Arow, Xr) - w.Brow
    num = R.abs().sum(2).amax(1)
    den = w.Arow.abs().sum(2).amax(1) * Xr.abs().sum(2).amax(1) + w.Brow.abs().sum(2).amax(1)
    berr = num / den
    its = it.cpu().numpy()
    return {"step_ms": step_ms, "fact_ms": fact_ms, "clocks": clocks,
            "berr_max": float(berr.max()), "berr_frac_1e13": float((berr <= 1e-13).double().mean()),
            "info_nonzero": int((info.cpu().numpy() != 0).sum()),
            "iter_mean": float(its[its >= 0].mean()) if (its >= 0).any() else None,
            "iter_max": int(its.max()), "fallbacks": int((its < 0).sum())}


E2E_CHUNKS = 8    # batch slices per step in the end-to-end run (large inputs only)
E2E_STREAMS = 2   # streams (one handle each) the slices alternate over
E2E_MIN_BYTES = 64 << 20  # smaller steps are one slice: there the per-slice launches and
                          # copies cost more than the overlap gains


class SlicedStep:
    """One end-to-end step as slices of the batch issued round-robin on E2E_STREAMS
    streams, each with its own handle (and so its own workspace): body(handle, c0, c1)
    copies members c0..c1-1 in, calls the library, copies the results out, all on the
    current (slice) stream.  Steps with at least E2E_MIN_BYTES of copies are cut into
    E2E_CHUNKS slices, so that one slice's copies overlap another slice's kernels and the
    two copy directions overlap each other, as a caller streaming batches from the host
    would; smaller steps are one slice.  step() spans the whole step: the slice streams
    wait for an event on the main stream and the main stream waits for all of them."""

    def __init__(self, torch, rs, bc, copy_bytes, body):
        self.torch, self.body, self.bc = torch, body, bc
        self.main = torch.cuda.current_stream()
        chunks = E2E_CHUNKS if copy_bytes >= E2E_MIN_BYTES else 1
        per = (bc + chunks - 1) // chunks
        self.bounds = [(c0, min(bc, c0 + per)) for c0 in range(0, bc, per)]
        self.streams = ([self.main] if len(self.bounds) == 1
                        else [torch.cuda.Stream() for _ in range(E2E_STREAMS)])
        self.handles = [rs.Handle(st.cuda_stream) for st in self.streams]
        self.desc = (f"{len(self.bounds)} slices of <= {per} members over "
                     f"{len(self.streams)} streams")

    def step(self):
        torch = self.torch
        if len(self.bounds) == 1:  # one slice: the whole batch on the main stream
            self.body(self.handles[0].value, 0, self.bc)
            return
        start = torch.cuda.Event()
        start.record(self.main)
        for i, (c0, c1) in enumerate(self.bounds):
            st = self.streams[i % E2E_STREAMS]
            st.wait_event(start)
            with torch.cuda.stream(st):
                self.body(self.handles[i % E2E_STREAMS].value, c0, c1)
        for st in self.streams:
            self.main.wait_stream(st)

    def close(self):
        self.torch.cuda.synchronize()
        for h in self.handles:
            h.close()


def run_e2e(w, torch, rs, dev, handle, steps):
    """Same step through the public C ABI with host buffers: every step copies the pinned
    A and B to the device, factors and solves, and copies the solutions and info back
    (streamed in slices, SlicedStep); all copies are inside the timed region."""
    n, bc, nrhs = w.n, w.bc, w.nrhs
    hA = w.A0.cpu().pin_memory()
    hB = w.B0.cpu().pin_memory()
    hX = torch.empty_like(hB).pin_memory()
    hI = torch.empty(bc, dtype=torch.int32).pin_memory()
    dA = torch.empty_like(w.A0)
    dB = torch.empty_like(w.B0)
    dX = torch.empty_like(w.B0)
    ipiv = torch.zeros(bc, n, dtype=torch.int32, device=dev)
    info = torch.zeros(bc, dtype=torch.int32, device=dev)
    it = torch.zeros(bc, dtype=torch.int32, device=dev)
    P = rs.ptr
    h2d, d2h = hA.numel() * 8 + hB.numel() * 8, hX.numel() * 8 + bc * 4

    def body(h, c0, c1):
        m = c1 - c0
        cut = (lambda t: t) if m == bc else (lambda t: t[c0:c1])
        a, b, x = cut(dA), cut(dB), cut(dX)
        pv, inf, itr = cut(ipiv), cut(info), cut(it)
        a.copy_(cut(hA), non_blocking=True)
        b.copy_(cut(hB), non_blocking=True)
        if w.name == "dsgesv_n256":
            rs.check(rs.call("rocsolver_dsgesv_strided_batched", h, n, nrhs, P(a), n, n * n,
                             P(pv), n, P(b), n, n * nrhs, P(x), n, n * nrhs, P(itr), P(inf),
                             m), "dsgesv")
            out = x
        elif w.name == "potrf_n64":
            rs.check(rs.call("rocsolver_dposv_strided_batched", h, rs.FILL_LOWER, n, nrhs,
                             P(a), n, n * n, P(b), n, n * nrhs, P(inf), m), "posv")
            out = b
        else:
            rs.check(rs.call("rocsolver_dgetrf_strided_batched", h, n, n, P(a), n, n * n,
                             P(pv), n, P(inf), m), "getrf")
            rs.check(rs.call("rocsolver_dgetrs_strided_batched", h, rs.OP_N, n, nrhs, P(a), n,
                             n * n, P(pv), n, P(b), n, n * nrhs, m), "getrs")
            out = b
        cut(hX).copy_(out, non_blocking=True)
        cut(hI).copy_(inf, non_blocking=True)

    sl = SlicedStep(torch, rs, bc, h2d + d2h, body)
    try:
        for _ in range(2):
            sl.step()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k = max(3, min(steps, 10))
        a.record(sl.main)
        for _ in range(k):
            sl.step()
        b.record(sl.main)
        torch.cuda.synchronize()
    finally:
        sl.close()
    ms = a.elapsed_time(b) / k
    return {"ms": ms, "h2d": h2d, "d2h": d2h, "pipeline": sl.desc}


# ----------------------------------------------------------------------------- CPU side
def _host_inputs(w):
    """Host copies of the workload's inputs (column-major members, flat buffers)."""
    if not hasattr(w, "host"):
        if w.name == "vbatched_4096":
            w.host = (w.sizes.cpu().numpy().astype(np.int32), w.rhs.cpu().numpy().astype(np.int32),
                      w.A0.cpu().numpy(), w.B0.cpu().numpy())
        elif w.name.startswith("adjoint"):
            w.host = (w.A0.double().cpu().numpy(), w.X0.double().cpu().numpy(),
                      w.G0.double().cpu().numpy())
        elif w.name == "getri_n64":
            w.host = (w.A0.cpu().numpy(),)
        else:
            w.host = (w.A0.cpu().numpy(), w.B0.cpu().numpy())
    return w.host


def _lapack_run(w, routine, cnt, threads):
    """One host-LAPACK pass over the first cnt members; returns seconds."""
    import oracle
    cnt = min(cnt, w.bc)
    if w.name == "vbatched_4096":
        sz, kk, A0, B0 = _host_inputs(w)
        nmax = w.nmax
        A = A0[:cnt].reshape(-1).copy()
        B = B0[:cnt].reshape(-1).copy()
        ipiv = np.zeros(cnt * nmax, np.int32)
        info = np.zeros(cnt, np.int32)
        t0 = time.perf_counter()
        oracle.lapack_batch(oracle.LH_VGESV, nmax, 16, A, nmax, nmax * nmax, ipiv, nmax, B, nmax,
                            16 * nmax, info=info, nv=sz, rv=kk, ld=nmax, bc=cnt, nthreads=threads)
        return time.perf_counter() - t0
    if w.name.startswith("adjoint"):
        A0, X0, G0 = _host_inputs(w)
        n, k = w.n, w.nrhs
        if not hasattr(w, "host_lu"):  # factored once, outside the timing, like the GPU arm
            LU = A0.reshape(-1).copy()
            piv = np.zeros(w.bc * n, np.int32)
            inf = np.zeros(w.bc, np.int32)
            oracle.lapack_batch(oracle.LH_GETRF_GETRS, n, 0, LU, n, n * n, piv, n, None, n, 0,
                                info=inf, bc=w.bc, nthreads=oracle.physical_cores())
            w.host_lu = (LU, piv)
        LU, piv = w.host_lu
        gB = G0[:cnt].reshape(-1).copy()
        gA = np.empty(cnt * n * n)
        t0 = time.perf_counter()
        oracle.lapack_batch(oracle.LH_ADJOINT, n, k, LU, n, n * n, piv, n, gB, n, n * k,
                            bc=cnt, nthreads=threads)
        oracle.lapack_outer(n, k, gB, X0[:cnt].reshape(-1), gA, cnt, nthreads=threads)
        return time.perf_counter() - t0
    if w.name == "zgesv_n64":
        A0, B0 = _host_inputs(w)
        n, k = w.n, w.nrhs
        A = A0[:cnt].reshape(-1).view(np.float64).copy()
        B = B0[:cnt].reshape(-1).view(np.float64).copy()
        ipiv = np.zeros(cnt * n, np.int32)
        info = np.zeros(cnt, np.int32)
        t0 = time.perf_counter()
        oracle.lapack_batch(oracle.LH_ZGESV, n, k, A, n, 2 * n * n, ipiv, n, B, n, 2 * n * k,
                            info=info, bc=cnt, nthreads=threads)
        return time.perf_counter() - t0
    if w.name == "getri_n64":
        (A0,) = _host_inputs(w)
        n = w.n
        if not hasattr(w, "host_lu"):  # factored once, outside the timing, like the GPU arm
            LU = A0.reshape(-1).copy()
            piv = np.zeros(w.bc * n, np.int32)
            inf = np.zeros(w.bc, np.int32)
            oracle.lapack_batch(oracle.LH_GETRF_GETRS, n, 0, LU, n, n * n, piv, n, None, n, 0,
                                info=inf, bc=w.bc, nthreads=oracle.physical_cores())
            w.host_lu = (LU, piv)
        LU, piv = w.host_lu
        A = LU[:cnt * n * n].copy()
        info = np.zeros(cnt, np.int32)
        t0 = time.perf_counter()
        oracle.lapack_batch(oracle.LH_GETRI, n, 0, A, n, n * n, piv, n, None, n, 0, info=info,
                            bc=cnt, nthreads=threads)
        return time.perf_counter() - t0
    A0, B0 = _host_inputs(w)
    n, k = w.n, w.nrhs
    A = A0[:cnt].reshape(-1).copy()
    B = B0[:cnt].reshape(-1).copy()
    ipiv = np.zeros(cnt * n, np.int32)
    info = np.zeros(cnt, np.int32)
    X = np.zeros_like(B) if routine == "dsgesv" else None
    it = np.zeros(cnt, np.int32) if routine == "dsgesv" else None
    op = {"getrf+getrs": oracle.LH_GETRF_GETRS, "potrf+potrs": oracle.LH_POTRF_POTRS,
          "gesv": oracle.LH_GESV, "dsgesv": oracle.LH_DSGESV}[routine]
    t0 = time.perf_counter()
    oracle.lapack_batch(op, n, k, A, n, n * n, ipiv, n, B, n, n * k, X, n, n * k, info, it,
                        bc=cnt, nthreads=threads)
    return time.perf_counter() - t0


def _lapack_rate(w, routine, threads, target_s):
    """Members per second of one routine on a bounded sample: a calibration pass, then
    enough members (repeating the whole batch if needed) to take about target_s."""
    c = max(threads * 2, 8)
    t = _lapack_run(w, routine, c, threads)
    c = min(c, w.bc)
    want = max(c, min(w.bc, int(c * max(1.0, target_s / max(t, 1e-6)))))
    t = _lapack_run(w, routine, want, threads)
    reps, tot = 1, t
    if want == w.bc and t < target_s:
        reps = max(1, int(target_s / max(t, 1e-6)))
        tot = sum(_lapack_run(w, routine, want, threads) for _ in range(reps))
    return reps * want / tot, f"{want} of {w.bc} members" + (f" x {reps}" if reps > 1 else "") \
        + f" in {tot:.1f} s"


def _lapack_routines(w):
    """Host-LAPACK routines timed for a workload (the reference's CPU path for it)."""
    return {"dsgesv_n256": ["dsgesv", "gesv"], "gesv_n256": ["gesv"],
            "getrf_n32": ["getrf+getrs"], "potrf_n64": ["potrf+potrs"],
            "vbatched_4096": ["gesv (per-member n, nrhs)"],
            "adjoint_n128": ["getrs (trans T) + dgemm"],
            "adjoint_n128_fp32": ["getrs (trans T) + dgemm"],
            "zgesv_n64": ["zgesv"], "getri_n64": ["getri (factors given)"]}[w.name]


def cpu_sample(w, target_s, one_core_s=None):
    """Host LAPACK (scipy's bundled OpenBLAS, loaded with dlopen; one call per member on one
    thread, the batch split statically over all physical cores) on a bounded sample of the
    same inputs, plus the 1-core figure (the reference client's serial loop).  For the
    mixed-precision headline both LAPACK dsgesv (the CPU analogue of the mixed path) and
    dgesv are timed and the faster is the value."""
    import oracle
    if not oracle.lapack_available():
        raise RuntimeError("host LAPACK (scipy's OpenBLAS) is not available on this host")
    cores = oracle.physical_cores()
    one_core_s = target_s / 4 if one_core_s is None else one_core_s
    routines = _lapack_routines(w)
    per = {}
    for r in routines:
        key = r.split(" ")[0]
        v, samp = _lapack_rate(w, key, cores, target_s / len(routines))
        v1, samp1 = _lapack_rate(w, key, 1, one_core_s / len(routines))
        per[r] = {"value": v, "sample": samp, "one_core": v1, "one_core_sample": samp1}
    best = max(per, key=lambda r: per[r]["value"])
    return {"value": per[best]["value"], "unit": w.unit, "cores": cores, "kind": "lapack",
            "routine": best, "one_core": per[best]["one_core"],
            "library": f"OpenBLAS bundled with scipy ({oracle.lapack_library_name()}), dlopen",
            "cpu_model": oracle.cpu_model(), "nproc": os.cpu_count(),
            "sample": f"host LAPACK {best}: {per[best]['sample']}, {cores} threads "
                      f"(one member per call); 1 core: {per[best]['one_core_sample']}",
            "routines": per}


# ----------------------------------------------------------------------------- main
class Ctx:
    """What every workload runner shares: torch, the library, the device, the process group
    (None on one GPU), the handle on the current stream, and this process's rank."""
    pass


def fp64_peak_tflops(torch, dev):
    """FP64 dense peak measured in this run: cuBLAS dgemm 8192^3 (torch.matmul), best of 3
    CUDA-event timings.  Only the denominator of the FP64 compute fraction."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    best = None
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    return 2.0 * 8192 ** 3 / (best / 1e3) / 1e12


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return main_reference(args, rank, world)

    import torch
    import rocsolver_b200 as rs
    torch.cuda.set_device(local)
    ctx = Ctx()
    ctx.torch, ctx.rs = torch, rs
    ctx.dev = torch.device("cuda", local)
    ctx.rank, ctx.world, ctx.local = rank, world, local
    ctx.pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        ctx.pg = dist
    ctx.handle = rs.Handle(torch.cuda.current_stream().cuda_stream)
    ctx.peaks = load_peaks()
    ctx.peaks["fp64_tflops"] = fp64_peak_tflops(torch, ctx.dev)
    headline = "dsgesv_n256" if args.workload == "all" else args.workload
    line = run_workload(headline, args, ctx, args.steps, args.warmup, args.cpu_seconds)
    if args.workload == "all":
        # the other configurations, measured in the same run (fewer steps; same contract)
        nested = {}
        for name in NESTED:
            sub = run_workload(name, args, ctx, min(args.steps, 10), max(3, min(args.warmup, 3)),
                               args.cpu_seconds_extra)
            for k in ("n_gpus", "higher_is_better", "scaling", "vs_baseline", "data"):
                sub.pop(k, None)
            nested[name] = sub
            torch.cuda.empty_cache()
        line["configs"] = nested
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.handle.close()
    if ctx.pg:
        ctx.pg.barrier()
        ctx.pg.destroy_process_group()


def run_workload(name, args, ctx, steps, warmup, cpu_seconds):
    if name in WIDE_WORKLOADS:
        return run_wide(name, args, ctx, steps, warmup, cpu_seconds)
    if name in EXTRA_WORKLOADS:
        return run_extra(name, args, ctx, steps, warmup, cpu_seconds)
    return run_core(name, args, ctx, steps, warmup, cpu_seconds)


def run_core(name, args, ctx, steps, warmup, cpu_seconds):
    """The strided-batched workloads (C1, C2, C3): one JSON line as a dict."""
    torch, rs, dev, pg, handle = ctx.torch, ctx.rs, ctx.dev, ctx.pg, ctx.handle
    world, rank = ctx.world, ctx.rank
    w = build_workload(name, torch, rs, dev, handle)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    plain = None
    if w.name == "dsgesv_n256":
        plain = run_ours(w, torch, rs, dev, handle, steps, warmup)
        res = run_mixed(w, torch, rs, dev, handle, steps, warmup)
    else:
        res = run_ours(w, torch, rs, dev, handle, steps, warmup)
    total_ms = sum(res["step_ms"])
    total_ms = max_over_ranks(torch, pg, total_ms, dev)
    e2e = run_e2e(w, torch, rs, dev, handle, steps)
    e2e["ms"] = max_over_ranks(torch, pg, e2e["ms"], dev)
    ms_per_step = total_ms / steps
    units = w.bc * world
    value = units / (ms_per_step / 1e3)
    peaks = ctx.peaks
    fact_s = res["fact_ms"] / 1e3
    achieved_gbs = w.bytes_per_unit_getrf * w.bc / fact_s / 1e9
    fp64_tf = w.flops_per_unit * w.bc / fact_s / 1e12
    line = {
        "metric": w.metric, "value": value, "unit": w.unit, "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": w.dtype,
        "data": "synthetic (seeded, generated on device)", "config": w.config,
        "gpu_launches": w.launches_per_step * steps,
        "e2e": {"value": units / (e2e["ms"] / 1e3), "unit": w.unit,
                "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                "pipeline": e2e["pipeline"]},
        "roofline": {"bound": "hbm", "limiter": w.limiter, "kernel": w.dominant, "achieved": achieved_gbs,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved_gbs / peaks["hbm_gbs"],
                     "traffic": w.traffic_per_unit * w.bc,
                     "peak_source": peaks["source"],
                     "kernel_ms": res["fact_ms"],
                     "compute": {"achieved_tflops": fp64_tf, "peak_tflops": peaks["fp64_tflops"],
                                 "frac": fp64_tf / peaks["fp64_tflops"],
                                 "peak": "FP64 dgemm measured in this run (cuBLAS 8192^3)"}},
        "clocks": res["clocks"],
        "accuracy": {"backward_err_max": res["berr_max"],
                     "frac_backward_err_le_1e-13": res["berr_frac_1e13"],
                     "info_nonzero": res["info_nonzero"]},
    }
    if plain is not None:
        plain_ms = sum(plain["step_ms"]) / steps
        plain_ms = max_over_ranks(torch, pg, plain_ms, dev)
        pf_tf = w.flops_per_unit * w.bc / (plain["fact_ms"] / 1e3) / 1e12
        line["plain_fp64"] = {"value": units / (plain_ms / 1e3), "unit": w.unit,
                              "ms_per_step": plain_ms, "getrf_ms": plain["fact_ms"],
                              "getrf_fp64_tflops": pf_tf,
                              "getrf_fp64_frac": pf_tf / peaks["fp64_tflops"],
                              "backward_err_max": plain["berr_max"],
                              "frac_backward_err_le_1e-13": plain["berr_frac_1e13"]}
        line["mixed_over_plain"] = plain_ms / ms_per_step
        line["accuracy"].update({"iter_mean": res["iter_mean"], "iter_max": res["iter_max"],
                                 "fp64_fallbacks": res["fallbacks"]})
        fbytes = (2 * w.n * w.n * 4 + 4 * w.n + 4) * w.bc
        fgbs = fbytes / (res["fact_ms"] / 1e3) / 1e9
        tf = w.flops_per_unit * w.bc / (res["fact_ms"] / 1e3) / 1e12
        tf32_peak = peaks["bf16_tflops"] / 2
        line["roofline"] = {"bound": "hbm", "limiter": w.limiter, "kernel": w.dominant, "achieved": fgbs,
                            "peak": peaks["hbm_gbs"], "unit": "GB/s",
                            "frac": fgbs / peaks["hbm_gbs"],
                            "traffic": w.traffic_per_unit * w.bc,
                            "peak_source": peaks["source"], "kernel_ms": res["fact_ms"],
                            "compute": {"achieved_tflops": tf, "peak_tflops": tf32_peak,
                                        "frac": 3 * tf / tf32_peak,
                                        "peak": "dense TF32 tensor rate = half the measured "
                                                "bf16 figure; frac counts the 3 split-TF32 "
                                                "products per FP32 multiply-add"}}
        if "stages_ms" in res:
            line["mixed_stages_ms"] = res["stages_ms"]
    if rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_sample(w, cpu_seconds)
    del w
    return line


def main_reference(args, rank, world):
    """Reference arm: the reference's own path is HIP/rocBLAS for AMD GPUs and cannot run
    here; its CPU implementation of the path is host LAPACK (its clients' oracle and CPU
    timing).  Rank 0 times host LAPACK (scipy's OpenBLAS, dlopen) on all physical host cores
    over a bounded sample of the same workload; the other ranks exit without work."""
    if rank != 0:
        return
    import torch
    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    name = "dsgesv_n256" if args.workload == "all" else args.workload
    w = (_extra_workload(name, torch, dev) if name in EXTRA_WORKLOADS
         else build_workload(name, torch, None, dev, None))
    w.dtype = getattr(w, "dtype", "f64")
    vals = []
    r = None
    for i in range(args.warmup + args.steps):
        r = cpu_sample(w, max(1.0, args.cpu_seconds / max(1, args.steps)),
                       one_core_s=0.5 if i < args.warmup + args.steps - 1 else 2.0)
        if i >= args.warmup:
            vals.append(r["value"])
    v = statistics.median(vals)
    cb = dict(r)
    cb["value"] = v
    line = {"metric": w.metric, "value": v, "unit": w.unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * w.bc / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": w.dtype,
            "data": "synthetic (seeded)", "config": w.config, "impl": "reference",
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": w.unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- extra rows
def run_wide(name, args, ctx, steps, warmup, cpu_seconds):
    """The complex solve (zgesv_n64) and the inverse (getri_n64): same contract as run_core
    (device time of the API call per step, max over ranks; e2e through the C ABI with host
    buffers; roofline of the dominant kernel; host LAPACK beside it)."""
    torch, rs, dev, pg, handle = ctx.torch, ctx.rs, ctx.dev, ctx.pg, ctx.handle
    world, rank = ctx.world, ctx.rank
    h = handle.value
    P = rs.ptr
    stream = torch.cuda.current_stream()
    w = Workload()
    w.name = name
    g = torch.Generator(device=dev)
    if name == "zgesv_n64":
        n, bc, nrhs = 64, 8192, 1
        g.manual_seed(13)
        re = lambda *sh: torch.rand(*sh, generator=g, device=dev, dtype=torch.float64) * 2 - 1
        A = torch.complex(re(bc, n, n), re(bc, n, n))
        B = torch.complex(re(bc, n, nrhs), re(bc, n, nrhs))
        w.A0, w.B0 = colmajor(torch, A), colmajor(torch, B)
        es = 16
        w.metric = "batched complex solves/s (zgesv_strided_batched, n=64)"
        w.unit = "solves/s"
        w.dtype = "c128"
        w.config = {"workload": "rocsolver_zgesv_strided_batched, n=64, batch 8192, nrhs 1, "
                                "re/im of A and b ~ U[-1,1]", "n": n, "batch": bc, "nrhs": nrhs,
                    "l2": "inputs 537 MB > L2; A and B restored between steps outside the "
                          "timed events"}
        w.bytes_per_unit = 2 * n * n * es + 4 * n + 4        # zgetrf: A in and out, ipiv, info
        w.flops_per_unit = 8.0 * n ** 3 / 3 + 8.0 * n * n * nrhs
        w.kernel = ("cgetrf_reg_kernel<rocblas_double_complex, 8, 2, true> (member in "
                    "registers, one CTA barrier per column)")
        # 217.1 MB per 2048 members from `ncu --set full --clock-control none -k
        # regex:cgetrf_reg -c 1 python -m rocsolver_b200.demo --case getrf --dtype z --n 64
        # --batch 2048 --reps 2`
        w.traffic_per_unit = (134357248 + 82747648) / 2048
        A_, B_ = w.A0.clone(), w.B0.clone()
        ipiv = torch.zeros(bc * n, dtype=torch.int32, device=dev)
        info = torch.zeros(bc, dtype=torch.int32, device=dev)

        def call():
            rs.check(rs.call("rocsolver_zgesv_strided_batched", h, n, nrhs, P(A_), n, n * n,
                             P(ipiv), n, P(B_), n, n * nrhs, P(info), bc), "zgesv")

        def kernel_only():
            rs.check(rs.call("rocsolver_zgetrf_strided_batched", h, n, n, P(A_), n, n * n,
                             P(ipiv), n, P(info), bc), "zgetrf")

        def restore():
            A_.copy_(w.A0)
            B_.copy_(w.B0)
        launches = 2
    else:
        n, bc, nrhs = 64, 16384, 0
        g.manual_seed(14)
        A = torch.rand(bc, n, n, generator=g, device=dev, dtype=torch.float64) * 2 - 1
        A += 4 * torch.eye(n, device=dev, dtype=torch.float64)
        w.A0 = colmajor(torch, A)
        es = 8
        w.metric = "batched inverses/s (dgetri_strided_batched from the LU factors, n=64)"
        w.unit = "inverses/s"
        w.dtype = "f64"
        w.config = {"workload": "rocsolver_dgetri_strided_batched in place, n=64, batch 16384, "
                                "A ~ U[-1,1] + 4 I factored by dgetrf once outside the timing",
                    "n": n, "batch": bc,
                    "l2": "factors 537 MB > L2; restored between steps outside the timed events"}
        w.bytes_per_unit = 2 * n * n * es + 4 * n + 4        # LU in, inverse out, ipiv, info
        w.flops_per_unit = 4.0 * n ** 3 / 3
        w.kernel = "getri_small_kernel<double, 64> (the whole inverse in shared memory)"
        # 480.7 MB per 8192 members from `ncu --set full --clock-control none -k
        # regex:getri_small -c 1 python -m rocsolver_b200.demo --case getri --n 64 --batch 8192
        # --reps 2`
        w.traffic_per_unit = (270556928 + 210124800) / 8192
        LU0 = w.A0.clone()
        ipiv = torch.zeros(bc * n, dtype=torch.int32, device=dev)
        info = torch.zeros(bc, dtype=torch.int32, device=dev)
        rs.check(rs.call("rocsolver_dgetrf_strided_batched", h, n, n, P(LU0), n, n * n, P(ipiv),
                         n, P(info), bc), "dgetrf")
        A_ = LU0.clone()

        def call():
            rs.check(rs.call("rocsolver_dgetri_strided_batched", h, n, P(A_), n, n * n, P(ipiv),
                             n, P(info), bc), "dgetri")
        kernel_only = call

        def restore():
            A_.copy_(LU0)
        launches = 1
    w.n, w.bc, w.nrhs = n, bc, nrhs
    for _ in range(warmup):
        restore()
        call()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    time.sleep(0.3)
    for i in range(steps):
        restore()
        ev[i][0].record(stream)
        call()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = max_over_ranks(torch, pg, sum(a.elapsed_time(b) for a, b in ev), dev)
    ms = total_ms / steps
    kev = []
    for _ in range(min(steps, 10)):
        restore()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        kernel_only()
        b.record(stream)
        kev.append((a, b))
    torch.cuda.synchronize()
    kms = statistics.median([a.elapsed_time(b) for a, b in kev])
    # accuracy of one more call
    restore()
    call()
    torch.cuda.synchronize()
    if name == "zgesv_n64":
        Ar = w.A0.view(bc, n, n).transpose(1, 2)
        X = B_.view(bc, nrhs, n).transpose(1, 2)
        Bm = w.B0.view(bc, nrhs, n).transpose(1, 2)
        R = torch.bmm(Ar, X) - Bm
        num = R.abs().sum(2).amax(1)
        den = Ar.abs().sum(2).amax(1) * X.abs().sum(2).amax(1) + Bm.abs().sum(2).amax(1)
        berr = num / den
        acc = {"backward_err_max": float(berr.max()),
               "frac_backward_err_le_1e-13": float((berr <= 1e-13).double().mean()),
               "info_nonzero": int((info != 0).sum())}
    else:
        Ar = w.A0.view(bc, n, n).transpose(1, 2)
        Inv = A_.view(bc, n, n).transpose(1, 2)
        E = torch.bmm(Ar, Inv) - torch.eye(n, device=dev, dtype=torch.float64)
        rel = E.abs().amax((1, 2)) / (Ar.abs().sum(2).amax(1) * Inv.abs().sum(2).amax(1))
        acc = {"residual_AinvA_minus_I_rel_max": float(rel.max()),
               "info_nonzero": int((info != 0).sum())}
    # e2e: inputs from pinned host memory, results back, every step (sliced over 2 streams)
    if name == "zgesv_n64":
        hA, hB = w.A0.cpu().pin_memory(), w.B0.cpu().pin_memory()
        hX, hI = torch.empty_like(hB).pin_memory(), torch.empty(bc, dtype=torch.int32).pin_memory()
        dA, dB = torch.empty_like(w.A0), torch.empty_like(w.B0)
        h2d, d2h = (hA.numel() + hB.numel()) * es, hX.numel() * es + bc * 4

        def body(hs, c0, c1):
            sl_ = slice(c0, c1)
            dA[sl_].copy_(hA[sl_], non_blocking=True)
            dB[sl_].copy_(hB[sl_], non_blocking=True)
            rs.check(rs.call("rocsolver_zgesv_strided_batched", hs, n, nrhs, P(dA[sl_]), n,
                             n * n, P(ipiv.view(bc, n)[sl_]), n, P(dB[sl_]), n, n * nrhs,
                             P(info[sl_]), c1 - c0), "zgesv")
            hX[sl_].copy_(dB[sl_], non_blocking=True)
            hI[sl_].copy_(info[sl_], non_blocking=True)
    else:
        hLU, hP = LU0.cpu().pin_memory(), ipiv.cpu().pin_memory()
        hInv, hI = torch.empty_like(hLU).pin_memory(), torch.empty(bc, dtype=torch.int32).pin_memory()
        dA, dP = torch.empty_like(LU0), torch.empty_like(ipiv)
        h2d, d2h = hLU.numel() * es + hP.numel() * 4, hInv.numel() * es + bc * 4

        def body(hs, c0, c1):
            sl_ = slice(c0, c1)
            dA[sl_].copy_(hLU[sl_], non_blocking=True)
            dP.view(bc, n)[sl_].copy_(hP.view(bc, n)[sl_], non_blocking=True)
            rs.check(rs.call("rocsolver_dgetri_strided_batched", hs, n, P(dA[sl_]), n, n * n,
                             P(dP.view(bc, n)[sl_]), n, P(info[sl_]), c1 - c0), "dgetri")
            hInv[sl_].copy_(dA[sl_], non_blocking=True)
            hI[sl_].copy_(info[sl_], non_blocking=True)
    sl = SlicedStep(torch, rs, bc, h2d + d2h, body)
    try:
        for _ in range(2):
            sl.step()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k = max(3, min(steps, 5))
        a.record(sl.main)
        for _ in range(k):
            sl.step()
        b.record(sl.main)
        torch.cuda.synchronize()
    finally:
        sl.close()
    e2e_ms = max_over_ranks(torch, pg, a.elapsed_time(b) / k, dev)
    peaks = ctx.peaks
    gbs = w.bytes_per_unit * bc / (kms / 1e3) / 1e9
    tf = w.flops_per_unit * bc / (kms / 1e3) / 1e12
    line = {"metric": w.metric, "value": bc * world / (ms / 1e3), "unit": w.unit,
            "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": w.dtype,
            "data": "synthetic (seeded, generated on device)", "config": w.config,
            "gpu_launches": launches * steps,
            "e2e": {"value": bc * world / (e2e_ms / 1e3), "unit": w.unit,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "pipeline": sl.desc},
            "roofline": {"bound": "hbm",
                         "limiter": "latency: the per-column pivot chain of the warp holding "
                                    "the column, 2 members (16 warps) per SM"
                         if name == "zgesv_n64" else
                         "latency: dependent dot-product chains in shared memory, 12 warps/SM",
                         "kernel": w.kernel, "achieved": gbs, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": gbs / peaks["hbm_gbs"],
                         "traffic": w.traffic_per_unit * bc,
                         "peak_source": peaks["source"], "kernel_ms": kms,
                         "compute": {"achieved_tflops": tf, "peak_tflops": peaks["fp64_tflops"],
                                     "frac": tf / peaks["fp64_tflops"],
                                     "peak": "FP64 dgemm measured in this run (cuBLAS 8192^3)"}},
            "clocks": clocks, "accuracy": acc}
    if rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_sample(w, cpu_seconds)
    return line


def _vb_inputs(torch, dev, bc, nmax, seed):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    sizes = torch.randint(8, nmax + 1, (bc,), generator=g, device=dev, dtype=torch.int32)
    rhs = torch.randint(1, 17, (bc,), generator=g, device=dev, dtype=torch.int32)
    A = torch.rand(bc, nmax, nmax, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    A += 0.1 * sizes.double()[:, None, None] * torch.eye(nmax, device=dev, dtype=torch.float64)
    B = torch.rand(bc, 16, nmax, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    # member b: n_b x n_b column-major in an nmax x nmax slot (lda = nmax); B: nmax x 16
    return sizes, rhs, A.transpose(1, 2).contiguous(), B.contiguous()


def _extra_workload(name, torch, dev):
    w = Workload()
    w.name = name
    if name == "vbatched_4096":
        w.bc, w.nmax = 4096, 512
        w.sizes, w.rhs, w.A0, w.B0 = _vb_inputs(torch, dev, w.bc, w.nmax, 11)
        w.metric = "variable-size batched solves/s (FP64 gesv_vbatched, n~U[8,512], nrhs~U[1,16])"
        w.unit = "solves/s"
        w.config = {"workload": "rocsolver_dgesv_vbatched, 4096 members, n ~ U[8,512], "
                                "nrhs ~ U[1,16], A ~ U[-1,1] + 0.1 n I, one persistent launch "
                                "(plus the plan kernel) replayed from a CUDA graph",
                    "batch": w.bc, "n_max": w.nmax,
                    "l2": "inputs 8.6 GB > L2; A and B restored between steps outside the "
                          "timed events"}
        n = w.sizes.double()
        k = w.rhs.double()
        w.bytes_total = float((2 * n * n * 8 + 2 * n * k * 8 + 4 * n + 4).sum())
        w.flops_total = float((2 * n ** 3 / 3 + 2 * n * n * k).sum())
        # DRAM bytes per member: 4464.1 MB per 512 members of the same distribution from
        # `ncu --set full --clock-control none -c 1 -k regex:vb_persistent python -m
        # rocsolver_b200.demo --case vbatched --n 512 --batch 512 --nrhs 16 --reps 2`
        w.traffic_per_unit = 4464067000 / 512
    else:
        w.bc, w.n, w.nrhs = 8192, 128, 8
        w.prec = "s" if name.endswith("fp32") else "d"
        dt = torch.float32 if w.prec == "s" else torch.float64
        es = 4 if w.prec == "s" else 8
        w.dtype = "f32" if w.prec == "s" else "f64"
        g = torch.Generator(device=dev)
        g.manual_seed(12)
        n, bc, nrhs = w.n, w.bc, w.nrhs
        A = torch.rand(bc, n, n, generator=g, device=dev, dtype=torch.float64) * 2 - 1
        A += 4 * torch.eye(n, device=dev, dtype=torch.float64)
        w.Arow = A
        w.A0 = A.to(dt).transpose(1, 2).contiguous()
        w.X0 = torch.randn(bc, nrhs, n, generator=g, device=dev, dtype=torch.float64).to(dt)
        w.G0 = torch.randn(bc, nrhs, n, generator=g, device=dev, dtype=torch.float64).to(dt)
        w.metric = (f"batched solve adjoints/s ({'FP32' if w.prec == 's' else 'FP64'} "
                    f"getrs_adjoint: gB = A^-T G, gA = -gB X')")
        w.unit = "adjoints/s"
        w.config = {"workload": f"rocsolver_{w.prec}getrs_adjoint_strided_batched, n=128, "
                                "batch 8192, nrhs 8, A ~ U[-1,1] + 4 I factored once (not "
                                "timed), G ~ N(0,1)", "n": n, "batch": bc, "nrhs": nrhs,
                    "l2": f"factors {bc * n * n * es / 2**30:.1f} GiB > L2"}
        w.bytes_total = bc * (2 * n * n * es + 4 * n * nrhs * es + 4 * n)
        w.flops_total = bc * (4.0 * n * n * nrhs)
        # 245.5 MB per 1024 FP64 members from `ncu --set full --clock-control none -c 1
        # -k regex:solve_adjoint python -m rocsolver_b200.demo --case adjoint --n 128
        # --batch 1024 --nrhs 8 --reps 2` (FP32 scaled by the element size)
        w.traffic_per_unit = 245479424 / 1024 * es / 8
    return w


def run_extra(name, args, ctx, steps, warmup, cpu_seconds):
    """The variable-size and adjoint rows (C4, C5): same contract as run_core (one JSON line
    as a dict, device time = max over ranks, e2e through the C ABI with host buffers)."""
    torch, rs, dev, pg, handle = ctx.torch, ctx.rs, ctx.dev, ctx.pg, ctx.handle
    world, rank = ctx.world, ctx.rank
    h = handle.value
    extra_handles = []
    graph = None
    w = _extra_workload(name, torch, dev)
    stream = torch.cuda.current_stream()
    P = rs.ptr
    bc = w.bc
    extra = {}
    if w.name == "vbatched_4096":
        nmax = w.nmax
        A, B = w.A0.clone(), w.B0.clone()
        ld = torch.full((bc,), nmax, dtype=torch.int32, device=dev)
        ipiv = torch.zeros(bc * nmax, dtype=torch.int32, device=dev)
        info = torch.zeros(bc, dtype=torch.int32, device=dev)
        ar = torch.arange(bc, device=dev, dtype=torch.int64)
        pa = ar * (nmax * nmax * 8) + A.data_ptr()
        pb = ar * (16 * nmax * 8) + B.data_ptr()
        pp = ar * (nmax * 4) + ipiv.data_ptr()

        # captured on a side stream with its own handle (a graph cannot capture the legacy
        # default stream); replays run on the current stream
        cap = torch.cuda.Stream()
        hcap = rs.Handle(cap.cuda_stream)
        extra_handles = [hcap]

        def call():
            rs.check(rs.call("rocsolver_dgesv_vbatched", hcap.value, P(w.sizes), P(w.rhs), P(pa),
                             P(ld), P(pp), P(pb), P(ld), P(info), nmax, 16, bc), "gesv_vbatched")

        def restore():
            A.copy_(w.A0)
            B.copy_(w.B0)

        restore()
        torch.cuda.synchronize()
        with torch.cuda.stream(cap):
            call()  # sizes the workspace before capture
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=cap):
            call()
        torch.cuda.synchronize()
        run = graph.replay
        launches = 2
    else:
        n, nrhs = w.n, w.nrhs
        LU = w.A0.clone()
        ipiv = torch.zeros(bc * n, dtype=torch.int32, device=dev)
        info = torch.zeros(bc, dtype=torch.int32, device=dev)
        rs.check(rs.call(f"rocsolver_{w.prec}getrf_strided_batched", h, n, n, P(LU), n, n * n,
                         P(ipiv), n, P(info), bc), "getrf")
        gA = torch.empty_like(LU)
        gB = torch.empty_like(w.G0)

        def call():
            rs.check(rs.call(f"rocsolver_{w.prec}getrs_adjoint_strided_batched", h, n, nrhs, P(LU), n,
                             n * n, P(ipiv), n, P(w.X0), n, n * nrhs, P(w.G0), n, n * nrhs,
                             P(gA), n, n * n, P(gB), n, n * nrhs, bc), "adjoint")

        def restore():
            pass

        run = call
        launches = 1
    for _ in range(warmup):
        restore()
        run()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    time.sleep(0.3)
    for i in range(steps):
        restore()
        ev[i][0].record(stream)
        run()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in ev)
    total_ms = max_over_ranks(torch, pg, total_ms, dev)
    ms = total_ms / steps
    peaks = ctx.peaks
    gbs = w.bytes_total / (ms / 1e3) / 1e9
    # accuracy and the comparison arm
    if w.name == "vbatched_4096":
        restore()
        run()
        torch.cuda.synchronize()
        sz, kk = w.sizes.cpu().numpy(), w.rhs.cpu().numpy()
        A0, B0, X = w.A0.cpu().numpy(), w.B0.cpu().numpy(), B.cpu().numpy()
        worst = 0.0
        for b in range(0, bc, 16):  # every 16th member, host check
            nb, kb = int(sz[b]), int(kk[b])
            Ab = A0[b][:nb, :nb].T  # A0[b][j][i] holds a_ij (column-major, lda = nmax)
            xb = X[b][:kb, :nb].T
            bb = B0[b][:kb, :nb].T
            r = np.abs(Ab @ xb - bb).max() / (np.abs(Ab).sum(1).max() * np.abs(xb).max()
                                               + np.abs(bb).max())
            worst = max(worst, r)
        extra["accuracy"] = {"backward_err_max_sampled": worst,
                             "info_nonzero": int((info.cpu().numpy() != 0).sum())}
        # per-size launches: dgetrf_batched + dgetrs_batched per distinct n (nrhs = the
        # largest nrhs among that size's members; the others solve spare columns)
        groups = {}
        for b in range(bc):
            groups.setdefault(int(sz[b]), []).append(b)
        plans = []
        for nb, mem in sorted(groups.items()):
            idx = torch.tensor(mem, device=dev, dtype=torch.int64)
            # pointer-array batches take ONE pivot array with stride strideP = n
            plans.append((nb, int(kk[mem].max()), pa[idx].contiguous(), pb[idx].contiguous(),
                          torch.zeros(len(mem) * nb, dtype=torch.int32, device=dev), len(mem)))

        def per_size():
            for nb, kmax, qa, qb, qp, cnt in plans:
                rs.check(rs.call("rocsolver_dgetrf_batched", h, nb, nb, P(qa), nmax, P(qp), nb,
                                 P(info), cnt), "getrf_batched")
                rs.check(rs.call("rocsolver_dgetrs_batched", h, rs.OP_N, nb, kmax, P(qa), nmax,
                                 P(qp), nb, P(qb), nmax, cnt), "getrs_batched")

        restore()
        per_size()
        torch.cuda.synchronize()
        pev = []
        for _ in range(3):
            restore()
            a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            per_size()
            b2.record(stream)
            pev.append((a, b2))
        torch.cuda.synchronize()
        pms = statistics.median([a.elapsed_time(b2) for a, b2 in pev])
        extra["per_size_launches"] = {"value": bc / (pms / 1e3), "unit": w.unit, "ms": pms,
                                      "launches": 2 * len(plans)}
        # e2e: A and B from pinned host memory, solutions and info back, every step
        hA, hB = w.A0.cpu().pin_memory(), w.B0.cpu().pin_memory()
        hX, hI = torch.empty_like(hB).pin_memory(), torch.empty(bc, dtype=torch.int32).pin_memory()

        def e2e_step():
            A.copy_(hA, non_blocking=True)
            B.copy_(hB, non_blocking=True)
            run()
            hX.copy_(B, non_blocking=True)
            hI.copy_(info, non_blocking=True)
        h2d, d2h = (hA.numel() + hB.numel()) * 8, hX.numel() * 8 + bc * 4
        e2e_pipeline = "one graph replay of the whole batch on one stream"
    else:
        n, nrhs = w.n, w.nrhs
        call()
        torch.cuda.synchronize()
        # gB against A^{-T} G and gA against -gB X' computed with torch (FP64)
        Gt = w.G0.double().transpose(1, 2)
        gBt = gB.double().transpose(1, 2)
        Aw = w.A0.double().transpose(1, 2)  # the matrix as factored (rounded for FP32)
        res = torch.bmm(Aw.transpose(1, 2), gBt) - Gt
        rel_b = float((res.abs().amax((1, 2)) / (Aw.abs().sum(1).amax(1)
                                                 * gBt.abs().amax((1, 2)))).max())
        gA_ref = -torch.bmm(gBt, w.X0.double())
        rel_a = float(((gA.double().transpose(1, 2) - gA_ref).abs().amax((1, 2))
                       / gA_ref.abs().amax((1, 2))).max())
        extra["accuracy"] = {"gB_backward_err_max": rel_b, "gA_rel_err_max": rel_a}
        hLU, hP = LU.cpu().pin_memory(), ipiv.cpu().pin_memory()
        hX, hG = w.X0.cpu().pin_memory(), w.G0.cpu().pin_memory()
        hgA, hgB = torch.empty_like(hLU).pin_memory(), torch.empty_like(hG).pin_memory()
        dLU, dP = torch.empty_like(LU), torch.empty_like(ipiv)
        dX, dG = torch.empty_like(w.X0), torch.empty_like(w.G0)

        es = LU.element_size()
        h2d = (hLU.numel() + hX.numel() + hG.numel()) * es + hP.numel() * 4
        d2h = (hgA.numel() + hgB.numel()) * es

        def body(hs, c0, c1):
            sl_ = slice(c0, c1)
            dLU[sl_].copy_(hLU[sl_], non_blocking=True)
            dP.view(bc, n)[sl_].copy_(hP.view(bc, n)[sl_], non_blocking=True)
            dX[sl_].copy_(hX[sl_], non_blocking=True)
            dG[sl_].copy_(hG[sl_], non_blocking=True)
            rs.check(rs.call(f"rocsolver_{w.prec}getrs_adjoint_strided_batched", hs, n, nrhs,
                             P(dLU[sl_]), n, n * n, P(dP.view(bc, n)[sl_]), n, P(dX[sl_]), n,
                             n * nrhs, P(dG[sl_]), n, n * nrhs, P(gA[sl_]), n, n * n,
                             P(gB[sl_]), n, n * nrhs, c1 - c0), "adjoint")
            hgA[sl_].copy_(gA[sl_], non_blocking=True)
            hgB[sl_].copy_(gB[sl_], non_blocking=True)
        sliced = SlicedStep(torch, rs, bc, h2d + d2h, body)
        extra_handles += sliced.handles
        e2e_step = sliced.step
        e2e_pipeline = sliced.desc
    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k = max(3, min(steps, 5))
    a.record(stream)
    for _ in range(k):
        e2e_step()
    b2.record(stream)
    torch.cuda.synchronize()
    e2e_ms = a.elapsed_time(b2) / k
    e2e_ms = max_over_ranks(torch, pg, e2e_ms, dev)
    line = {"metric": w.metric, "value": bc * world / (ms / 1e3), "unit": w.unit,
            "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": getattr(w, "dtype", "f64"),
            "data": "synthetic (seeded, generated on device)", "config": w.config,
            "gpu_launches": launches * steps,
            "e2e": {"value": bc * world / (e2e_ms / 1e3), "unit": w.unit,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "pipeline": e2e_pipeline},
            "roofline": {"bound": "hbm", "limiter": "latency: per-column chains of the CTA LU",
                         "kernel": "vb_persistent_kernel<double>"
                         if w.name == "vbatched_4096" else
                         f"solve_adjoint_kernel<{'float' if w.prec == 's' else 'double'}>",
                         "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": gbs / peaks["hbm_gbs"],
                         "traffic": w.traffic_per_unit * bc,
                         "peak_source": peaks["source"],
                         "compute": {"achieved_tflops": w.flops_total / (ms / 1e3) / 1e12,
                                     "peak_tflops": peaks["fp64_tflops"],
                                     "frac": w.flops_total / (ms / 1e3) / 1e12
                                     / peaks["fp64_tflops"],
                                     "peak": "FP64 dgemm measured in this run (cuBLAS 8192^3); "
                                             "the FP32 adjoint is also compared with it"}},
            "clocks": clocks}
    line.update(extra)
    if rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_sample(w, cpu_seconds)
    del graph
    torch.cuda.synchronize()
    for hh in extra_handles:
        hh.close()
    del w
    return line


if __name__ == "__main__":
    main()
