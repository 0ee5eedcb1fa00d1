"""Run one library entry point on seeded synthetic data, a few times.

    python -m rocsolver_b200.demo --case getrf --n 256 --batch 512 [--dtype d] [--reps 3]

Cases: getrf, getrs, gesv, potrf, potrs, getri (in place, from factors computed once before
the timing), dsgesv, adjoint, vbatched, sgetrf_tf32 (the FP32 LU with split-TF32 trailing
updates; its kernel configuration, the tcgen05 engine included, follows the tuning table,
e.g. one named by $ROCSOLVER_B200_TUNING).  --dtype c / z runs the complex precisions of
getrf, getrs, gesv, potrf and potrs.  Used to drive
profilers (one small, fixed workload per kernel) and as a usage example of the C ABI from
Python.  Prints the median device time per call.
"""
import argparse
import statistics

import torch

import rocsolver_b200 as rs


def cond_matrices(torch, n, bc, g, dev, lo, hi):
    """A = U diag(s) V' (U, V from QR of Gaussians), s log-spaced from 1 to 1/kappa,
    log10(kappa) uniform in [lo, hi] per member."""
    A = torch.empty(bc, n, n, dtype=torch.float64, device=dev)
    t = torch.linspace(0, 1, n, device=dev, dtype=torch.float64)[None, :]
    for c0 in range(0, bc, 256):
        m = min(bc, c0 + 256) - c0
        U, _ = torch.linalg.qr(torch.randn(m, n, n, generator=g, device=dev, dtype=torch.float64))
        V, _ = torch.linalg.qr(torch.randn(m, n, n, generator=g, device=dev, dtype=torch.float64))
        lk = lo + (hi - lo) * torch.rand(m, 1, generator=g, device=dev, dtype=torch.float64)
        A[c0:c0 + m] = (U * torch.pow(10.0, -lk * t)[:, None, :]) @ V.transpose(1, 2)
    return A


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", required=True,
                    choices=["getrf", "getrs", "gesv", "potrf", "potrs", "dsgesv", "adjoint",
                             "vbatched", "sgetrf_tf32", "getri"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--dtype", default="d", choices=["s", "d", "c", "z"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--cond", type=float, default=0.0,
                    help="dsgesv: A = U diag(s) V' with log10(cond) uniform in [1, COND]")
    a = ap.parse_args()
    if a.case == "sgetrf_tf32":
        a.dtype = "s"
    dt = {"d": torch.float64, "s": torch.float32, "z": torch.complex128,
          "c": torch.complex64}[a.dtype]
    rdt = torch.float64 if a.dtype in "dz" else torch.float32
    dev = torch.device("cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    n, bc, nrhs = a.n, a.batch, a.nrhs
    def rnd(*shape):
        x = torch.rand(*shape, generator=g, device=dev, dtype=rdt) * 2 - 1
        if dt.is_complex:
            x = torch.complex(x, torch.rand(*shape, generator=g, device=dev, dtype=rdt) * 2 - 1)
        return x

    A0 = rnd(bc, n, n)
    if a.case in ("potrf", "potrs"):
        A0 = A0 @ A0.conj().transpose(1, 2) + n * torch.eye(n, device=dev, dtype=dt)
    elif a.case == "dsgesv" and a.cond > 0:
        A0 = cond_matrices(torch, n, bc, g, dev, 1.0, a.cond)
    elif a.case in ("dsgesv", "adjoint", "getri"):
        A0 = A0 + 4 * torch.eye(n, device=dev, dtype=dt)
    A0 = A0.transpose(1, 2).contiguous()
    B0 = rnd(bc, nrhs, n).contiguous()
    A, B = A0.clone(), B0.clone()
    X = torch.empty_like(B)
    gA = torch.empty_like(A)
    ipiv = torch.zeros(bc * n, dtype=torch.int32, device=dev)
    info = torch.zeros(bc, dtype=torch.int32, device=dev)
    it = torch.zeros(bc, dtype=torch.int32, device=dev)
    p = a.dtype
    h = rs.Handle(torch.cuda.current_stream().cuda_stream)
    P = rs.ptr
    if a.case in ("getrs", "adjoint", "getri"):
        rs.check(rs.call(f"rocsolver_{p}getrf_strided_batched", h.value, n, n, P(A), n, n * n,
                         P(ipiv), n, P(info), bc), "getrf")
        A0 = A.clone()
    if a.case == "potrs":
        rs.check(rs.call(f"rocsolver_{p}potrf_strided_batched", h.value, rs.FILL_LOWER, n, P(A),
                         n, n * n, P(info), bc), "potrf")
        A0 = A.clone()
    vb = None
    if a.case == "vbatched":
        sizes = torch.randint(8, n + 1, (bc,), generator=g, device=dev, dtype=torch.int32)
        rhs = torch.randint(1, max(nrhs, 1) + 1, (bc,), generator=g, device=dev,
                            dtype=torch.int32)
        ld = torch.full((bc,), n, dtype=torch.int32, device=dev)
        es = A.element_size()
        pa = torch.arange(bc, device=dev, dtype=torch.int64) * (n * n * es) + A.data_ptr()
        pb = torch.arange(bc, device=dev, dtype=torch.int64) * (n * nrhs * es) + B.data_ptr()
        pp = torch.arange(bc, device=dev, dtype=torch.int64) * (n * 4) + ipiv.data_ptr()
        vb = (sizes, rhs, ld, pa, pb, pp)

    def call():
        if a.case == "getrf":
            st = rs.call(f"rocsolver_{p}getrf_strided_batched", h.value, n, n, P(A), n, n * n,
                         P(ipiv), n, P(info), bc)
        elif a.case == "sgetrf_tf32":
            st = rs.call("rocsolver_sgetrf_tf32_strided_batched", h.value, n, n, P(A), n, n * n,
                         P(ipiv), n, P(info), bc)
        elif a.case == "getrs":
            st = rs.call(f"rocsolver_{p}getrs_strided_batched", h.value, rs.OP_N, n, nrhs, P(A),
                         n, n * n, P(ipiv), n, P(B), n, n * nrhs, bc)
        elif a.case == "gesv":
            st = rs.call(f"rocsolver_{p}gesv_strided_batched", h.value, n, nrhs, P(A), n, n * n,
                         P(ipiv), n, P(B), n, n * nrhs, P(info), bc)
        elif a.case == "potrf":
            st = rs.call(f"rocsolver_{p}potrf_strided_batched", h.value, rs.FILL_LOWER, n, P(A),
                         n, n * n, P(info), bc)
        elif a.case == "potrs":
            st = rs.call(f"rocsolver_{p}potrs_strided_batched", h.value, rs.FILL_LOWER, n, nrhs,
                         P(A), n, n * n, P(B), n, n * nrhs, bc)
        elif a.case == "getri":
            st = rs.call(f"rocsolver_{p}getri_strided_batched", h.value, n, P(A), n, n * n,
                         P(ipiv), n, P(info), bc)
        elif a.case == "dsgesv":
            st = rs.call("rocsolver_dsgesv_strided_batched", h.value, n, nrhs, P(A), n, n * n,
                         P(ipiv), n, P(B), n, n * nrhs, P(X), n, n * nrhs, P(it), P(info), bc)
        elif a.case == "adjoint":
            st = rs.call(f"rocsolver_{p}getrs_adjoint_strided_batched", h.value, n, nrhs, P(A), n,
                         n * n, P(ipiv), n, P(B), n, n * nrhs, P(B0), n, n * nrhs, P(gA), n,
                         n * n, P(X), n, n * nrhs, bc)
        else:
            sizes, rhs, ld, pa, pb, pp = vb
            st = rs.call(f"rocsolver_{p}gesv_vbatched", h.value, P(sizes), P(rhs), P(pa), P(ld),
                         P(pp), P(pb), P(ld), P(info), n, nrhs, bc)
        rs.check(st, a.case)

    times = []
    for _ in range(a.reps):
        A.copy_(A0)
        B.copy_(B0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        call()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    h.close()
    print(f"{a.case} {a.dtype} n={n} batch={bc} nrhs={nrhs}: median {statistics.median(times):.4f} ms"
          f" over {a.reps} calls; info nonzero {int((info != 0).sum())}")
    if a.case == "dsgesv":
        vals, cnt = torch.unique(it, return_counts=True)
        print("iter histogram:", dict(zip(vals.tolist(), cnt.tolist())))


if __name__ == "__main__":
    main()
