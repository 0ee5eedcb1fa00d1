"""Autotuner for the CTA LU kernels and the persistent variable-size kernel.

    python -m rocsolver_b200.tune [--out PATH] [--quick] [--classes 64,128,256,...]

Replaces the reference's hand-set compile-time tables (library/src/include/ideal_sizes.hpp:
166-240, roclapack_getrf.hpp:17-166) with measurement on the GPU the library runs on.
For every size class and precision it times each compiled configuration that can take
the class's largest size -- (threads, rows per thread, panel width), trailing-update
column chunk, and whether the panel's row interchanges are folded into the trailing
update -- on seeded uniform[-1, 1] batches, and keeps the fastest.  For the variable-size
kernel it also tunes the number of resident CTAs per SM, on batches with n uniform in
[8, n_max] and nrhs uniform in [1, 16].  Precision t is the FP32 LU with split-TF32
trailing updates (rocsolver_sgetrf_tf32_strided_batched, the factorisation of dsgesv); its
candidates include the tcgen05 trailing update (fold = 2) for the variants compiled with it.

The table (format in include/rocsolver.h, rocsolver_b200_tuning_set) is written to
rocsolver_b200/tuning_b200.txt by default, where the library reads it when the first
handle is created.  Every candidate's pivots are compared with the built-in
configuration's on the same input; results do not depend on the table, only speed does.
"""
import argparse
import datetime
import os
import statistics

import torch

import rocsolver_b200 as rs

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "tuning_b200.txt")

# compiled CTA variants: (threads, rows per thread, panel width)
LU_VARIANTS = [(64, 1, 32), (128, 1, 32), (128, 2, 32), (128, 2, 16), (128, 4, 16),
               (256, 1, 32), (256, 2, 16), (256, 2, 32), (256, 4, 8), (256, 4, 16),
               (256, 8, 4), (256, 8, 8)]
VB_VARIANTS = [(256, 1, 32), (256, 2, 16), (256, 2, 32), (256, 4, 8), (256, 4, 16),
               (256, 8, 4)]
# variants compiled with the tcgen05 trailing update (precision t, fold = 2) and with the
# two-level LU (outer panels of 64 columns, K = 64 tcgen05 updates; fold = 3)
UM_VARIANTS = [(128, 1, 32), (128, 2, 32), (256, 1, 32), (256, 2, 32), (256, 2, 16),
               (256, 4, 16), (256, 4, 8), (256, 8, 8)]
LU2_VARIANTS = [(256, 2, 32), (256, 2, 16), (256, 4, 16), (256, 4, 8), (256, 8, 8)]
# batch per getrf size class (enough CTAs for several waves on 148 SMs)
GETRF_CLASSES = {64: 16384, 128: 8192, 256: 2048, 512: 592, 1024: 296, 2048: 148}
VB_CLASSES = {256: 4096, 512: 4096, 1024: 1024}


def _time(fn, reset, reps):
    ts = []
    for _ in range(reps + 1):
        reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts[1:])


def _lu_candidates(n, quick, prec="d"):
    out = []
    for nt, r, jb in LU_VARIANTS:
        if nt * r < n or nt * r >= 4 * n:
            continue  # too few rows for n, or mostly idle threads
        for cw in ((64, 128) if quick else (32, 64, 96, 128)):
            if cw > ((n + 31) // 32) * 32:
                continue
            folds = (0, 1)
            if prec == "t" and (nt, r, jb) in UM_VARIANTS:
                folds += (2,)
            if prec == "t" and (nt, r, jb) in LU2_VARIANTS and n >= 256:
                folds += (3,)
            for fold in folds:
                out.append((nt, r, jb, cw, fold))
    return out


def tune_getrf(prec, n, bc, reps, quick, log):
    dt = torch.float64 if prec == "d" else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(1000 + n)
    A0 = (torch.rand(bc, n, n, generator=g, device="cuda", dtype=dt) * 2 - 1).contiguous()
    A = torch.empty_like(A0)
    ipiv = torch.zeros(bc * n, dtype=torch.int32, device="cuda")
    info = torch.zeros(bc, dtype=torch.int32, device="cuda")
    h = rs.Handle(torch.cuda.current_stream().cuda_stream)
    fn_name = ("rocsolver_sgetrf_tf32_strided_batched" if prec == "t"
               else f"rocsolver_{prec}getrf_strided_batched")

    def call():
        st = rs.call(fn_name, h.value, n, n, rs.ptr(A), n, n * n, rs.ptr(ipiv), n,
                     rs.ptr(info), bc)
        rs.check(st, fn_name)

    def reset():
        A.copy_(A0)

    try:
        rs.set_tuning_table("")
        t_builtin = _time(call, reset, reps)
        piv_ref = ipiv.clone()
        best = None
        for cand in _lu_candidates(n, quick, prec):
            nt, r, jb, cw, fold = cand
            rs.set_tuning_table(f"getrf {prec} {n} {nt} {r} {jb} {cw} {fold}\n")
            t = _time(call, reset, reps)
            mism = int((ipiv != piv_ref).sum())
            bad = int((info != 0).sum()) + int((~torch.isfinite(A)).sum())
            log(f"  getrf {prec} n={n} bc={bc} {cand}: {t:.3f} ms  pivot mismatches {mism}"
                f"  bad {bad}")
            if bad == 0 and (best is None or t < best[0]):
                best = (t, cand)
        log(f"getrf {prec} n={n}: built-in {t_builtin:.3f} ms, best {best[1]} {best[0]:.3f} ms")
        return best[1], best[0], t_builtin
    finally:
        h.close()


def _vb_batch(prec, nmax, bc, seed):
    dt = torch.float64 if prec == "d" else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    sizes = torch.randint(8, nmax + 1, (bc,), generator=g, device="cuda", dtype=torch.int32)
    rhs = torch.randint(1, 17, (bc,), generator=g, device="cuda", dtype=torch.int32)
    A0 = torch.rand(bc, nmax, nmax, generator=g, device="cuda", dtype=dt) * 2 - 1
    A0 = A0 + 0.1 * sizes.to(dt)[:, None, None] * torch.eye(nmax, device="cuda", dtype=dt)
    B0 = torch.rand(bc, 16, nmax, generator=g, device="cuda", dtype=dt) * 2 - 1
    return sizes, rhs, A0.contiguous(), B0.contiguous()


def tune_vbatched(prec, nmax, bc, reps, quick, log):
    sizes, rhs, A0, B0 = _vb_batch(prec, nmax, bc, 2000 + nmax)
    A, B = torch.empty_like(A0), torch.empty_like(B0)
    es = A.element_size()
    ld = torch.full((bc,), nmax, dtype=torch.int32, device="cuda")
    ipiv = torch.zeros(bc * nmax, dtype=torch.int32, device="cuda")
    info = torch.zeros(bc, dtype=torch.int32, device="cuda")
    ar = torch.arange(bc, device="cuda", dtype=torch.int64)
    pa = ar * (nmax * nmax * es) + A.data_ptr()
    pb = ar * (16 * nmax * es) + B.data_ptr()
    pp = ar * (nmax * 4) + ipiv.data_ptr()
    h = rs.Handle(torch.cuda.current_stream().cuda_stream)
    fn_name = f"rocsolver_{prec}gesv_vbatched"
    P = rs.ptr

    def call():
        st = rs.call(fn_name, h.value, P(sizes), P(rhs), P(pa), P(ld), P(pp), P(pb), P(ld),
                     P(info), nmax, 16, bc)
        rs.check(st, fn_name)

    def reset():
        A.copy_(A0)
        B.copy_(B0)

    try:
        rs.set_tuning_table("")
        t_builtin = _time(call, reset, reps)
        piv_ref = ipiv.clone()
        best = None
        for nt, r, jb in VB_VARIANTS:
            if nt * r < nmax or nt * r >= 4 * nmax:
                continue
            for cw in ((0,) if quick else (32, 64, 128)):
                for fold in (0, 1):
                    for per_sm in (0, 1):
                        cand = (nt, r, jb, cw, fold, per_sm)
                        rs.set_tuning_table(f"vbatched {prec} {nmax} " +
                                            " ".join(map(str, cand)) + "\n")
                        t = _time(call, reset, reps)
                        mism = int((ipiv != piv_ref).sum())
                        bad = int((info != 0).sum())
                        log(f"  vbatched {prec} n_max={nmax} bc={bc} {cand}: {t:.3f} ms  "
                            f"pivot mismatches {mism}  bad {bad}")
                        if bad == 0 and (best is None or t < best[0]):
                            best = (t, cand)
        log(f"vbatched {prec} n_max={nmax}: built-in {t_builtin:.3f} ms, best {best[1]} "
            f"{best[0]:.3f} ms")
        return best[1], best[0], t_builtin
    finally:
        h.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--log", default=None, help="also append the measurements to this file")
    ap.add_argument("--classes", default=",".join(map(str, GETRF_CLASSES)))
    ap.add_argument("--vb-classes", default=",".join(map(str, VB_CLASSES)))
    ap.add_argument("--precisions", default="d,s,t")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--quick", action="store_true", help="fewer chunk widths")
    ap.add_argument("--merge", action="store_true",
                    help="keep the --out file's rows of the precisions not tuned now")
    a = ap.parse_args()
    logf = open(a.log, "a") if a.log else None

    def log(msg):
        print(msg, flush=True)
        if logf:
            logf.write(msg + "\n")
            logf.flush()

    old = rs.tuning_table()
    lines = [f"# written by python -m rocsolver_b200.tune on {torch.cuda.get_device_name()} "
             f"({datetime.date.today().isoformat()})",
             "# getrf    <s|d|t> <m_max> <threads> <rows/thread> <panel> <chunk> <fold>"
             "    # ms: tuned / built-in",
             "# vbatched <s|d> <n_max> <threads> <rows/thread> <panel> <chunk> <fold> "
             "<ctas/SM>"]
    try:
        for prec in a.precisions.split(","):
            for n in [int(x) for x in a.classes.split(",") if x]:
                cand, t, tb = tune_getrf(prec, n, GETRF_CLASSES.get(n, 256), a.reps, a.quick,
                                         log)
                lines.append(f"getrf {prec} {n} " + " ".join(map(str, cand))
                             + f"    # {t:.3f} / {tb:.3f} ms, batch {GETRF_CLASSES.get(n, 256)}")
            for n in [int(x) for x in a.vb_classes.split(",") if x and prec != "t"]:
                cand, t, tb = tune_vbatched(prec, n, VB_CLASSES.get(n, 1024), a.reps, a.quick,
                                            log)
                lines.append(f"vbatched {prec} {n} " + " ".join(map(str, cand))
                             + f"    # {t:.3f} / {tb:.3f} ms, batch {VB_CLASSES.get(n, 1024)}")
    finally:
        rs.set_tuning_table(old)
    if a.merge and os.path.exists(a.out):
        tuned = set(a.precisions.split(","))
        with open(a.out) as f:
            kept = [ln.rstrip("\n") for ln in f
                    if ln.split()[:1] in (["getrf"], ["vbatched"]) and ln.split()[1] not in tuned]
        lines = lines[:3] + kept + lines[3:]
    text = "\n".join(lines) + "\n"
    with open(a.out, "w") as f:
        f.write(text)
    log(f"wrote {a.out}")


if __name__ == "__main__":
    main()
