"""Generate the golden LAPACK fixtures that pin the oracle.

The reference keeps no golden vectors: its tests run host LAPACK at test time
(clients/common/lapack_host_reference.cpp:5052-5392).  Reference-LAPACK 3.9.1
(install.sh:182) is not installed here; the LAPACK that is, is OpenBLAS as
bundled with scipy (scipy.linalg.lapack).  This script runs it on

  * the reference's own test inputs (mt19937(69069) integers 1..10, +400 on the
    diagonal and -4 off it, rows reversed, zeroed columns in the "singular"
    members; clients/include/testing_getf2_getrf.hpp:128-180,
    testing_getrs.hpp:125-160, testing_potf2_potrf.hpp:103-140,
    testing_gesv.hpp:138-180) over the sizes of the reference's check-in
    suites (clients/gtest/getf2_getrf_gtest.cpp:24-56, getrs_gtest.cpp,
    potf2_potrf_gtest.cpp, potrs_gtest.cpp, gesv_gtest.cpp, posv_gtest.cpp);
  * uniform[-1,1] matrices at the sizes of the benchmarked configurations
    (scaled down in batch), and edge sizes n = 1, 2, 31, 33, 63, 65;
  * getri on the reference's getri inputs (testing_getri.hpp:102-166: the host
    getrf factors of a scaled, row-reversed integer matrix, with zeroed U
    diagonal entries in the singular members) over its check-in sizes
    (clients/gtest/getri_gtest.cpp:24-37): the factors and pivots given to
    getri, and the inverse and info LAPACK dgetri returns;
  * large members at the benchmarked orders (uniform n = 256 and 512, and the
    mixed-precision configuration's cond-graded matrices at n = 256): ipiv and
    info in full, the factors as projections (LU V, W^T LU for seeded Gaussian
    V, W; tests/refcases.py projections) so the fixture stays small, and an
    nrhs = 4 solve at n = 256;

and stores the LAPACK outputs in lapack_golden.npz (the inputs are regenerated
from the same seeded generators in tests/refcases.py).

The complex precisions go to lapack_golden_complex.npz: LAPACK zgetrf / zgetrs (N, T, C) /
zpotrf / zpotrs / zgesv (and the c routines on a subset) on the reference's complex test
inputs (each element two draws of the integer stream, real part first) at a subset of the
same suite sizes, on complex uniform matrices and on Hermitian positive definite Gram
matrices.  Run it with
``python tests/golden/make_golden.py`` from the repository root.
"""
import os
import sys

import numpy as np
import scipy.linalg.lapack as la

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tests.refcases import (ref_getrf_input, ref_getrs_input, ref_potrf_input,  # noqa: E402
                            ref_gesv_input, uniform_general, spd_gram, cond_graded,
                            projections, ref_getri_matrix, ref_getri_singular,
                            uniform_complex, hpd_gram)

BC = 3  # batched variants of the reference suites use batch_count = 3


def lapack_getrf(A):
    lu, piv, info = la.dgetrf(A, overwrite_a=0)
    return lu, (piv + 1).astype(np.int32), int(info)


def lapack_potrf(A, lower):
    c, info = la.dpotrf(A, lower=int(lower), clean=0, overwrite_a=0)
    return c, int(info)


def main():
    out = {}
    cases = []

    # ---- getrf: reference suite sizes (m x n), lda = m, regular + singular
    for m in (32, 50, 70):
        for n in (16, 20, 40, 100):
            for singular in (False, True):
                A = ref_getrf_input(m, n, m, BC, singular)
                key = f"getrf_ref_m{m}_n{n}_s{int(singular)}"
                lus, pivs, infos = [], [], []
                for b in range(BC):
                    lu, piv, info = lapack_getrf(A[b])
                    lus.append(lu); pivs.append(piv); infos.append(info)
                out[key + "_LU"] = np.stack(lus)
                out[key + "_ipiv"] = np.stack(pivs)
                out[key + "_info"] = np.array(infos, np.int32)
                cases.append(key)

    # ---- getrf: uniform[-1,1], square and edge sizes
    for n in (1, 2, 5, 31, 32, 33, 63, 64, 65, 100, 128):
        A = uniform_general(n, n, 4, seed=100 + n)
        key = f"getrf_uni_n{n}"
        lus, pivs, infos = [], [], []
        for b in range(A.shape[0]):
            lu, piv, info = lapack_getrf(A[b])
            lus.append(lu); pivs.append(piv); infos.append(info)
        out[key + "_LU"] = np.stack(lus)
        out[key + "_ipiv"] = np.stack(pivs)
        out[key + "_info"] = np.array(infos, np.int32)
        cases.append(key)

    # ---- getrs: reference suite (n x nrhs, trans N/T)
    for n in (20, 30, 50):
        for nrhs in (10, 20, 30):
            A, B = ref_getrs_input(n, nrhs, BC)
            for trans in (0, 1):
                key = f"getrs_ref_n{n}_r{nrhs}_t{trans}"
                lus, pivs, xs = [], [], []
                for b in range(BC):
                    lu, piv, info = lapack_getrf(A[b])
                    x, info2 = la.dgetrs(lu, piv - 1, B[b], trans=trans)
                    assert info2 == 0
                    lus.append(lu); pivs.append(piv); xs.append(x)
                out[key + "_LU"] = np.stack(lus)
                out[key + "_ipiv"] = np.stack(pivs)
                out[key + "_X"] = np.stack(xs)
                cases.append(key)

    # ---- potrf: reference suite (n in 10,20,50,70), uplo L/U, regular + singular
    for n in (10, 20, 50, 70):
        for lower in (True, False):
            for singular in (False, True):
                A = ref_potrf_input(n, BC, singular)
                key = f"potrf_ref_n{n}_L{int(lower)}_s{int(singular)}"
                cs, infos = [], []
                for b in range(BC):
                    c, info = lapack_potrf(A[b], lower)
                    cs.append(c); infos.append(info)
                out[key + "_C"] = np.stack(cs)
                out[key + "_info"] = np.array(infos, np.int32)
                cases.append(key)

    # ---- potrf / potrs on SPD Gram matrices (configuration shape n=64, nrhs=4)
    for n in (1, 2, 31, 33, 64, 65):
        A = spd_gram(n, 4, seed=200 + n)
        rng = np.random.default_rng(300 + n)
        B = rng.standard_normal((4, n, 4))
        for lower in (True, False):
            key = f"potrs_spd_n{n}_L{int(lower)}"
            cs, xs, infos = [], [], []
            for b in range(4):
                c, info = lapack_potrf(A[b], lower)
                x, info2 = la.dpotrs(c, B[b], lower=int(lower))
                cs.append(c); xs.append(x); infos.append(info)
            out[key + "_C"] = np.stack(cs)
            out[key + "_info"] = np.array(infos, np.int32)
            out[key + "_X"] = np.stack(xs)
            cases.append(key)

    # ---- gesv: reference suite (n, nrhs), regular + singular
    for n in (20, 35, 50):
        for nrhs in (1, 10):
            for singular in (False, True):
                A, B = ref_gesv_input(n, nrhs, BC, singular)
                key = f"gesv_ref_n{n}_r{nrhs}_s{int(singular)}"
                lus, pivs, xs, infos = [], [], [], []
                for b in range(BC):
                    lu, piv, x, info = la.dgesv(A[b], B[b])
                    if info != 0:  # LAPACK leaves B untouched on failure
                        x = B[b].copy()
                    lus.append(lu); pivs.append((piv + 1).astype(np.int32)); xs.append(x)
                    infos.append(int(info))
                out[key + "_ipiv"] = np.stack(pivs)
                out[key + "_X"] = np.stack(xs)
                out[key + "_info"] = np.array(infos, np.int32)
                cases.append(key)

    # ---- getri: reference suite (n, singular) with lda = n
    for n, singular in ((32, False), (50, True), (70, False), (100, True)):
        A = ref_getri_matrix(n, n, BC)
        lus, pivs, invs, infos = [], [], [], []
        for b in range(BC):
            lu, piv, info = lapack_getrf(A[b])
            assert info == 0
            if singular:
                for i in ref_getri_singular(b, BC, n):
                    lu[i, i] = 0.0
            inv, info2 = la.dgetri(lu, piv - 1)
            lus.append(lu); pivs.append(piv); infos.append(int(info2))
            invs.append(inv if info2 == 0 else lu)
        key = f"getri_ref_n{n}_s{int(singular)}"
        out[key + "_LU"] = np.stack(lus)
        out[key + "_ipiv"] = np.stack(pivs)
        out[key + "_inv"] = np.stack(invs)
        out[key + "_info"] = np.array(infos, np.int32)
        cases.append(key)

    # ---- large members: ipiv / info in full, factors as projections
    big = [("bigrf_uni_n256", uniform_general(256, 256, 2, seed=1256)),
           ("bigrf_uni_n512", uniform_general(512, 512, 1, seed=1512)),
           ("bigrf_cond_n256", cond_graded(256, 3, seed=2256))]
    for key, A in big:
        pivs, infos, ps, qs = [], [], [], []
        for b in range(A.shape[0]):
            lu, piv, info = lapack_getrf(A[b])
            p, q, _, _ = projections(lu)
            pivs.append(piv); infos.append(info); ps.append(p); qs.append(q)
        out[key + "_ipiv"] = np.stack(pivs)
        out[key + "_info"] = np.array(infos, np.int32)
        out[key + "_P"] = np.stack(ps)
        out[key + "_Q"] = np.stack(qs)
        cases.append(key)
    A = uniform_general(256, 256, 2, seed=1256)
    B = np.random.default_rng(1257).uniform(-1, 1, (2, 256, 4))
    xs = []
    for b in range(2):
        lu, piv, info = lapack_getrf(A[b])
        x, info2 = la.dgetrs(lu, piv - 1, B[b])
        assert info2 == 0
        xs.append(x)
    out["bigrs_uni_n256_r4_X"] = np.stack(xs)
    cases.append("bigrs_uni_n256_r4")

    out["cases"] = np.array(cases)
    path = os.path.join(HERE, "lapack_golden.npz")
    np.savez_compressed(path, **out)
    print(path, len(cases), "cases", os.path.getsize(path) // 1024, "KiB")


def main_complex():
    out = {}
    cases = []
    for P, cdt in (("z", np.complex128), ("c", np.complex64)):
        getrf, getrs = getattr(la, P + "getrf"), getattr(la, P + "getrs")
        potrf, potrs, gesv = getattr(la, P + "potrf"), getattr(la, P + "potrs"), getattr(la, P + "gesv")
        full = P == "z"

        def lu_of(A):
            lu, piv, info = getrf(A.astype(cdt), overwrite_a=0)
            return lu, (piv + 1).astype(np.int32), int(info)

        def put(key, **arrs):
            for k, v in arrs.items():
                out[key + "_" + k] = v
            cases.append(key)

        for m, n in (((32, 16), (50, 40), (70, 100)) if full else ((50, 40),)):
            for singular in (False, True):
                A = ref_getrf_input(m, n, m, BC, singular, cplx=True)
                r = [lu_of(A[b]) for b in range(BC)]
                put(f"{P}getrf_ref_m{m}_n{n}_s{int(singular)}", LU=np.stack([x[0] for x in r]),
                    ipiv=np.stack([x[1] for x in r]), info=np.array([x[2] for x in r], np.int32))
        for n in ((1, 2, 31, 33, 65) if full else (33, 65)):
            A = uniform_complex(n, n, 4, seed=400 + n)
            r = [lu_of(A[b]) for b in range(4)]
            put(f"{P}getrf_uni_n{n}", LU=np.stack([x[0] for x in r]),
                ipiv=np.stack([x[1] for x in r]), info=np.array([x[2] for x in r], np.int32))
        for n, nrhs in (((20, 10), (50, 30)) if full else ((20, 10),)):
            A, B = ref_getrs_input(n, nrhs, BC, cplx=True)
            r = [lu_of(A[b]) for b in range(BC)]
            out[f"{P}getrs_ref_n{n}_r{nrhs}_LU"] = np.stack([x[0] for x in r])
            out[f"{P}getrs_ref_n{n}_r{nrhs}_ipiv"] = np.stack([x[1] for x in r])
            for trans in (0, 1, 2):
                xs = []
                for b in range(BC):
                    x, info2 = getrs(r[b][0], r[b][1] - 1, B[b].astype(cdt), trans=trans)
                    assert info2 == 0
                    xs.append(x)
                put(f"{P}getrs_ref_n{n}_r{nrhs}_t{trans}", X=np.stack(xs))
        for n in ((10, 50) if full else (10,)):
            for lower in (True, False):
                for singular in (False, True):
                    A = ref_potrf_input(n, BC, singular, cplx=True)
                    cs, infos = [], []
                    for b in range(BC):
                        c, info = potrf(A[b].astype(cdt), lower=int(lower), clean=0, overwrite_a=0)
                        cs.append(c); infos.append(int(info))
                    put(f"{P}potrf_ref_n{n}_L{int(lower)}_s{int(singular)}", C=np.stack(cs),
                        info=np.array(infos, np.int32))
        for n in ((1, 33, 64) if full else (33,)):
            A = hpd_gram(n, 4, seed=500 + n)
            B = uniform_complex(n, 3, 4, seed=600 + n)
            for lower in (True, False):
                cs, xs, infos = [], [], []
                for b in range(4):
                    c, info = potrf(A[b].astype(cdt), lower=int(lower), clean=0, overwrite_a=0)
                    x, info2 = potrs(c, B[b].astype(cdt), lower=int(lower))
                    cs.append(c); xs.append(x); infos.append(int(info))
                put(f"{P}potrs_hpd_n{n}_L{int(lower)}", C=np.stack(cs), X=np.stack(xs),
                    info=np.array(infos, np.int32))
        for n, nrhs in (((20, 1), (50, 10)) if full else ((20, 1),)):
            for singular in (False, True):
                A, B = ref_gesv_input(n, nrhs, BC, singular, cplx=True)
                pivs, xs, infos = [], [], []
                for b in range(BC):
                    lu, piv, x, info = gesv(A[b].astype(cdt), B[b].astype(cdt))
                    if info != 0:
                        x = B[b].astype(cdt)
                    pivs.append((piv + 1).astype(np.int32)); xs.append(x); infos.append(int(info))
                put(f"{P}gesv_ref_n{n}_r{nrhs}_s{int(singular)}", ipiv=np.stack(pivs),
                    X=np.stack(xs), info=np.array(infos, np.int32))
    # getri (zgetri / cgetri) on the reference's getri inputs, zeroed U diagonal entries in
    # the singular members
    for P, cdt, sizes in (("z", np.complex128, ((32, False), (50, True))),
                          ("c", np.complex64, ((32, False),))):
        getrf, getri = getattr(la, P + "getrf"), getattr(la, P + "getri")
        for n, singular in sizes:
            A = ref_getri_matrix(n, n, BC, cplx=True).astype(cdt)
            lus, pivs, invs, infos = [], [], [], []
            for b in range(BC):
                lu, piv, info = getrf(A[b], overwrite_a=0)
                assert info == 0
                if singular:
                    for i in ref_getri_singular(b, BC, n):
                        lu[i, i] = 0.0
                inv, info2 = getri(lu, piv)
                lus.append(lu); pivs.append((piv + 1).astype(np.int32)); infos.append(int(info2))
                invs.append(inv if info2 == 0 else lu)
            key = f"{P}getri_ref_n{n}_s{int(singular)}"
            out[key + "_LU"] = np.stack(lus)
            out[key + "_ipiv"] = np.stack(pivs)
            out[key + "_inv"] = np.stack(invs)
            out[key + "_info"] = np.array(infos, np.int32)
            cases.append(key)
    out["cases"] = np.array(cases)
    path = os.path.join(HERE, "lapack_golden_complex.npz")
    np.savez_compressed(path, **out)
    print(path, len(cases), "cases", os.path.getsize(path) // 1024, "KiB")


if __name__ == "__main__":
    if "--complex-only" not in sys.argv:
        main()
    main_complex()
