/* oracle_complex.c -- CPU restatement of the complex (c/z) LU / Cholesky factor-and-solve
 * path.  TEST INFRASTRUCTURE ONLY: the checker the CUDA library is compared against; never
 * linked into the product library.
 *
 * Same routines and conventions as oracle.c for the complex types the reference
 * instantiates (library/src/lapack/roclapack_getf2.hpp, roclapack_getrs.hpp:117-150,
 * roclapack_potf2.hpp:16-75,185-248, roclapack_potrs.hpp:87-152; its clients check them
 * against host LAPACK zgetrf/zgetrs/zpotrf/zpotrs, clients/common/lapack_host_reference.cpp):
 *   zgetf2 : pivot = first index of the largest |re| + |im| (LAPACK izamax / dcabs1, strict
 *            '>' so a NaN never wins unless it is the first candidate); scaling by the
 *            reciprocal when |pivot| >= sfmin (modulus), else by division; info = first
 *            exactly-zero pivot
 *   zgetrs : trans 0 = N (laswp, L unit, U), 1 = T, 2 = C (conjugate transpose: U^H, L^H,
 *            laswp backwards)
 *   zpotf2 : A = L L^H (lower) or U^H U (upper); ajj = real(a_jj) - sum |l_jk|^2; info = first
 *            j with ajj <= 0 or NaN (a_jj set to ajj, then stop)
 *   zpotrs : lower L Y = B, L^H X = Y; upper U^H Y = B, U X = Y
 *   gesv / posv: B left unchanged where info > 0
 *   zgetri : inverse from the LU factors (ztrti2 + unblocked zgetri, as oracle.c's dgetri)
 * Pinned against scipy's bundled OpenBLAS LAPACK by tests/golden/make_golden.py.
 * Arrays are interleaved (re, im) pairs, column-major, member b at A + b*strideA elements.
 */
#include <complex.h>
#include <float.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>

#define IDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

#define DEFINE_CORACLE(P, R, C, SFMIN, SQRT, FABS, CABS)                                     \
    static R P##_cabs1(C z) { return FABS(creal##P(z)) + FABS(cimag##P(z)); }               \
    static void P##_getf2(int m, int n, C* A, int lda, int* ipiv, int* info, int pivot)      \
    {                                                                                        \
        *info = 0;                                                                           \
        int mn = m < n ? m : n;                                                              \
        for(int j = 0; j < mn; ++j)                                                          \
        {                                                                                    \
            int jp = j;                                                                      \
            if(pivot)                                                                        \
            {                                                                                \
                R bv = P##_cabs1(A[IDX(j, j, lda)]);                                         \
                for(int i = j + 1; i < m; ++i)                                               \
                {                                                                            \
                    R v = P##_cabs1(A[IDX(i, j, lda)]);                                      \
                    if(v > bv)                                                               \
                    {                                                                        \
                        bv = v;                                                              \
                        jp = i;                                                              \
                    }                                                                        \
                }                                                                            \
                ipiv[j] = jp + 1;                                                            \
            }                                                                                \
            C piv = A[IDX(jp, j, lda)];                                                      \
            if(piv != (C)0)                                                                  \
            {                                                                                \
                if(jp != j)                                                                  \
                    for(int c = 0; c < n; ++c)                                               \
                    {                                                                        \
                        C t = A[IDX(j, c, lda)];                                             \
                        A[IDX(j, c, lda)] = A[IDX(jp, c, lda)];                              \
                        A[IDX(jp, c, lda)] = t;                                              \
                    }                                                                        \
                if(CABS(piv) >= SFMIN)                                                       \
                {                                                                            \
                    C r = (C)1 / piv;                                                        \
                    for(int i = j + 1; i < m; ++i)                                           \
                        A[IDX(i, j, lda)] *= r;                                              \
                }                                                                            \
                else                                                                         \
                    for(int i = j + 1; i < m; ++i)                                           \
                        A[IDX(i, j, lda)] /= piv;                                            \
            }                                                                                \
            else if(*info == 0)                                                              \
                *info = j + 1;                                                               \
            for(int c = j + 1; c < n; ++c)                                                   \
            {                                                                                \
                C u = A[IDX(j, c, lda)];                                                     \
                if(u != (C)0)                                                                \
                    for(int i = j + 1; i < m; ++i)                                           \
                        A[IDX(i, c, lda)] -= A[IDX(i, j, lda)] * u;                          \
            }                                                                                \
        }                                                                                    \
    }                                                                                        \
    static void P##_laswp(int n, int nrhs, C* B, int ldb, const int* ipiv, int fwd)          \
    {                                                                                        \
        for(int c = 0; c < nrhs; ++c)                                                        \
            for(int s = 0; s < n; ++s)                                                       \
            {                                                                                \
                int k = fwd ? s : n - 1 - s;                                                 \
                int p = ipiv[k] - 1;                                                         \
                if(p != k)                                                                   \
                {                                                                            \
                    C t = B[IDX(k, c, ldb)];                                                 \
                    B[IDX(k, c, ldb)] = B[IDX(p, c, ldb)];                                   \
                    B[IDX(p, c, ldb)] = t;                                                   \
                }                                                                            \
            }                                                                                \
    }                                                                                        \
    /* op(M) = M (cj = 0) or conj(M) (cj = 1) entries; lower/upper, (un)transposed */       \
    static C P##_e(const C* A, int lda, int i, int j, int cj)                                \
    {                                                                                        \
        C v = A[IDX(i, j, lda)];                                                             \
        return cj ? conj##P(v) : v;                                                          \
    }                                                                                        \
    /* solve op(T) x = b column by column: T lower (tl) or upper, op = transpose (tr) with  \
       conjugation (cj), unit diagonal (unit) */                                             \
    static void P##_trsv(int n, int nrhs, const C* A, int lda, C* B, int ldb, int tl,        \
                         int tr, int cj, int unit)                                           \
    {                                                                                        \
        /* effective lower-triangular solve when (tl && !tr) || (!tl && tr) */              \
        int lower = (tl && !tr) || (!tl && tr);                                              \
        for(int c = 0; c < nrhs; ++c)                                                        \
        {                                                                                    \
            C* b = &B[IDX(0, c, ldb)];                                                       \
            if(lower)                                                                        \
                for(int k = 0; k < n; ++k)                                                   \
                {                                                                            \
                    C s = b[k];                                                              \
                    for(int i = 0; i < k; ++i)                                               \
                        s -= (tr ? P##_e(A, lda, i, k, cj) : P##_e(A, lda, k, i, cj)) * b[i];\
                    b[k] = unit ? s : s / (tr ? P##_e(A, lda, k, k, cj) : P##_e(A, lda, k, k, cj)); \
                }                                                                            \
            else                                                                             \
                for(int k = n - 1; k >= 0; --k)                                              \
                {                                                                            \
                    C s = b[k];                                                              \
                    for(int i = k + 1; i < n; ++i)                                           \
                        s -= (tr ? P##_e(A, lda, i, k, cj) : P##_e(A, lda, k, i, cj)) * b[i];\
                    b[k] = unit ? s : s / P##_e(A, lda, k, k, cj);                           \
                }                                                                            \
        }                                                                                    \
    }                                                                                        \
    static void P##_getrs(int trans, int n, int nrhs, const C* A, int lda, const int* ipiv,  \
                          C* B, int ldb)                                                     \
    {                                                                                        \
        if(trans == 0)                                                                       \
        {                                                                                    \
            P##_laswp(n, nrhs, B, ldb, ipiv, 1);                                             \
            P##_trsv(n, nrhs, A, lda, B, ldb, 1, 0, 0, 1);                                   \
            P##_trsv(n, nrhs, A, lda, B, ldb, 0, 0, 0, 0);                                   \
        }                                                                                    \
        else                                                                                 \
        {                                                                                    \
            int cj = trans == 2;                                                             \
            P##_trsv(n, nrhs, A, lda, B, ldb, 0, 1, cj, 0);                                  \
            P##_trsv(n, nrhs, A, lda, B, ldb, 1, 1, cj, 1);                                  \
            P##_laswp(n, nrhs, B, ldb, ipiv, 0);                                             \
        }                                                                                    \
    }                                                                                        \
    static void P##_potf2(int upper, int n, C* A, int lda, int* info)                        \
    {                                                                                        \
        *info = 0;                                                                           \
        for(int j = 0; j < n; ++j)                                                           \
        {                                                                                    \
            R ajj = creal##P(A[IDX(j, j, lda)]);                                             \
            for(int k = 0; k < j; ++k)                                                       \
            {                                                                                \
                C v = upper ? A[IDX(k, j, lda)] : A[IDX(j, k, lda)];                         \
                ajj -= creal##P(v) * creal##P(v) + cimag##P(v) * cimag##P(v);                \
            }                                                                                \
            if(ajj <= (R)0 || isnan(ajj))                                                    \
            {                                                                                \
                A[IDX(j, j, lda)] = ajj;                                                     \
                *info = j + 1;                                                               \
                return;                                                                      \
            }                                                                                \
            ajj = SQRT(ajj);                                                                 \
            A[IDX(j, j, lda)] = ajj;                                                         \
            for(int i = j + 1; i < n; ++i)                                                   \
            {                                                                                \
                C s = upper ? A[IDX(j, i, lda)] : A[IDX(i, j, lda)];                         \
                for(int k = 0; k < j; ++k)                                                   \
                    s -= upper ? conj##P(A[IDX(k, j, lda)]) * A[IDX(k, i, lda)]              \
                               : A[IDX(i, k, lda)] * conj##P(A[IDX(j, k, lda)]);             \
                s *= (R)1 / ajj;                                                             \
                if(upper)                                                                    \
                    A[IDX(j, i, lda)] = s;                                                   \
                else                                                                         \
                    A[IDX(i, j, lda)] = s;                                                   \
            }                                                                                \
        }                                                                                    \
    }                                                                                        \
    static void P##_potrs(int upper, int n, int nrhs, const C* A, int lda, C* B, int ldb)    \
    {                                                                                        \
        if(upper)                                                                            \
        {                                                                                    \
            P##_trsv(n, nrhs, A, lda, B, ldb, 0, 1, 1, 0);                                   \
            P##_trsv(n, nrhs, A, lda, B, ldb, 0, 0, 0, 0);                                   \
        }                                                                                    \
        else                                                                                 \
        {                                                                                    \
            P##_trsv(n, nrhs, A, lda, B, ldb, 1, 0, 0, 0);                                   \
            P##_trsv(n, nrhs, A, lda, B, ldb, 1, 1, 1, 0);                                   \
        }                                                                                    \
    }                                                                                        \
    /* inverse from the LU factors (LAPACK zgetri unblocked, as oracle.c's dgetri): info =  \
       first zero U(i,i) with A untouched; inv(U) by ztrti2; X L = inv(U) from the right;    \
       column interchanges in reverse order (none when pivot = 0) */                          \
    static void P##_getri(int n, C* A, int lda, const int* ipiv, int* info, int pivot)       \
    {                                                                                        \
        *info = 0;                                                                           \
        for(int i = 0; i < n; ++i)                                                           \
            if(A[IDX(i, i, lda)] == (C)0)                                                    \
            {                                                                                \
                *info = i + 1;                                                               \
                return;                                                                      \
            }                                                                                \
        for(int j = 0; j < n; ++j)                                                           \
        {                                                                                    \
            A[IDX(j, j, lda)] = (C)1 / A[IDX(j, j, lda)];                                    \
            C ajj = -A[IDX(j, j, lda)];                                                      \
            for(int jj = 0; jj < j; ++jj)                                                    \
            {                                                                                \
                C t = A[IDX(jj, j, lda)];                                                    \
                if(t != (C)0)                                                                \
                {                                                                            \
                    for(int i = 0; i < jj; ++i)                                              \
                        A[IDX(i, j, lda)] += t * A[IDX(i, jj, lda)];                         \
                    A[IDX(jj, j, lda)] = t * A[IDX(jj, jj, lda)];                            \
                }                                                                            \
            }                                                                                \
            for(int i = 0; i < j; ++i)                                                       \
                A[IDX(i, j, lda)] *= ajj;                                                    \
        }                                                                                    \
        C* work = (C*)malloc(sizeof(C) * (size_t)(n > 0 ? n : 1));                           \
        for(int j = n - 1; j >= 0; --j)                                                      \
        {                                                                                    \
            for(int i = j + 1; i < n; ++i)                                                   \
            {                                                                                \
                work[i] = A[IDX(i, j, lda)];                                                 \
                A[IDX(i, j, lda)] = (C)0;                                                    \
            }                                                                                \
            for(int jj = j + 1; jj < n; ++jj)                                                \
            {                                                                                \
                C t = -work[jj];                                                             \
                if(t != (C)0)                                                                \
                    for(int i = 0; i < n; ++i)                                               \
                        A[IDX(i, j, lda)] += t * A[IDX(i, jj, lda)];                         \
            }                                                                                \
        }                                                                                    \
        free(work);                                                                          \
        if(pivot)                                                                            \
            for(int j = n - 2; j >= 0; --j)                                                  \
            {                                                                                \
                int jp = ipiv[j] - 1;                                                        \
                if(jp != j)                                                                  \
                    for(int i = 0; i < n; ++i)                                               \
                    {                                                                        \
                        C t = A[IDX(i, j, lda)];                                             \
                        A[IDX(i, j, lda)] = A[IDX(i, jp, lda)];                              \
                        A[IDX(i, jp, lda)] = t;                                              \
                    }                                                                        \
            }                                                                                \
    }                                                                                        \
    /* batch driver: op 0 getrf, 1 getrs, 2 potrf, 3 potrs, 4 gesv, 5 posv, 6 getri */       \
    void oracle_##P##batch(int op, int m, int n, int nrhs, int trans, int upper, int pivot,  \
                           C* A, int lda, int64_t sA, int* ipiv, int64_t sP, C* B, int ldb,  \
                           int64_t sB, int* info, int bc)                                    \
    {                                                                                        \
        for(int b = 0; b < bc; ++b)                                                          \
        {                                                                                    \
            C* a = A + (size_t)b * sA;                                                       \
            int* p = ipiv ? ipiv + (size_t)b * sP : 0;                                       \
            C* x = B ? B + (size_t)b * sB : 0;                                               \
            int dummy = 0;                                                                   \
            int* inf = info ? info + b : &dummy;                                             \
            switch(op)                                                                       \
            {                                                                                \
            case 0: P##_getf2(m, n, a, lda, p, inf, pivot); break;                           \
            case 1: P##_getrs(trans, n, nrhs, a, lda, p, x, ldb); break;                     \
            case 2: P##_potf2(upper, n, a, lda, inf); break;                                 \
            case 3: P##_potrs(upper, n, nrhs, a, lda, x, ldb); break;                        \
            case 4:                                                                          \
                P##_getf2(n, n, a, lda, p, inf, 1);                                          \
                if(*inf == 0)                                                                \
                    P##_getrs(0, n, nrhs, a, lda, p, x, ldb);                                \
                break;                                                                       \
            case 5:                                                                          \
                P##_potf2(upper, n, a, lda, inf);                                            \
                if(*inf == 0)                                                                \
                    P##_potrs(upper, n, nrhs, a, lda, x, ldb);                               \
                break;                                                                       \
            case 6: P##_getri(n, a, lda, p, inf, pivot); break;                              \
            }                                                                                \
        }                                                                                    \
    }

#define crealz creal
#define cimagz cimag
#define conjz conj
#define crealc crealf
#define cimagc cimagf
#define conjc conjf
DEFINE_CORACLE(z, double, double complex, DBL_MIN, sqrt, fabs, cabs)
DEFINE_CORACLE(c, float, float complex, FLT_MIN, sqrtf, fabsf, cabsf)
