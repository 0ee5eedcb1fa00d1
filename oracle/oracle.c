/* oracle.c -- CPU restatement of the batched LU / Cholesky factor-and-solve
 * path.  TEST INFRASTRUCTURE ONLY: this file is the checker that the CUDA
 * library is compared against (and the timed CPU baseline); it is never linked
 * into, or called by, the product library.
 *
 * The reference (rocSOLVER 3.23) checks its GPU results against host LAPACK
 * (clients/common/lapack_host_reference.cpp:5052-5392 -> dgetrf_, dgetrs_,
 * dpotrf_, dpotrs_, dgesv_, dposv_).  This file restates the unblocked LAPACK
 * algorithms those routines reduce to, with the same pivot rule, the same
 * scaling rule and the same info conventions:
 *   getf2  : LAPACK dgetf2 == rocSOLVER getf2 (library/src/lapack/roclapack_getf2.hpp:42-99
 *            check_singularity, :133-156 iamax; specialized/roclapack_getf2_specialized_kernels.hpp:83-124)
 *   getrs  : library/src/lapack/roclapack_getrs.hpp:117-150 (laswp, L, U / U', L', laswp back)
 *   laswp  : library/src/auxiliary/rocauxiliary_laswp.hpp:18-64,195-216
 *   potf2  : LAPACK dpotf2 == library/src/lapack/roclapack_potf2.hpp:16-43 (first non-positive
 *            minor gives info), :218-248 (lower), :185-216 (upper)
 *   potrs  : library/src/lapack/roclapack_potrs.hpp:87-152
 *   gesv/posv : library/src/lapack/roclapack_gesv.hpp:105-178, roclapack_posv.hpp:101-170
 *               (B is left unchanged where info > 0)
 *   getri  : LAPACK dgetri / dtrti2 (unblocked), the reference's cpu_getri
 *            (clients/common/lapack_host_reference.cpp; library/src/lapack/roclapack_getri.hpp:265-390
 *            computes the same inverse by blocks)
 * Pinned against scipy's bundled OpenBLAS LAPACK by tests/golden/make_golden.py.
 *
 * Every routine exists for float (prefix s) and double (prefix d); batch
 * drivers split the batch statically across pthreads.
 */
#include <math.h>
#include <float.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

/* ---------------------------------------------------------------------- */
#define DEFINE_ORACLE(P, T, SFMIN, SQRT)                                                    \
    /* first index of max |x| (LAPACK idamax: strict '>' so the first max wins and a NaN   \
       never replaces the running maximum).  Returns 0-based offset. */                     \
    static int P##_iamax(int n, const T* x)                                                 \
    {                                                                                       \
        int best = 0;                                                                       \
        T bv = (T)fabs((double)x[0]);                                                       \
        for(int i = 1; i < n; ++i)                                                          \
        {                                                                                   \
            T v = (T)fabs((double)x[i]);                                                    \
            if(v > bv)                                                                      \
            {                                                                               \
                bv = v;                                                                     \
                best = i;                                                                   \
            }                                                                               \
        }                                                                                   \
        return best;                                                                        \
    }                                                                                       \
                                                                                            \
    /* unblocked LU with (pivot=1) or without (pivot=0) partial pivoting, LAPACK dgetf2.    \
       ipiv 1-based, info = first exactly-zero pivot (1-based) or 0. */                     \
    void oracle_##P##getf2(int m, int n, T* A, int lda, int* ipiv, int* info, int pivot)    \
    {                                                                                       \
        *info = 0;                                                                          \
        int mn = m < n ? m : n;                                                             \
        for(int j = 0; j < mn; ++j)                                                         \
        {                                                                                   \
            int jp = j;                                                                     \
            if(pivot)                                                                       \
            {                                                                               \
                jp = j + P##_iamax(m - j, &A[IDX(j, j, lda)]);                              \
                ipiv[j] = jp + 1;                                                           \
            }                                                                               \
            T piv = A[IDX(jp, j, lda)];                                                     \
            if(piv != (T)0)                                                                 \
            {                                                                               \
                if(jp != j)                                                                 \
                    for(int c = 0; c < n; ++c)                                              \
                    {                                                                       \
                        T t = A[IDX(j, c, lda)];                                            \
                        A[IDX(j, c, lda)] = A[IDX(jp, c, lda)];                             \
                        A[IDX(jp, c, lda)] = t;                                             \
                    }                                                                       \
                if((T)fabs((double)piv) >= SFMIN)                                           \
                {                                                                           \
                    T r = (T)1 / piv;                                                       \
                    for(int i = j + 1; i < m; ++i)                                          \
                        A[IDX(i, j, lda)] *= r;                                             \
                }                                                                           \
                else                                                                        \
                {                                                                           \
                    for(int i = j + 1; i < m; ++i)                                          \
                        A[IDX(i, j, lda)] /= piv;                                           \
                }                                                                           \
            }                                                                               \
            else if(*info == 0)                                                             \
                *info = j + 1;                                                              \
            for(int c = j + 1; c < n; ++c)                                                  \
            {                                                                               \
                T u = A[IDX(j, c, lda)];                                                    \
                if(u != (T)0)                                                               \
                    for(int i = j + 1; i < m; ++i)                                          \
                        A[IDX(i, c, lda)] -= A[IDX(i, j, lda)] * u;                         \
            }                                                                               \
        }                                                                                   \
    }                                                                                       \
                                                                                            \
    /* row interchanges on the nrhs columns of B, forward (inc>0) or backward (inc<0). */   \
    void oracle_##P##laswp(int n, int nrhs, T* B, int ldb, const int* ipiv, int inc)        \
    {                                                                                       \
        for(int c = 0; c < nrhs; ++c)                                                       \
        {                                                                                   \
            for(int s = 0; s < n; ++s)                                                      \
            {                                                                               \
                int k = inc > 0 ? s : n - 1 - s;                                            \
                int p = ipiv[k] - 1;                                                        \
                if(p != k)                                                                  \
                {                                                                           \
                    T t = B[IDX(k, c, ldb)];                                                \
                    B[IDX(k, c, ldb)] = B[IDX(p, c, ldb)];                                  \
                    B[IDX(p, c, ldb)] = t;                                                  \
                }                                                                           \
            }                                                                               \
        }                                                                                   \
    }                                                                                       \
                                                                                            \
    /* triangular solves in the column-oriented form of reference BLAS dtrsm (side=L). */   \
    static void P##_trsm_lower_n(int n, int nrhs, const T* A, int lda, T* B, int ldb,       \
                                 int unit)                                                  \
    {                                                                                       \
        for(int c = 0; c < nrhs; ++c)                                                       \
            for(int k = 0; k < n; ++k)                                                      \
            {                                                                               \
                T* b = &B[IDX(0, c, ldb)];                                                  \
                if(b[k] != (T)0)                                                            \
                {                                                                           \
                    if(!unit)                                                               \
                        b[k] /= A[IDX(k, k, lda)];                                          \
                    for(int i = k + 1; i < n; ++i)                                          \
                        b[i] -= b[k] * A[IDX(i, k, lda)];                                   \
                }                                                                           \
            }                                                                               \
    }                                                                                       \
    static void P##_trsm_upper_n(int n, int nrhs, const T* A, int lda, T* B, int ldb,       \
                                 int unit)                                                  \
    {                                                                                       \
        for(int c = 0; c < nrhs; ++c)                                                       \
            for(int k = n - 1; k >= 0; --k)                                                 \
            {                                                                               \
                T* b = &B[IDX(0, c, ldb)];                                                  \
                if(b[k] != (T)0)                                                            \
                {                                                                           \
                    if(!unit)                                                               \
                        b[k] /= A[IDX(k, k, lda)];                                          \
                    for(int i = 0; i < k; ++i)                                              \
                        b[i] -= b[k] * A[IDX(i, k, lda)];                                   \
                }                                                                           \
            }                                                                               \
    }                                                                                       \
    /* op(A) = A^T with A upper: forward substitution over rows */                          \
    static void P##_trsm_upper_t(int n, int nrhs, const T* A, int lda, T* B, int ldb,       \
                                 int unit)                                                  \
    {                                                                                       \
        for(int c = 0; c < nrhs; ++c)                                                       \
            for(int i = 0; i < n; ++i)                                                      \
            {                                                                               \
                T* b = &B[IDX(0, c, ldb)];                                                  \
                T t = b[i];                                                                 \
                for(int k = 0; k < i; ++k)                                                  \
                    t -= A[IDX(k, i, lda)] * b[k];                                          \
                if(!unit)                                                                   \
                    t /= A[IDX(i, i, lda)];                                                 \
                b[i] = t;                                                                   \
            }                                                                               \
    }                                                                                       \
    /* op(A) = A^T with A lower: backward substitution over rows */                         \
    static void P##_trsm_lower_t(int n, int nrhs, const T* A, int lda, T* B, int ldb,       \
                                 int unit)                                                  \
    {                                                                                       \
        for(int c = 0; c < nrhs; ++c)                                                       \
            for(int i = n - 1; i >= 0; --i)                                                 \
            {                                                                               \
                T* b = &B[IDX(0, c, ldb)];                                                  \
                T t = b[i];                                                                 \
                for(int k = i + 1; k < n; ++k)                                              \
                    t -= A[IDX(k, i, lda)] * b[k];                                          \
                if(!unit)                                                                   \
                    t /= A[IDX(i, i, lda)];                                                 \
                b[i] = t;                                                                   \
            }                                                                               \
    }                                                                                       \
                                                                                            \
    /* trans: 0 = none, 1 = transpose (conjugate transpose is the same for real T) */       \
    void oracle_##P##getrs(int trans, int n, int nrhs, const T* A, int lda, const int* ipiv,\
                           T* B, int ldb)                                                   \
    {                                                                                       \
        if(n == 0 || nrhs == 0)                                                             \
            return;                                                                         \
        if(!trans)                                                                          \
        {                                                                                   \
            if(ipiv)                                                                        \
                oracle_##P##laswp(n, nrhs, B, ldb, ipiv, 1);                                \
            P##_trsm_lower_n(n, nrhs, A, lda, B, ldb, 1);                                   \
            P##_trsm_upper_n(n, nrhs, A, lda, B, ldb, 0);                                   \
        }                                                                                   \
        else                                                                                \
        {                                                                                   \
            P##_trsm_upper_t(n, nrhs, A, lda, B, ldb, 0);                                   \
            P##_trsm_lower_t(n, nrhs, A, lda, B, ldb, 1);                                   \
            if(ipiv)                                                                        \
                oracle_##P##laswp(n, nrhs, B, ldb, ipiv, -1);                               \
        }                                                                                   \
    }                                                                                       \
                                                                                            \
    /* unblocked Cholesky, LAPACK dpotf2; upper=1 computes U^T U, else L L^T.  On the      \
       first non-positive (or NaN) pivot the value is stored, info = j+1, and the routine   \
       returns, as LAPACK does. */                                                          \
    void oracle_##P##potf2(int upper, int n, T* A, int lda, int* info)                      \
    {                                                                                       \
        *info = 0;                                                                          \
        for(int j = 0; j < n; ++j)                                                          \
        {                                                                                   \
            T dot = (T)0; /* DDOT, accumulated then subtracted */                           \
            for(int k = 0; k < j; ++k)                                                      \
            {                                                                               \
                T v = upper ? A[IDX(k, j, lda)] : A[IDX(j, k, lda)];                        \
                dot += v * v;                                                               \
            }                                                                               \
            T ajj = A[IDX(j, j, lda)] - dot;                                                \
            if(ajj <= (T)0 || ajj != ajj)                                                   \
            {                                                                               \
                A[IDX(j, j, lda)] = ajj;                                                    \
                *info = j + 1;                                                              \
                return;                                                                     \
            }                                                                               \
            ajj = SQRT(ajj);                                                                \
            A[IDX(j, j, lda)] = ajj;                                                        \
            T r = (T)1 / ajj;                                                               \
            for(int i = j + 1; i < n; ++i)                                                  \
            {                                                                               \
                T s;                                                                        \
                if(upper)                                                                   \
                { /* DGEMV('T'): dot accumulated, then subtracted */                        \
                    T t = (T)0;                                                             \
                    for(int k = 0; k < j; ++k)                                              \
                        t += A[IDX(k, i, lda)] * A[IDX(k, j, lda)];                         \
                    s = A[IDX(j, i, lda)] - t;                                              \
                }                                                                           \
                else                                                                        \
                { /* DGEMV('N'): column-by-column axpy */                                   \
                    s = A[IDX(i, j, lda)];                                                  \
                    for(int k = 0; k < j; ++k)                                              \
                        s -= A[IDX(i, k, lda)] * A[IDX(j, k, lda)];                         \
                }                                                                           \
                if(upper)                                                                   \
                    A[IDX(j, i, lda)] = s * r;                                              \
                else                                                                        \
                    A[IDX(i, j, lda)] = s * r;                                              \
            }                                                                               \
        }                                                                                   \
    }                                                                                       \
                                                                                            \
    void oracle_##P##potrs(int upper, int n, int nrhs, const T* A, int lda, T* B, int ldb)  \
    {                                                                                       \
        if(n == 0 || nrhs == 0)                                                             \
            return;                                                                         \
        if(upper)                                                                           \
        {                                                                                   \
            P##_trsm_upper_t(n, nrhs, A, lda, B, ldb, 0);                                   \
            P##_trsm_upper_n(n, nrhs, A, lda, B, ldb, 0);                                   \
        }                                                                                   \
        else                                                                                \
        {                                                                                   \
            P##_trsm_lower_n(n, nrhs, A, lda, B, ldb, 0);                                   \
            P##_trsm_lower_t(n, nrhs, A, lda, B, ldb, 0);                                   \
        }                                                                                   \
    }                                                                                       \
                                                                                            \
    void oracle_##P##gesv(int n, int nrhs, T* A, int lda, int* ipiv, T* B, int ldb,         \
                          int* info)                                                        \
    {                                                                                       \
        oracle_##P##getf2(n, n, A, lda, ipiv, info, 1);                                     \
        if(*info == 0)                                                                      \
            oracle_##P##getrs(0, n, nrhs, A, lda, ipiv, B, ldb);                            \
    }                                                                                       \
                                                                                            \
    void oracle_##P##posv(int upper, int n, int nrhs, T* A, int lda, T* B, int ldb,         \
                          int* info)                                                        \
    {                                                                                       \
        oracle_##P##potf2(upper, n, A, lda, info);                                          \
        if(*info == 0)                                                                      \
            oracle_##P##potrs(upper, n, nrhs, A, lda, B, ldb);                              \
    }                                                                                       \
                                                                                            \
    /* inverse from the LU factors, LAPACK dgetri unblocked (the reference's oracle,       \
       clients/common/lapack_host_reference.cpp cpu_getri): dtrtri's singularity test      \
       (info = first zero U(i,i); A untouched), inv(U) by dtrti2 (dtrmv + dscal per         \
       column), then inv(A) L = inv(U) column by column from the right (dgemv), then the    \
       column interchanges in reverse order.  pivot = 0: no interchanges (npvt).            \
       work: n elements. */                                                                 \
    void oracle_##P##getri(int n, T* A, int lda, const int* ipiv, int* info, T* work,       \
                           int pivot)                                                       \
    {                                                                                       \
        *info = 0;                                                                          \
        for(int i = 0; i < n; ++i)                                                          \
            if(A[IDX(i, i, lda)] == (T)0)                                                   \
            {                                                                               \
                *info = i + 1;                                                              \
                return;                                                                     \
            }                                                                               \
        for(int j = 0; j < n; ++j)                                                          \
        {                                                                                   \
            A[IDX(j, j, lda)] = (T)1 / A[IDX(j, j, lda)];                                   \
            T ajj = -A[IDX(j, j, lda)];                                                     \
            /* x = U(0:j,0:j) x for x = A(0:j, j) (dtrmv, upper, no transpose) */           \
            for(int jj = 0; jj < j; ++jj)                                                   \
            {                                                                               \
                T t = A[IDX(jj, j, lda)];                                                   \
                if(t != (T)0)                                                               \
                {                                                                           \
                    for(int i = 0; i < jj; ++i)                                             \
                        A[IDX(i, j, lda)] += t * A[IDX(i, jj, lda)];                        \
                    A[IDX(jj, j, lda)] = t * A[IDX(jj, jj, lda)];                           \
                }                                                                           \
            }                                                                               \
            for(int i = 0; i < j; ++i)                                                      \
                A[IDX(i, j, lda)] *= ajj;                                                   \
        }                                                                                   \
        for(int j = n - 1; j >= 0; --j)                                                     \
        {                                                                                   \
            for(int i = j + 1; i < n; ++i)                                                  \
            {                                                                               \
                work[i] = A[IDX(i, j, lda)];                                                \
                A[IDX(i, j, lda)] = (T)0;                                                   \
            }                                                                               \
            for(int jj = j + 1; jj < n; ++jj)                                               \
            {                                                                               \
                T t = -work[jj];                                                            \
                if(t != (T)0)                                                               \
                    for(int i = 0; i < n; ++i)                                              \
                        A[IDX(i, j, lda)] += t * A[IDX(i, jj, lda)];                        \
            }                                                                               \
        }                                                                                   \
        if(pivot)                                                                           \
            for(int j = n - 2; j >= 0; --j)                                                 \
            {                                                                               \
                int jp = ipiv[j] - 1;                                                       \
                if(jp != j)                                                                 \
                    for(int i = 0; i < n; ++i)                                              \
                    {                                                                       \
                        T t = A[IDX(i, j, lda)];                                            \
                        A[IDX(i, j, lda)] = A[IDX(i, jp, lda)];                             \
                        A[IDX(i, jp, lda)] = t;                                             \
                    }                                                                       \
            }                                                                               \
    }

DEFINE_ORACLE(d, double, DBL_MIN, sqrt)
DEFINE_ORACLE(s, float, FLT_MIN, sqrtf)

/* ---------------------------------------------------------------------- */
/* Batch drivers: member b of a strided batch starts at X + b*strideX.  The
 * batch is split statically over nthreads pthreads (one LAPACK-style call per
 * member, as the reference's host-LAPACK test path, testing_getf2_getrf.hpp:290-296,
 * does). */
typedef struct
{
    int op; /* 0 getrf, 1 getrs, 2 potrf, 3 potrs, 4 gesv, 5 posv, 6 getri */
    int dbl;
    int m, n, nrhs, trans, upper, pivot;
    void* A;
    int lda;
    int64_t sA;
    int* ipiv;
    int64_t sP;
    void* B;
    int ldb;
    int64_t sB;
    int* info;
    int b0, b1;
} job_t;

static void run_one(const job_t* j, int b)
{
    size_t es = j->dbl ? sizeof(double) : sizeof(float);
    char* A = (char*)j->A + (size_t)b * (size_t)j->sA * es;
    char* B = j->B ? (char*)j->B + (size_t)b * (size_t)j->sB * es : NULL;
    int* ipiv = j->ipiv ? j->ipiv + (size_t)b * (size_t)j->sP : NULL;
    int* info = j->info ? j->info + b : NULL;
    int dummy = 0;
    if(!info)
        info = &dummy;
    switch(j->op)
    {
    case 0:
        if(j->dbl)
            oracle_dgetf2(j->m, j->n, (double*)A, j->lda, ipiv, info, j->pivot);
        else
            oracle_sgetf2(j->m, j->n, (float*)A, j->lda, ipiv, info, j->pivot);
        break;
    case 1:
        if(j->dbl)
            oracle_dgetrs(j->trans, j->n, j->nrhs, (double*)A, j->lda, ipiv, (double*)B, j->ldb);
        else
            oracle_sgetrs(j->trans, j->n, j->nrhs, (float*)A, j->lda, ipiv, (float*)B, j->ldb);
        break;
    case 2:
        if(j->dbl)
            oracle_dpotf2(j->upper, j->n, (double*)A, j->lda, info);
        else
            oracle_spotf2(j->upper, j->n, (float*)A, j->lda, info);
        break;
    case 3:
        if(j->dbl)
            oracle_dpotrs(j->upper, j->n, j->nrhs, (double*)A, j->lda, (double*)B, j->ldb);
        else
            oracle_spotrs(j->upper, j->n, j->nrhs, (float*)A, j->lda, (float*)B, j->ldb);
        break;
    case 4:
        if(j->dbl)
            oracle_dgesv(j->n, j->nrhs, (double*)A, j->lda, ipiv, (double*)B, j->ldb, info);
        else
            oracle_sgesv(j->n, j->nrhs, (float*)A, j->lda, ipiv, (float*)B, j->ldb, info);
        break;
    case 5:
        if(j->dbl)
            oracle_dposv(j->upper, j->n, j->nrhs, (double*)A, j->lda, (double*)B, j->ldb, info);
        else
            oracle_sposv(j->upper, j->n, j->nrhs, (float*)A, j->lda, (float*)B, j->ldb, info);
        break;
    case 6:
    {
        void* w = malloc(es * (size_t)(j->n > 0 ? j->n : 1));
        if(j->dbl)
            oracle_dgetri(j->n, (double*)A, j->lda, ipiv, info, (double*)w, j->pivot);
        else
            oracle_sgetri(j->n, (float*)A, j->lda, ipiv, info, (float*)w, j->pivot);
        free(w);
        break;
    }
    }
}

static void* worker(void* arg)
{
    const job_t* j = (const job_t*)arg;
    for(int b = j->b0; b < j->b1; ++b)
        run_one(j, b);
    return NULL;
}

/* Generic batch entry point used by the Python test harness (ctypes) and the
 * CPU baseline.  nthreads <= 1 runs serially on the calling thread. */
void oracle_batch(int op, int dbl, int m, int n, int nrhs, int trans, int upper, int pivot,
                  void* A, int lda, int64_t sA, int* ipiv, int64_t sP, void* B, int ldb,
                  int64_t sB, int* info, int bc, int nthreads)
{
    job_t base = {op, dbl, m, n, nrhs, trans, upper, pivot, A, lda, sA, ipiv, sP, B, ldb, sB,
                  info, 0, bc};
    if(nthreads <= 1 || bc <= 1)
    {
        worker(&base);
        return;
    }
    if(nthreads > bc)
        nthreads = bc;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
    job_t* jobs = (job_t*)malloc(sizeof(job_t) * (size_t)nthreads);
    for(int t = 0; t < nthreads; ++t)
    {
        jobs[t] = base;
        jobs[t].b0 = (int)((int64_t)bc * t / nthreads);
        jobs[t].b1 = (int)((int64_t)bc * (t + 1) / nthreads);
        pthread_create(&th[t], NULL, worker, &jobs[t]);
    }
    for(int t = 0; t < nthreads; ++t)
        pthread_join(th[t], NULL);
    free(th);
    free(jobs);
}
