/* lapack_host.c -- host LAPACK over a batch: the timed CPU baseline.
 * TEST AND BENCH INFRASTRUCTURE ONLY: never linked into, or called by, the product library.
 *
 * The reference's CPU implementation of this path is host LAPACK: its clients time
 * cpu_getrf / cpu_getrs / cpu_potrf / cpu_potrs / cpu_gesv in a serial loop over the batch
 * (clients/include/testing_getf2_getrf.hpp:290-296, clients/common/lapack_host_reference.cpp
 * dgetrf_/dgetrs_/dpotrf_/dpotrs_/dgesv_).  Reference-LAPACK is not installed in this
 * image; the LAPACK that is, OpenBLAS as bundled with scipy (libscipy_openblas, symbols
 * prefixed scipy_), is loaded here with dlopen.  Each LAPACK call runs on one thread
 * (scipy_openblas_set_num_threads(1)) and the batch is split statically over nthreads
 * pthreads, one contiguous slice each; nthreads = 1 is the reference's serial loop.
 *
 * Operations (all FP64, column-major, member b of X at X + b*strideX):
 *   LH_GETRF_GETRS : dgetrf + dgetrs ('N') per member (B overwritten by X)
 *   LH_POTRF_POTRS : dpotrf + dpotrs ('L') per member
 *   LH_GESV        : dgesv per member
 *   LH_DSGESV      : dsgesv per member (LAPACK's mixed-precision iterative refinement;
 *                    A and B are not modified, X receives the solution, iter[] the ITER)
 *   LH_ADJOINT     : dgetrs ('T') on G in the B slot (gB = A^-T G, A holding LU factors
 *                    and ipiv); the outer product gA = -gB X^T is lapack_host_outer (dgemm)
 *   LH_GETRI       : dgetri per member (A holding LU factors and ipiv)
 *   LH_ZGESV       : zgesv per member (complex double, interleaved re/im: A, B, the strides
 *                    sA / sB counted in doubles, lda / ldb in complex elements)
 *   LH_VGESV       : dgesv per member with per-member order n[b] and nrhs[b] (members in
 *                    fixed slots of strideA / strideB elements, lda = ldb = ld)
 */
#include <dlfcn.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum
{
    LH_GETRF_GETRS = 0,
    LH_POTRF_POTRS = 1,
    LH_GESV = 2,
    LH_DSGESV = 3,
    LH_ADJOINT = 4,
    LH_GETRI = 5,
    LH_VGESV = 6,
    LH_ZGESV = 7
};

typedef void (*getrf_t)(const int*, const int*, double*, const int*, int*, int*);
typedef void (*getrs_t)(const char*, const int*, const int*, const double*, const int*,
                        const int*, double*, const int*, int*, size_t);
typedef void (*potrf_t)(const char*, const int*, double*, const int*, int*, size_t);
typedef void (*potrs_t)(const char*, const int*, const int*, const double*, const int*,
                        double*, const int*, int*, size_t);
typedef void (*gesv_t)(const int*, const int*, double*, const int*, int*, double*, const int*,
                       int*);
typedef void (*dsgesv_t)(const int*, const int*, double*, const int*, int*, double*,
                         const int*, double*, const int*, double*, float*, int*, int*);
typedef void (*getri_t)(const int*, double*, const int*, const int*, double*, const int*, int*);
typedef void (*gemm_t)(const char*, const char*, const int*, const int*, const int*,
                       const double*, const double*, const int*, const double*, const int*,
                       const double*, double*, const int*, size_t, size_t);
typedef void (*setnt_t)(int);

static struct
{
    void* h;
    getrf_t getrf;
    getrs_t getrs;
    potrf_t potrf;
    potrs_t potrs;
    gesv_t gesv;
    dsgesv_t dsgesv;
    getri_t getri;
    gemm_t gemm;
    setnt_t setnt;
    gesv_t zgesv; /* same argument list with complex (interleaved) arrays */
} L;

/* Load the LAPACK library at path (once).  Returns 0 on success, else the number of the
 * first symbol that was not found (1-based), or -1 if dlopen failed. */
int lapack_host_open(const char* path)
{
    if(L.h)
        return 0;
    void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if(!h)
        return -1;
    const char* names[] = {"scipy_dgetrf_", "scipy_dgetrs_", "scipy_dpotrf_", "scipy_dpotrs_",
                           "scipy_dgesv_",  "scipy_dsgesv_", "scipy_dgetri_", "scipy_dgemm_",
                           "scipy_openblas_set_num_threads", "scipy_zgesv_"};
    void* f[10];
    for(int i = 0; i < 10; ++i)
    {
        f[i] = dlsym(h, names[i]);
        if(!f[i])
        {
            dlclose(h);
            return i + 1;
        }
    }
    L.getrf = (getrf_t)f[0];
    L.getrs = (getrs_t)f[1];
    L.potrf = (potrf_t)f[2];
    L.potrs = (potrs_t)f[3];
    L.gesv = (gesv_t)f[4];
    L.dsgesv = (dsgesv_t)f[5];
    L.getri = (getri_t)f[6];
    L.gemm = (gemm_t)f[7];
    L.setnt = (setnt_t)f[8];
    L.zgesv = (gesv_t)f[9];
    L.setnt(1);
    L.h = h;
    return 0;
}

typedef struct
{
    int op, n, nrhs, ld;
    double* A;
    int lda;
    int64_t sA;
    int* ipiv;
    int64_t sP;
    double* B;
    int ldb;
    int64_t sB;
    double* X;
    int ldx;
    int64_t sX;
    int* info;
    int* iter;
    const int* nv;
    const int* rv;
    int b0, b1;
} Job;

static void* run_slice(void* arg)
{
    Job* j = (Job*)arg;
    const int n = j->n, nrhs = j->nrhs;
    double* work = NULL;
    float* swork = NULL;
    if(j->op == LH_DSGESV)
    {
        work = (double*)malloc(sizeof(double) * (size_t)n * nrhs);
        swork = (float*)malloc(sizeof(float) * (size_t)n * (n + nrhs));
    }
    if(j->op == LH_GETRI)
        work = (double*)malloc(sizeof(double) * (size_t)n * 64);
    const int lwork = n * 64;
    for(int b = j->b0; b < j->b1; ++b)
    {
        double* a = j->A + (int64_t)b * j->sA;
        int* p = j->ipiv ? j->ipiv + (int64_t)b * j->sP : NULL;
        double* bb = j->B ? j->B + (int64_t)b * j->sB : NULL;
        double* x = j->X ? j->X + (int64_t)b * j->sX : NULL;
        int inf = 0, it = 0;
        switch(j->op)
        {
        case LH_GETRF_GETRS:
            L.getrf(&n, &n, a, &j->lda, p, &inf);
            if(inf == 0)
            {
                int i2 = 0;
                L.getrs("N", &n, &nrhs, a, &j->lda, p, bb, &j->ldb, &i2, 1);
            }
            break;
        case LH_POTRF_POTRS:
            L.potrf("L", &n, a, &j->lda, &inf, 1);
            if(inf == 0)
            {
                int i2 = 0;
                L.potrs("L", &n, &nrhs, a, &j->lda, bb, &j->ldb, &i2, 1);
            }
            break;
        case LH_GESV: L.gesv(&n, &nrhs, a, &j->lda, p, bb, &j->ldb, &inf); break;
        case LH_ZGESV: L.zgesv(&n, &nrhs, a, &j->lda, p, bb, &j->ldb, &inf); break;
        case LH_DSGESV:
            L.dsgesv(&n, &nrhs, a, &j->lda, p, bb, &j->ldb, x, &j->ldx, work, swork, &it, &inf);
            if(j->iter)
                j->iter[b] = it;
            break;
        case LH_ADJOINT:
        {
            int i2 = 0; /* G in the B slot becomes gB = A^-T G */
            L.getrs("T", &n, &nrhs, a, &j->lda, p, bb, &j->ldb, &i2, 1);
            break;
        }
        case LH_GETRI: L.getri(&n, a, &j->lda, p, work, &lwork, &inf); break;
        case LH_VGESV:
        {
            const int nb = j->nv[b], rb = j->rv[b];
            L.gesv(&nb, &rb, a, &j->ld, p, bb, &j->ld, &inf);
            break;
        }
        default: break;
        }
        if(j->info)
            j->info[b] = inf;
    }
    free(work);
    free(swork);
    return NULL;
}

/* Run op over members 0..bc-1 on nthreads pthreads.  Returns 0, or -1 if the library is
 * not loaded. */
int lapack_host_batch(int op, int n, int nrhs, double* A, int lda, int64_t sA, int* ipiv,
                      int64_t sP, double* B, int ldb, int64_t sB, double* X, int ldx,
                      int64_t sX, int* info, int* iter, const int* nv, const int* rv, int ld,
                      int bc, int nthreads)
{
    if(!L.h)
        return -1;
    if(nthreads < 1)
        nthreads = 1;
    if(nthreads > bc)
        nthreads = bc > 0 ? bc : 1;
    Job* jobs = (Job*)calloc((size_t)nthreads, sizeof(Job));
    pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
    const int per = (bc + nthreads - 1) / nthreads;
    for(int t = 0; t < nthreads; ++t)
    {
        Job* j = &jobs[t];
        j->op = op;
        j->n = n;
        j->nrhs = nrhs;
        j->ld = ld;
        j->A = A;
        j->lda = lda;
        j->sA = sA;
        j->ipiv = ipiv;
        j->sP = sP;
        j->B = B;
        j->ldb = ldb;
        j->sB = sB;
        j->X = X;
        j->ldx = ldx;
        j->sX = sX;
        j->info = info;
        j->iter = iter;
        j->nv = nv;
        j->rv = rv;
        j->b0 = t * per < bc ? t * per : bc;
        j->b1 = (t + 1) * per < bc ? (t + 1) * per : bc;
    }
    for(int t = 1; t < nthreads; ++t)
        pthread_create(&th[t], NULL, run_slice, &jobs[t]);
    run_slice(&jobs[0]);
    for(int t = 1; t < nthreads; ++t)
        pthread_join(th[t], NULL);
    free(jobs);
    free(th);
    return 0;
}

/* gA = -gB X^T per member (the adjoint's outer product) with dgemm, members split over
 * nthreads pthreads: gB n x nrhs (ld n), X n x nrhs (ld n), gA n x n (ld n). */
typedef struct
{
    int n, nrhs;
    const double* gB;
    const double* X;
    double* gA;
    int b0, b1;
} OJob;

static void* run_outer(void* arg)
{
    OJob* j = (OJob*)arg;
    const double alpha = -1.0, beta = 0.0;
    const int n = j->n, k = j->nrhs;
    for(int b = j->b0; b < j->b1; ++b)
        L.gemm("N", "T", &n, &n, &k, &alpha, j->gB + (size_t)b * n * k, &n,
               j->X + (size_t)b * n * k, &n, &beta, j->gA + (size_t)b * n * n, &n, 1, 1);
    return NULL;
}

int lapack_host_outer(int n, int nrhs, const double* gB, const double* X, double* gA, int bc,
                      int nthreads)
{
    if(!L.h)
        return -1;
    if(nthreads < 1)
        nthreads = 1;
    if(nthreads > bc)
        nthreads = bc > 0 ? bc : 1;
    OJob* jobs = (OJob*)calloc((size_t)nthreads, sizeof(OJob));
    pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
    const int per = (bc + nthreads - 1) / nthreads;
    for(int t = 0; t < nthreads; ++t)
    {
        OJob j = {n, nrhs, gB, X, gA, t * per < bc ? t * per : bc,
                  (t + 1) * per < bc ? (t + 1) * per : bc};
        jobs[t] = j;
    }
    for(int t = 1; t < nthreads; ++t)
        pthread_create(&th[t], NULL, run_outer, &jobs[t]);
    run_outer(&jobs[0]);
    for(int t = 1; t < nthreads; ++t)
        pthread_join(th[t], NULL);
    free(jobs);
    free(th);
    return 0;
}
