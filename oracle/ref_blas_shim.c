/*
 * ref_blas_shim.c -- TEST INFRASTRUCTURE for oracle/_ref only.
 *
 * The reference's BLAS/LAPACK backend (src/linalg/linalg_blas_lapack.cpp:9-44)
 * binds the Fortran symbols zgemm_/zgemv_/zgetrf_/zgetrs_.  This image has no
 * system BLAS/LAPACK; scipy ships OpenBLAS 0.3.x with the same LP64 Fortran ABI
 * under a "scipy_" prefix.  These four forwarders let the reference's own backend
 * link against it unchanged.
 */
typedef struct { double re, im; } zc_t;

void scipy_zgemm_(const char*, const char*, const int*, const int*, const int*, const zc_t*, const zc_t*,
                  const int*, const zc_t*, const int*, const zc_t*, zc_t*, const int*);
void scipy_zgemv_(const char*, const int*, const int*, const zc_t*, const zc_t*, const int*, const zc_t*,
                  const int*, const zc_t*, zc_t*, const int*);
void scipy_zgetrf_(const int*, const int*, zc_t*, const int*, int*, int*);
void scipy_zgetrs_(const char*, const int*, const int*, const zc_t*, const int*, const int*, zc_t*, const int*,
                   int*);
void scipy_openblas_set_num_threads(int);
int scipy_openblas_get_num_threads(void);

void zgemm_(const char* ta, const char* tb, const int* m, const int* n, const int* k, const zc_t* alpha,
            const zc_t* a, const int* lda, const zc_t* b, const int* ldb, const zc_t* beta, zc_t* c,
            const int* ldc) {
    scipy_zgemm_(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

void zgemv_(const char* t, const int* m, const int* n, const zc_t* alpha, const zc_t* a, const int* lda,
            const zc_t* x, const int* incx, const zc_t* beta, zc_t* y, const int* incy) {
    scipy_zgemv_(t, m, n, alpha, a, lda, x, incx, beta, y, incy);
}

void zgetrf_(const int* m, const int* n, zc_t* a, const int* lda, int* ipiv, int* info) {
    scipy_zgetrf_(m, n, a, lda, ipiv, info);
}

void zgetrs_(const char* t, const int* n, const int* nrhs, const zc_t* a, const int* lda, const int* ipiv,
             zc_t* b, const int* ldb, int* info) {
    scipy_zgetrs_(t, n, nrhs, a, lda, ipiv, b, ldb, info);
}

void ref_blas_set_threads(int n) { scipy_openblas_set_num_threads(n); }
int ref_blas_get_threads(void) { return scipy_openblas_get_num_threads(); }
