/*
 * Minimal BLAS/LAPACK entry points for the reference-oracle build.
 *
 * TEST INFRASTRUCTURE ONLY. The ProteinDF reference objects linked into the
 * oracle harness (oracle/_ref/pdfxc_ref) reference a handful of BLAS/LAPACK
 * symbols through their dense-matrix containers. The XC quadrature path itself
 * calls none of them; the only call made at run time is from
 * DfGenerateGrid's constructor (src/libpdf/DfGenerateGrid.cpp:1739-1809,
 * getOMatrix: a 3x3 product and a 3x3 symmetric eigen-decomposition), whose
 * result the harness does not use (it passes the identity orientation to the
 * sphere generator explicitly). So this file provides plain column-major
 * reference implementations of the level-1/2/3 routines and a Jacobi
 * eigensolver for the packed symmetric case, and an abort for the rest.
 * Fortran calling convention: every argument by pointer, hidden string
 * lengths ignored.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int lsame(const char* a, char b) {
    char c = *a;
    if (c >= 'a' && c <= 'z') c = (char)(c - 'a' + 'A');
    if (b >= 'a' && b <= 'z') b = (char)(b - 'a' + 'A');
    return c == b;
}

void dscal_(const int* n, const double* a, double* x, const int* incx) {
    for (int i = 0; i < *n; ++i) x[(long)i * *incx] *= *a;
}

void daxpy_(const int* n, const double* a, const double* x, const int* incx,
            double* y, const int* incy) {
    for (int i = 0; i < *n; ++i) y[(long)i * *incy] += *a * x[(long)i * *incx];
}

double ddot_(const int* n, const double* x, const int* incx, const double* y,
             const int* incy) {
    double s = 0.0;
    for (int i = 0; i < *n; ++i) s += x[(long)i * *incx] * y[(long)i * *incy];
    return s;
}

void dgemv_(const char* trans, const int* m, const int* n, const double* alpha,
            const double* a, const int* lda, const double* x, const int* incx,
            const double* beta, double* y, const int* incy) {
    const int t = !lsame(trans, 'N');
    const int ny = t ? *n : *m, nx = t ? *m : *n;
    for (int i = 0; i < ny; ++i) {
        double s = 0.0;
        for (int k = 0; k < nx; ++k) {
            const double aik = t ? a[(long)k + (long)i * *lda] : a[(long)i + (long)k * *lda];
            s += aik * x[(long)k * *incx];
        }
        double* yi = &y[(long)i * *incy];
        *yi = (*beta == 0.0 ? 0.0 : *beta * *yi) + *alpha * s;
    }
}

void dgemm_(const char* ta, const char* tb, const int* m, const int* n,
            const int* k, const double* alpha, const double* a, const int* lda,
            const double* b, const int* ldb, const double* beta, double* c,
            const int* ldc) {
    const int at = !lsame(ta, 'N'), bt = !lsame(tb, 'N');
    for (int j = 0; j < *n; ++j) {
        for (int i = 0; i < *m; ++i) {
            double s = 0.0;
            for (int l = 0; l < *k; ++l) {
                const double ail = at ? a[(long)l + (long)i * *lda] : a[(long)i + (long)l * *lda];
                const double blj = bt ? b[(long)j + (long)l * *ldb] : b[(long)l + (long)j * *ldb];
                s += ail * blj;
            }
            double* cij = &c[(long)i + (long)j * *ldc];
            *cij = (*beta == 0.0 ? 0.0 : *beta * *cij) + *alpha * s;
        }
    }
}

void dspmv_(const char* uplo, const int* n, const double* alpha, const double* ap,
            const double* x, const int* incx, const double* beta, double* y,
            const int* incy) {
    const int up = lsame(uplo, 'U');
    const int nn = *n;
    for (int i = 0; i < nn; ++i) {
        double s = 0.0;
        for (int j = 0; j < nn; ++j) {
            int r = i < j ? i : j, c = i < j ? j : i; /* r <= c */
            long idx = up ? (long)r + (long)c * (c + 1) / 2
                          : (long)c + (long)r * (2 * nn - r - 1) / 2;
            s += ap[idx] * x[(long)j * *incx];
        }
        double* yi = &y[(long)i * *incy];
        *yi = (*beta == 0.0 ? 0.0 : *beta * *yi) + *alpha * s;
    }
}

/* Packed symmetric eigenproblem by cyclic Jacobi rotations; eigenvalues
 * ascending, eigenvectors as columns of z (column-major, leading dim ldz). */
void dspev_(const char* jobz, const char* uplo, const int* n, double* ap, double* w,
            double* z, const int* ldz, double* work, int* info) {
    (void)work;
    const int nn = *n, up = lsame(uplo, 'U'), vec = lsame(jobz, 'V');
    double* a = (double*)calloc((size_t)nn * nn, sizeof(double));
    double* v = (double*)calloc((size_t)nn * nn, sizeof(double));
    for (int c = 0; c < nn; ++c)
        for (int r = 0; r <= c; ++r) {
            long idx = up ? (long)r + (long)c * (c + 1) / 2 : (long)c + (long)r * (2 * nn - r - 1) / 2;
            a[r * nn + c] = a[c * nn + r] = ap[idx];
        }
    for (int i = 0; i < nn; ++i) v[i * nn + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < nn; ++p)
            for (int q = p + 1; q < nn; ++q) off += a[p * nn + q] * a[p * nn + q];
        if (off < 1e-300) break;
        for (int p = 0; p < nn; ++p)
            for (int q = p + 1; q < nn; ++q) {
                const double apq = a[p * nn + q];
                if (fabs(apq) < 1e-300) continue;
                const double theta = (a[q * nn + q] - a[p * nn + p]) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < nn; ++k) {
                    const double akp = a[k * nn + p], akq = a[k * nn + q];
                    a[k * nn + p] = cs * akp - sn * akq;
                    a[k * nn + q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < nn; ++k) {
                    const double apk = a[p * nn + k], aqk = a[q * nn + k];
                    a[p * nn + k] = cs * apk - sn * aqk;
                    a[q * nn + k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < nn; ++k) {
                    const double vkp = v[k * nn + p], vkq = v[k * nn + q];
                    v[k * nn + p] = cs * vkp - sn * vkq;
                    v[k * nn + q] = sn * vkp + cs * vkq;
                }
            }
    }
    int* order = (int*)malloc(sizeof(int) * nn);
    for (int i = 0; i < nn; ++i) order[i] = i;
    for (int i = 0; i < nn; ++i)
        for (int j = i + 1; j < nn; ++j)
            if (a[order[j] * nn + order[j]] < a[order[i] * nn + order[i]]) {
                int t = order[i]; order[i] = order[j]; order[j] = t;
            }
    for (int i = 0; i < nn; ++i) {
        w[i] = a[order[i] * nn + order[i]];
        if (vec)
            for (int k = 0; k < nn; ++k) z[(long)k + (long)i * *ldz] = v[k * nn + order[i]];
    }
    free(order); free(a); free(v);
    *info = 0;
}

/* Full (column-major, leading dim lda) <-> packed triangular copies. */
static long packed_index(int up, int n, int r, int c) { /* requires r<=c (U) or r>=c (L) */
    return up ? (long)r + (long)c * (c + 1) / 2 : (long)r + (long)c * (2L * n - c - 1) / 2;
}

void dtrttp_(const char* uplo, const int* n, const double* a, const int* lda, double* ap, int* info) {
    const int up = lsame(uplo, 'U');
    for (int c = 0; c < *n; ++c)
        for (int r = up ? 0 : c; up ? r <= c : r < *n; ++r)
            ap[packed_index(up, *n, r, c)] = a[(long)r + (long)c * *lda];
    *info = 0;
}

void dtpttr_(const char* uplo, const int* n, const double* ap, double* a, const int* lda, int* info) {
    const int up = lsame(uplo, 'U');
    for (int c = 0; c < *n; ++c)
        for (int r = up ? 0 : c; up ? r <= c : r < *n; ++r)
            a[(long)r + (long)c * *lda] = ap[packed_index(up, *n, r, c)];
    *info = 0;
}

#define PDFXC_UNUSED_LAPACK(name)                                                  \
    void name(void) {                                                              \
        fprintf(stderr, "oracle harness: unexpected call to " #name "\n");        \
        abort();                                                                   \
    }
PDFXC_UNUSED_LAPACK(dsptri_)
PDFXC_UNUSED_LAPACK(dsptrf_)
PDFXC_UNUSED_LAPACK(dgetri_)
PDFXC_UNUSED_LAPACK(dgetrf_)
PDFXC_UNUSED_LAPACK(dgelss_)
