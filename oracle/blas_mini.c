/*
 * blas_mini.c -- the eleven BLAS/LAPACK routines the FABIPB reference calls,
 * written from their published netlib definitions in plain C (column-major,
 * Fortran calling convention, LP64 integers).
 *
 * TEST INFRASTRUCTURE ONLY.  This file exists so the reference CPU solver can
 * be compiled from its own sources into oracle/_ref/ without any external
 * BLAS/LAPACK library.  It is linked only into the oracle binaries that the
 * tests and the CPU-baseline leg of bench.py run as a checker.
 *
 * Callers in the reference: gmres.c:14-25 (dcopy, dnrm2, dscal, drot, drotg,
 * ddot, daxpy, dtrsv, dgemv), fmm.c:28 and treecode.c:15 (dgemv),
 * precond_fmm.c:20-21 (dgetrf, dgetrs).
 */
#include <math.h>
#include <stddef.h>

#define A_(i, j) a[(size_t)(j) * (size_t)lda_ + (size_t)(i)]

static int lsame(const char *c, char u) {
  char x = *c;
  if (x >= 'a' && x <= 'z') x = (char)(x - 'a' + 'A');
  return x == u;
}

/* y := alpha*op(A)*x + beta*y */
void dgemv_(const char *trans, const int *m, const int *n, const double *alpha,
            const double *a, const int *lda, const double *x, const int *incx,
            const double *beta, double *y, const int *incy) {
  int M = *m, N = *n, lda_ = *lda, ix = *incx, iy = *incy;
  int leny = lsame(trans, 'N') ? M : N;
  int lenx = lsame(trans, 'N') ? N : M;
  int i, j;
  double al = *alpha, be = *beta;
  int kx = ix > 0 ? 0 : -(lenx - 1) * ix;
  int ky = iy > 0 ? 0 : -(leny - 1) * iy;
  if (M == 0 || N == 0 || (al == 0.0 && be == 1.0)) return;
  if (be != 1.0) {
    for (i = 0; i < leny; i++) {
      double *yi = &y[ky + i * iy];
      *yi = (be == 0.0) ? 0.0 : be * (*yi);
    }
  }
  if (al == 0.0) return;
  if (lsame(trans, 'N')) {
    for (j = 0; j < N; j++) {
      double t = al * x[kx + j * ix];
      for (i = 0; i < M; i++) y[ky + i * iy] += t * A_(i, j);
    }
  } else {
    for (j = 0; j < N; j++) {
      double t = 0.0;
      for (i = 0; i < M; i++) t += A_(i, j) * x[kx + i * ix];
      y[ky + j * iy] += al * t;
    }
  }
}

double ddot_(const int *n, const double *x, const int *incx, const double *y,
             const int *incy) {
  int i, N = *n, ix = *incx, iy = *incy;
  double s = 0.0;
  int kx = ix > 0 ? 0 : -(N - 1) * ix, ky = iy > 0 ? 0 : -(N - 1) * iy;
  for (i = 0; i < N; i++) s += x[kx + i * ix] * y[ky + i * iy];
  return s;
}

void daxpy_(const int *n, const double *alpha, const double *x, const int *incx,
            double *y, const int *incy) {
  int i, N = *n, ix = *incx, iy = *incy;
  int kx = ix > 0 ? 0 : -(N - 1) * ix, ky = iy > 0 ? 0 : -(N - 1) * iy;
  if (*alpha == 0.0) return;
  for (i = 0; i < N; i++) y[ky + i * iy] += (*alpha) * x[kx + i * ix];
}

void dscal_(const int *n, const double *alpha, double *x, const int *incx) {
  int i, N = *n, ix = *incx;
  if (ix <= 0) return;
  for (i = 0; i < N; i++) x[i * ix] *= *alpha;
}

void dcopy_(const int *n, const double *x, const int *incx, double *y, const int *incy) {
  int i, N = *n, ix = *incx, iy = *incy;
  int kx = ix > 0 ? 0 : -(N - 1) * ix, ky = iy > 0 ? 0 : -(N - 1) * iy;
  for (i = 0; i < N; i++) y[ky + i * iy] = x[kx + i * ix];
}

/* Euclidean norm with the running scale of the netlib routine (no overflow). */
double dnrm2_(const int *n, const double *x, const int *incx) {
  int i, N = *n, ix = *incx;
  double scale = 0.0, ssq = 1.0;
  if (N < 1 || ix < 1) return 0.0;
  if (N == 1) return fabs(x[0]);
  for (i = 0; i < N; i++) {
    double v = x[i * ix];
    if (v != 0.0) {
      double av = fabs(v);
      if (scale < av) {
        ssq = 1.0 + ssq * (scale / av) * (scale / av);
        scale = av;
      } else {
        ssq += (av / scale) * (av / scale);
      }
    }
  }
  return scale * sqrt(ssq);
}

void drot_(const int *n, double *x, const int *incx, double *y, const int *incy,
           const double *c, const double *s) {
  int i, N = *n, ix = *incx, iy = *incy;
  int kx = ix > 0 ? 0 : -(N - 1) * ix, ky = iy > 0 ? 0 : -(N - 1) * iy;
  for (i = 0; i < N; i++) {
    double xv = x[kx + i * ix], yv = y[ky + i * iy];
    x[kx + i * ix] = (*c) * xv + (*s) * yv;
    y[ky + i * iy] = (*c) * yv - (*s) * xv;
  }
}

/* Givens rotation: r = sign * sqrt(a^2+b^2), sign taken from the larger of |a|,|b|. */
void drotg_(double *a, double *b, double *c, double *s) {
  double aa = *a, bb = *b;
  double roe = (fabs(aa) > fabs(bb)) ? aa : bb;
  double scale = fabs(aa) + fabs(bb);
  double r, z;
  if (scale == 0.0) {
    *c = 1.0; *s = 0.0; r = 0.0; z = 0.0;
  } else {
    r = scale * sqrt((aa / scale) * (aa / scale) + (bb / scale) * (bb / scale));
    if (roe < 0.0) r = -r;
    *c = aa / r;
    *s = bb / r;
    z = 1.0;
    if (fabs(aa) > fabs(bb)) z = *s;
    if (fabs(bb) >= fabs(aa) && *c != 0.0) z = 1.0 / (*c);
  }
  *a = r;
  *b = z;
}

/* Triangular solve op(A) x = b, in place. */
void dtrsv_(const char *uplo, const char *trans, const char *diag, const int *n,
            const double *a, const int *lda, double *x, const int *incx) {
  int N = *n, lda_ = *lda, ix = *incx, i, j;
  int nounit = lsame(diag, 'N');
  int kx = ix > 0 ? 0 : -(N - 1) * ix;
#define X_(k) x[kx + (k) * ix]
  if (N == 0) return;
  if (lsame(trans, 'N')) {
    if (lsame(uplo, 'U')) {
      for (j = N - 1; j >= 0; j--) {
        if (X_(j) != 0.0) {
          if (nounit) X_(j) /= A_(j, j);
          for (i = j - 1; i >= 0; i--) X_(i) -= X_(j) * A_(i, j);
        }
      }
    } else {
      for (j = 0; j < N; j++) {
        if (X_(j) != 0.0) {
          if (nounit) X_(j) /= A_(j, j);
          for (i = j + 1; i < N; i++) X_(i) -= X_(j) * A_(i, j);
        }
      }
    }
  } else {
    if (lsame(uplo, 'U')) {
      for (j = 0; j < N; j++) {
        double t = X_(j);
        for (i = 0; i < j; i++) t -= A_(i, j) * X_(i);
        if (nounit) t /= A_(j, j);
        X_(j) = t;
      }
    } else {
      for (j = N - 1; j >= 0; j--) {
        double t = X_(j);
        for (i = N - 1; i > j; i--) t -= A_(i, j) * X_(i);
        if (nounit) t /= A_(j, j);
        X_(j) = t;
      }
    }
  }
#undef X_
}

/* LU with partial pivoting (right-looking, unblocked), 1-based pivots. */
void dgetrf_(int *m, int *n, double *a, int *lda, int *ipiv, int *info) {
  int M = *m, N = *n, lda_ = *lda, j, i, k, p;
  int mn = M < N ? M : N;
  *info = 0;
  for (j = 0; j < mn; j++) {
    double amax = -1.0;
    p = j;
    for (i = j; i < M; i++) {
      double v = fabs(A_(i, j));
      if (v > amax) { amax = v; p = i; }
    }
    ipiv[j] = p + 1;
    if (A_(p, j) != 0.0) {
      if (p != j) {
        for (k = 0; k < N; k++) {
          double t = A_(j, k); A_(j, k) = A_(p, k); A_(p, k) = t;
        }
      }
      {
        double inv = 1.0 / A_(j, j);
        for (i = j + 1; i < M; i++) A_(i, j) *= inv;
      }
    } else if (*info == 0) {
      *info = j + 1;
    }
    for (k = j + 1; k < N; k++) {
      double t = A_(j, k);
      if (t != 0.0) {
        double *colk = &A_(0, k);
        const double *colj = &A_(0, j);
        for (i = j + 1; i < M; i++) colk[i] -= t * colj[i];
      }
    }
  }
}

/* Solve A X = B with the factors of dgetrf (no-transpose only is used). */
void dgetrs_(char *trans, int *n, int *nrhs, double *a, int *lda, int *ipiv,
             double *b, int *ldb, int *info) {
  int N = *n, lda_ = *lda, L = *ldb, r, i, j;
  *info = 0;
  for (r = 0; r < *nrhs; r++) {
    double *x = &b[(size_t)r * (size_t)L];
    if (lsame(trans, 'N')) {
      for (i = 0; i < N; i++) {
        int p = ipiv[i] - 1;
        if (p != i) { double t = x[i]; x[i] = x[p]; x[p] = t; }
      }
      for (j = 0; j < N; j++) {
        double xj = x[j];
        if (xj != 0.0) for (i = j + 1; i < N; i++) x[i] -= xj * A_(i, j);
      }
      for (j = N - 1; j >= 0; j--) {
        if (x[j] != 0.0) {
          x[j] /= A_(j, j);
          for (i = 0; i < j; i++) x[i] -= x[j] * A_(i, j);
        }
      }
    } else {
      for (j = 0; j < N; j++) {
        double t = x[j];
        for (i = 0; i < j; i++) t -= A_(i, j) * x[i];
        x[j] = t / A_(j, j);
      }
      for (j = N - 1; j >= 0; j--) {
        double t = x[j];
        for (i = j + 1; i < N; i++) t -= A_(i, j) * x[i];
        x[j] = t;
      }
      for (i = N - 1; i >= 0; i--) {
        int p = ipiv[i] - 1;
        if (p != i) { double t = x[i]; x[i] = x[p]; x[p] = t; }
      }
    }
  }
}
