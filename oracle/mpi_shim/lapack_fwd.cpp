// LAPACK entry points the reference program links against (dgesv_ in its
// quintic-spline refresh, dsysvx_ in its Powell optimizer).  Neither is on
// the spline3eq objective path; they are forwarded at first use to the
// OpenBLAS build that ships inside scipy (loaded with dlopen from the path
// given at compile time).  Test-oracle infrastructure only.
#include <cstdio>
#include <cstdlib>
#include <dlfcn.h>

#ifndef MZ_SCIPY_OPENBLAS
#define MZ_SCIPY_OPENBLAS ""
#endif

static void *mz_sym(const char *name) {
  static void *lib = nullptr;
  if (!lib) {
    lib = dlopen(MZ_SCIPY_OPENBLAS, RTLD_NOW | RTLD_LOCAL);
    if (!lib) {
      std::fprintf(stderr, "oracle lapack forwarder: cannot open %s\n", MZ_SCIPY_OPENBLAS);
      std::exit(4);
    }
  }
  void *p = dlsym(lib, name);
  if (!p) {
    std::fprintf(stderr, "oracle lapack forwarder: missing %s\n", name);
    std::exit(4);
  }
  return p;
}

extern "C" {

typedef void (*dgesv_t)(int *, int *, double *, int *, int *, double *, int *, int *);
void dgesv_(int *n, int *nrhs, double *a, int *lda, int *ipiv, double *b, int *ldb, int *info) {
  static dgesv_t f = (dgesv_t)mz_sym("scipy_dgesv_");
  f(n, nrhs, a, lda, ipiv, b, ldb, info);
}

typedef void (*dsysvx_t)(char *, char *, int *, int *, double *, int *, double *, int *, int *,
                         double *, int *, double *, int *, double *, double *, double *, double *,
                         int *, int *, int *);
void dsysvx_(char *fact, char *uplo, int *n, int *nrhs, double *a, int *lda, double *af, int *ldaf,
             int *ipiv, double *b, int *ldb, double *x, int *ldx, double *rcond, double *ferr,
             double *berr, double *work, int *lwork, int *iwork, int *info) {
  static dsysvx_t f = (dsysvx_t)mz_sym("scipy_dsysvx_");
  f(fact, uplo, n, nrhs, a, lda, af, ldaf, ipiv, b, ldb, x, ldx, rcond, ferr, berr, work, lwork,
    iwork, info);
}

}  // extern "C"
