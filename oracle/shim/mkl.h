/*
 * oracle/shim/mkl.h -- test infrastructure only.
 *
 * A project-written stand-in for the subset of Intel MKL that the reference's
 * double-precision CPU path includes as "mkl.h".  It lets oracle/Makefile compile
 * the reference's own sources, unmodified, into oracle/_ref/ so that the oracle
 * and the golden fixtures can be pinned against the reference itself.
 *
 * MKL is not installed here.  The dense linear algebra is forwarded to the
 * `scipy_`-prefixed exports of the OpenBLAS that ships inside scipy
 * (LAPACKE_zheevd/cheevd, cblas_zgemm3m/cgemm3m, cblas_zdotc_sub/cdotc_sub).
 * The VSL random-number subset used by rlm/disorder_potential.cpp:3-21 and
 * hlm/main_hlm_cpu.cpp:66-67,79 is implemented here from the published MT19937
 * algorithm (Matsumoto & Nishimura, ACM TOMACS 8(1), 1998):
 *   - vslNewStream(MT19937, seed): state seeded with init_genrand(seed mod 2^32);
 *   - vslSkipAheadStream(n): discards n 32-bit outputs;
 *   - viRngUniformBits: raw 32-bit tempered outputs;
 *   - vdRngUniform/vsRngUniform(a,b): one 32-bit output x per value,
 *     u = a + (b - a) * (x * 2^-32).
 * MKL's exact integer->double mapping is not part of the reference tree, so this
 * generator pins "same seed -> same disorder" inside this repository only.  The
 * product's host generator (random-landau-model_b200/csrc/host_tables.cpp)
 * implements the same published algorithm and mapping independently.
 */
#ifndef RLMB_ORACLE_MKL_SHIM_H
#define RLMB_ORACLE_MKL_SHIM_H

#include <complex>
#include <cstdint>
#include <cstdlib>

#ifndef MKL_Complex16
#define MKL_Complex16 std::complex<double>
#endif
#ifndef MKL_Complex8
#define MKL_Complex8 std::complex<float>
#endif

/* ---------------------------------------------------------------- LAPACKE */
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

extern "C" {
int scipy_LAPACKE_zheevd(int layout, char jobz, char uplo, int n, void* a, int lda, double* w);
int scipy_LAPACKE_cheevd(int layout, char jobz, char uplo, int n, void* a, int lda, float* w);
void scipy_cblas_zgemm3m(int layout, int ta, int tb, int m, int n, int k, const void* alpha,
                         const void* a, int lda, const void* b, int ldb, const void* beta,
                         void* c, int ldc);
void scipy_cblas_cgemm3m(int layout, int ta, int tb, int m, int n, int k, const void* alpha,
                         const void* a, int lda, const void* b, int ldb, const void* beta,
                         void* c, int ldc);
void scipy_cblas_zdotc_sub(int n, const void* x, int incx, const void* y, int incy, void* dotc);
void scipy_cblas_cdotc_sub(int n, const void* x, int incx, const void* y, int incy, void* dotc);
}

static inline int LAPACKE_zheevd(int layout, char jobz, char uplo, int n, MKL_Complex16* a,
                                 int lda, double* w) {
    return scipy_LAPACKE_zheevd(layout, jobz, uplo, n, (void*)a, lda, w);
}
static inline int LAPACKE_cheevd(int layout, char jobz, char uplo, int n, MKL_Complex8* a,
                                 int lda, float* w) {
    return scipy_LAPACKE_cheevd(layout, jobz, uplo, n, (void*)a, lda, w);
}

/* ------------------------------------------------------------------ CBLAS */
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

static inline void cblas_zgemm3m(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                                 int m, int n, int k, const void* alpha, const void* a, int lda,
                                 const void* b, int ldb, const void* beta, void* c, int ldc) {
    scipy_cblas_zgemm3m((int)layout, (int)ta, (int)tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
static inline void cblas_cgemm3m(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                                 int m, int n, int k, const void* alpha, const void* a, int lda,
                                 const void* b, int ldb, const void* beta, void* c, int ldc) {
    scipy_cblas_cgemm3m((int)layout, (int)ta, (int)tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

/* MKL's Fortran-style dot products: result returned through the first argument. */
static inline void zdotc(MKL_Complex16* res, const int* n, const MKL_Complex16* x, const int* incx,
                         const MKL_Complex16* y, const int* incy) {
    scipy_cblas_zdotc_sub(*n, x, *incx, y, *incy, res);
}
static inline void cdotc(MKL_Complex8* res, const int* n, const MKL_Complex8* x, const int* incx,
                         const MKL_Complex8* y, const int* incy) {
    scipy_cblas_cdotc_sub(*n, x, *incx, y, *incy, res);
}

/* -------------------------------------------------------------------- VSL */
#define VSL_BRNG_MT19937 0x00D00000
#define VSL_RNG_METHOD_UNIFORM_STD 0
#define VSL_RNG_METHOD_UNIFORMBITS_STD 0

struct RlmbShimMT19937 {
    uint32_t mt[624];
    int idx;
};
typedef RlmbShimMT19937* VSLStreamStatePtr;

static inline void rlmb_shim_mt_seed(RlmbShimMT19937* s, uint32_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->idx = 624;
}

static inline uint32_t rlmb_shim_mt_next(RlmbShimMT19937* s) {
    if (s->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (s->mt[i] & 0x80000000u) | (s->mt[(i + 1) % 624] & 0x7fffffffu);
            uint32_t v = s->mt[(i + 397) % 624] ^ (y >> 1);
            if (y & 1u) v ^= 0x9908b0dfu;
            s->mt[i] = v;
        }
        s->idx = 0;
    }
    uint32_t y = s->mt[s->idx++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= (y >> 18);
    return y;
}

static inline int vslNewStream(VSLStreamStatePtr* stream, int brng, unsigned long seed) {
    (void)brng;
    *stream = (VSLStreamStatePtr)std::malloc(sizeof(RlmbShimMT19937));
    rlmb_shim_mt_seed(*stream, (uint32_t)seed);
    return 0;
}
static inline int vslSkipAheadStream(VSLStreamStatePtr stream, long long nskip) {
    for (long long i = 0; i < nskip; ++i) (void)rlmb_shim_mt_next(stream);
    return 0;
}
static inline int vslDeleteStream(VSLStreamStatePtr* stream) {
    std::free(*stream);
    *stream = 0;
    return 0;
}
static inline int viRngUniformBits(int method, VSLStreamStatePtr stream, int n, unsigned int* r) {
    (void)method;
    for (int i = 0; i < n; ++i) r[i] = rlmb_shim_mt_next(stream);
    return 0;
}
static inline int vdRngUniform(int method, VSLStreamStatePtr stream, int n, double* r, double a,
                               double b) {
    (void)method;
    for (int i = 0; i < n; ++i) {
        double u = (double)rlmb_shim_mt_next(stream) * (1.0 / 4294967296.0);
        r[i] = a + (b - a) * u;
    }
    return 0;
}
static inline int vsRngUniform(int method, VSLStreamStatePtr stream, int n, float* r, float a,
                               float b) {
    (void)method;
    for (int i = 0; i < n; ++i) {
        float u = (float)((double)rlmb_shim_mt_next(stream) * (1.0 / 4294967296.0));
        r[i] = a + (b - a) * u;
    }
    return 0;
}

#endif
