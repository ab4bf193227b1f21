// Small dense Hermitian eigenproblems in one thread (double precision).
#pragma once
#include <cfloat>

#include "common.cuh"

namespace rlmb {

// Cyclic complex Jacobi: diagonalises the k x k Hermitian a (column-major, both triangles
// stored, leading dimension k) in place and accumulates the rotations into v (v <- v G),
// until the off-diagonal mass falls below 1e-32 of the diagonal mass (at most 50 sweeps).
// On return diag(a) holds the eigenvalues (unsorted) and the columns of v (if v started
// as I) the eigenvectors.
__device__ __forceinline__ void herm_jacobi(cplx* a, cplx* v, int k) {
    for (int sweep = 0; sweep < 50; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int cc = 0; cc < k; ++cc)
            for (int r = 0; r < k; ++r) {
                if (r != cc) off += cabs2(a[r + cc * k]);
                else diag += cabs2(a[r + cc * k]);
            }
        if (off <= 1e-32 * fmax(diag, DBL_MIN)) break;
        for (int p = 0; p < k - 1; ++p)
            for (int q = p + 1; q < k; ++q) {
                const cplx apq = a[p + q * k];
                const double r = sqrt(cabs2(apq));
                if (r < 1e-300) continue;
                const cplx e = mk(apq.x / r, apq.y / r);   // apq = r e
                const double app = a[p + p * k].x, aqq = a[q + q * k].x;
                const double tau = (aqq - app) / (2.0 * r);
                const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                const double cs = 1.0 / sqrt(1.0 + t * t), sn = t * cs;
                // G = diag(1, conj(e)) R, R = [[c, s], [-s, c]]; columns p, q of G:
                // G[:,p] = (c, -s conj(e)), G[:,q] = (s, c conj(e))
                const cplx gpp = mk(cs, 0.0), gpq = mk(sn, 0.0);
                const cplx gqp = cscale(cconj(e), -sn), gqq = cscale(cconj(e), cs);
                for (int m = 0; m < k; ++m) {   // A <- A G (columns p, q)
                    const cplx akp = a[m + p * k], akq = a[m + q * k];
                    a[m + p * k] = cadd(cmul(akp, gpp), cmul(akq, gqp));
                    a[m + q * k] = cadd(cmul(akp, gpq), cmul(akq, gqq));
                    const cplx vkp = v[m + p * k], vkq = v[m + q * k];
                    v[m + p * k] = cadd(cmul(vkp, gpp), cmul(vkq, gqp));
                    v[m + q * k] = cadd(cmul(vkp, gpq), cmul(vkq, gqq));
                }
                for (int m = 0; m < k; ++m) {   // A <- G^H A (rows p, q)
                    const cplx apk = a[p + m * k], aqk = a[q + m * k];
                    a[p + m * k] = cadd(cmulc(gpp, apk), cmulc(gqp, aqk));
                    a[q + m * k] = cadd(cmulc(gpq, apk), cmulc(gqq, aqk));
                }
                a[p + q * k] = mk(0, 0);
                a[q + p * k] = mk(0, 0);
                a[p + p * k].y = 0.0;
                a[q + q * k].y = 0.0;
            }
    }
}

}  // namespace rlmb
