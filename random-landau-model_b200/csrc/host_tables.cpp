// Host-side inputs of the pipeline: the disorder-independent rlm coefficient tables and
// the disorder generators.  They stay on the host because they must match the
// reference bit for bit (same libm calls, same order of operations) and cost nothing
// next to the eigensolves.
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/rlm_b200.h"

namespace {

// MT19937 (Matsumoto & Nishimura, ACM TOMACS 8(1), 1998): init_genrand seeding and the
// tempered 32-bit output; this is the generator behind the reference's
// vslNewStream(VSL_BRNG_MT19937, seed) calls.
struct Mt19937 {
    uint32_t mt[624];
    int idx;
    explicit Mt19937(uint32_t seed) {
        mt[0] = seed;
        for (int i = 1; i < 624; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
        idx = 624;
    }
    void twist() {
        for (int i = 0; i < 624; ++i) {
            const uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
            uint32_t v = mt[(i + 397) % 624] ^ (y >> 1);
            if (y & 1u) v ^= 0x9908b0dfu;
            mt[i] = v;
        }
        idx = 0;
    }
    uint32_t next() {
        if (idx >= 624) twist();
        uint32_t y = mt[idx++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        return y;
    }
    void skip(long long n) {
        while (n > 0) {
            if (idx >= 624) twist();
            const long long take = std::min<long long>(n, 624 - idx);
            idx += (int)take;
            n -= take;
        }
    }
    // vdRngUniform(a, b): one 32-bit output per value
    double uniform(double a, double b) { return a + (b - a) * ((double)next() * (1.0 / 4294967296.0)); }
};

}  // namespace

extern "C" int rlmb_rlm_coeff_tables(int n_phi, int off_head, int dim, int n_mesh, double L1,
                                     double L2, double* coeff_mn, double* coeff_m_theta,
                                     double* coeff_jm) {
    if (n_phi <= 0 || dim != 2 * off_head + 1 || n_mesh <= 0 || !coeff_mn || !coeff_m_theta || !coeff_jm)
        return RLMB_ERR_ARG;
    // rlm/matrix_coefficients.cpp:9-11 -- note the single-precision expf and 1.0f/n_phi of the
    // reference's double build, promoted to double exactly as the reference multiplies them.
    const double pi2 = M_PI * 2.0;
    const float inv_n = 1.0f / n_phi;
    for (int m = 0; m < dim; ++m)
        for (int n = 0; n < dim; ++n) {
            const double a = M_PI * (m - off_head) * (n - off_head) / n_phi;
            const float ex = expf(-M_PI * ((m - off_head) * (m - off_head) * L2 / L1 +
                                           (n - off_head) * (n - off_head) * L1 / L2) / 2.0 / n_phi);
            const double re = cos(a), im = -sin(a);
            coeff_mn[2 * (m * dim + n)] = re * (double)ex * (double)inv_n;
            coeff_mn[2 * (m * dim + n) + 1] = im * (double)ex * (double)inv_n;
        }
    // rlm/matrix_coefficients.cpp:14-19
    for (int t = 0; t <= n_mesh; ++t) {
        const double dtheta = t * pi2 / n_mesh;
        for (int m = 0; m < dim; ++m) {
            const double a = (m - off_head) * dtheta / n_phi;
            coeff_m_theta[2 * (t * dim + m)] = cos(a);
            coeff_m_theta[2 * (t * dim + m) + 1] = sin(a);
        }
    }
    // rlm/matrix_coefficients.cpp:21-24
    for (int j = 0; j < n_phi; ++j)
        for (int m = 0; m < dim; ++m) {
            const double a = pi2 * (m - off_head) * (j + 1) / n_phi;
            coeff_jm[2 * (j * dim + m)] = cos(a);
            coeff_jm[2 * (j * dim + m) + 1] = -sin(a);
        }
    return RLMB_OK;
}

extern "C" int rlmb_rlm_disorder(int impurity_num, double L1, double L2, unsigned long seed,
                                 int sample, double* x, double* y, double* s) {
    if (impurity_num <= 0 || sample < 0 || !x || !y || !s) return RLMB_ERR_ARG;
    // rlm/disorder_potential.cpp:3-21: a fresh stream per sample, skipped by 3*N_imp*sample
    Mt19937 g((uint32_t)seed);
    g.skip((long long)impurity_num * 3 * sample);
    for (int i = 0; i < impurity_num; ++i) x[i] = g.uniform(0.0, L1);
    for (int i = 0; i < impurity_num; ++i) y[i] = g.uniform(0.0, L2);
    for (int i = 0; i < impurity_num; ++i) s[i] = (g.next() % 2 == 0) ? 1.0 : -1.0;
    return RLMB_OK;
}

extern "C" int rlmb_hlm_potentials(unsigned long seed, int n_sites, int n_sample, double* out) {
    if (n_sites <= 0 || n_sample < 0 || (!out && n_sample > 0)) return RLMB_ERR_ARG;
    // hlm/main_hlm_cpu.cpp:66-67,79: one stream for the whole run
    Mt19937 g((uint32_t)seed);
    for (long long k = 0; k < (long long)n_sample * n_sites; ++k) out[k] = g.uniform(-1.0, 1.0);
    return RLMB_OK;
}
