// Calls the reference-named C++ entry points of include/diag_wrappers_b200.h the way the
// reference's own call sites do, on inputs written by tests/test_wrappers.py, and writes the
// results back for comparison.  Built and run by that test only.
//
//   wrappers_check heevd    in out n        mkl_heevd on a host col-major matrix ('U')
//   wrappers_check cusolver in out n        cusolver_diag_hamil on a device complex64 matrix
//   wrappers_check magma    in out n        magma_diag_hamil (device matrix, host eigenvalues)
//   wrappers_check chern    in out n_phi dim_vec n_mesh theta_1     cal_Chern on a host ring
//   wrappers_check peer     in out n_phi dim_vec n_mesh theta_1     peer_cal_Chern, odd m only
//   wrappers_check tables   out n_phi off_head n_mesh L             prepare_coeff
//   wrappers_check disorder out n_imp L seed sample                 generate_disorder_potential
//   wrappers_check vmn      in out n_imp dim off_head               get_potential_coeff
//   wrappers_check vmngpu   in out n_imp dim off_head               prepare_potential_coeff (device, float)
//   wrappers_check sethamil in out n_phi off_head                   set_hamil_matrix (device, float)
//   wrappers_check chernio  dir out n_phi dim_vec n_mesh theta_1    cal_Chern_wfs_IO on files in dir
#include <cuda_runtime.h>

#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <vector>

#include <unistd.h>

#include "diag_wrappers_b200.h"

typedef std::complex<double> cd;
typedef std::complex<float> cf;

template <typename T>
static std::vector<T> slurp(const char* path, size_t count) {
    std::vector<T> v(count);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char*>(v.data()), count * sizeof(T));
    return v;
}
template <typename T>
static void dump(std::ofstream& f, const T* p, size_t count) {
    f.write(reinterpret_cast<const char*>(p), count * sizeof(T));
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    const std::string mode = argv[1];
    if (mode == "heevd") {
        const int n = atoi(argv[4]);
        auto h = slurp<cd>(argv[2], (size_t)n * n);
        std::vector<double> w(n);
        mkl_heevd(h.data(), w.data(), n);
        std::ofstream f(argv[3], std::ios::binary);
        dump(f, w.data(), n);
        dump(f, h.data(), (size_t)n * n);
    } else if (mode == "cusolver" || mode == "magma") {
        const int n = atoi(argv[4]);
        auto h = slurp<cf>(argv[2], (size_t)n * n);
        cuFloatComplex* d = nullptr;
        float* dw = nullptr;
        cudaMalloc(&d, (size_t)n * n * sizeof(cf));
        cudaMalloc(&dw, n * sizeof(float));
        cudaMemcpy(d, h.data(), (size_t)n * n * sizeof(cf), cudaMemcpyHostToDevice);
        std::vector<float> w(n);
        if (mode == "cusolver") {
            cusolver_diag_hamil(d, dw, n);
            cudaMemcpy(w.data(), dw, n * sizeof(float), cudaMemcpyDeviceToHost);
        } else {
            magma_diag_hamil(d, w.data(), n);
        }
        cudaMemcpy(h.data(), d, (size_t)n * n * sizeof(cf), cudaMemcpyDeviceToHost);
        std::ofstream f(argv[3], std::ios::binary);
        dump(f, w.data(), n);
        dump(f, h.data(), (size_t)n * n);
        cudaFree(d);
        cudaFree(dw);
    } else if (mode == "chern" || mode == "peer") {
        const int n_phi = atoi(argv[4]), dim_vec = atoi(argv[5]), g = atoi(argv[6]), t1 = atoi(argv[7]);
        auto wfs = slurp<cd>(argv[2], (size_t)2 * (g + 1) * n_phi * dim_vec);
        std::vector<double> ct((size_t)g * n_phi, -7.0);
        if (mode == "chern") {
            cal_Chern(wfs.data(), ct.data(), n_phi, dim_vec, g, t1);
        } else {
            std::vector<int> odd;
            for (int m = 1; m < g; m += 2) odd.push_back(m);
            struct_Chern p{n_phi, dim_vec, g, t1, odd.data(), (int)odd.size(), wfs.data(), ct.data()};
            peer_cal_Chern(&p);
        }
        std::ofstream f(argv[3], std::ios::binary);
        dump(f, ct.data(), ct.size());
    } else if (mode == "tables") {
        const int n_phi = atoi(argv[3]), o = atoi(argv[4]), g = atoi(argv[5]);
        const double L = atof(argv[6]);
        const int dim = 2 * o + 1;
        std::vector<cd> cmn(dim * dim), cmt((g + 1) * dim), cjm(n_phi * dim);
        prepare_coeff(cmn.data(), cmt.data(), cjm.data(), n_phi, o, dim, dim, g, L, L);
        std::ofstream f(argv[2], std::ios::binary);
        dump(f, cmn.data(), cmn.size());
        dump(f, cmt.data(), cmt.size());
        dump(f, cjm.data(), cjm.size());
    } else if (mode == "disorder") {
        const int nimp = atoi(argv[3]), sample = atoi(argv[6]);
        const double L = atof(argv[4]);
        const unsigned long seed = strtoul(argv[5], nullptr, 10);
        std::vector<double> x(nimp), y(nimp), s(nimp);
        generate_disorder_potential(x.data(), y.data(), s.data(), nimp, L, L, seed, sample);
        std::ofstream f(argv[2], std::ios::binary);
        dump(f, x.data(), nimp);
        dump(f, y.data(), nimp);
        dump(f, s.data(), nimp);
    } else if (mode == "vmn") {
        const int nimp = atoi(argv[4]), dim = atoi(argv[5]), o = atoi(argv[6]);
        auto in = slurp<double>(argv[2], 3 * (size_t)nimp + 2 * (size_t)dim * dim);
        std::vector<cd> cmn(dim * dim), v(dim * dim);
        std::memcpy(cmn.data(), in.data() + 3 * (size_t)nimp, (size_t)dim * dim * sizeof(cd));
        get_potential_coeff(in.data(), in.data() + nimp, in.data() + 2 * (size_t)nimp, v.data(), cmn.data(), dim, dim,
                            o, nimp);
        std::ofstream f(argv[3], std::ios::binary);
        dump(f, v.data(), v.size());
    } else if (mode == "vmngpu") {
        // in: x, y, s (float, n_imp each), coeff_mn (complex float, dim*dim)
        const int nimp = atoi(argv[4]), dim = atoi(argv[5]), o = atoi(argv[6]);
        const size_t dd = (size_t)dim * dim;
        auto xyz = slurp<float>(argv[2], 3 * (size_t)nimp + 2 * dd);
        float* d = nullptr;
        cudaMalloc(&d, (3 * (size_t)nimp + 4 * dd) * sizeof(float));
        cudaMemcpy(d, xyz.data(), (3 * (size_t)nimp + 2 * dd) * sizeof(float), cudaMemcpyHostToDevice);
        cuFloatComplex* dc = reinterpret_cast<cuFloatComplex*>(d + 3 * (size_t)nimp);
        cuFloatComplex* dv = dc + dd;
        prepare_potential_coeff(d, d + nimp, d + 2 * (size_t)nimp, dv, dc, dim, dim, o, nimp);
        std::vector<cf> v(dd);
        cudaMemcpy(v.data(), dv, dd * sizeof(cf), cudaMemcpyDeviceToHost);
        std::ofstream f(argv[3], std::ios::binary);
        dump(f, v.data(), dd);
        cudaFree(d);
    } else if (mode == "sethamil") {
        // in: ct1 (dim), ct2 (dim), coeff_jm (n_phi*dim), Vmn (dim*dim), complex float
        const int n_phi = atoi(argv[4]), o = atoi(argv[5]);
        const int dim = 2 * o + 1;
        const size_t nin = 2 * (size_t)dim + (size_t)n_phi * dim + (size_t)dim * dim;
        auto in = slurp<cf>(argv[2], nin);
        cuFloatComplex* d = nullptr;
        cudaMalloc(&d, (nin + (size_t)n_phi * n_phi) * sizeof(cf));
        cudaMemcpy(d, in.data(), nin * sizeof(cf), cudaMemcpyHostToDevice);
        cuFloatComplex* wfs = d + nin;
        set_hamil_matrix(d, d + dim, d + 2 * dim, d + 2 * dim + (size_t)n_phi * dim, wfs, n_phi, dim, o);
        std::vector<cf> h((size_t)n_phi * n_phi);
        cudaMemcpy(h.data(), wfs, h.size() * sizeof(cf), cudaMemcpyDeviceToHost);
        std::ofstream f(argv[3], std::ios::binary);
        dump(f, h.data(), h.size());
        cudaFree(d);
    } else if (mode == "chernio") {
        const int n_phi = atoi(argv[4]), dim_vec = atoi(argv[5]), g = atoi(argv[6]), t1 = atoi(argv[7]);
        std::vector<double> ct((size_t)g * n_phi, -7.0);
        const std::string out = argv[3];
        if (chdir(argv[2]) != 0) return 3;
        cal_Chern_wfs_IO(ct.data(), n_phi, dim_vec, g, t1);
        std::ofstream f(out, std::ios::binary);
        dump(f, ct.data(), ct.size());
    } else {
        return 2;
    }
    return 0;
}
