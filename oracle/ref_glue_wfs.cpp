// oracle/ref_glue_wfs.cpp -- test infrastructure only: a command-line front end to the
// reference's write_wfs (diag_wrappers/wfs_file.cpp:2-11), compiled with it into
// oracle/_ref/wfs_ref.  Usage: wfs_ref <theta_1> <theta_2> <input.bin>; reads the raw
// complex<double> values of input.bin and writes wfs_<theta_1>_<theta_2>.bin in the
// current directory through the reference function.
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

void write_wfs(int theta_1, int theta_2, std::complex<double>* wfs, unsigned long size);

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    FILE* f = fopen(argv[3], "rb");
    if (!f) return 1;
    std::vector<std::complex<double>> v;
    std::complex<double> z;
    while (fread(&z, sizeof(z), 1, f) == 1) v.push_back(z);
    fclose(f);
    write_wfs(atoi(argv[1]), atoi(argv[2]), v.data(), v.size());
    return 0;
}
