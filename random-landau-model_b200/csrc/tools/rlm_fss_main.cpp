// rlm_fss -- finite-size-scaling driver: the rlm twist-mesh pipeline for several n_phi in one
// run, one output file per size, resumable by sample index.
//
// Options (those of rlm where they overlap, rlm/init_rlm.cpp:4-89):
//   -n  comma-separated list of n_phi (e.g. 64,128,192,256,384,512)
//   -q  quanta concentration          -i  impurity concentration
//   -g  theta mesh griding size       -c  # of disorder configurations per size
//   -s  seed                          -b  samples per pipeline call (default 16)
//   -p  precision: fp64 (default) or mixed
// Every size N writes energy_Chern_No_n<N>.txt in the line format of the reference's
// energy_Chern_No.txt (rlm/main_rlm_cpu.cpp:241-242), appending each batch as it finishes.
// On restart the complete samples already in a file are kept (an incomplete last sample is
// dropped) and the run continues from the next sample index; sample k always uses the
// disorder of sample k of the seed, so a resumed file equals an uninterrupted one.
#include <unistd.h>

#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "driver_common.h"

using namespace std;

static void usage(char* target) {
    cout << "Usage: " << target << " -[OPTIONS]" << endl;
    cout << "Options:\n";
    cout << "  -n  comma-separated list of n_phi\n";
    cout << "  -q  quanta concentration \n";
    cout << "  -i  impurity concentration\n";
    cout << "  -g  theta mesh griding size (n_mesh)\n";
    cout << "  -c  # of disorder configurations(n_sample) per n_phi\n";
    cout << "  -s  seed to generate seeds\n";
    cout << "  -b  # of samples per pipeline call\n";
    cout << "  -p  precision: fp64 or mixed\n";
}

// Complete samples (n_phi lines each) at the head of `path`; rewrites the file without an
// incomplete trailing sample.
static long resume_count(const string& path, long n_phi) {
    ifstream in(path);
    if (!in) return 0;
    vector<string> lines;
    string ln;
    while (getline(in, ln)) lines.push_back(ln);
    in.close();
    const long done = (long)lines.size() / n_phi;
    if ((long)lines.size() != done * n_phi) {
        ofstream out(path, ios::trunc);
        for (long i = 0; i < done * n_phi; ++i) out << lines[i] << "\n";
    }
    return done;
}

int main(int argc, char* argv[]) {
    string sizes = "64,128,192,256,384,512";
    long n_mesh = 16, n_sample = 16, batch = 16;
    double qc = 1, ic = 16;
    unsigned long seed = 1;
    string prec = "fp64";
    int ch, err_flag = 0;
    while ((ch = getopt(argc, argv, "n:q:i:g:c:s:b:p:h:")) != -1) {
        switch (ch) {
            case 'n': sizes = optarg; break;
            case 'q': qc = atof(optarg); break;
            case 'i': ic = atof(optarg); break;
            case 'g': n_mesh = atoi(optarg); break;
            case 'c': n_sample = atoi(optarg); break;
            case 's': seed = strtoul(optarg, nullptr, 10); break;
            case 'b': batch = atoi(optarg); break;
            case 'p': prec = optarg; break;
            default: err_flag++; break;
        }
    }
    vector<long> list;
    {
        stringstream ss(sizes);
        string tok;
        while (getline(ss, tok, ','))
            if (!tok.empty()) list.push_back(atol(tok.c_str()));
    }
    if (err_flag || list.empty() || n_mesh <= 0 || n_sample < 0 || batch <= 0 || (prec != "fp64" && prec != "mixed")) {
        usage(argv[0]);
        exit(2);
    }
    for (long n : list)
        if (n <= 0) {
            usage(argv[0]);
            exit(2);
        }
    rlmb_context* ctx = nullptr;
    int rc = rlmb_create(&ctx, 0);
    if (rc) return driver::fail("rlmb_create", rc);
    if (prec == "mixed" && (rc = rlmb_set_precision(ctx, RLMB_PRECISION_MIXED))) return driver::fail("rlmb_set_precision", rc);
    for (long n_phi : list) {
        const string path = "energy_Chern_No_n" + to_string(n_phi) + ".txt";
        const long start = resume_count(path, n_phi);
        ofstream out(path, ios::app);
        const double t0 = driver::now_s();
        vector<double> e, c;
        for (long s0 = start; s0 < n_sample; s0 += batch) {
            const long cnt = min(batch, n_sample - s0);
            e.assign(cnt * n_phi, 0.0);
            c.assign(cnt * n_phi, 0.0);
            rc = rlmb_rlm_mesh_solve(ctx, (int)n_phi, qc, ic, (int)n_mesh, seed, (int)s0, (int)cnt, e.data(), c.data());
            if (rc < 0) return driver::fail("rlmb_rlm_mesh_solve", rc);
            for (long n = 0; n < cnt; ++n)
                for (long i = 0; i < n_phi; ++i)
                    out << std::left << setw(8) << s0 + n << " " << setw(15) << setprecision(8) << e[n * n_phi + i]
                        << " " << c[n * n_phi + i] << endl;
            out.flush();
        }
        const double dt = driver::now_s() - t0;
        cerr << std::left << "n_phi " << setw(6) << n_phi << " samples " << start << ".." << n_sample - 1 << "  "
             << dt << " s";
        if (n_sample > start && dt > 0) cerr << "  (" << (n_sample - start) / (dt / 3600.0) << " samples/hour)";
        cerr << endl;
    }
    rlmb_destroy(ctx);
    return 0;
}
