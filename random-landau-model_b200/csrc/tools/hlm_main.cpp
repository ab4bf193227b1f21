// hlm -- drop-in for the reference's hlm_cpu_dp program on one B200.
//
// Options, usage text, log_hlm.txt and energy_Chern_No.txt are those of
// hlm/init_hlm.cpp:4-94 and hlm/main_hlm_cpu.cpp:22-197 (-h needs an argument, as in the
// reference).  -t is accepted and has no effect.  The stderr report keeps the reference's
// lines; its per-k-point times are the device times of the batched kernels for sample 0.
#include <unistd.h>

#include <cstdlib>
#include <fstream>
#include <vector>

#include "driver_common.h"

using namespace std;

static void usage(char* target) {
    cout << "Usage: " << target << " -[OPTIONS]" << endl;
    cout << "Options:\n";
    cout << "  -x  lx\n";
    cout << "  -y  ly \n";
    cout << "  -q  q [p/q, p set to 1] \n";
    cout << "  -g  theta mesh griding size (n_mesh)\n";
    cout << "  -b  band to be projected onto\n";
    cout << "  -c  # of disorder configurations (n_sample)\n";
    cout << "  -s  seed to generate seeds\n";
    cout << "  -t  # of threads\n";
}

int main(int argc, char* argv[]) {
    int lx = 3, ly = 3, n_mesh = 32, n_sample = 1, Q = 3, band = 0, num_threads = 1;
    unsigned long seed = std::chrono::high_resolution_clock::now().time_since_epoch().count();
    int ch, err_flag = 0;
    while ((ch = getopt(argc, argv, "x:y:b:q:g:c:s:h:t:")) != -1) {
        switch (ch) {
            case 'x': lx = atoi(optarg); break;
            case 'y': ly = atoi(optarg); break;
            case 'b': band = atoi(optarg); break;
            case 'q': Q = atoi(optarg); break;
            case 'g': n_mesh = atoi(optarg); break;
            case 'c': n_sample = atoi(optarg); break;
            case 's': seed = atoi(optarg); break;
            case 't': num_threads = atoi(optarg); break;
            default: err_flag++; break;
        }
    }
    if (err_flag) {
        usage(argv[0]);
        exit(2);
    }
    {
        ofstream flog("log_hlm.txt");
        flog << "########################################################" << endl;
        flog << setw(25) << "seed: " << seed << endl;
        flog << setw(25) << "lx: " << lx << endl;
        flog << setw(25) << "ly: " << ly << endl;
        flog << setw(25) << "Q: " << Q << endl;
        flog << setw(25) << "n_mesh: " << n_mesh << endl;
        flog << setw(25) << "n_sample: " << n_sample << endl;
        flog << setw(25) << "n_thread: " << num_threads << endl;
        flog << "########################################################" << endl;
    }
    const int n_sites = lx * ly, n_phi = n_sites / Q;
    ofstream fchern("energy_Chern_No.txt");
    rlmb_context* ctx = nullptr;
    int rc = rlmb_create(&ctx, 0);
    if (rc) return driver::fail("rlmb_create", rc);
    // on-site potentials of every sample from the run-long stream (hlm/main_hlm_cpu.cpp:66-67,79)
    vector<double> pots((size_t)n_sample * n_sites);
    rc = rlmb_hlm_potentials(seed, n_sites, n_sample, pots.data());
    if (rc) return driver::fail("rlmb_hlm_potentials", rc);
    vector<double> e((size_t)n_phi * n_sample), c((size_t)n_phi * n_sample);
    if (n_sample > 0) {
        rlmb_profile_enable(ctx, 1);
        rc = rlmb_hlm_mesh_solve(ctx, lx, ly, Q, band, n_mesh, pots.data(), 1, e.data(), c.data());
        if (rc < 0) return driver::fail("rlmb_hlm_mesh_solve", rc);
        const double diag_time = driver::kernel_seconds(ctx, {"k_hlm_bloch", "k_hlm_vtilde", "k_hlm_project",
                                                              "k_hetrd", "k_stebz", "k_stein", "k_larft",
                                                              "k_ormtr"}) / (n_mesh + 1);   // per theta_1 line
        const double chern_time = driver::kernel_seconds(ctx, {"k_hlm_links", "k_plaquettes"}) / n_mesh;
        rlmb_profile_enable(ctx, 0);
        cerr << std::left << setw(40) << "diagonalization time/k-point: " << diag_time / (n_mesh + 1) << " s\n";
        const long total_time = lround((chern_time * n_mesh + diag_time * (n_mesh + 1)) * n_sample);
        cerr << setw(40) << "Chern No. calculation time/k-point: " << chern_time / (n_mesh + 1) << " s\n";
        cerr << setw(40) << "estimated total time:";
        driver::print_hms(total_time);
        cerr << std::left << setw(40) << "estimated # of samples/hour:" << n_sample / (total_time / 3600.0) << endl;
        cerr << setw(40) << "# module" << "%(time)" << endl;
        cerr << setw(40) << "diagonalization" << diag_time * (n_mesh + 1) * n_sample / total_time * 100.0 << endl;
        cerr << setw(40) << "Chern No. calculation" << chern_time * n_mesh * n_sample / total_time * 100.0 << endl;
        if (n_sample > 1) {
            rc = rlmb_hlm_mesh_solve(ctx, lx, ly, Q, band, n_mesh, pots.data() + n_sites, n_sample - 1,
                                     e.data() + n_phi, c.data() + n_phi);
            if (rc < 0) return driver::fail("rlmb_hlm_mesh_solve", rc);
        }
    }
    // energy_Chern_No.txt exactly as hlm/main_hlm_cpu.cpp:194-196 writes it
    for (int n = 0; n < n_sample; ++n)
        for (int i = 0; i < n_phi; ++i)
            fchern << setw(8) << n << " " << setw(15) << setprecision(8) << e[(size_t)n * n_phi + i] << " "
                   << c[(size_t)n * n_phi + i] << endl;
    fchern.close();
    rlmb_destroy(ctx);
    return 0;
}
