// rlm -- drop-in for the reference's rlm_cpu_dp / rlm_gpu_* programs on one B200.
//
// Options, usage text, log_rlm.txt and energy_Chern_No.txt are those of
// rlm/init_rlm.cpp:4-89 and rlm/main_rlm_cpu.cpp:96-243 (-h needs an argument and -d is
// listed but not accepted, as in the reference).  -t is accepted and has no effect: the
// twist mesh runs batched on the GPU.  The stderr report keeps the reference's lines; its
// per-k-point times are the device times of the batched kernels for sample 0.
#include <unistd.h>

#include <cstdlib>
#include <fstream>
#include <vector>

#include "driver_common.h"

using namespace std;

static void usage(char* target) {
    cout << "Usage: " << target << " -[OPTIONS]" << endl;
    cout << "Options:\n";
    cout << "  -n  n_phi\n";
    cout << "  -q  quanta concentration \n";
    cout << "  -i  impurity concentration\n";
    cout << "  -g  theta mesh griding size (n_mesh)\n";
    cout << "  -d  disorder potential K-space cut (offhead)\n";
    cout << "  -c  # of disorder configurations(n_sample)\n";
    cout << "  -s  seed to generate seeds\n";
    cout << "  -t  # of threads\n";
}

int main(int argc, char* argv[]) {
    long n_phi = 32, n_mesh = 32, n_sample = 1, num_threads = 1;
    double quanta_concentration = 1, impurity_concentration = 16;
    unsigned long seed = std::chrono::high_resolution_clock::now().time_since_epoch().count();
    int ch, err_flag = 0;
    while ((ch = getopt(argc, argv, "n:q:i:g:c:s:h:t:")) != -1) {
        switch (ch) {
            case 'n': n_phi = atoi(optarg); break;
            case 'q': quanta_concentration = atof(optarg); break;
            case 'i': impurity_concentration = atof(optarg); break;
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
    (void)num_threads;
    {
        ofstream flog("log_rlm.txt");
        flog << "########################################################" << endl;
        flog << setw(25) << "seed: " << seed << endl;
        flog << setw(25) << "n_phi: " << n_phi << endl;
        flog << setw(25) << "n_mesh: " << n_mesh << endl;
        flog << setw(25) << "n_sample: " << n_sample << endl;
        flog << setw(25) << "quanta_concentration: " << quanta_concentration << endl;
        flog << setw(25) << "impurity_concentration: " << impurity_concentration << endl;
        flog << "########################################################" << endl;
    }
    // derived sizes (rlm/main_rlm_cpu.cpp:29-33)
    const double L1 = sqrt(n_phi * quanta_concentration), L2 = L1;
    const long impurity_num = (long)(impurity_concentration * n_phi / quanta_concentration);
    const long off_head = (long)(sqrt((double)impurity_num) / 2 + 1);
    const long dim = off_head * 2 + 1;

    ofstream fchern("energy_Chern_No.txt");
    rlmb_context* ctx = nullptr;
    int rc = rlmb_create(&ctx, 0);
    if (rc) return driver::fail("rlmb_create", rc);

    // coefficient tables (host, rlm/matrix_coefficients.cpp:3-25)
    double t0 = driver::now_s();
    vector<double> cmn(2 * dim * dim), cmt(2 * (n_mesh + 1) * dim), cjm(2 * n_phi * dim);
    rc = rlmb_rlm_coeff_tables((int)n_phi, (int)off_head, (int)dim, (int)n_mesh, L1, L2, cmn.data(), cmt.data(),
                               cjm.data());
    if (rc) return driver::fail("rlmb_rlm_coeff_tables", rc);
    const double coeff_time = driver::now_s() - t0;
    cerr << std::left << setw(40) << "coefficients initialization time: " << coeff_time << " s\n";

    vector<double> e(n_phi * n_sample), c(n_phi * n_sample);
    double pot_time = 0, diag_time = 0, chern_time = 0;
    if (n_sample > 0) {
        // sample 0 alone, with the per-kernel profile for the report
        rlmb_profile_enable(ctx, 1);
        rc = rlmb_rlm_mesh_solve(ctx, (int)n_phi, quanta_concentration, impurity_concentration, (int)n_mesh, seed,
                                 0, 1, e.data(), c.data());
        if (rc < 0) return driver::fail("rlmb_rlm_mesh_solve", rc);
        pot_time = driver::kernel_seconds(ctx, {"k_vmn"});
        diag_time = driver::kernel_seconds(ctx, {"k_rlm_assemble", "k_hetrd", "k_stebz", "k_stein", "k_larft",
                                                 "k_ormtr"}) / (n_mesh + 1);   // per theta_1 line
        chern_time = driver::kernel_seconds(ctx, {"k_rlm_links", "k_plaquettes"}) / n_mesh;
        rlmb_profile_enable(ctx, 0);
        cerr << setw(40) << "potential initialization time: " << pot_time << " s\n";
        cerr << setw(40) << "diagonalization time/k-point: " << diag_time / (n_mesh + 1) << " s\n";
        const double total_time = coeff_time + (pot_time + (chern_time * n_mesh + diag_time * (n_mesh + 1))) * n_sample;
        cerr << setw(40) << "Chern No. calculation time/k-point: " << chern_time / (n_mesh + 1) << " s\n";
        cerr << setw(40) << "estimated total time:";
        driver::print_hms((long)total_time);
        cerr << std::left << setw(40) << "estimated # of samples/hour:" << n_sample / (total_time / 3600.0) << endl;
        cerr << setw(40) << "# module" << "%(time)" << endl;
        cerr << setw(40) << "coefficients" << coeff_time / total_time * 100.0 << "\n";
        cerr << setw(40) << "potential" << pot_time * n_sample / total_time * 100.0 << "\n";
        cerr << setw(40) << "diagonalization" << diag_time * (n_mesh + 1) * n_sample / total_time * 100.0 << endl;
        cerr << setw(40) << "Chern No. calculation" << chern_time * n_mesh * n_sample / total_time * 100.0 << endl;
        if (n_sample > 1) {
            rc = rlmb_rlm_mesh_solve(ctx, (int)n_phi, quanta_concentration, impurity_concentration, (int)n_mesh, seed,
                                     1, (int)n_sample - 1, e.data() + n_phi, c.data() + n_phi);
            if (rc < 0) return driver::fail("rlmb_rlm_mesh_solve", rc);
        }
    }
    // energy_Chern_No.txt exactly as rlm/main_rlm_cpu.cpp:241-242 writes it
    for (long n = 0; n < n_sample; ++n)
        for (long i = 0; i < n_phi; ++i)
            fchern << std::left << setw(8) << n << " " << setw(15) << setprecision(8) << e[n * n_phi + i] << " "
                   << c[n * n_phi + i] << endl;
    fchern.close();
    rlmb_destroy(ctx);
    return 0;
}
