// Shared parts of the rlm / hlm command-line drivers: per-phase device times read from the
// library's kernel profile, and the reference's stderr timing report.
#pragma once
#include <chrono>
#include <cmath>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <string>

#include "../../../include/rlm_b200.h"

namespace driver {

inline double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device seconds spent in kernels whose names start with any of `prefixes`.
inline double kernel_seconds(rlmb_context* ctx, std::initializer_list<const char*> prefixes) {
    double ms = 0.0;
    const int n = rlmb_profile_count(ctx);
    for (int i = 0; i < n; ++i) {
        char name[128];
        double t = 0.0;
        long long cnt = 0;
        if (rlmb_profile_entry(ctx, i, name, sizeof(name), &t, &cnt) != RLMB_OK) continue;
        for (const char* p : prefixes)
            if (std::strncmp(name, p, std::strlen(p)) == 0) ms += t;
    }
    return ms * 1e-3;
}

inline const char* kDiagKernels[] = {"k_hetrd", "k_stebz", "k_stein", "k_larft", "k_ormtr"};

// "estimated total time:" hh:mm:ss as the reference prints it (rlm/main_rlm_cpu.cpp:217-219).
inline void print_hms(long total) {
    std::cerr << std::right << std::setw(3) << std::setfill('0') << total / 3600 << std::setw(1) << ":";
    std::cerr << std::setw(2) << std::setfill('0') << (total % 3600) / 60 << std::setw(1) << ":";
    std::cerr << std::setw(2) << std::setfill('0') << total % 60 << std::endl << std::setfill(' ');
}

inline int fail(const char* what, int rc) {
    std::cerr << what << " failed: " << rlmb_status_string(rc) << " (status " << rc << ")\n";
    return 1;
}

}  // namespace driver
