// harness_common.h — flag parsing and checks shared by the two harnesses.
//
// Flags keep the reference's `--name=value` form and names
// (common/helper_string.h:17-65; test.cu:26-29; benchmark.cu:29-39).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sgemm_b200.h"

namespace harness {

inline const char* find_flag(int argc, char** argv, const char* name) {
    const size_t len = std::strlen(name);
    for (int i = 1; i < argc; ++i) {
        const char* a = argv[i];
        while (*a == '-') ++a;
        if (strncasecmp(a, name, len) == 0 && a[len] == '=') return a + len + 1;
    }
    return nullptr;
}

inline int flag_int(int argc, char** argv, const char* name, int def) {
    const char* v = find_flag(argc, argv, name);
    return (v && *v) ? std::atoi(v) : def;
}

inline double flag_double(int argc, char** argv, const char* name, double def) {
    const char* v = find_flag(argc, argv, name);
    return (v && *v) ? std::atof(v) : def;
}

inline std::string flag_str(int argc, char** argv, const char* name, const char* def) {
    const char* v = find_flag(argc, argv, name);
    return (v && *v) ? std::string(v) : std::string(def);
}

inline int parse_path(const std::string& s) {
    if (s == "bf16x6") return SGEMM_B200_PATH_BF16X6;
    if (s == "tf32x3") return SGEMM_B200_PATH_TF32X3;
    return SGEMM_B200_PATH_PLAIN;
}

inline int parse_dist(const std::string& s) {
    if (s == "upm1") return SGEMM_B200_DIST_UNIFORM_PM1;
    if (s == "pow2") return SGEMM_B200_DIST_SIGNED_POW2;
    return SGEMM_B200_DIST_UNIFORM_01;
}

#define HCHECK(x)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) {                                                           \
            std::fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
                         __LINE__);                                                        \
            std::exit(2);                                                                  \
        }                                                                                  \
    } while (0)

#define SCHECK(x)                                                                          \
    do {                                                                                   \
        int s_ = (x);                                                                      \
        if (s_ != SGEMM_B200_OK) {                                                         \
            std::fprintf(stderr, "sgemm_b200 error %s at %s:%d\n",                         \
                         sgemm_b200_status_string(s_), __FILE__, __LINE__);                \
            std::exit(2);                                                                  \
        }                                                                                  \
    } while (0)

// The reference's comparison (common/helper_matrix.h:51-86): elementwise
// relative error |(ref - x) / ref| <= eps, NaN and Inf in x count as failures.
struct CmpResult {
    bool equal;
    long n_false, n_inf, n_nan, n_bit_exact;
};

inline CmpResult compare_mats(const float* ref, const float* x, size_t n, float eps) {
    CmpResult r{true, 0, 0, 0, 0};
    for (size_t i = 0; i < n; ++i) {
        if (std::isnan(x[i])) {
            ++r.n_nan;
            ++r.n_false;
            continue;
        }
        if (std::isinf(x[i])) {
            ++r.n_inf;
            ++r.n_false;
            continue;
        }
        if (x[i] == ref[i]) ++r.n_bit_exact;
        if (std::fabs((ref[i] - x[i]) / ref[i]) > eps) ++r.n_false;
    }
    r.equal = r.n_false == 0;
    return r;
}

}  // namespace harness
