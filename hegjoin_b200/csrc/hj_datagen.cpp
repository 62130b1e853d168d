// hj_datagen.cpp -- seeded synthetic datasets on the host (OpenMP).
//
// The same counter-based generator as hegjoin_b200/workloads.py (Exp(rate=40)
// per coordinate, redrawn until the value cast to the dataset type is < 1),
// written in C++ so request streams of many datasets can be produced quickly.
// It stands in for the reference's generator (datasets/
// dataset_gen_fixed_len_expo_dist.cpp:24-91), keeping its distribution.  This
// file is the definition of the workloads' data: it uses only IEEE operations
// and glibc's log1p/sqrt/cos, compiled without FMA contraction, so every
// machine running this image produces the same bits.
#include <cmath>
#include <cstdint>

#include "hegjoin_datagen.h"

namespace {
constexpr uint64_t kSalt = 0xD1B54A32D192ED03ull;
inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline uint64_t stream_base(uint64_t seed, uint64_t stream) {
    return mix64(seed ^ kSalt ^ (stream * 0x632BE59BD9B4E019ull));
}
inline double uniform(uint64_t base, uint64_t i, uint32_t attempt) {
    return (double)(mix64(base + i * 64u + attempt) >> 11) * 0x1.0p-53;
}

template <typename T>
void exp40_fill(uint64_t seed, uint64_t stream, uint64_t count, T* out) {
    const uint64_t base = stream_base(seed, stream);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)count; ++i) {
        T v = T(0);
        for (uint32_t a = 0; a < 64; ++a) {
            double x = -std::log1p(-uniform(base, (uint64_t)i, a)) / 40.0;
            v = (T)x;
            if (v < T(1)) break;
        }
        out[i] = v;
    }
}

// 80% Exp(40) points, then 20% from n_clusters Gaussian clusters (sigma) with
// centres uniform in [0,1)^d, clipped to [0, 1).
template <typename T>
void skewed_fill(uint64_t seed, uint64_t n, uint32_t d, uint32_t n_clusters, double sigma, double frac, T* out) {
    const uint64_t n_c = (uint64_t)std::llround((double)n * frac);
    const uint64_t n_e = n - n_c;
    exp40_fill<T>(seed, 0, n_e * d, out);
    const uint64_t b1 = stream_base(seed, 1), b2 = stream_base(seed, 2), b3 = stream_base(seed, 3);
    const double two_pi = 6.283185307179586;
    const double top = std::nextafter(1.0, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (int64_t)n_c; ++p) {
        uint64_t cid = mix64((uint64_t)p + seed * 7919u) % n_clusters;
        for (uint32_t l = 0; l < d; ++l) {
            uint64_t idx = (uint64_t)p * d + l;
            double centre = uniform(b1, cid * d + l, 0);
            double g = std::sqrt(-2.0 * std::log1p(-uniform(b2, idx, 0))) * std::cos(two_pi * uniform(b3, idx, 0));
            double x = std::fmin(std::fmax(centre + sigma * g, 0.0), top);
            T v = (T)x;
            if (!(v < T(1))) v = std::nextafter(T(1), T(0));
            out[(n_e + p) * d + l] = v;
        }
    }
}

}  // namespace

extern "C" hj_status hj_generate_exp40(uint64_t seed, uint64_t stream, uint64_t n, uint32_t d, int dtype, void* out) {
    if (!out || d == 0) return HJ_ERR_INVALID;
    if (dtype == HJ_F32) exp40_fill<float>(seed, stream, n * d, static_cast<float*>(out));
    else exp40_fill<double>(seed, stream, n * d, static_cast<double*>(out));
    return HJ_OK;
}

extern "C" hj_status hj_generate_skewed(uint64_t seed, uint64_t n, uint32_t d, uint32_t n_clusters, double sigma,
                                        double frac_clustered, int dtype, void* out) {
    if (!out || d == 0 || n_clusters == 0) return HJ_ERR_INVALID;
    if (dtype == HJ_F32) skewed_fill<float>(seed, n, d, n_clusters, sigma, frac_clustered, static_cast<float*>(out));
    else skewed_fill<double>(seed, n, d, n_clusters, sigma, frac_clustered, static_cast<double*>(out));
    return HJ_OK;
}
