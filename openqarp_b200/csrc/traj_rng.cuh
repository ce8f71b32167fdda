// traj_rng.cuh — the per-shot random streams of the trajectory path, restated for the device.
//
// Shot s of the reference's trajectory loop draws from std::mt19937(seed + s)
// (qarp_simulator.cpp:1150), through std::uniform_real_distribution<double>(0, 1) for
// measurements, the final sample and noise channels, and through
// std::uniform_int_distribution<uint64_t> for the k-qubit depolarizing string
// (noise_model.cpp:115-121).  The engine keeps one MT19937 state per shot in device memory and
// draws exactly what the reference's shot draws, in the same order:
//   * MT19937: Matsumoto & Nishimura (1998), 32-bit parameters (n = 624, m = 397,
//     a = 0x9908b0df, tempering (11, 7/0x9d2c5680, 15/0xefc60000, 18)), seeding
//     x_i = 1812433253 (x_{i-1} ^ (x_{i-1} >> 30)) + i, first output after one full twist;
//   * generate_canonical<double, 53> over a 32-bit engine: two outputs w0, w1, the 64-bit
//     integer w0 + 2^32 w1 rounded once to double, times 2^-64, and 1 - 2^-53 when that
//     rounds up to 1;
//   * uniform integers in [0, range) for range <= 2^32: Lemire's multiply-and-reject method
//     (ACM TOMACS 29(1), 2019), one 32 x 32 -> 64-bit product per draw, redrawn while the low
//     word is below (2^32 - range) mod range; wider ranges compose a high word drawn that way
//     with one raw output, rejecting results above the range.
// The state is stored shot-minor (word i of shot s at i * stride + s) so that a warp of shots
// reads and twists consecutive words.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define QSV_HD __host__ __device__ __forceinline__
#else
#define QSV_HD inline
#endif

namespace qsv {

constexpr int kMtN = 624;
constexpr int kMtM = 397;

// A view of one shot's engine inside the shot-minor state array.
struct MtView {
    uint32_t* w;          // word i at w[i * stride]
    uint64_t stride;
    uint32_t* idx;        // next word to temper (kMtN: twist first)

    QSV_HD uint32_t& at(int i) const { return w[static_cast<uint64_t>(i) * stride]; }

    QSV_HD void seed(uint32_t s) const {
        uint32_t x = s;
        at(0) = x;
        for (int i = 1; i < kMtN; ++i) {
            x = 1812433253u * (x ^ (x >> 30)) + static_cast<uint32_t>(i);
            at(i) = x;
        }
        *idx = kMtN;
    }

    QSV_HD void twist() const {
        constexpr uint32_t upper = 0x80000000u, lower = 0x7fffffffu, a = 0x9908b0dfu;
        for (int k = 0; k < kMtN - kMtM; ++k) {
            const uint32_t y = (at(k) & upper) | (at(k + 1) & lower);
            at(k) = at(k + kMtM) ^ (y >> 1) ^ ((y & 1u) ? a : 0u);
        }
        for (int k = kMtN - kMtM; k < kMtN - 1; ++k) {
            const uint32_t y = (at(k) & upper) | (at(k + 1) & lower);
            at(k) = at(k + kMtM - kMtN) ^ (y >> 1) ^ ((y & 1u) ? a : 0u);
        }
        const uint32_t y = (at(kMtN - 1) & upper) | (at(0) & lower);
        at(kMtN - 1) = at(kMtM - 1) ^ (y >> 1) ^ ((y & 1u) ? a : 0u);
        *idx = 0;
    }

    QSV_HD uint32_t next() const {
        if (*idx >= static_cast<uint32_t>(kMtN)) twist();
        uint32_t y = at(static_cast<int>((*idx)++));
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        return y;
    }

    // std::uniform_real_distribution<double>(0, 1) over std::mt19937
    QSV_HD double canonical() const {
        const uint64_t w0 = next();
        const uint64_t w1 = next();
        const uint64_t v = w0 | (w1 << 32);
#ifdef __CUDA_ARCH__
        const double d = __ull2double_rn(v);
#else
        const double d = static_cast<double>(v);   // round to nearest, as the library's sum
#endif
        const double u = d * 0x1p-64;
        return u >= 1.0 ? 0x1.fffffffffffffp-1 : u;
    }

    // uniform integer in [0, range), 1 <= range <= 2^32
    QSV_HD uint64_t below32(uint64_t range) const {
        const uint32_t r32 = static_cast<uint32_t>(range);   // 2^32 wraps to 0: raw output
        if (r32 == 0) return next();
        uint64_t product = static_cast<uint64_t>(next()) * r32;
        uint32_t low = static_cast<uint32_t>(product);
        if (low < r32) {
            const uint32_t threshold = (0u - r32) % r32;
            while (low < threshold) {
                product = static_cast<uint64_t>(next()) * r32;
                low = static_cast<uint32_t>(product);
            }
        }
        return product >> 32;
    }

    // std::uniform_int_distribution<uint64_t>(lo, hi) over std::mt19937, hi - lo < 2^62
    QSV_HD uint64_t uniform(uint64_t lo, uint64_t hi) const {
        const uint64_t urange = hi - lo;
        if (urange < 0xffffffffull) return lo + below32(urange + 1);
        if (urange == 0xffffffffull) return lo + next();
        uint64_t ret, tmp;
        do {
            tmp = below32((urange >> 32) + 1) << 32;
            ret = tmp + next();
        } while (ret > urange || ret < tmp);
        return lo + ret;
    }
};

}  // namespace qsv
