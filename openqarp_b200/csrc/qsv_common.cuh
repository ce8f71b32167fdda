// qsv_common.cuh — shared device/host definitions of the B200 statevector engine.
//
// Amplitudes live in HBM as interleaved complex: double2 (complex128) or float2
// (complex64 bulk mode).  Index bit q is qubit q (LSB-first), the reference's convention
// (docs/contracts/qarp_conventions.md:42-49).  Every reduction accumulates in FP64
// whatever the storage type.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace qsv {

// ------------------------------------------------------------------ complex helpers
template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };
template <typename T> using vec2_t = typename Vec2<T>::type;

// A complex coefficient as passed to kernels (always the storage precision).
template <typename T> struct cplx { T re, im; };

template <typename T>
__host__ __device__ __forceinline__ vec2_t<T> mk(T re, T im) {
    vec2_t<T> v; v.x = re; v.y = im; return v;
}

// a * b
template <typename T>
__device__ __forceinline__ vec2_t<T> cmul(cplx<T> a, vec2_t<T> b) {
    return mk<T>(a.re * b.x - a.im * b.y, a.re * b.y + a.im * b.x);
}
// acc + a * b
template <typename T>
__device__ __forceinline__ vec2_t<T> cfma(cplx<T> a, vec2_t<T> b, vec2_t<T> acc) {
    acc.x = fma(a.re, b.x, acc.x);
    acc.x = fma(-a.im, b.y, acc.x);
    acc.y = fma(a.re, b.y, acc.y);
    acc.y = fma(a.im, b.x, acc.y);
    return acc;
}

// FP64 complex accumulator used by every reduction.
struct dcplx { double re, im; };

__device__ __forceinline__ void dacc_conj_mul(dcplx& acc, double ar, double ai, double br, double bi) {
    // acc += conj(a) * b
    acc.re = fma(ar, br, acc.re);
    acc.re = fma(ai, bi, acc.re);
    acc.im = fma(ar, bi, acc.im);
    acc.im = fma(-ai, br, acc.im);
}

// ------------------------------------------------------------------ index helpers
// Insert a zero bit at each of the `k` ascending positions `pos[0..k)`.
__device__ __forceinline__ uint64_t insert_zeros(uint64_t g, const uint8_t* pos, int k) {
#pragma unroll 8
    for (int b = 0; b < 8; ++b) {
        if (b >= k) break;
        const uint64_t p = pos[b];
        const uint64_t low = g & ((1ull << p) - 1ull);
        g = ((g >> p) << (p + 1)) | low;
    }
    return g;
}

// Insert a one bit at each ascending position.
__device__ __forceinline__ uint64_t insert_ones(uint64_t g, const uint8_t* pos, int k) {
#pragma unroll 8
    for (int b = 0; b < 8; ++b) {
        if (b >= k) break;
        const uint64_t p = pos[b];
        const uint64_t low = g & ((1ull << p) - 1ull);
        g = ((g >> p) << (p + 1)) | (1ull << p) | low;
    }
    return g;
}

// ------------------------------------------------------------------ launch geometry
constexpr int kThreads = 256;
int sm_count(int device);
// grid for `work` items with `per_thread` items per thread, capped for grid-stride loops
inline unsigned grid_for(uint64_t work, int per_thread = 1, unsigned cap = 1u << 30) {
    uint64_t threads = (work + per_thread - 1) / per_thread;
    uint64_t blocks = (threads + kThreads - 1) / kThreads;
    if (blocks < 1) blocks = 1;
    if (blocks > cap) blocks = cap;
    return static_cast<unsigned>(blocks);
}

}  // namespace qsv

#include "debug_bounds.cuh"
