// Population storage codecs.
//
// Populations are stored shifted and weight-normalised:
//     g_i = (f_i / w_i - rho0) * scale
// so that the stored numbers are O(|u|) instead of O(w_i).  1/w_i is exact
// for every velocity set, bounce-back keeps its meaning (w_i == w_opp(i)),
// and the collision is done on g directly (no cancellation against w_i*rho0).
// FP16/BF16 use a power-of-two scale; FP32/FP64 use scale 1.
#pragma once
#include <cuda_fp16.h>
#include <cuda_bf16.h>

namespace lbm {

// Rounding of the 2-byte formats.  Rounding to nearest gives every node of a
// uniform region the same error in every tick, and those errors add up: a
// uniformly forced fluid stored as FP16 drifts by ~1e-3 of its velocity over
// a few hundred ticks.  The stores of the tick therefore round
// stochastically: the fraction below the kept bits is rounded up when it
// exceeds a dither drawn from a hash of the destination cell, the direction
// and the kept bits themselves.  Over the nodes of a flow the dithers are
// uniform, so the rounding errors have zero mean and no longer add up
// coherently; the dither is a pure function of (cell, direction, value), so
// every launch path gives bit-identical results.
constexpr unsigned kDitherCell = 0x85EBCA77u;

// odd multiplier of direction `dir`, cell `k` (0..3) of an aligned group of four
__host__ __device__ __forceinline__ constexpr unsigned dither_mul(int dir, int k) {
    return 0x9E3779B1u + (unsigned)(4 * dir + k) * 0x632BE5A6u;
}

// v with its low DROP bits rounded away stochastically (DROP = 13: the kept
// bits are exactly an IEEE half in its normal range; 16: a bfloat16)
template <int DROP>
__device__ __forceinline__ float round_dither(float v, unsigned key, unsigned mul) {
    constexpr unsigned M = ~((1u << DROP) - 1u);
    const unsigned b = __float_as_uint(v);
    const unsigned h = ((b & M) ^ key) * mul;
    return __uint_as_float((b + (h >> (32 - DROP))) & M);
}

enum StoreKind { ST_F32 = 0, ST_F16 = 1, ST_BF16 = 2, ST_F64 = 3 };

template <int S> struct Store;

template <> struct Store<ST_F32> {
    using T = float;   // stored type
    using R = float;   // arithmetic type of the collision
    static __device__ __forceinline__ R dec(T v, R) { return v; }
    static __device__ __forceinline__ T enc(R v, R) { return v; }
    static __device__ __forceinline__ T enc_sr(R v, R, unsigned, int) { return v; }
    static constexpr int bytes = 4;
};
template <> struct Store<ST_F64> {
    using T = double;
    using R = double;
    static __device__ __forceinline__ R dec(T v, R) { return v; }
    static __device__ __forceinline__ T enc(R v, R) { return v; }
    static __device__ __forceinline__ T enc_sr(R v, R, unsigned, int) { return v; }
    static constexpr int bytes = 8;
};
template <> struct Store<ST_F16> {
    using T = __half;
    using R = float;
    static __device__ __forceinline__ R dec(T v, R inv_scale) { return __half2float(v) * inv_scale; }
    static __device__ __forceinline__ T enc(R v, R scale) { return __float2half_rn(v * scale); }
    // stochastic rounding of a value stored at (cell, dir) of the tick
    static __device__ __forceinline__ T enc_sr(R v, R scale, unsigned cell, int dir) {
        return __float2half_rn(round_dither<13>(v * scale, (cell & ~3u) * kDitherCell, dither_mul(dir, cell & 3u)));
    }
    static constexpr int bytes = 2;
};
template <> struct Store<ST_BF16> {
    using T = __nv_bfloat16;
    using R = float;
    static __device__ __forceinline__ R dec(T v, R inv_scale) { return __bfloat162float(v) * inv_scale; }
    static __device__ __forceinline__ T enc(R v, R scale) { return __float2bfloat16_rn(v * scale); }
    static __device__ __forceinline__ T enc_sr(R v, R scale, unsigned cell, int dir) {
        return __float2bfloat16_rn(
            round_dither<16>(v * scale, (cell & ~3u) * kDitherCell, dither_mul(dir, cell & 3u)));
    }
    static constexpr int bytes = 2;
};

}  // namespace lbm
