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

// Random bits of a thread's group of four cells (the vector bulk kernels):
// one well-mixed 32-bit word from the group's first cell and the kept bits of
// three of its post-collision values (which change from tick to tick as the
// flow evolves), spread into four independent 32-bit words (rs_words).  The
// pair of cells (2p, 2p+1) of direction i is converted by the hardware's
// stochastic-rounding conversion (cvt.rs) with word (i + 2p) mod 4 as its
// random bits.  For every (p, i) the word is uniform over the nodes of a flow,
// so the rounding is unbiased, at one instruction per two values.
__device__ __forceinline__ unsigned group_dither(int cell0, float v1, float v2, float v3) {
    unsigned x = ((__float_as_uint(v1) ^ __float_as_uint(v2) ^ __float_as_uint(v3)) & 0xFFFFE000u) ^
                 ((unsigned)cell0 * kDitherCell);
    x *= 0x9E3779B1u;
    x ^= x >> 15;
    x *= 0x2C1B3C6Du;
    x ^= x >> 13;
    return x;
}

// four independent 32-bit words from a group's word (multiply-xorshift steps)
__device__ __forceinline__ void rs_words(unsigned x, unsigned* w) {
    unsigned y = x * 0x85EBCA6Bu;
    y ^= y >> 13;
    unsigned z = y * 0xC2B2AE35u;
    z ^= z >> 16;
    unsigned u = z * 0x27D4EB2Fu;
    u ^= u >> 15;
    w[0] = x;
    w[1] = y;
    w[2] = z;
    w[3] = u;
}

// two floats to a packed half2 / bfloat162 (lo in the low half), rounded
// stochastically by the conversion with the random bits `rbits` (sm_100a);
// finite values saturate at the largest finite value, as rounding toward
// zero does
__device__ __forceinline__ unsigned pack_half2_rs(float lo, float hi, unsigned rbits) {
    unsigned r;
    asm("cvt.rs.satfinite.f16x2.f32 %0, %1, %2, %3;" : "=r"(r) : "f"(hi), "f"(lo), "r"(rbits));
    return r;
}
__device__ __forceinline__ unsigned pack_bf162_rs(float lo, float hi, unsigned rbits) {
    unsigned r;
    asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(r) : "f"(hi), "f"(lo), "r"(rbits));
    return r;
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
    static constexpr int drop = 0;
};
template <> struct Store<ST_F64> {
    using T = double;
    using R = double;
    static __device__ __forceinline__ R dec(T v, R) { return v; }
    static __device__ __forceinline__ T enc(R v, R) { return v; }
    static __device__ __forceinline__ T enc_sr(R v, R, unsigned, int) { return v; }
    static constexpr int bytes = 8;
    static constexpr int drop = 0;
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
    static constexpr int drop = 13;  // FP32 mantissa bits below an IEEE half's
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
    static constexpr int drop = 16;  // FP32 mantissa bits below a bfloat16's
};

}  // namespace lbm
