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

enum StoreKind { ST_F32 = 0, ST_F16 = 1, ST_BF16 = 2, ST_F64 = 3 };

template <int S> struct Store;

template <> struct Store<ST_F32> {
    using T = float;   // stored type
    using R = float;   // arithmetic type of the collision
    static __device__ __forceinline__ R dec(T v, R) { return v; }
    static __device__ __forceinline__ T enc(R v, R) { return v; }
    static constexpr int bytes = 4;
};
template <> struct Store<ST_F64> {
    using T = double;
    using R = double;
    static __device__ __forceinline__ R dec(T v, R) { return v; }
    static __device__ __forceinline__ T enc(R v, R) { return v; }
    static constexpr int bytes = 8;
};
template <> struct Store<ST_F16> {
    using T = __half;
    using R = float;
    static __device__ __forceinline__ R dec(T v, R inv_scale) { return __half2float(v) * inv_scale; }
    static __device__ __forceinline__ T enc(R v, R scale) { return __float2half_rn(v * scale); }
    static constexpr int bytes = 2;
};
template <> struct Store<ST_BF16> {
    using T = __nv_bfloat16;
    using R = float;
    static __device__ __forceinline__ R dec(T v, R inv_scale) { return __bfloat162float(v) * inv_scale; }
    static __device__ __forceinline__ T enc(R v, R scale) { return __float2bfloat16_rn(v * scale); }
    static constexpr int bytes = 2;
};

}  // namespace lbm
