// Bulk stream-collide pass with its loads on the Tensor Memory Accelerator.
//
// The vector bulk kernel (k_bulk_v4, kernels.cuh) loads its populations with
// ordinary vector loads: a warp has one batch of loads in flight, then
// collides, then stores, so the bytes in flight per SM depend on how many
// warps happen to be between their loads and their collision.  Here the loads
// are taken off the warps: persistent CTAs walk their tiles (blocks of whole
// x-rows of one z-slice) through a ring of `stages` shared-memory buffers.
// One thread issues, per tile, one 1-D bulk copy (cp.async.bulk) per
// population plane -- the tile's rows are contiguous in every plane of the
// [Q][z][y][x] layout -- that completes on the stage's mbarrier; the warps
// read the stage, release it (the next tile's copies go out at once) and
// collide while the copies of the following stages are in flight.  So the
// memory system always holds the next stages' loads, whatever the warps do.
//
// The arithmetic is that of bulk_v4_tile: four consecutive x-nodes per
// thread, the same collide() on the same values, the same pushes with
// streaming vector stores; results are bit-identical.  The value that leaves
// a thread's 4-node segment along +-x goes to its neighbour by a warp shuffle
// (a row is RT = nx/4 consecutive lanes, RT a power of two up to 32, so the
// periodic x-wrap is the shuffle's wrap inside its segment).
//
// Every mbarrier wait is bounded; a wait that gives up sets kErrSpinTimeout,
// the CTA stops, waits (bounded again) for the copies it has in flight and
// returns.  Only this GPU's own population buffers are read; no multicast.
#pragma once
#include "kernels.cuh"

namespace lbm {

constexpr int kTmaMaxStages = 4;
constexpr long long kTmaWaitLimit = 1LL << 22;  // try_wait polls per stage (each may suspend briefly)

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned phase) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// wait for the phase `phase` of `bar` to complete, at most kTmaWaitLimit polls
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned phase) {
    for (long long it = 0; it < kTmaWaitLimit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

// L2 policy for data read once per pass: evict first
__device__ __forceinline__ unsigned long long policy_evict_first() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`
// (addresses 16-byte aligned, size a multiple of 16: checked by the host)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar,
                                          unsigned long long policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}

// four consecutive stored populations from shared memory, as floats
template <int ST> struct SmemVec4;
template <> struct SmemVec4<ST_F32> {
    static __device__ __forceinline__ void load(const void* p, float* v) {
        const float4 q = *reinterpret_cast<const float4*>(p);
        v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    }
};
template <> struct SmemVec4<ST_F16> {
    static __device__ __forceinline__ void load(const void* p, float* v) {
        const uint2 q = *reinterpret_cast<const uint2*>(p);
        const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&q.x));
        const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&q.y));
        v[0] = lo.x; v[1] = lo.y; v[2] = hi.x; v[3] = hi.y;
    }
};
template <> struct SmemVec4<ST_BF16> {
    static __device__ __forceinline__ void load(const void* p, float* v) {
        const uint2 q = *reinterpret_cast<const uint2*>(p);
        const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&q.x));
        const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&q.y));
        v[0] = lo.x; v[1] = lo.y; v[2] = hi.x; v[3] = hi.y;
    }
};

// Shape of a TMA bulk launch (chosen by the host).
struct TmaShape {
    int rows;      // x-rows per tile (threads = rows * nx / 4)
    int stages;    // shared-memory buffers in the ring (2 .. kTmaMaxStages)
    int grid;      // persistent CTAs
    int smem;      // dynamic shared memory bytes
};

// dynamic shared memory of a launch: stages x Q planes x rows x nx values, then the mbarriers
inline int tma_smem_bytes(int q, int nx, int rows, int stages, int esz) {
    const size_t data = (size_t)stages * q * rows * nx * esz;
    return (int)(((data + 15) / 16) * 16 + 8 * kTmaMaxStages);
}

template <class L, int ST, bool TRT, bool SR>
__global__ void __launch_bounds__(512, 1) k_bulk_tma(const StepArgs a, const int rows_max, const int stages) {
    extern __shared__ __align__(128) unsigned char smem[];
    using T = typename Store<ST>::T;
    using R = float;
    constexpr int Q = L::Q;
    constexpr int esz = (int)sizeof(T);
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int RT = nx >> 2;  // threads per x-row, a power of two <= 32
    const int tid = threadIdx.x;
    const int row = tid / RT, j = tid - row * RT;
    const int nyb = (ny + rows_max - 1) / rows_max;
    const long long tiles = (long long)nyb * nz;
    const size_t slot = (size_t)rows_max * nx;  // values per plane in a stage
    const size_t stage_vals = slot * Q;
    T* ring = reinterpret_cast<T*>(smem);
    unsigned long long* bars =
        reinterpret_cast<unsigned long long*>(smem + ((stage_vals * stages * esz + 15) / 16) * 16);
    const long long G = gridDim.x;
    const long long t0 = blockIdx.x;
    if (tid == 0) {
        for (int s = 0; s < stages; ++s) mbar_init(&bars[s], 1);
        mbar_init_fence();
    }
    __syncthreads();
    const unsigned long long pol = policy_evict_first();
    // copies of tile t into stage s (thread 0)
    auto issue = [&](long long t, int s) {
        const int z = (int)(t / nyb), y0 = (int)(t - (long long)z * nyb) * rows_max;
        const int rows = min(rows_max, ny - y0);
        const unsigned bytes = (unsigned)(rows * nx * esz);
        mbar_expect_tx(&bars[s], bytes * Q);
        const long long off = ((long long)z * ny + y0) * nx;
        T* dst = ring + s * stage_vals;
#pragma unroll
        for (int i = 0; i < Q; ++i)
            bulk_load(dst + i * slot, static_cast<const T*>(a.srcq[i]) + off, bytes, &bars[s], pol);
    };
    if (tid == 0)
        for (int s = 0; s < stages; ++s)
            if (t0 + s * G < tiles) issue(t0 + s * G, s);
    const R Fx = a.kf.F[0], Fy = a.kf.F[1], Fz = a.kf.F[2];
    const unsigned lanes = 0xffffffffu;
    long long k = 0;
    bool aborted = false;
    for (long long t = t0; t < tiles; t += G, ++k) {
        const int s = (int)(k % stages);
        const unsigned phase = (unsigned)((k / stages) & 1);
        if (t + G >= tiles) grid_dep_trigger();  // last tile: the fix-up may start its stores-free part
        const bool ok = mbar_wait_bounded(&bars[s], phase);
        const int z = (int)(t / nyb), y0 = (int)(t - (long long)z * nyb) * rows_max;
        const int y = y0 + row;
        const bool valid = ok && row < rows_max && y < ny;
        const int x0 = 4 * j;
        R g[4][Q];
        const T* st = ring + s * stage_vals + (size_t)row * nx + x0;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            R v[4] = {0, 0, 0, 0};
            if (valid) SmemVec4<ST>::load(st + i * slot, v);
            g[0][i] = v[0];
            g[1][i] = v[1];
            g[2][i] = v[2];
            g[3][i] = v[3];
        }
        // every thread has read stage s: refill it (or stop if a wait gave up)
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(a.err, kErrSpinTimeout);
            aborted = true;
            break;
        }
        if (tid == 0 && t + stages * G < tiles) issue(t + stages * G, s);
        bool bad = false;
#pragma unroll
        for (int c = 0; c < 4; ++c) bad |= bad_density(collide<L, R, TRT>(a, g[c], Fx, Fy, Fz, false));
        report_density(valid && bad, a.err);
        constexpr bool sr = SR && Store<ST>::bytes == 2;
        unsigned dw[4];
        if (sr) rs_words(group_dither((int)(x0 + nx * (y + (long long)ny * z)), g[0][1], g[0][2],
                                                           g[0][3]), dw);
        const unsigned* dither = sr ? dw : nullptr;
        const int ys[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
        const int zs[3] = {z == 0 ? nz - 1 : z - 1, z, z == nz - 1 ? 0 : z + 1};
        const int left = (j + RT - 1) & (RT - 1), right = (j + 1) & (RT - 1);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int tq = x0 + nx * (ys[L::cy(i) + 1] + ny * zs[L::cz(i) + 1]);
            if (L::cx(i) == 0) {
                if (valid) Vec4<ST>::store(a.dstq[i], tq, i, g[0][i], g[1][i], g[2][i], g[3][i], dither);
            } else if (L::cx(i) == 1) {
                const R in = __shfl_sync(lanes, g[3][i], left, RT);
                if (valid) Vec4<ST>::store(a.dstq[i], tq, i, in, g[0][i], g[1][i], g[2][i], dither);
            } else {
                const R in = __shfl_sync(lanes, g[0][i], right, RT);
                if (valid) Vec4<ST>::store(a.dstq[i], tq, i, g[1][i], g[2][i], g[3][i], in, dither);
            }
        }
    }
    if (aborted && tid == 0) {  // copies of this and the next stages may still be in flight
        for (long long kk = k; kk < k + stages; ++kk) {
            const long long t = t0 + kk * G;
            if (t < tiles) (void)mbar_wait_bounded(&bars[kk % stages], (unsigned)((kk / stages) & 1));
        }
    }
}

}  // namespace lbm
