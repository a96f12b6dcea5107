// One persistent kernel per tick (B200): the bulk pass, the boundary fix-up
// and the particle update of one tick (tick!, src/gpu/fluids.jl:132-226, and
// moveParticles!, src/gpu/particles.jl:7-92) as items of one work queue.
//
// The fix-up and the particle update are latency-bound chains that move
// almost no bytes; run as separate kernels after the bulk pass they add their
// whole latency to the tick.  Here CTAs take items in queue order:
//   A  near tiles: bulk tiles within two nodes of a region the fix-up reads
//      or writes (static wall tiles, and the tile slots that cover each
//      particle's solid box grown by two nodes);
//   B  fix-up CTAs, each waiting until every A item is done (their link slots
//      and re-collided nodes lie inside the A tiles' reach);
//   C  particle updates, each waiting until every B item is done (they reduce
//      the fix-up's momentum-exchange partials);
//   D  far tiles: every other bulk tile.  A D tile neither reads nor writes a
//      node that B or C touch, so D items need no wait and the A -> B -> C
//      chain runs while the D tiles stream at memory speed.
// An item only waits for items earlier in the queue, which CTAs already hold
// and finish without waiting on later ones, so the waits always end; each
// wait is bounded anyway and reports kErrSpinTimeout if it gives up.
// Replicas of a batch simply contribute their items to the same four phases.
// The same kernel also runs subsets of the queue (only D items over every
// tile, only B items, only C items) as three launches in stream order.
//
// The particle update of tick n runs while the D tiles of tick n still test
// particle boxes, so it publishes its boxes into the other of two buffers:
// the kernel of tick n reads nbox[1 - src] and the update writes nbox[src].
#pragma once
#include "fixup.cuh"
#include "particles.cuh"

namespace lbm {

constexpr int kTickBlock = kFixBlock;  // fix-up items use the CTA as it is
constexpr long long kSpinLimit = 1LL << 22;  // polls of >= 128 ns: about a second (the largest limit)

struct TickItems {
    const int4* amap;  // {replica, kind (0 static tile, 1 particle slot), tile or particle, dy | dz << 16}
    const int2* bmap;  // {replica, fix-up block}
    const int2* cmap;  // {replica, particle}
    const int2* dmap;  // {replica, tile}
    long long na, nb, nc, nd;
    int d_test;  // 1: D items skip tiles near boundary work (A covers them); 0: D is every tile
    int wait_extra;        // added to the target of the B items' wait: 0, except in a test that makes
                           // that wait run out (a target no count reaches)
    long long spin_limit;  // polls before a wait gives up, in [1, kSpinLimit]
};

struct TickCounters {
    int next;   // next queue position
    int done;   // CTAs finished
    int cnt_a;  // A items done
    int cnt_b;  // B items done
};

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// the CTA waits (thread 0 polls, at most `limit` times) until *ctr >= target
__device__ __forceinline__ void cta_wait(const int* ctr, int target, int* err, long long limit) {
    if (threadIdx.x == 0) {
        long long it = 0;
        if (limit < 1 || limit > kSpinLimit) limit = kSpinLimit;
        while (ld_acquire_gpu(ctr) < target) {
            if (++it > limit) {
                atomicOr(err, kErrSpinTimeout);
                break;
            }
            __nanosleep(128);
        }
    }
    __syncthreads();
}

// publish a finished item: every thread's writes, then the counter
__device__ __forceinline__ void cta_done(int* ctr) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctr, 1);
    }
}

// Tile of near slot (dy, dz) of particle p: rows [lo1 - 2, hi1 + 2] and
// slices [lo2 - 2, hi2 + 2] of its published box, periodic; -1 if the slot
// lies past the box.  A y-range that wraps is covered as two segments.
template <int D>
__device__ __forceinline__ long long near_slot_tile(const StepArgs& a, int p, int dy, int dz) {
    const int* b = a.nbox + 6 * p;
    if (b[0] > b[3] || b[1] > b[4] || b[2] > b[5]) return -1;
    const int ny = a.g.n[1], nz = a.g.n[2], vr = a.vrows;
    const int leny = b[4] - b[1] + 5;
    int ty;
    if (leny >= ny) {
        if (dy >= a.vnt1) return -1;
        ty = dy;
    } else {
        const int y0 = wrap_idx(b[1] - 2, ny);
        const int e = y0 + leny;  // exclusive end, unwrapped
        const int t0 = y0 / vr, c1 = (min(e, ny) - 1) / vr - t0 + 1;
        if (dy < c1) {
            ty = t0 + dy;
        } else {
            if (e <= ny || dy - c1 >= (e - ny - 1) / vr + 1) return -1;
            ty = dy - c1;
        }
    }
    int tz = 0;
    if (D == 3) {
        const int lenz = b[5] - b[2] + 5;
        if (lenz >= nz) {
            if (dz >= nz) return -1;
            tz = dz;
        } else {
            if (dz >= lenz) return -1;
            tz = wrap_idx(b[2] - 2 + dz, nz);
        }
    } else if (dz > 0) {
        return -1;
    }
    return ty + (long long)a.vnt1 * tz;
}

template <class L, int ST, bool TRT, bool SR>
__global__ void __launch_bounds__(kTickBlock, 8) k_tick(const StepArgs* __restrict__ args,
                                                       const ParticleArgs* __restrict__ pargs, const TickItems it,
                                                       TickCounters* q, int* err) {
    constexpr int B = kTickBlock;
    __shared__ float s_ex[x_moving_dirs<L>()][B];
    __shared__ int s_next;
    const long long nab = it.na + it.nb, nabc = nab + it.nc, total = nabc + it.nd;
    if (threadIdx.x == 0) s_next = atomicAdd(&q->next, 1);
    __syncthreads();
    long long t = s_next;
    int nxt = 0;
    while (t < total) {
        // the next position is fetched now and used after this item; it is
        // later than everything this item waits for
        if (threadIdx.x == 0) nxt = atomicAdd(&q->next, 1);
        if (t < it.na) {
            const int4 m = it.amap[t];
            const StepArgs& A = args[m.x];
            const long long tile =
                m.y == 0 ? (long long)m.z : near_slot_tile<L::D>(A, m.z, m.w & 0xffff, m.w >> 16);
            if (tile >= 0) bulk_v4_tile<L, ST, TRT, B, SR>(A, tile, s_ex);
            cta_done(&q->cnt_a);
        } else if (t < nab) {
            cta_wait(&q->cnt_a, (int)it.na + it.wait_extra, err, it.spin_limit);
            const int2 m = it.bmap[t - it.na];
            fixup_body<L, ST, TRT, kTickBlock>(args[m.x], m.y);
            cta_done(&q->cnt_b);
        } else if (t < nabc) {
            cta_wait(&q->cnt_b, (int)it.nb, err, it.spin_limit);
            const int2 m = it.cmap[t - nab];
            particles_body<L, 128>(pargs[m.x], m.y);
        } else {
            const int2 m = it.dmap[t - nabc];
            const StepArgs& A = args[m.x];
            bool skip = false;
            if (it.d_test) {
                bool nr = threadIdx.x == 0 && A.vnear && A.vnear[m.y];
                for (int p = threadIdx.x; p < A.nparts; p += B) nr = nr || tile_meets_box<L::D>(A, m.y, p);
                skip = __syncthreads_or(nr);
            }
            if (!skip) bulk_v4_tile<L, ST, TRT, B, SR>(A, m.y, s_ex);
        }
        if (threadIdx.x == 0) s_next = nxt;
        __syncthreads();
        t = s_next;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&q->done, 1) == (int)gridDim.x - 1) {  // last CTA: reset for the next tick
            q->next = 0;
            q->done = 0;
            q->cnt_a = 0;
            q->cnt_b = 0;
            __threadfence();
        }
    }
}

// The bulk tiles of a batch, one CTA per item of the D map (no queue): the
// replicas' arguments come from `args[dmap[i].x]`.
template <class L, int ST, bool TRT, bool SR>
__global__ void __launch_bounds__(kTickBlock, bulk_threads_per_sm<L, ST, SR>() / kTickBlock)
    k_bulk_batch(const StepArgs* __restrict__ args, const int2* __restrict__ dmap, int reverse) {
    __shared__ float s_ex[x_moving_dirs<L>()][kTickBlock];
    // every other tick the map is walked last to first (see k_bulk_v4)
    const int2 m = dmap[reverse ? gridDim.x - 1 - blockIdx.x : blockIdx.x];
    bulk_v4_tile<L, ST, TRT, kTickBlock, SR>(args[m.x], m.y, s_ex);
}

}  // namespace lbm
