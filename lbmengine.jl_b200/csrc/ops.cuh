// Launch table: one entry per (velocity set, storage, collision) instantiation.
#pragma once
#include <cuda_runtime.h>
#include "kernels.cuh"
#include "bulk_tma.cuh"
#include "fixup.cuh"
#include "particles.cuh"
#include "aux_kernels.cuh"
#include "tick.cuh"
#include "adjoint.cuh"

namespace lbm {

struct Ops {
    void (*bulk)(const StepArgs&, unsigned grid, dim3 block, cudaStream_t);
    // early: launch with programmatic stream serialization (the fix-up may
    // start while the kernel before it in the stream still runs)
    // walk: the chunk-walking kernel (k_fixup_walk), whose grid is fixup_walk_grid
    void (*fixup)(const StepArgs&, unsigned grid, cudaStream_t, bool early, bool walk);
    void (*particles)(const ParticleArgs&, unsigned grid, cudaStream_t);
    // link-list rebuild of flagged particles: two passes of blocks_per_particle
    // CTAs per particle; counts holds nparts * blocks_per_particle ints
    void (*links)(const ParticleArgs&, int nparts, int blocks_per_particle, int* counts, cudaStream_t);
    void (*encode)(const CodecArgs&, cudaStream_t);
    void (*decode)(const CodecArgs&, cudaStream_t);
    void (*macro)(const CodecArgs&, cudaStream_t);
    void (*stress)(const CodecArgs&, cudaStream_t);
    // global FP64 sums: rho and rho u into out[4] (part: one slot of 4 per kTotBlock cells)
    void (*totals)(const CodecArgs&, double* part, double* out, cudaStream_t);
    void (*init)(const InitArgs&, cudaStream_t);
    void (*mask)(const MaskArgs&, cudaStream_t);
    // vector bulk pass over all tiles, CTAs of `block` threads (64..512); null for FP64
    void (*bulk_v4)(const StepArgs&, long long tiles, int block, cudaStream_t);
    // the same pass with TMA bulk loads through a shared-memory ring (bulk_tma.cuh); null for FP64
    void (*bulk_tma)(const StepArgs&, const TmaShape&, cudaStream_t);
    // one persistent kernel per tick over the A/B/C/D item queue (tick.cuh);
    // sr: the 2-byte stores round stochastically
    void (*tick)(const StepArgs* args, const ParticleArgs* pargs, const TickItems& items, TickCounters* q,
                 int* err, unsigned grid, cudaStream_t, bool sr);
    // a batch's bulk tiles, one CTA per entry of dmap
    void (*bulk_batch)(const StepArgs* args, const int2* dmap, long long tiles, cudaStream_t, bool sr, bool reverse);
    // discrete adjoint of one tick, and of the initial condition (adjoint.cuh)
    void (*adjoint)(const AdjArgs&, cudaStream_t);
    void (*adjoint_init)(const AdjArgs&, cudaStream_t);
    const void* bulk_fn;      // kernel symbols (occupancy queries, attributes)
    const void* bulk_tma_fn;
    const void* fixup_fn;
    const void* tick_fn;      // the round-to-nearest variants (occupancy queries)
    const void* tick_fn_sr;   // the stochastic-rounding variant
    const void* bulk_tma_fn_sr;
};

constexpr int kBulkBlocks[5] = {64, 96, 128, 256, 512};  // CTA sizes of the vector bulk kernel (and 32 on request)

inline unsigned blocks_for(long long n, int b) { return (unsigned)((n + b - 1) / b); }

template <class L, int ST, bool TRT>
struct OpsImpl {
    static void bulk(const StepArgs& a, unsigned grid, dim3 block, cudaStream_t s) {
        k_bulk<L, ST, TRT><<<grid, block, 0, s>>>(a);
    }
    static void fixup(const StepArgs& a, unsigned grid, cudaStream_t s, bool early, bool walk) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(kFixThreads);
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = early ? 1 : 0;
        if (walk) cudaLaunchKernelEx(&cfg, k_fixup_walk<L, ST, TRT>, a);
        else cudaLaunchKernelEx(&cfg, k_fixup<L, ST, TRT>, a);
    }
    static void particles(const ParticleArgs& a, unsigned grid, cudaStream_t s) {
        k_particles<L><<<grid, kPartBlock, 0, s>>>(a);
    }
    static void links(const ParticleArgs& a, int nparts, int bpp, int* counts, cudaStream_t s) {
        if (nparts <= 0) return;
        k_links_count<L><<<(unsigned)(nparts * bpp), kLinkBlock, 0, s>>>(a, bpp, counts);
        k_links_write<L><<<(unsigned)(nparts * bpp), kLinkBlock, 0, s>>>(a, bpp, counts);
    }
    static constexpr bool kTwo = Store<ST>::bytes == 2;  // stochastic variants exist for 2-byte storage
    template <bool SR>
    static void bulk_v4_sr(const StepArgs& a, long long tiles, int block, cudaStream_t s) {
        const unsigned g = (unsigned)tiles;
        if (block <= 32) k_bulk_v4<L, ST, TRT, 32, SR><<<g, 32, 0, s>>>(a);
        else if (block <= 64) k_bulk_v4<L, ST, TRT, 64, SR><<<g, 64, 0, s>>>(a);
        else if (block <= 96) k_bulk_v4<L, ST, TRT, 96, SR><<<g, 96, 0, s>>>(a);
        else if (block <= 128) k_bulk_v4<L, ST, TRT, 128, SR><<<g, 128, 0, s>>>(a);
        else if (block <= 256) k_bulk_v4<L, ST, TRT, 256, SR><<<g, 256, 0, s>>>(a);
        else k_bulk_v4<L, ST, TRT, 512, SR><<<g, 512, 0, s>>>(a);
    }
    static void bulk_v4(const StepArgs& a, long long tiles, int block, cudaStream_t s) {
        if constexpr (ST != ST_F64) {
            if constexpr (kTwo)
                if (a.stochastic) return bulk_v4_sr<true>(a, tiles, block, s);
            bulk_v4_sr<false>(a, tiles, block, s);
        }
    }
    static void bulk_tma(const StepArgs& a, const TmaShape& sh, cudaStream_t s) {
        if constexpr (ST != ST_F64) {
            const dim3 g((unsigned)sh.grid), b((unsigned)(sh.rows * (a.g.n[0] / 4)));
            if constexpr (kTwo)
                if (a.stochastic) {
                    k_bulk_tma<L, ST, TRT, true><<<g, b, (size_t)sh.smem, s>>>(a, sh.rows, sh.stages);
                    return;
                }
            k_bulk_tma<L, ST, TRT, false><<<g, b, (size_t)sh.smem, s>>>(a, sh.rows, sh.stages);
        }
    }
    static void tick(const StepArgs* args, const ParticleArgs* pargs, const TickItems& items, TickCounters* q,
                     int* err, unsigned grid, cudaStream_t s, bool sr) {
        if constexpr (ST != ST_F64) {
            if constexpr (kTwo)
                if (sr) {
                    k_tick<L, ST, TRT, true><<<grid, kTickBlock, 0, s>>>(args, pargs, items, q, err);
                    return;
                }
            k_tick<L, ST, TRT, false><<<grid, kTickBlock, 0, s>>>(args, pargs, items, q, err);
        }
    }
    static void bulk_batch(const StepArgs* args, const int2* dmap, long long tiles, cudaStream_t s, bool sr,
                           bool reverse) {
        if constexpr (ST != ST_F64) {
            if constexpr (kTwo)
                if (sr) {
                    k_bulk_batch<L, ST, TRT, true><<<(unsigned)tiles, kTickBlock, 0, s>>>(args, dmap, reverse ? 1 : 0);
                    return;
                }
            k_bulk_batch<L, ST, TRT, false><<<(unsigned)tiles, kTickBlock, 0, s>>>(args, dmap, reverse ? 1 : 0);
        }
    }
    static void adjoint(const AdjArgs& a, cudaStream_t s) {
        k_adjoint<L, ST, TRT><<<blocks_for(a.g.N, kAdjBlock), kAdjBlock, 0, s>>>(a);
    }
    static void adjoint_init(const AdjArgs& a, cudaStream_t s) {
        k_adjoint_init<L, ST><<<blocks_for(a.g.N, kAdjBlock), kAdjBlock, 0, s>>>(a);
    }
    static void encode(const CodecArgs& a, cudaStream_t s) { k_encode<L, ST><<<blocks_for(a.N, 256), 256, 0, s>>>(a); }
    static void decode(const CodecArgs& a, cudaStream_t s) { k_decode<L, ST><<<blocks_for(a.N, 256), 256, 0, s>>>(a); }
    static void macro(const CodecArgs& a, cudaStream_t s) { k_macro<L, ST><<<blocks_for(a.N, 256), 256, 0, s>>>(a); }
    static void stress(const CodecArgs& a, cudaStream_t s) { k_stress<L, ST><<<blocks_for(a.N, 256), 256, 0, s>>>(a); }
    static void totals(const CodecArgs& a, double* part, double* out, cudaStream_t s) {
        const unsigned nb = blocks_for(a.N, kTotBlock);
        k_totals<L, ST><<<nb, kTotBlock, 0, s>>>(a, part);
        k_totals_final<<<1, kTotBlock, 0, s>>>(part, (long long)nb, out);
    }
    static void init(const InitArgs& a, cudaStream_t s) { k_init<L, ST><<<blocks_for(a.N, 256), 256, 0, s>>>(a); }
    static void mask(const MaskArgs& a, cudaStream_t s) { k_mask<L::D><<<blocks_for(a.N, 256), 256, 0, s>>>(a); }
    static Ops make() {
        Ops o;
        o.bulk = bulk;
        o.fixup = fixup;
        o.particles = particles;
        o.links = links;
        o.encode = encode;
        o.decode = decode;
        o.macro = macro;
        o.stress = stress;
        o.totals = totals;
        o.init = init;
        o.mask = mask;
        o.bulk_v4 = ST == ST_F64 ? nullptr : bulk_v4;
        o.bulk_tma = ST == ST_F64 ? nullptr : bulk_tma;
        o.bulk_tma_fn = o.bulk_tma_fn_sr = nullptr;
        if constexpr (ST != ST_F64) {
            o.bulk_tma_fn = (const void*)k_bulk_tma<L, ST, TRT, false>;
            o.bulk_tma_fn_sr = kTwo ? (const void*)k_bulk_tma<L, ST, TRT, kTwo> : o.bulk_tma_fn;
        }
        o.tick = ST == ST_F64 ? nullptr : tick;
        o.bulk_batch = ST == ST_F64 ? nullptr : bulk_batch;
        o.adjoint = adjoint;
        o.adjoint_init = adjoint_init;
        o.bulk_fn = (const void*)k_bulk<L, ST, TRT>;
        o.fixup_fn = (const void*)k_fixup<L, ST, TRT>;
        o.tick_fn = o.tick_fn_sr = nullptr;
        if constexpr (ST != ST_F64) {
            o.tick_fn = (const void*)k_tick<L, ST, TRT, false>;
            o.tick_fn_sr = kTwo ? (const void*)k_tick<L, ST, TRT, kTwo> : o.tick_fn;
        }
        return o;
    }
};

template <class L>
bool ops_for(int storage, int trt, Ops* out) {
    switch (storage * 2 + (trt ? 1 : 0)) {
        case ST_F32 * 2: *out = OpsImpl<L, ST_F32, false>::make(); return true;
        case ST_F32 * 2 + 1: *out = OpsImpl<L, ST_F32, true>::make(); return true;
        case ST_F16 * 2: *out = OpsImpl<L, ST_F16, false>::make(); return true;
        case ST_F16 * 2 + 1: *out = OpsImpl<L, ST_F16, true>::make(); return true;
        case ST_BF16 * 2: *out = OpsImpl<L, ST_BF16, false>::make(); return true;
        case ST_BF16 * 2 + 1: *out = OpsImpl<L, ST_BF16, true>::make(); return true;
        case ST_F64 * 2: *out = OpsImpl<L, ST_F64, false>::make(); return true;
        case ST_F64 * 2 + 1: *out = OpsImpl<L, ST_F64, true>::make(); return true;
        default: return false;
    }
}

// defined in inst_<lattice>.cu
bool ops_d2q9(int storage, int trt, Ops* out);
bool ops_d3q15(int storage, int trt, Ops* out);
bool ops_d3q19(int storage, int trt, Ops* out);
bool ops_d3q27(int storage, int trt, Ops* out);

}  // namespace lbm
