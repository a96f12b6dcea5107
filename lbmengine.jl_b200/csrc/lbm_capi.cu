// C ABI of the B200 lattice-Boltzmann library (include/lbm_b200.h).
//
// Host side of the drop-in boundary: validates the resolved modelInit /
// addSquirmer! keyword sets, owns all device memory of a model, and runs
// LBMpropagate! as CUDA-graph replays of the tick
//     k_tick (one persistent kernel: bulk, fix-up and particle update items)
// or, where it does not apply, k_bulk(_v4) -> k_fixup on the main stream with
// k_particles on a side stream (see enqueue_tick).
#include "lbm_b200.h"
#include "ops.cuh"
#include "interactions.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <charconv>
#include <chrono>
#include <thread>
#include <unordered_map>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

using namespace lbm;

namespace {

thread_local std::string g_global_err;

const char* kBuildInfo =
    "lbm_b200: sm_100a vectorised push collide-stream (BGK/TRT + Guo), boundary-link fix-up "
    "(halfway bounce-back, moving walls, Ladd squirmers); storage f32/f16/bf16/f64";

struct Graph {
    cudaGraphExec_t exec = nullptr;
};

constexpr int kGraphSteps = 16;  // ticks per CUDA graph of a batch
// Ticks per CUDA graph of one model, longest first: a call of n ticks replays
// the longest graphs that fit, so every tick count runs from graphs.  Each
// graph ends by joining the side stream (the last particle update), a bubble
// that longer graphs amortise.
constexpr int kModelGraphSizes[4] = {64, 16, 4, 1};
constexpr int kModelGraphTicks = kModelGraphSizes[0];
// A model's first lbm_step call of at most this many ticks launches them one
// by one instead of building the graphs it would need: on the 128^3 D3Q19
// model building the 16- and 4-tick graphs takes about 1.4 ms, and a tick
// launched alone costs about 10 us more than one replayed in a graph.
// Later calls build and replay graphs.
constexpr int kFirstCallDirectTicks = 32;
static_assert(kFirstCallDirectTicks <= kModelGraphTicks, "profiling slots");

}  // namespace

struct lbm_handle {
    // configuration
    int device = 0;
    int dims = 0, q = 0, lattice = 0, storage = 0, trt = 0;
    int schedule = 0;  // LBM_SCHEDULE_* (resolved: never AUTO)
    int n[3] = {1, 1, 1};
    long long N = 0;
    GridDesc g{};
    double dx = 1, dt = 1, tau = 1, tau_minus = 1;
    double rho0 = 1, scale = 1;
    int force_mode = 0;
    int particle_rules = LBM_RULES_GPU_MODULE;
    int rounding = LBM_ROUND_STOCHASTIC;
    double F[3] = {0, 0, 0};
    int incompressible = 0;
    double rho_inc = 1;
    bool has_walls = false;
    std::vector<double> X[3];
    Ops ops{};
    // device state: the main stream and a side stream for the particle update
    cudaStream_t stream = nullptr, side = nullptr;
    cudaEvent_t ev_fix = nullptr, ev_part = nullptr;
    bool part_pending = false;
    // vector bulk pass: tiles of vrows full x-rows, vblock threads per tile
    int vrows = 0, vnt1 = 0, vblock = 0;
    // TMA bulk pass (bulk_tma.cuh): its launch shape, valid when tma_ok
    int bulk_kind = LBM_BULK_AUTO;
    bool in_batch = false;  // a replica of an lbm_batch: its tiles belong to the batch's queue
    TmaShape tma{};
    bool tma_ok = false;
    long long vtiles = 0;
    std::vector<unsigned char> vnear;  // static near flags of the tiles (walls)
    unsigned char* d_vnear = nullptr;
    int* d_nbox[2] = {nullptr, nullptr};  // published solid boxes, [pcap][6] each
    // persistent tick kernel: item maps, per-parity arguments, queue counters
    bool tick_ready = false;
    unsigned tick_grid = 0;
    TickItems items{};
    int4* d_amap = nullptr;
    int2 *d_bmap = nullptr, *d_cmap = nullptr, *d_dmap = nullptr;
    StepArgs* d_targs = nullptr;      // [2]: by source buffer
    ParticleArgs* d_pargs = nullptr;  // [2]
    TickCounters* d_tq = nullptr;
    long long spin_limit = kSpinLimit;  // polls before a wait of the tick kernel gives up
    int wait_extra = 0;                 // test knob: added to the fix-up items' wait target
    void* pop[2] = {nullptr, nullptr};
    int cur = 0;
    double* d_coord[3] = {nullptr, nullptr, nullptr};
    unsigned char* d_wall = nullptr;
    double* d_uw = nullptr;
    double* d_ffield = nullptr;
    int2* d_wlinks = nullptr;   // static wall-link entries (cell, mask)
    int* d_wnodes = nullptr;    // static wall nodes
    int nwlinks = 0, nwnodes = 0;
    unsigned long long* d_tilebits = nullptr;
    int words = 1;
    ParticleDev* d_parts = nullptr;
    int pcap = 0;
    std::vector<ParticleDev> hparts;  // host copy of the static fields (offsets, capacities)
    int2* d_ivl = nullptr;
    long long ivl_slots = 0;
    int2* d_links = nullptr;
    long long link_slots = 0;
    double* d_partial = nullptr;
    long long partial_slots = 0;
    int maxchunks = 0;
    int link_bpp = 1;  // link-rebuild CTAs per particle (largest near box / kLinkBlock)
    int* d_linkcnt = nullptr;  // [particle capacity][link_bpp] per-CTA link counts
    long long linkcnt_slots = 0;
    int* d_err = nullptr;
    double* d_tmp = nullptr;  // FP64 read-back / upload scratch
    // particle interactions (lbm_set_interactions)
    std::vector<lbm_interaction> inter;
    InterItem* d_items = nullptr;
    int* d_coff = nullptr;
    int* d_cent = nullptr;
    double* d_pf = nullptr;
    double* d_fint = nullptr;
    // trajectory recording (lbm_record_trajectories): ring of trj_cap ticks
    double* d_trj = nullptr;
    long long trj_cap = 0, trj_read = 0;
    // asynchronous writer of fluid snapshots (lbm_write_fluid_csv)
    std::thread writer;
    std::string writer_err;
    size_t tmp_bytes = 0;
    size_t device_bytes = 0;
    // time
    long long tick = 0;
    double time = 0;
    long long calls = 0;  // lbm_step calls made
    // graphs of kModelGraphSizes[k] ticks: [profiling][starting buffer][k]
    Graph graphs[2][2][4];
    // profiling: per graph slot, events before/after the bulk kernel, after
    // the fix-up and after the particle kernel; plus the whole call
    int profiling = 0;  // 0 off, 1 whole-call time, 2 also per-kernel event nodes
    std::vector<cudaEvent_t> pev;
    cudaEvent_t t_begin = nullptr, t_end = nullptr;
    lbm_profile prof{};
    std::string err;
};

namespace {

int set_err(lbm_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    else g_global_err = msg;
    return code;
}

#define CUDA_TRY(h, call)                                                                              \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            return set_err((h), e_ == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,          \
                           std::string(#call) + ": " + cudaGetErrorString(e_));                         \
        }                                                                                              \
    } while (0)

// every entry point runs on the handle's device, whatever the caller's current device
#define BIND(h)                                                                                        \
    do {                                                                                               \
        if (cudaSetDevice((h)->device) != cudaSuccess) {                                               \
            cudaGetLastError();                                                                        \
            return set_err((h), LBM_ERR_CUDA, "cannot select the handle's CUDA device");               \
        }                                                                                              \
    } while (0)

// process-wide cap on the device bytes one handle or batch may hold (0: none)
std::atomic<long long> g_mem_limit{0};

// Device memory: cudaMalloc, with freed blocks kept (up to kKeepBytes over
// all devices) for later allocations of the same size.  cudaMalloc and
// cudaFree of a 128^3 D3Q19 FP32 model's buffers take about 1.3 ms each, a
// kept block is handed out in microseconds, so a process that builds models
// one after another (parameter sweeps, replicas, the end-to-end path of a
// short run) does not pay for them again.  A stream-ordered memory pool gave
// the same saving, but the bulk pass ran 1-1.5 % slower on its memory.  A
// freed block is kept only after its device has finished its queued work,
// as cudaFree waits for it.
constexpr size_t kKeepBytes = size_t(4) << 30;
struct BlockCache {
    std::mutex mu;
    std::multimap<size_t, std::pair<int, void*>> kept;        // capacity -> (device, block)
    std::unordered_map<void*, std::pair<int, size_t>> live;  // block -> (device, capacity)
    size_t kept_bytes = 0;
};
BlockCache g_blocks;

// cudaFree the kept blocks of device `dev` (the current device)
void release_kept(int dev) {
    std::vector<void*> drop;
    {
        std::lock_guard<std::mutex> lk(g_blocks.mu);
        for (auto it = g_blocks.kept.begin(); it != g_blocks.kept.end();) {
            if (it->second.first == dev) {
                drop.push_back(it->second.second);
                g_blocks.kept_bytes -= it->first;
                it = g_blocks.kept.erase(it);
            } else {
                ++it;
            }
        }
    }
    for (void* q : drop) cudaFree(q);
}

// `bytes` (at least 1) on the current device: a kept block of this device
// holding them with at most an eighth to spare, else cudaMalloc
cudaError_t block_alloc(void** p, size_t bytes) {
    bytes = bytes ? bytes : 1;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lk(g_blocks.mu);
        for (auto it = g_blocks.kept.lower_bound(bytes);
             it != g_blocks.kept.end() && it->first <= bytes + bytes / 8; ++it) {
            if (it->second.first != dev) continue;
            *p = it->second.second;
            g_blocks.live[*p] = {dev, it->first};
            g_blocks.kept_bytes -= it->first;
            g_blocks.kept.erase(it);
            return cudaSuccess;
        }
    }
    e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation) {  // hand this device's kept blocks back and try once more
        cudaGetLastError();
        release_kept(dev);
        e = cudaMalloc(p, bytes);
    }
    if (e == cudaSuccess) {
        std::lock_guard<std::mutex> lk(g_blocks.mu);
        g_blocks.live[*p] = {dev, bytes};
    }
    return e;
}

// give back a block from block_alloc: kept when there is room, else cudaFree
void block_free(void* p) {
    int dev = -1;
    size_t cap = 0;
    {
        std::lock_guard<std::mutex> lk(g_blocks.mu);
        auto it = g_blocks.live.find(p);
        if (it != g_blocks.live.end()) {
            dev = it->second.first;
            cap = it->second.second;
            g_blocks.live.erase(it);
        }
    }
    if (dev < 0) {
        cudaFree(p);
        return;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (dev != cur) cudaSetDevice(dev);
    bool kept = false;
    if (cudaDeviceSynchronize() == cudaSuccess) {
        std::lock_guard<std::mutex> lk(g_blocks.mu);
        if (g_blocks.kept_bytes + cap <= kKeepBytes) {
            g_blocks.kept.emplace(cap, std::make_pair(dev, p));
            g_blocks.kept_bytes += cap;
            kept = true;
        }
    }
    if (!kept) {
        cudaGetLastError();
        cudaFree(p);
    }
    if (dev != cur) cudaSetDevice(cur);
}

template <class P>
int dev_alloc(lbm_handle* h, P** p, size_t bytes) {
    const long long cap = g_mem_limit.load();
    if (cap > 0 && (long long)(h->device_bytes + bytes) > cap) {
        *p = nullptr;
        return set_err(h, LBM_ERR_OOM, "device allocation of " + std::to_string(bytes) +
                                           " bytes would exceed the memory limit of " + std::to_string(cap) +
                                           " bytes (lbm_set_memory_limit)");
    }
    cudaError_t e = block_alloc((void**)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return set_err(h, LBM_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed: " +
                                           cudaGetErrorString(e));
    }
    h->device_bytes += bytes;
    return LBM_OK;
}

template <class P>
void dev_free(P*& p) {
    if (p) block_free((void*)p);
    p = nullptr;
}

bool get_ops(int lattice, int storage, int trt, Ops* o) {
    switch (lattice) {
        case LBM_D2Q9: return ops_d2q9(storage, trt, o);
        case LBM_D3Q15: return ops_d3q15(storage, trt, o);
        case LBM_D3Q19: return ops_d3q19(storage, trt, o);
        case LBM_D3Q27: return ops_d3q27(storage, trt, o);
        default: return false;
    }
}

// host copy of the lattice (link enumeration, Guo constants)
struct HostLattice {
    int q = 0, d = 0;
    std::vector<int> cx, cy, cz, opp;
    std::vector<double> w;
};

template <class L>
HostLattice host_lattice_of() {
    HostLattice hl;
    hl.q = L::Q;
    hl.d = L::D;
    for (int i = 0; i < L::Q; ++i) {
        hl.cx.push_back(L::cx(i));
        hl.cy.push_back(L::cy(i));
        hl.cz.push_back(L::cz(i));
        hl.opp.push_back(L::opp(i));
        hl.w.push_back(L::w(i));
    }
    return hl;
}

HostLattice host_lattice(int lattice) {
    switch (lattice) {
        case LBM_D2Q9: return host_lattice_of<D2Q9>();
        case LBM_D3Q15: return host_lattice_of<D3Q15>();
        case LBM_D3Q19: return host_lattice_of<D3Q19>();
        default: return host_lattice_of<D3Q27>();
    }
}

int storage_bytes(int storage) {
    switch (storage) {
        case LBM_STORE_F16:
        case LBM_STORE_BF16: return 2;
        case LBM_STORE_F64: return 8;
        default: return 4;
    }
}

int ensure_tmp(lbm_handle* h, size_t bytes) {
    if (h->tmp_bytes >= bytes) return LBM_OK;
    dev_free(h->d_tmp);
    h->device_bytes -= h->tmp_bytes;
    h->tmp_bytes = 0;
    int rc = dev_alloc(h, &h->d_tmp, bytes);
    if (rc) return rc;
    h->tmp_bytes = bytes;
    return LBM_OK;
}

void drop_graphs(lbm_handle* h) {
    h->tick_ready = false;  // the tick kernel's maps and arguments are rebuilt with the graphs
    for (auto& prof : h->graphs)
        for (auto& row : prof)
            for (auto& gr : row) {
                if (gr.exec) cudaGraphExecDestroy(gr.exec);
                gr.exec = nullptr;
            }
}

template <class L>
void lattice_vectors_of(int* cx, int* cy, int* cz, int* q) {
    *q = L::Q;
    for (int i = 0; i < L::Q; ++i) {
        cx[i] = L::cx(i);
        cy[i] = L::cy(i);
        cz[i] = L::cz(i);
    }
}

// lattice vectors of a velocity set into fixed arrays (no host heap use, so
// that the allocation-free entry point can build its arguments too)
void lattice_vectors(int lattice, int* cx, int* cy, int* cz, int* q) {
    switch (lattice) {
        case LBM_D2Q9: lattice_vectors_of<D2Q9>(cx, cy, cz, q); break;
        case LBM_D3Q15: lattice_vectors_of<D3Q15>(cx, cy, cz, q); break;
        case LBM_D3Q19: lattice_vectors_of<D3Q19>(cx, cy, cz, q); break;
        default: lattice_vectors_of<D3Q27>(cx, cy, cz, q); break;
    }
}

// Kernel arguments of one tick from buffer `src`, with the fix-up's
// momentum-exchange partials in `partial`.  Uses no host heap.
StepArgs make_step_args(const lbm_handle* h, int src, double* partial) {
    StepArgs a{};
    a.src = h->pop[src];
    a.dst = h->pop[1 - src];
    a.g = h->g;
    for (int k = 0; k < 3; ++k) a.coord[k] = h->d_coord[k];
    a.tilebits = h->d_tilebits;
    a.words = h->words;
    a.nparts = (int)h->hparts.size();
    a.wall = h->d_wall;
    a.uw = h->d_uw;
    a.ffield = h->d_ffield;
    a.parts = h->d_parts;
    a.ivl = h->d_ivl;
    a.links = h->d_links;
    a.wlinks = h->d_wlinks;
    a.wnodes = h->d_wnodes;
    a.nwlinks = h->nwlinks;
    a.nwnodes = h->nwnodes;
    a.maxchunks = h->maxchunks;
    a.nlinkoc = (int)std::min<size_t>(h->hparts.size(), kLinkOcParams);
    for (int p = 0; p < a.nlinkoc; ++p) {
        a.linkoc[p][0] = h->hparts[p].link_off;
        a.linkoc[p][1] = h->hparts[p].link_cap;
    }
    a.vrows = h->vrows;
    a.vnt1 = h->vnt1;
    a.vtiles = h->vtiles;
    a.nbox = h->d_nbox[src];
    a.vnear = h->d_vnear;
    a.partial = partial;
    a.err = h->d_err;
    a.rho0 = h->rho0;
    a.scale = h->scale;
    a.inv_scale = 1.0 / h->scale;
    a.omega = h->dt / h->tau;
    a.omega_p = h->dt / h->tau;
    a.omega_m = h->trt ? h->dt / h->tau_minus : 0.0;
    a.guo_k = h->dt * (1 - h->dt / (2 * h->tau));
    a.guo_kp = a.guo_k;
    a.guo_km = h->trt ? h->dt * (1 - h->dt / (2 * h->tau_minus)) : 0.0;
    for (int k = 0; k < 3; ++k) a.F[k] = h->F[k];
    a.half_dt = 0.5 * h->dt;
    a.coeff = std::pow(h->dx, h->dims) / h->dt;
    a.force_mode = h->force_mode;
    a.incompressible = h->incompressible;
    a.rho_inc = h->rho_inc;
    // Guo constants (collide(): BGK A_i + K0 + B_i cu ; TRT even K0 + B_i cu, odd A_i)
    // in storage units: collide() works on g' = S (f/w - rho0)
    const double kodd = (h->trt ? 3.0 * a.guo_km : 3.0 * a.guo_k) * h->scale;
    const double keven = (h->trt ? 9.0 * a.guo_kp : 9.0 * a.guo_k) * h->scale;
    a.gK0 = (h->trt ? -3.0 * a.guo_kp : -3.0 * a.guo_k) * h->scale;
    a.gkA = kodd;
    a.gkB = keven;
    int cx[27], cy[27], cz[27], q = 0;
    lattice_vectors(h->lattice, cx, cy, cz, &q);
    const size_t esz = storage_bytes(h->storage);
    for (int i = 0; i < 27; ++i) {
        a.gA[i] = a.gB[i] = 0.0;
        a.srcq[i] = nullptr;
        a.dstq[i] = nullptr;
    }
    for (int i = 0; i < q; ++i) {
        const double cF = cx[i] * h->F[0] + cy[i] * h->F[1] + cz[i] * h->F[2];
        a.gA[i] = kodd * cF;
        a.gB[i] = keven * cF;
        a.srcq[i] = static_cast<const char*>(a.src) + (size_t)i * h->N * esz;
        a.dstq[i] = static_cast<char*>(a.dst) + (size_t)i * h->N * esz;
    }
    a.trt = h->trt;
    a.stochastic = h->rounding == LBM_ROUND_STOCHASTIC ? 1 : 0;
    a.reverse = src;  // the tick after a forward pass (it wrote buffer 1) walks backwards
    fill_collide_consts(a);
    return a;
}

StepArgs step_args(const lbm_handle* h, int src) { return make_step_args(h, src, h->d_partial); }

bool use_vector_bulk(const lbm_handle* h) {
    return h->ops.bulk_v4 != nullptr && h->force_mode != LBM_FORCE_FIELD && h->vrows > 0;
}

// the TMA bulk pass is used where its shape is valid and the caller asked for it
bool use_tma_bulk(const lbm_handle* h) {
    return h->tma_ok && h->bulk_kind == LBM_BULK_TMA && use_vector_bulk(h);
}

// Launch shape of the TMA bulk pass for `threads` threads per CTA and
// `stages` ring buffers (0: chosen here); false where it does not apply:
// rows of nx = 4 RT nodes with RT a power of two up to 32 (a row is a
// shuffle segment of a warp), 16-byte aligned rows, no per-node force field.
bool choose_tma(lbm_handle* h, int threads, int stages, TmaShape* out) {
    const void* fn = h->rounding == LBM_ROUND_STOCHASTIC ? h->ops.bulk_tma_fn_sr : h->ops.bulk_tma_fn;
    if (!h->ops.bulk_tma || !fn || h->force_mode == LBM_FORCE_FIELD) return false;
    const int nx = h->n[0], ny = h->n[1], esz = storage_bytes(h->storage);
    if (nx % 4 != 0) return false;
    const int RT = nx / 4;
    if (RT > 32 || (RT & (RT - 1)) != 0 || (nx * esz) % 16 != 0) return false;
    if (threads <= 0) threads = esz == 4 ? 256 : 512;
    if (threads > 512 || threads % 32 != 0 || threads % RT != 0) return false;
    int rows = threads / RT;
    while (rows > ny && rows * RT > 32) rows /= 2;  // no more rows than the grid has
    threads = rows * RT;
    if (threads % 32 != 0) return false;
    const long long stage_bytes = (long long)h->q * rows * nx * esz;
    if (stage_bytes >= (1 << 20)) return false;  // an mbarrier's transaction count
    if (stages <= 0) stages = (int)std::min<long long>(kTmaMaxStages, (200 * 1024) / stage_bytes);
    if (stages < 2 || stages > kTmaMaxStages) return false;
    const int smem = tma_smem_bytes(h->q, nx, rows, stages, esz);
    if (smem > 227 * 1024) return false;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return false;
    }
    const long long tiles = (long long)((ny + rows - 1) / rows) * h->n[2];
    out->rows = rows;
    out->stages = stages;
    out->smem = smem;
    out->grid = (int)std::max<long long>(1, std::min<long long>(tiles, (long long)per_sm * sms));
    return true;
}

// the bulk pass over all tiles
void launch_bulk(const lbm_handle* h, const StepArgs& a, cudaStream_t s) {
    if (use_tma_bulk(h))
        h->ops.bulk_tma(a, h->tma, s);
    else if (use_vector_bulk(h))
        h->ops.bulk_v4(a, h->vtiles, h->vblock, s);
    else
        h->ops.bulk(a, (unsigned)h->g.ntiles, dim3(h->g.t[0], h->g.t[1], h->g.t[2]), s);
}

// `src`: population buffer of the tick (selects the published-box buffer);
// -1 publishes into both (setup)
ParticleArgs particle_args(const lbm_handle* h, int mode, int pid, int src = -1) {
    ParticleArgs a{};
    a.nbox_out[0] = src < 0 ? h->d_nbox[0] : h->d_nbox[src];
    a.nbox_out[1] = src < 0 ? h->d_nbox[1] : nullptr;
    a.parts = h->d_parts;
    a.nparts = (int)h->hparts.size();
    a.mode = mode;
    a.inline_links = mode != 0 ? 1 : 0;  // setup rebuilds its list at once
    a.setup_pid = pid;
    a.words = h->words;
    a.partial = h->d_partial;
    a.tilebits = h->d_tilebits;
    a.ivl = h->d_ivl;
    a.links = h->d_links;
    a.g = h->g;
    for (int k = 0; k < 3; ++k) {
        a.coord[k] = h->d_coord[k];
        a.x0[k] = h->X[k].empty() ? 0.0 : h->X[k][0];
    }
    a.dx = h->dx;
    a.dt = h->dt;
    a.err = h->d_err;
    a.trj = h->d_trj;
    a.trj_cap = h->trj_cap;
    a.fint = h->inter.empty() ? nullptr : h->d_fint;
    return a;
}

InterArgs inter_args(const lbm_handle* h) {
    InterArgs a{};
    a.items = h->d_items;
    a.nitems = (int)h->inter.size();
    a.nparts = (int)h->hparts.size();
    a.dims = h->dims;
    a.parts = h->d_parts;
    a.coff = h->d_coff;
    a.cent = h->d_cent;
    a.pf = h->d_pf;
    a.fint = h->d_fint;
    return a;
}

// the interactions of a tick, before its particle update (same stream)
void launch_interactions(const lbm_handle* h, cudaStream_t s) {
    if (h->inter.empty()) return;
    k_interactions<<<1, kInterThreads, 0, s>>>(inter_args(h));
}

CodecArgs codec_args(const lbm_handle* h) {
    CodecArgs c{};
    c.pop = h->pop[h->cur];
    c.N = h->N;
    c.wall = h->d_wall;
    c.ffield = h->d_ffield;
    c.rho0 = h->rho0;
    c.scale = h->scale;
    c.inv_scale = 1.0 / h->scale;
    c.half_dt = 0.5 * h->dt;
    for (int k = 0; k < 3; ++k) c.F[k] = h->F[k];
    c.force_mode = h->force_mode;
    return c;
}

long long fixup_blocks(const lbm_handle* h) {
    return (long long)h->hparts.size() * h->maxchunks + (h->nwlinks + kFixBlock - 1) / kFixBlock +
           (h->nwnodes + kFixBlock - 1) / kFixBlock;
}

// the fix-up walks the lists' chunks (k_fixup_walk) when a CTA per chunk of
// every list's capacity would be many CTAs
bool fixup_walk(const lbm_handle* h) { return (long long)h->hparts.size() * h->maxchunks >= kFixWalkMin; }

// CTAs of a fix-up launch
long long fixup_grid(const lbm_handle* h) {
    if (!fixup_walk(h)) return fixup_blocks(h);
    return (long long)h->hparts.size() * fixup_ctas_per_particle(h->maxchunks) +
           (h->nwlinks + kFixBlock - 1) / kFixBlock + (h->nwnodes + kFixBlock - 1) / kFixBlock;
}

// the persistent tick kernel applies to the vector bulk kernel with
// kTickBlock-thread tiles, when there is boundary work to overlap
bool use_tick_kernel(const lbm_handle* h) {
    return h->schedule == LBM_SCHEDULE_PERSISTENT && h->inter.empty() && use_vector_bulk(h) && h->ops.tick != nullptr &&
           h->vblock == kTickBlock && h->tick_grid > 0 && fixup_blocks(h) > 0;
}

// (Re)build the item maps and the per-parity arguments of the tick kernel.
int prepare_tick(lbm_handle* h) {
    if (h->tick_ready || !use_tick_kernel(h)) return LBM_OK;
    const int np = (int)h->hparts.size();
    std::vector<int4> am;
    for (long long t = 0; t < (long long)h->vnear.size(); ++t)
        if (h->vnear[t]) am.push_back(make_int4(0, 0, (int)t, 0));
    for (int p = 0; p < np; ++p) {
        // a solid box spans at most 2r/dx + 5 nodes per axis; grown by two on each side
        const long long len = (long long)std::floor(2.0 * h->hparts[p].radius / h->dx) + 9;
        const long long nys = std::min<long long>(h->vnt1 + 1, (len + h->vrows - 1) / h->vrows + 2);
        const long long nzs = h->dims == 3 ? std::min<long long>(h->n[2], len) : 1;
        if (nys >= 65536 || nzs >= 32768)
            return set_err(h, LBM_ERR_UNSUPPORTED, "particle too large for the tick kernel's tile slots");
        for (long long dz = 0; dz < nzs; ++dz)
            for (long long dy = 0; dy < nys; ++dy) am.push_back(make_int4(0, 1, p, (int)(dy | (dz << 16))));
    }
    std::vector<int2> bm, cm, dm;
    const long long nb = fixup_blocks(h);
    for (long long b = 0; b < nb; ++b) bm.push_back(make_int2(0, (int)b));
    for (int p = 0; p < np; ++p) cm.push_back(make_int2(0, p));
    for (long long t = 0; t < h->vtiles; ++t) dm.push_back(make_int2(0, (int)t));
    StepArgs ta[2];
    ParticleArgs pa[2];
    for (int s = 0; s < 2; ++s) {
        ta[s] = step_args(h, s);
        ta[s].nbox = h->d_nbox[1 - s];  // boxes of the previous tick's update (see tick.cuh)
        pa[s] = particle_args(h, 0, 0, s);
        pa[s].inline_links = 1;  // no separate link kernels inside the persistent tick
    }
    dev_free(h->d_amap);
    dev_free(h->d_bmap);
    dev_free(h->d_cmap);
    dev_free(h->d_dmap);
    int rc = dev_alloc(h, &h->d_amap, sizeof(int4) * std::max<size_t>(1, am.size()));
    if (!rc) rc = dev_alloc(h, &h->d_bmap, sizeof(int2) * std::max<size_t>(1, bm.size()));
    if (!rc) rc = dev_alloc(h, &h->d_cmap, sizeof(int2) * std::max<size_t>(1, cm.size()));
    if (!rc) rc = dev_alloc(h, &h->d_dmap, sizeof(int2) * std::max<size_t>(1, dm.size()));
    if (!rc && !h->d_targs) rc = dev_alloc(h, &h->d_targs, sizeof(StepArgs) * 2);
    if (!rc && !h->d_pargs) rc = dev_alloc(h, &h->d_pargs, sizeof(ParticleArgs) * 2);
    if (rc) return rc;
    if (!am.empty()) CUDA_TRY(h, cudaMemcpyAsync(h->d_amap, am.data(), sizeof(int4) * am.size(), cudaMemcpyHostToDevice, h->stream));
    if (!bm.empty()) CUDA_TRY(h, cudaMemcpyAsync(h->d_bmap, bm.data(), sizeof(int2) * bm.size(), cudaMemcpyHostToDevice, h->stream));
    if (!cm.empty()) CUDA_TRY(h, cudaMemcpyAsync(h->d_cmap, cm.data(), sizeof(int2) * cm.size(), cudaMemcpyHostToDevice, h->stream));
    if (!dm.empty()) CUDA_TRY(h, cudaMemcpyAsync(h->d_dmap, dm.data(), sizeof(int2) * dm.size(), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->d_targs, ta, sizeof(ta), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->d_pargs, pa, sizeof(pa), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->items.amap = h->d_amap;
    h->items.bmap = h->d_bmap;
    h->items.cmap = h->d_cmap;
    h->items.dmap = h->d_dmap;
    h->items.na = (long long)am.size();
    h->items.nb = (long long)bm.size();
    h->items.nc = (long long)cm.size();
    h->items.nd = (long long)dm.size();
    h->items.d_test = 1;
    h->items.spin_limit = h->spin_limit;
    h->items.wait_extra = h->wait_extra;
    h->tick_ready = true;
    return LBM_OK;
}

int launches_per_tick(const lbm_handle* h) {
    if (use_tick_kernel(h)) return 1;
    const bool fix = fixup_blocks(h) > 0;
    return 1 + (fix ? 1 : 0) + (h->hparts.empty() ? 0 : 1);  // the particle update rebuilds its links itself
}

// events of graph slot s: [0] before bulk, [1] after bulk, [2] after fix-up, [3] after particles
cudaEvent_t prof_event(lbm_handle* h, int slot, int k) { return h->pev[slot * 4 + k]; }

void prof_record(lbm_handle* h, int slot, int k, cudaStream_t s) {
    if (h->profiling < 2) return;
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &st);
    // inside a capture the record becomes an event node of the graph
    if (st == cudaStreamCaptureStatusActive)
        cudaEventRecordWithFlags(prof_event(h, slot, k), s, cudaEventRecordExternal);
    else
        cudaEventRecord(prof_event(h, slot, k), s);
}

// Inside a stream capture: the single node the next captured work on `s`
// depends on (null outside a capture or for several).
cudaGraphNode_t capture_tail(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    const cudaGraphNode_t* deps = nullptr;
    size_t n = 0;
    if (cudaStreamGetCaptureInfo_v3(s, &st, nullptr, nullptr, &deps, nullptr, &n) != cudaSuccess) return nullptr;
    return st == cudaStreamCaptureStatusActive && n == 1 ? deps[0] : nullptr;
}

// Inside a stream capture: the next captured kernel depends on kernel node
// `from` through a programmatic edge (its other dependencies stay full ones).
void programmatic_from(cudaStream_t s, cudaGraphNode_t from) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    const cudaGraphNode_t* deps = nullptr;
    size_t n = 0;
    if (cudaStreamGetCaptureInfo_v3(s, &st, nullptr, nullptr, &deps, nullptr, &n) != cudaSuccess ||
        st != cudaStreamCaptureStatusActive || n > 8)
        return;
    cudaGraphNode_t nodes[8];
    cudaGraphEdgeData edges[8] = {};
    for (size_t i = 0; i < n; ++i) {
        nodes[i] = deps[i];
        if (deps[i] == from) {
            edges[i].from_port = cudaGraphKernelNodePortProgrammatic;
            edges[i].type = cudaGraphDependencyTypeProgrammatic;
        }
    }
    cudaStreamUpdateCaptureDependencies_v2(s, nodes, edges, n, cudaStreamSetCaptureDependencies);
}

// Enqueue one tick (capturable); `slot` selects the profiling events.
// Persistent tick kernel: one launch.  Otherwise
//   main: bulk(n) -> [wait particles(n-1)] -> fixup(n) -> bulk(n+1) ...
//   side:                    particles(n) after fixup(n)
// The bulk pass never reads particle state, so the particle update of tick n
// runs concurrently with the bulk pass of tick n+1.
void enqueue_tick(lbm_handle* h, int src, int slot) {
    prof_record(h, slot, 0, h->stream);
    if (use_tick_kernel(h)) {
        h->ops.tick(h->d_targs + src, h->d_pargs + src, h->items, h->d_tq, h->d_err, h->tick_grid, h->stream,
                    h->rounding == LBM_ROUND_STOCHASTIC);
        prof_record(h, slot, 1, h->stream);
        return;
    }
    const StepArgs a = step_args(h, src);
    launch_bulk(h, a, h->stream);
    prof_record(h, slot, 1, h->stream);
    // The fix-up follows the bulk pass through a programmatic edge (it computes
    // during the bulk pass's last wave and stores after it) unless per-kernel
    // events sit between the two.  Inside a capture the edge is set by hand so
    // that the one from the particle update stays a full dependency; outside
    // one the launch attribute serves when no event wait comes between.
    const bool early = h->profiling < 2;
    const cudaGraphNode_t bulk_node = early ? capture_tail(h->stream) : nullptr;
    bool waited = false;
    if (h->part_pending) {
        cudaStreamWaitEvent(h->stream, h->ev_part, 0);
        h->part_pending = false;
        waited = true;
    }
    const long long nb = fixup_blocks(h);
    if (nb > 0) {
        if (bulk_node) programmatic_from(h->stream, bulk_node);
        h->ops.fixup(a, (unsigned)fixup_grid(h), h->stream, early && !bulk_node && !waited, fixup_walk(h));
    }
    if (a.nparts == 0) prof_record(h, slot, 2, h->stream);
    if (a.nparts > 0) {
        cudaEventRecord(h->ev_fix, h->stream);
        cudaStreamWaitEvent(h->side, h->ev_fix, 0);
        prof_record(h, slot, 2, h->side);
        ParticleArgs pa = particle_args(h, 0, 0, src);
        pa.inline_links = 1;
        launch_interactions(h, h->side);
        h->ops.particles(pa, (unsigned)a.nparts, h->side);
        prof_record(h, slot, 3, h->side);
        cudaEventRecord(h->ev_part, h->side);
        h->part_pending = true;
    }
}

// make the main stream wait for outstanding side-stream work
void join_particles(lbm_handle* h) {
    if (h->part_pending) {
        cudaStreamWaitEvent(h->stream, h->ev_part, 0);
        h->part_pending = false;
    }
}

int build_graph(lbm_handle* h, int start, int size_idx) {
    Graph& gr = h->graphs[h->profiling >= 2 ? 1 : 0][start][size_idx];
    if (gr.exec) return LBM_OK;
    cudaGraph_t graph = nullptr;
    CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int b = start;
    for (int s = 0; s < kModelGraphSizes[size_idx]; ++s) {
        enqueue_tick(h, b, s);
        b = 1 - b;
    }
    join_particles(h);  // a capture must end with every forked stream joined
    cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(h, LBM_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(e));
    }
    e = cudaGraphInstantiate(&gr.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        gr.exec = nullptr;
        return set_err(h, LBM_ERR_CUDA, std::string("graph instantiation failed: ") + cudaGetErrorString(e));
    }
    // upload now: a graph's first launch otherwise pays for it
    CUDA_TRY(h, cudaGraphUpload(gr.exec, h->stream));
    return LBM_OK;
}

// The graphs a call of `nsteps` ticks launches (the largest sizes first, as
// lbm_step does, from the current buffer), built before the call's first
// launch and before its profiling start event: a call pays only for the
// graphs it is the first to need, never in the middle of its launches.
int ensure_graphs(lbm_handle* h, int64_t nsteps) {
    static_assert(kModelGraphSizes[0] % 2 == 0, "the largest graph must leave the buffer unchanged");
    int64_t done = 0;
    int cur = h->cur;
    while (done < nsteps) {
        int k = 0;
        while (kModelGraphSizes[k] > nsteps - done) ++k;
        const int rc = build_graph(h, cur, k);
        if (rc) return rc;
        if (k == 0) {  // the largest graph repeats without changing the buffer
            done += (nsteps - done) / kModelGraphSizes[0] * kModelGraphSizes[0];
            continue;
        }
        done += kModelGraphSizes[k];
        if (kModelGraphSizes[k] & 1) cur = 1 - cur;
    }
    return LBM_OK;
}

// Read (and clear) the device error word after the work of a call.  The state
// of the model after any of these errors is undefined: restore a checkpoint
// (lbm_load_state) or destroy the handle.
int check_device_error(lbm_handle* h) {
    int err = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (err == 0) return LBM_OK;
    CUDA_TRY(h, cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (err & kErrLinkOverflow) return set_err(h, LBM_ERR_STATE, "particle boundary links exceeded their capacity");
    if (err & kErrIntervalOverflow) return set_err(h, LBM_ERR_STATE, "particle solid box exceeded its capacity");
    if (err & kErrSpinTimeout) return set_err(h, LBM_ERR_TIMEOUT, "a wait inside the tick kernel gave up");
    if (err & kErrNumeric)
        return set_err(h, LBM_ERR_NUMERIC,
                       "non-finite or negative density on the device (the simulation diverged near tick " +
                           std::to_string(h->tick) + ")");
    return set_err(h, LBM_ERR_STATE, "unknown device error word " + std::to_string(err));
}

// vector tiles of `B` threads: B / (nx/4) whole x-rows of one z-slice
void set_vector_block(lbm_handle* h, int B) {
    const int RT = h->n[0] / 4;
    h->vblock = B;
    h->vrows = std::max(1, std::min(B / RT, h->n[1]));
    h->vnt1 = (h->n[1] + h->vrows - 1) / h->vrows;
    h->vtiles = (long long)h->vnt1 * h->n[2];
}

// CTA tile: full x-rows up to 256 nodes (x-wrap stays inside the CTA)
void choose_tiles(lbm_handle* h) {
    GridDesc& g = h->g;
    for (int k = 0; k < 3; ++k) g.n[k] = h->n[k];
    const int t0 = std::min(256, ((h->n[0] + 31) / 32) * 32);
    const int t1 = std::max(1, std::min(256 / t0, h->n[1]));
    g.t[0] = t0;
    g.t[1] = t1;
    g.t[2] = 1;
    for (int k = 0; k < 3; ++k) g.nt[k] = (h->n[k] + g.t[k] - 1) / g.t[k];
    g.N = h->N;
    g.ntiles = (long long)g.nt[0] * g.nt[1] * g.nt[2];
    // vector tiles: whole x-rows, 4 nodes per thread, in the CTA size that
    // leaves the fewest idle threads (kTickBlock on a tie: 96 threads for rows
    // of 96 or 192 nodes, 64 for rows of 4*2^k <= 256).  The persistent tick
    // kernel and batch queues run kTickBlock-thread tiles: set_vector_block.
    h->vrows = h->vnt1 = h->vblock = 0;
    h->vtiles = 0;
    if (h->n[0] % 4 == 0 && h->n[0] / 4 <= 512) {
        const int RT = h->n[0] / 4;
        double best = -1.0;
        int pick = 0;
        for (int B : kBulkBlocks) {
            if (B < RT) continue;
            const int rows = std::min(B / RT, h->n[1]);
            const double use = (double)(rows * RT) / B;
            if (use > best + 1e-9 || (use > best - 1e-9 && B == kTickBlock)) {
                best = std::max(best, use);
                pick = B;
            }
        }
        if (h->schedule == LBM_SCHEDULE_PERSISTENT && RT <= kTickBlock) pick = kTickBlock;
        set_vector_block(h, pick);
    }
}

int upload(lbm_handle* h, void* dst, const void* src, size_t bytes) {
    CUDA_TRY(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream));
    return LBM_OK;
}

void destroy_all(lbm_handle* h) {
    if (!h) return;
    if (h->writer.joinable()) h->writer.join();
    cudaSetDevice(h->device);
    dev_free(h->d_trj);
    dev_free(h->d_items);
    dev_free(h->d_coff);
    dev_free(h->d_cent);
    dev_free(h->d_pf);
    dev_free(h->d_fint);
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_graphs(h);
    dev_free(h->pop[0]);
    dev_free(h->pop[1]);
    for (auto& c : h->d_coord) dev_free(c);
    dev_free(h->d_wall);
    dev_free(h->d_uw);
    dev_free(h->d_ffield);
    dev_free(h->d_wlinks);
    dev_free(h->d_wnodes);
    dev_free(h->d_tilebits);
    dev_free(h->d_parts);
    dev_free(h->d_ivl);
    dev_free(h->d_links);
    dev_free(h->d_linkcnt);
    dev_free(h->d_partial);
    dev_free(h->d_err);
    dev_free(h->d_tmp);
    dev_free(h->d_vnear);
    dev_free(h->d_nbox[0]);
    dev_free(h->d_nbox[1]);
    dev_free(h->d_amap);
    dev_free(h->d_bmap);
    dev_free(h->d_cmap);
    dev_free(h->d_dmap);
    dev_free(h->d_targs);
    dev_free(h->d_pargs);
    dev_free(h->d_tq);
    for (auto& e : h->pev) cudaEventDestroy(e);
    if (h->t_begin) cudaEventDestroy(h->t_begin);
    if (h->t_end) cudaEventDestroy(h->t_end);
    if (h->ev_fix) cudaEventDestroy(h->ev_fix);
    if (h->ev_part) cudaEventDestroy(h->ev_part);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

// grow a device array, keeping its first `keep` elements
template <class T>
int grow(lbm_handle* h, T** arr, long long* cap, long long need, long long keep) {
    if (need <= *cap && *arr) return LBM_OK;
    long long ncap = std::max<long long>(need, *cap * 2);
    T* na = nullptr;
    int rc = dev_alloc(h, &na, sizeof(T) * std::max<long long>(1, ncap));
    if (rc) return rc;
    CUDA_TRY(h, cudaMemsetAsync(na, 0, sizeof(T) * std::max<long long>(1, ncap), h->stream));
    if (*arr && keep > 0)
        CUDA_TRY(h, cudaMemcpyAsync(na, *arr, sizeof(T) * keep, cudaMemcpyDeviceToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    dev_free(*arr);
    *arr = na;
    *cap = ncap;
    return LBM_OK;
}

// grow device particle storage / tile-bit words
int ensure_particle_capacity(lbm_handle* h, int nparts_new) {
    if (nparts_new > h->pcap || !h->d_parts) {
        int cap = std::max(8, h->pcap * 2);
        while (cap < nparts_new) cap *= 2;
        ParticleDev* np = nullptr;
        int rc = dev_alloc(h, &np, sizeof(ParticleDev) * cap);
        if (rc) return rc;
        if (h->d_parts && !h->hparts.empty())
            CUDA_TRY(h, cudaMemcpyAsync(np, h->d_parts, sizeof(ParticleDev) * h->hparts.size(),
                                        cudaMemcpyDeviceToDevice, h->stream));
        int* nb[2] = {nullptr, nullptr};
        for (int b = 0; b < 2; ++b) {
            rc = dev_alloc(h, &nb[b], sizeof(int) * 6 * cap);
            if (rc) return rc;
            if (h->d_nbox[b] && !h->hparts.empty())
                CUDA_TRY(h, cudaMemcpyAsync(nb[b], h->d_nbox[b], sizeof(int) * 6 * h->hparts.size(),
                                            cudaMemcpyDeviceToDevice, h->stream));
        }
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        dev_free(h->d_parts);
        h->d_parts = np;
        for (int b = 0; b < 2; ++b) {
            dev_free(h->d_nbox[b]);
            h->d_nbox[b] = nb[b];
        }
        h->pcap = cap;
    }
    const int words_new = std::max(1, (nparts_new + 63) / 64);
    if (words_new > h->words || !h->d_tilebits) {
        const int w = std::max(words_new, h->words);
        unsigned long long* nb = nullptr;
        int rc = dev_alloc(h, &nb, sizeof(unsigned long long) * h->g.ntiles * w);
        if (rc) return rc;
        CUDA_TRY(h, cudaMemsetAsync(nb, 0, sizeof(unsigned long long) * h->g.ntiles * w, h->stream));
        if (h->d_tilebits)
            CUDA_TRY(h, cudaMemcpy2DAsync(nb, sizeof(unsigned long long) * w, h->d_tilebits,
                                          sizeof(unsigned long long) * h->words,
                                          sizeof(unsigned long long) * h->words, h->g.ntiles,
                                          cudaMemcpyDeviceToDevice, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        dev_free(h->d_tilebits);
        h->d_tilebits = nb;
        h->words = w;
    }
    return LBM_OK;
}

bool is_uniform_axis(const std::vector<double>& X, double dx) {
    for (size_t i = 1; i < X.size(); ++i) {
        const double expect = X[0] + (double)i * dx;
        if (std::fabs(X[i] - expect) > 1e-9 * (std::fabs(expect) + std::fabs(dx) + 1.0)) return false;
    }
    return true;
}

// (Re)allocate the trajectory ring for `cap` ticks of every particle and
// restart the count; cap 0 stops recording.
int trj_alloc(lbm_handle* h, long long cap) {
    if (h->d_trj) {
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        dev_free(h->d_trj);
        h->device_bytes -= sizeof(double) * 9 * (size_t)h->trj_cap * h->hparts.size();
    }
    h->trj_cap = 0;
    h->trj_read = 0;
    const long long np = (long long)h->hparts.size();
    for (long long p = 0; p < np; ++p) {
        const long long zero = 0;
        CUDA_TRY(h, cudaMemcpyAsync(&h->d_parts[p].nrec, &zero, sizeof(zero), cudaMemcpyHostToDevice, h->stream));
    }
    if (cap > 0 && np > 0) {
        const int rc = dev_alloc(h, &h->d_trj, sizeof(double) * 9 * (size_t)cap * np);
        if (rc) return rc;
        h->trj_cap = cap;
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);  // the graphs hold the particle kernel's arguments
    return LBM_OK;
}

// Upload the interaction items and each particle's ordered contributions.
int upload_interactions(lbm_handle* h) {
    const int n = (int)h->inter.size(), np = (int)h->hparts.size();
    dev_free(h->d_items);
    dev_free(h->d_coff);
    dev_free(h->d_cent);
    dev_free(h->d_pf);
    dev_free(h->d_fint);
    if (n == 0) return LBM_OK;
    std::vector<InterItem> items(n);
    std::vector<std::vector<int>> per(np);
    for (int t = 0; t < n; ++t) {
        const lbm_interaction& e = h->inter[t];
        InterItem& it = items[t];
        it.kind = e.kind;
        it.id1 = e.id1 - 1;
        it.id2 = e.id2 - 1;
        it.id3 = e.kind == LBM_INTERACTION_POLAR ? e.id3 - 1 : 0;
        for (int k = 0; k < 4; ++k) it.p[k] = e.p[k];
        // the order in which applyInteraction! adds to the force inputs
        if (e.kind == LBM_INTERACTION_POLAR) {
            per[it.id1].push_back(t << 3 | 0 << 1 | 0);
            per[it.id3].push_back(t << 3 | 1 << 1 | 0);
            per[it.id2].push_back(t << 3 | 2 << 1 | 1);
        } else {
            per[it.id1].push_back(t << 3 | 0 << 1 | 0);
            per[it.id2].push_back(t << 3 | 0 << 1 | 1);
        }
    }
    std::vector<int> coff(np + 1, 0), cent;
    for (int p = 0; p < np; ++p) {
        coff[p + 1] = coff[p] + (int)per[p].size();
        cent.insert(cent.end(), per[p].begin(), per[p].end());
    }
    int rc = dev_alloc(h, &h->d_items, sizeof(InterItem) * n);
    if (!rc) rc = dev_alloc(h, &h->d_coff, sizeof(int) * (np + 1));
    if (!rc) rc = dev_alloc(h, &h->d_cent, sizeof(int) * std::max<size_t>(1, cent.size()));
    if (!rc) rc = dev_alloc(h, &h->d_pf, sizeof(double) * 9 * n);
    if (!rc) rc = dev_alloc(h, &h->d_fint, sizeof(double) * 3 * std::max(1, np));
    if (rc) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(h->d_items, items.data(), sizeof(InterItem) * n, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->d_coff, coff.data(), sizeof(int) * (np + 1), cudaMemcpyHostToDevice, h->stream));
    if (!cent.empty())
        CUDA_TRY(h, cudaMemcpyAsync(h->d_cent, cent.data(), sizeof(int) * cent.size(), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

// Julia's print(::Float64) (what CSV.jl writes): the shortest digits that
// read back to x; plain notation for 1e-4 <= |x| < 1e6 with at least one
// decimal ("1.0", "0.0001"), else d.ddd e<exp> without padding ("1.0e-5",
// "1.234567e6"); "NaN", "Inf", "-Inf".
void julia_float(double x, std::string& out) {
    if (std::isnan(x)) {
        out += "NaN";
        return;
    }
    if (std::isinf(x)) {
        out += x < 0 ? "-Inf" : "Inf";
        return;
    }
    if (x == 0.0) {
        out += std::signbit(x) ? "-0.0" : "0.0";
        return;
    }
    char buf[48];
    const auto r = std::to_chars(buf, buf + sizeof(buf), x, std::chars_format::scientific);
    const std::string sci(buf, r.ptr);  // [-]d[.ddd]e[+-]XX
    const size_t epos = sci.find('e');
    const int e10 = std::atoi(sci.c_str() + epos + 1);
    std::string mant = sci.substr(0, epos);
    const bool neg = mant[0] == '-';
    if (neg) mant.erase(0, 1);
    std::string digits;
    for (char c : mant)
        if (c != '.') digits += c;
    if (neg) out += '-';
    if (e10 < -4 || e10 >= 6) {
        out += digits[0];
        out += '.';
        out += digits.size() > 1 ? digits.substr(1) : std::string("0");
        out += 'e';
        out += std::to_string(e10);
    } else if (e10 < 0) {
        out += "0.";
        out.append((size_t)(-e10 - 1), '0');
        out += digits;
    } else {
        const size_t ip = (size_t)e10 + 1;  // digits before the point
        if (digits.size() <= ip) {
            out += digits;
            out.append(ip - digits.size(), '0');
            out += ".0";
        } else {
            out += digits.substr(0, ip);
            out += '.';
            out += digits.substr(ip);
        }
    }
}

// static wall lists: wall nodes, and fluid nodes with a wall source in some direction
void wall_lists(const lbm_handle* h, const std::vector<unsigned char>& W, std::vector<int2>& wl,
                std::vector<int>& wn) {
    const HostLattice hl = host_lattice(h->lattice);
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const int c = x + nx * (y + ny * z);
                if (W[c]) {
                    wn.push_back(c);
                    continue;
                }
                unsigned mask = 0;
                for (int i = 1; i < hl.q; ++i) {
                    const int tx = (x + hl.cx[i] + nx) % nx, ty = (y + hl.cy[i] + ny) % ny, tz = (z + hl.cz[i] + nz) % nz;
                    if (W[tx + nx * (ty + ny * tz)]) mask |= 1u << hl.opp[i];  // link (x, j), x - c_j = x + c_i
                }
                if (mask) wl.push_back(make_int2(c, (int)mask));
            }
}

}  // namespace

extern "C" {

int32_t lbm_abi_version(void) { return LBM_ABI_VERSION; }
const char* lbm_build_info(void) { return kBuildInfo; }
const char* lbm_last_global_error(void) { return g_global_err.c_str(); }
const char* lbm_last_error(lbm_handle* h) { return h ? h->err.c_str() : g_global_err.c_str(); }

int lbm_create(const lbm_config* cfg, lbm_handle** out) {
    if (!cfg || !out) return set_err(nullptr, LBM_ERR_INVALID, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_err(nullptr, LBM_ERR_NO_DEVICE, "no CUDA device is available");
    }
    int device = cfg->device;
    if (device >= ndev) return set_err(nullptr, LBM_ERR_INVALID, "no CUDA device with that ordinal");
    if (device < 0) {
        if (cudaGetDevice(&device) != cudaSuccess) return set_err(nullptr, LBM_ERR_CUDA, "cudaGetDevice failed");
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return set_err(nullptr, LBM_ERR_CUDA, "cudaSetDevice failed");
    }
    if (cfg->dims != 2 && cfg->dims != 3) return set_err(nullptr, LBM_ERR_INVALID, "dims must be 2 or 3");
    const int vd = cfg->lattice == LBM_D2Q9 ? 2 : 3;
    if (cfg->lattice != LBM_D2Q9 && cfg->lattice != LBM_D3Q15 && cfg->lattice != LBM_D3Q19 &&
        cfg->lattice != LBM_D3Q27)
        return set_err(nullptr, LBM_ERR_INVALID,
                       "If a default velocity set is chosen, it must be one of the following: [:D2Q9, :D3Q15, :D3Q19, :D3Q27]");
    if (vd != cfg->dims)
        return set_err(nullptr, LBM_ERR_INVALID,
                       "The chosen velocity must be " + std::to_string(cfg->dims) + "-dimensional!");
    if (cfg->collision != LBM_BGK && cfg->collision != LBM_TRT)
        return set_err(nullptr, LBM_ERR_INVALID, "Collision model is not implemented!");
    if (cfg->storage < LBM_STORE_F32 || cfg->storage > LBM_STORE_F64)
        return set_err(nullptr, LBM_ERR_INVALID, "unknown storage format");
    if (!(cfg->dx > 0) || !std::isfinite(cfg->dx)) return set_err(nullptr, LBM_ERR_INVALID, "latticeParameter must be positive");
    if (!(cfg->tau > 0.5 * cfg->dx)) return set_err(nullptr, LBM_ERR_INVALID, "relaxation time must exceed dt/2");
    if (cfg->collision == LBM_TRT && !(cfg->tau_minus > 0.5 * cfg->dx))
        return set_err(nullptr, LBM_ERR_INVALID, "TRT tau- must exceed dt/2");
    long long N = 1;
    for (int a = 0; a < 3; ++a) {
        const long long na = a < cfg->dims ? cfg->n[a] : 1;
        if (na < 1 || na > (1 << 20)) return set_err(nullptr, LBM_ERR_INVALID, "grid sizes must be in [1, 2^20]");
        N *= na;
    }
    if (N >= (1LL << 31)) return set_err(nullptr, LBM_ERR_UNSUPPORTED, "more than 2^31 lattice nodes");
    if (cfg->schedule < LBM_SCHEDULE_AUTO || cfg->schedule > LBM_SCHEDULE_PERSISTENT || cfg->schedule == 2)
        return set_err(nullptr, LBM_ERR_INVALID, "unknown schedule");
    if (cfg->force_mode < LBM_FORCE_NONE || cfg->force_mode > LBM_FORCE_FIELD)
        return set_err(nullptr, LBM_ERR_INVALID, "unknown force mode");
    if (cfg->force_mode == LBM_FORCE_FIELD && !cfg->force_field)
        return set_err(nullptr, LBM_ERR_INVALID, "force density does not have consistent dimensions!");
    if (!cfg->compressible && cfg->rho_init)
        return set_err(nullptr, LBM_ERR_UNSUPPORTED, "incompressible equilibrium with a non-uniform initial density");
    if (cfg->particle_rules != LBM_RULES_GPU_MODULE && cfg->particle_rules != LBM_RULES_CPU_MODULE)
        return set_err(nullptr, LBM_ERR_INVALID, "unknown particle rules");
    if (cfg->rounding != LBM_ROUND_STOCHASTIC && cfg->rounding != LBM_ROUND_NEAREST)
        return set_err(nullptr, LBM_ERR_INVALID, "unknown rounding");

    lbm_handle* h = new lbm_handle();
    h->device = device;
    h->dims = cfg->dims;
    h->lattice = cfg->lattice;
    h->q = cfg->lattice;
    h->storage = cfg->storage;
    h->trt = cfg->collision == LBM_TRT;
    for (int a = 0; a < 3; ++a) h->n[a] = a < cfg->dims ? (int)cfg->n[a] : 1;
    h->N = N;
    h->dx = cfg->dx;
    h->dt = cfg->dx;
    h->tau = cfg->tau;
    h->tau_minus = cfg->tau_minus;
    h->rho0 = cfg->rho_ref > 0 ? cfg->rho_ref : 1.0;
    h->scale = (cfg->storage == LBM_STORE_F16 || cfg->storage == LBM_STORE_BF16)
                   ? (cfg->store_scale > 0 ? cfg->store_scale : 4096.0)
                   : 1.0;
    h->force_mode = cfg->force_mode;
    h->particle_rules = cfg->particle_rules;
    h->rounding = cfg->rounding;
    h->schedule = cfg->schedule == LBM_SCHEDULE_AUTO ? LBM_SCHEDULE_STREAM : cfg->schedule;
    if (cfg->force_mode == LBM_FORCE_UNIFORM)
        for (int k = 0; k < cfg->dims; ++k) h->F[k] = cfg->force[k];
    h->incompressible = cfg->compressible ? 0 : 1;
    h->rho_inc = cfg->rho_uniform;
    if (!get_ops(h->lattice, h->storage, h->trt, &h->ops)) {
        delete h;
        return set_err(nullptr, LBM_ERR_INVALID, "no kernel instantiation for this configuration");
    }
    for (int a = 0; a < 3; ++a) {
        h->X[a].resize(h->n[a]);
        for (int i = 0; i < h->n[a]; ++i)
            h->X[a][i] = (a < cfg->dims && cfg->coords[a]) ? cfg->coords[a][i] : cfg->x0[a] + (double)i * h->dx;
        if (a < cfg->dims && !is_uniform_axis(h->X[a], h->dx)) {
            delete h;
            return set_err(nullptr, LBM_ERR_INVALID, "node coordinates must form a uniform grid with spacing dx");
        }
    }
    choose_tiles(h);
    if (!h->ops.bulk_v4 || h->force_mode == LBM_FORCE_FIELD) {  // scalar bulk kernel
        h->vrows = h->vnt1 = h->vblock = 0;
        h->vtiles = 0;
    }
    int rc = LBM_OK;
#define TRY(x)                       \
    do {                             \
        rc = (x);                    \
        if (rc != LBM_OK) {          \
            g_global_err = h->err;   \
            destroy_all(h);          \
            return rc;               \
        }                            \
    } while (0)
    TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess
            ? LBM_OK : set_err(h, LBM_ERR_CUDA, "stream creation failed"));
    {  // the side stream (fix-up, particle update) takes SM slots ahead of the bulk pass
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        TRY(cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, hi) == cudaSuccess
                ? LBM_OK : set_err(h, LBM_ERR_CUDA, "stream creation failed"));
    }
    TRY(cudaEventCreateWithFlags(&h->ev_fix, cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&h->ev_part, cudaEventDisableTiming) == cudaSuccess
            ? LBM_OK : set_err(h, LBM_ERR_CUDA, "event creation failed"));
    TRY(dev_alloc(h, &h->d_tq, sizeof(TickCounters)));
    if (cudaMemsetAsync(h->d_tq, 0, sizeof(TickCounters), h->stream) != cudaSuccess)
        TRY(set_err(h, LBM_ERR_CUDA, "memset failed"));
    if (h->vtiles > 0 && h->vblock == kTickBlock && h->ops.tick_fn) {  // persistent grid: all resident CTAs
        int per_sm = 0, sms = 0;
        const void* tfn = h->rounding == LBM_ROUND_STOCHASTIC ? h->ops.tick_fn_sr : h->ops.tick_fn;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tfn, kTickBlock, 0) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
            TRY(set_err(h, LBM_ERR_CUDA, "occupancy query failed"));
        h->tick_grid = (unsigned)std::max(0, per_sm * sms);
    }
    h->tma_ok = choose_tma(h, 0, 0, &h->tma);
    const size_t pop_bytes = (size_t)N * h->q * storage_bytes(h->storage);
    TRY(dev_alloc(h, &h->pop[0], pop_bytes));
    TRY(dev_alloc(h, &h->pop[1], pop_bytes));
    for (int a = 0; a < 3; ++a) {
        TRY(dev_alloc(h, &h->d_coord[a], sizeof(double) * h->n[a]));
        TRY(upload(h, h->d_coord[a], h->X[a].data(), sizeof(double) * h->n[a]));
    }
    TRY(dev_alloc(h, &h->d_err, sizeof(int)));
    if (cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream) != cudaSuccess)
        TRY(set_err(h, LBM_ERR_CUDA, "memset failed"));

    // walls (initMethods.jl:568-628): mask | {|u_w| > 0}
    std::vector<unsigned char> W;
    if (cfg->wall_mask || cfg->wall_velocity) {
        W.assign(N, 0);
        if (cfg->wall_mask)
            for (long long c = 0; c < N; ++c) W[c] = cfg->wall_mask[c] ? 1 : 0;
        if (cfg->wall_velocity) {
            for (long long c = 0; c < N; ++c)
                for (int k = 0; k < h->dims; ++k)
                    if (cfg->wall_velocity[k * N + c] != 0.0) W[c] = 1;
            TRY(dev_alloc(h, &h->d_uw, sizeof(double) * N * h->dims));
            TRY(upload(h, h->d_uw, cfg->wall_velocity, sizeof(double) * N * h->dims));
        }
        h->has_walls = true;
        TRY(dev_alloc(h, &h->d_wall, N));
        TRY(upload(h, h->d_wall, W.data(), N));
        std::vector<int2> wl;
        std::vector<int> wn;
        wall_lists(h, W, wl, wn);
        h->nwlinks = (int)wl.size();
        h->nwnodes = (int)wn.size();
        TRY(dev_alloc(h, &h->d_wlinks, sizeof(int2) * std::max<size_t>(1, wl.size())));
        TRY(dev_alloc(h, &h->d_wnodes, sizeof(int) * std::max<size_t>(1, wn.size())));
        if (!wl.empty()) TRY(upload(h, h->d_wlinks, wl.data(), sizeof(int2) * wl.size()));
        if (!wn.empty()) TRY(upload(h, h->d_wnodes, wn.data(), sizeof(int) * wn.size()));
        if (h->vtiles > 0) {  // vector tiles within one node of a wall node or wall link
            std::vector<unsigned char>& vn = h->vnear;
            vn.assign(h->vtiles, 0);
            auto mark = [&](long long c) {
                const int y = (int)((c / h->n[0]) % h->n[1]), z = (int)(c / ((long long)h->n[0] * h->n[1]));
                for (int dz = -1; dz <= 1; ++dz) {
                    if (h->dims == 2 && dz != 0) continue;
                    for (int dy = -1; dy <= 1; ++dy) {
                        const int yy = (y + dy + h->n[1]) % h->n[1], zz = (z + dz + h->n[2]) % h->n[2];
                        vn[yy / h->vrows + (long long)h->vnt1 * zz] = 1;
                    }
                }
            };
            for (const int2& e : wl) mark(e.x);
            for (int c : wn) mark(c);
            TRY(dev_alloc(h, &h->d_vnear, h->vtiles));
            TRY(upload(h, h->d_vnear, vn.data(), h->vtiles));
        }
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) TRY(set_err(h, LBM_ERR_CUDA, "upload failed"));
    }
    TRY(ensure_particle_capacity(h, 0));

    // force field, zeroed on walls (initMethods.jl:639-650)
    if (cfg->force_mode == LBM_FORCE_FIELD) {
        std::vector<double> ff(cfg->force_field, cfg->force_field + N * h->dims);
        if (h->has_walls)
            for (int k = 0; k < h->dims; ++k)
                for (long long c = 0; c < N; ++c)
                    if (W[c]) ff[k * N + c] = 0.0;
        TRY(dev_alloc(h, &h->d_ffield, sizeof(double) * N * h->dims));
        TRY(upload(h, h->d_ffield, ff.data(), sizeof(double) * N * h->dims));
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) TRY(set_err(h, LBM_ERR_CUDA, "upload failed"));
    }
    // initial populations on the device (findInitialConditions)
    size_t need = 0;
    if (cfg->rho_init) need += sizeof(double) * N;
    if (cfg->u_init) need += sizeof(double) * N * h->dims;
    if (need) TRY(ensure_tmp(h, need));
    InitArgs ia{};
    ia.pop = h->pop[0];
    ia.N = N;
    double* tp = h->d_tmp;
    if (cfg->rho_init) {
        TRY(upload(h, tp, cfg->rho_init, sizeof(double) * N));
        ia.rho = tp;
        tp += N;
    }
    if (cfg->u_init) {
        TRY(upload(h, tp, cfg->u_init, sizeof(double) * N * h->dims));
        ia.u = tp;
    }
    ia.wall = h->d_wall;
    ia.ffield = h->d_ffield;
    ia.rho_uniform = cfg->rho_uniform;
    for (int k = 0; k < 3; ++k) {
        ia.u_uniform[k] = cfg->u_uniform[k];
        ia.F[k] = h->F[k];
    }
    ia.dt = h->dt;
    ia.rho0 = h->rho0;
    ia.scale = h->scale;
    ia.zero_walls = (h->has_walls || h->trt) ? 1 : 0;
    ia.force_mode = h->force_mode;
    h->ops.init(ia, h->stream);
    if (cudaGetLastError() != cudaSuccess) TRY(set_err(h, LBM_ERR_CUDA, "initialisation kernel failed"));
    if (cudaMemsetAsync(h->pop[1], 0, pop_bytes, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
        TRY(set_err(h, LBM_ERR_CUDA, "initialisation failed"));
#undef TRY
    h->cur = 0;
    *out = h;
    return LBM_OK;
}

int lbm_add_particle(lbm_handle* h, const lbm_particle_params* p, int32_t* id_out) {
    if (!h || !p) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    if (p->kind != LBM_BEAD && p->kind != LBM_SQUIRMER) return set_err(h, LBM_ERR_INVALID, "unknown particle kind");
    if ((int)h->hparts.size() >= 255)
        return set_err(h, LBM_ERR_INVALID, "particle ids are UInt8 in the reference: at most 255 particles");
    if (!(p->radius > 0) || !std::isfinite(p->radius)) return set_err(h, LBM_ERR_INVALID, "radius must be positive");
    const int d = h->dims;
    // mass (initMethods.jl:18/108): node count of the origin-centred sphere
    const double r2 = p->radius * p->radius;
    long long count = 0;
    {
        std::vector<int> ax[3];
        for (int a = 0; a < 3; ++a) {
            if (a >= d) {
                ax[a].push_back(0);
                continue;
            }
            for (int i = 0; i < h->n[a]; ++i) {
                const double v = h->X[a][i];
                if (v * v < r2) ax[a].push_back(i);
            }
        }
        for (int z : ax[2])
            for (int y : ax[1])
                for (int x : ax[0]) {
                    const double a0 = h->X[0][x], a1 = h->X[1][y];
                    volatile double s = a0 * a0;
                    volatile double t1 = a1 * a1;
                    double s2 = s + t1;
                    if (d == 3) {
                        const double a2 = h->X[2][z];
                        volatile double t2 = a2 * a2;
                        s2 = s2 + t2;
                    }
                    if (s2 < r2) ++count;
                }
    }
    const double mass = p->mass_density * (double)count * std::pow(h->dx, d);
    const double inertia = d == 2 ? 0.5 * mass * r2 : 0.4 * mass * r2;
    ParticleDev P{};
    for (int k = 0; k < 3; ++k) {
        P.R[k] = k < d ? p->position[k] : 0.0;
        P.v[k] = k < d ? p->velocity[k] : 0.0;
        P.w[k] = d == 2 ? (k == 0 ? p->angular_velocity[0] : 0.0) : p->angular_velocity[k];
        P.e[k] = (p->kind == LBM_SQUIRMER && k < d) ? p->swimming_direction[k] : 0.0;
    }
    P.radius = p->radius;
    P.r2 = r2;
    P.B1 = p->kind == LBM_SQUIRMER ? p->B1 : 0.0;
    P.B2 = p->kind == LBM_SQUIRMER ? p->B2 : 0.0;
    P.inv_mass = 1.0 / mass;
    P.inv_inertia = 1.0 / inertia;
    P.kind = p->kind;
    P.coupleF = p->couple_forces ? 1 : 0;
    P.coupleT = p->couple_torques ? 1 : 0;
    P.valid = 0;
    P.rules = h->particle_rules;
    for (int k = 0; k < 3; ++k) {
        P.slo[k] = 1;
        P.shi[k] = 0;
    }
    // capacities from the widest index box of the sphere: solid box <= 2r/dx + 5
    // nodes per axis, near box (links) 2 more
    long long span = (long long)std::floor(2.0 * p->radius / h->dx) + 6;
    long long rows = 1, near = 1;
    for (int a = 0; a < 3; ++a) {
        if (a >= d) continue;
        if (a > 0) rows *= std::min<long long>(span, h->n[a]);
        near *= std::min<long long>(span + 2, h->n[a]);
    }
    if (near >= (1LL << 28)) return set_err(h, LBM_ERR_UNSUPPORTED, "particle too large for the link lists");
    const int pid = (int)h->hparts.size();
    long long ivl_off = 0, link_off = 0, part_off = 0;
    for (const auto& q : h->hparts) {
        ivl_off = std::max<long long>(ivl_off, (long long)q.ivl_off + q.ivl_cap);
        link_off = std::max<long long>(link_off, (long long)q.link_off + q.link_cap);
        part_off = std::max<long long>(part_off, (long long)q.part_off + (q.link_cap + kFixBlock - 1) / kFixBlock);
    }
    P.ivl_off = (int)ivl_off;
    P.ivl_cap = (int)rows;
    P.link_off = (int)link_off;
    P.link_cap = (int)near;
    P.part_off = (int)part_off;
    P.nlinks = 0;
    const long long chunks = (near + kFixBlock - 1) / kFixBlock;
    int rc = ensure_particle_capacity(h, pid + 1);
    if (rc) return rc;
    rc = grow(h, &h->d_ivl, &h->ivl_slots, ivl_off + rows, ivl_off);
    if (rc) return rc;
    rc = grow(h, &h->d_links, &h->link_slots, link_off + near, link_off);
    if (rc) return rc;
    rc = grow(h, &h->d_partial, &h->partial_slots, (part_off + chunks) * kPartialStride, 0);
    if (rc) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(h->d_parts + pid, &P, sizeof(P), cudaMemcpyHostToDevice, h->stream));
    h->hparts.push_back(P);
    h->maxchunks = std::max<int>(h->maxchunks, (int)chunks);
    h->link_bpp = std::max<int>(h->link_bpp, (int)((near + kLinkBlock - 1) / kLinkBlock));
    rc = grow(h, &h->d_linkcnt, &h->linkcnt_slots, (long long)(pid + 1) * h->link_bpp, 0);
    if (rc) return rc;
    drop_graphs(h);
    if (!h->inter.empty()) {  // the contribution lists cover every particle
        rc = upload_interactions(h);
        if (rc) return rc;
    }
    if (h->trj_cap > 0) {  // the ring holds every particle: start it again with this one
        rc = trj_alloc(h, h->trj_cap);
        if (rc) return rc;
    }
    // initial setup: moveParticles!(initialSetup = true)
    h->ops.particles(particle_args(h, 1, pid), 1, h->stream);
    CUDA_TRY(h, cudaGetLastError());
    rc = check_device_error(h);
    if (rc) return rc;
    if (id_out) *id_out = pid + 1;
    return LBM_OK;
}

int lbm_step(lbm_handle* h, int64_t nsteps) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    if (nsteps < 0) return set_err(h, LBM_ERR_INVALID, "ticks must be non-negative");
    BIND(h);
    {
        const int rc = prepare_tick(h);
        if (rc) return rc;
    }
    const bool direct = h->calls++ == 0 && nsteps <= kFirstCallDirectTicks;
    if (nsteps > 0 && !direct) {
        const int rc = ensure_graphs(h, nsteps);
        if (rc) return rc;
    }
    if (h->profiling) CUDA_TRY(h, cudaEventRecord(h->t_begin, h->stream));
    int64_t done = 0;
    int slots_used = 0;
    if (direct) {
        for (; done < nsteps; ++done) {
            enqueue_tick(h, h->cur, (int)done);
            h->cur = 1 - h->cur;
        }
        slots_used = (int)nsteps;
    }
    while (done < nsteps) {
        int k = 0;
        while (kModelGraphSizes[k] > nsteps - done) ++k;  // the last size is 1
        CUDA_TRY(h, cudaGraphLaunch(h->graphs[h->profiling >= 2 ? 1 : 0][h->cur][k].exec, h->stream));
        done += kModelGraphSizes[k];
        if (kModelGraphSizes[k] & 1) h->cur = 1 - h->cur;
        slots_used = std::max(slots_used, kModelGraphSizes[k]);
    }
    join_particles(h);
    if (h->profiling) CUDA_TRY(h, cudaEventRecord(h->t_end, h->stream));
    CUDA_TRY(h, cudaGetLastError());
    for (int64_t s = 0; s < nsteps; ++s) h->time += h->dt;
    h->tick += nsteps;
    int rc = check_device_error(h);
    lbm_profile& p = h->prof;
    p = lbm_profile{};
    p.steps = nsteps;
    p.launches = nsteps * launches_per_tick(h);
    p.bulk_cells = h->N;
    if (h->profiling && nsteps > 0) {
        float ms = 0;
        CUDA_TRY(h, cudaEventElapsedTime(&ms, h->t_begin, h->t_end));
        p.total_ms = ms;
        const bool fused = use_tick_kernel(h);  // one kernel: its time is reported as bulk_ms
        const bool fix = !fused && fixup_blocks(h) > 0;
        double sb = 0, sf = 0, sp = 0;
        if (h->profiling < 2) slots_used = 0;  // per-kernel events were not recorded
        for (int s = 0; s < slots_used; ++s) {
            CUDA_TRY(h, cudaEventElapsedTime(&ms, prof_event(h, s, 0), prof_event(h, s, 1)));
            sb += ms;
            if (fix) {
                CUDA_TRY(h, cudaEventElapsedTime(&ms, prof_event(h, s, 1), prof_event(h, s, 2)));
                sf += ms;
            }
            if (!fused && !h->hparts.empty()) {
                CUDA_TRY(h, cudaEventElapsedTime(&ms, prof_event(h, s, 2), prof_event(h, s, 3)));
                sp += ms;
            }
        }
        p.bulk_ms = slots_used ? sb / slots_used : 0.0;
        p.fixup_ms = slots_used ? sf / slots_used : 0.0;
        p.particles_ms = slots_used ? sp / slots_used : 0.0;
        p.profiled_steps = slots_used;
        long long entries = h->nwlinks;
        if (!h->hparts.empty()) {
            std::vector<ParticleDev> tmp(h->hparts.size());
            CUDA_TRY(h, cudaMemcpy(tmp.data(), h->d_parts, sizeof(ParticleDev) * tmp.size(), cudaMemcpyDeviceToHost));
            for (const auto& q : tmp) entries += q.nlinks;
        }
        p.fixup_entries = entries;
    }
    return rc;
}

int lbm_set_profiling(lbm_handle* h, int32_t on) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    BIND(h);
    if (on && h->pev.empty()) {
        h->pev.resize(4 * kModelGraphTicks);
        for (auto& e : h->pev) CUDA_TRY(h, cudaEventCreate(&e));
        CUDA_TRY(h, cudaEventCreate(&h->t_begin));
        CUDA_TRY(h, cudaEventCreate(&h->t_end));
    }
    h->profiling = on < 0 ? 0 : (on > 2 ? 2 : on);
    return LBM_OK;
}

int lbm_get_profile(lbm_handle* h, lbm_profile* out) {
    if (!h || !out) return set_err(h, LBM_ERR_INVALID, "null argument");
    *out = h->prof;
    return LBM_OK;
}

int lbm_set_wait_limit(lbm_handle* h, int64_t polls, int32_t target_offset) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    if (polls < 1 || polls > kSpinLimit)
        return set_err(h, LBM_ERR_INVALID, "the wait limit must lie in [1, " + std::to_string(kSpinLimit) + "] polls");
    if (target_offset < 0 || target_offset > 1) return set_err(h, LBM_ERR_INVALID, "target_offset must be 0 or 1");
    BIND(h);
    h->spin_limit = polls;
    h->wait_extra = target_offset;
    drop_graphs(h);  // the graphs hold the tick kernel's arguments
    return LBM_OK;
}

int lbm_set_bulk_kernel(lbm_handle* h, int32_t kind, int32_t threads, int32_t stages) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    if (kind != LBM_BULK_AUTO && kind != LBM_BULK_VECTOR && kind != LBM_BULK_TMA)
        return set_err(h, LBM_ERR_INVALID, "unknown bulk kernel");
    if (h->in_batch) return set_err(h, LBM_ERR_STATE, "a batch replica's kernels belong to its batch");
    BIND(h);
    if (kind == LBM_BULK_VECTOR && !use_vector_bulk(h))
        return set_err(h, LBM_ERR_UNSUPPORTED, "the vector bulk kernel does not apply to this model");
    if (kind == LBM_BULK_VECTOR && threads != 0) {  // CTA size of the vector kernel (tiles of whole x-rows)
        const int RT = h->n[0] / 4;
        if ((threads != 32 && threads != 64 && threads != 96 && threads != 128 && threads != 256 && threads != 512) ||
            threads < RT || threads % RT != 0 || h->schedule == LBM_SCHEDULE_PERSISTENT)
            return set_err(h, LBM_ERR_UNSUPPORTED,
                           "vector kernel CTAs hold whole x-rows: 32, 64, 96, 128, 256 or 512 threads, a multiple of "
                           "nx/4 (stream schedule)");
        set_vector_block(h, threads);
    }
    if (kind != LBM_BULK_VECTOR) {
        TmaShape sh{};
        if (!choose_tma(h, threads, stages, &sh)) {
            if (kind == LBM_BULK_TMA)
                return set_err(h, LBM_ERR_UNSUPPORTED,
                               "the TMA bulk kernel does not apply to this model or launch shape (x-rows of 4*2^k "
                               "<= 128 nodes, 16-byte aligned rows, no force field, shared memory <= 227 KB)");
            h->tma_ok = false;
        } else {
            h->tma = sh;
            h->tma_ok = true;
        }
    }
    h->bulk_kind = kind;
    drop_graphs(h);
    return LBM_OK;
}

int lbm_set_memory_limit(int64_t bytes) {
    if (bytes < 0) return set_err(nullptr, LBM_ERR_INVALID, "the memory limit must be non-negative");
    g_mem_limit.store(bytes);
    return LBM_OK;
}

int lbm_time_kernel(lbm_handle* h, int32_t kernel, int32_t launches, double* avg_ms) {
    if (!h || !avg_ms) return set_err(h, LBM_ERR_INVALID, "null argument");
    if (kernel < LBM_KERNEL_BULK || kernel > LBM_KERNEL_TICK || launches < 1)
        return set_err(h, LBM_ERR_INVALID, "unknown kernel or launch count");
    BIND(h);
    const int np = (int)h->hparts.size();
    if (kernel == LBM_KERNEL_FIXUP && fixup_blocks(h) == 0) return set_err(h, LBM_ERR_STATE, "model has no boundary links");
    if (kernel == LBM_KERNEL_PARTICLES && np == 0) return set_err(h, LBM_ERR_STATE, "model has no particles");
    if (kernel == LBM_KERNEL_TICK) {
        if (!use_tick_kernel(h)) return set_err(h, LBM_ERR_STATE, "the persistent tick kernel does not apply");
        const int rc0 = prepare_tick(h);
        if (rc0) return rc0;
    }
    // save everything the launches touch
    const size_t pop_bytes = (size_t)h->N * h->q * storage_bytes(h->storage);
    const size_t parts_b = sizeof(ParticleDev) * np, ivl_b = sizeof(int2) * h->ivl_slots,
                 link_b = sizeof(int2) * h->link_slots, bits_b = sizeof(unsigned long long) * h->g.ntiles * h->words,
                 box_b = sizeof(int) * 6 * np;
    const size_t save_b = 2 * pop_bytes + parts_b + ivl_b + link_b + bits_b + 2 * box_b;
    char* save = nullptr;
    int rc = dev_alloc(h, &save, save_b);
    if (rc) return rc;
    char* sp = save;
    const void* srcs[8] = {h->pop[0], h->pop[1], h->d_parts, h->d_ivl, h->d_links, h->d_tilebits, h->d_nbox[0], h->d_nbox[1]};
    const size_t sizes[8] = {pop_bytes, pop_bytes, parts_b, ivl_b, link_b, bits_b, box_b, box_b};
    for (int k = 0; k < 8; ++k) {
        if (sizes[k] && srcs[k]) CUDA_TRY(h, cudaMemcpyAsync(sp, srcs[k], sizes[k], cudaMemcpyDeviceToDevice, h->stream));
        sp += sizes[k];
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUDA_TRY(h, cudaEventCreate(&e0));
    CUDA_TRY(h, cudaEventCreate(&e1));
    int b = h->cur;
    CUDA_TRY(h, cudaEventRecord(e0, h->stream));
    for (int l = 0; l < launches; ++l) {
        const StepArgs a = step_args(h, b);
        if (kernel == LBM_KERNEL_BULK) {
            launch_bulk(h, a, h->stream);
            b = 1 - b;
        } else if (kernel == LBM_KERNEL_FIXUP) {
            h->ops.fixup(a, (unsigned)fixup_grid(h), h->stream, false, fixup_walk(h));
        } else if (kernel == LBM_KERNEL_TICK) {
            h->ops.tick(h->d_targs + b, h->d_pargs + b, h->items, h->d_tq, h->d_err, h->tick_grid, h->stream,
                        h->rounding == LBM_ROUND_STOCHASTIC);
            b = 1 - b;
        } else {
            const ParticleArgs pa = particle_args(h, 0, 0, b);
            h->ops.particles(pa, (unsigned)np, h->stream);
            h->ops.links(pa, np, h->link_bpp, h->d_linkcnt, h->stream);
        }
    }
    CUDA_TRY(h, cudaEventRecord(e1, h->stream));
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaEventSynchronize(e1));
    float ms = 0;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *avg_ms = ms / launches;
    sp = save;
    void* dsts[8] = {h->pop[0], h->pop[1], h->d_parts, h->d_ivl, h->d_links, h->d_tilebits, h->d_nbox[0], h->d_nbox[1]};
    for (int k = 0; k < 8; ++k) {
        if (sizes[k] && dsts[k]) CUDA_TRY(h, cudaMemcpyAsync(dsts[k], sp, sizes[k], cudaMemcpyDeviceToDevice, h->stream));
        sp += sizes[k];
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    dev_free(save);
    h->device_bytes -= save_b;
    return check_device_error(h);
}

int lbm_get_fields(lbm_handle* h, double* rho, double* u) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    BIND(h);
    const size_t nb = sizeof(double) * h->N * (1 + h->dims);
    int rc = ensure_tmp(h, nb);
    if (rc) return rc;
    CodecArgs c = codec_args(h);
    c.rho = h->d_tmp;
    c.u = h->d_tmp + h->N;
    h->ops.macro(c, h->stream);
    CUDA_TRY(h, cudaGetLastError());
    if (rho) CUDA_TRY(h, cudaMemcpyAsync(rho, c.rho, sizeof(double) * h->N, cudaMemcpyDeviceToHost, h->stream));
    if (u) CUDA_TRY(h, cudaMemcpyAsync(u, c.u, sizeof(double) * h->N * h->dims, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

int lbm_get_stress(lbm_handle* h, double* sigma) {
    if (!h || !sigma) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    const size_t nb = sizeof(double) * h->N * h->dims * h->dims;
    int rc = ensure_tmp(h, nb);
    if (rc) return rc;
    CodecArgs c = codec_args(h);
    c.stress = h->d_tmp;
    c.stress_coeff = 1.0 - 0.5 * h->dt / h->tau;
    c.incompressible = h->incompressible;
    c.rho_inc = h->rho_inc;
    h->ops.stress(c, h->stream);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaMemcpyAsync(sigma, c.stress, nb, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

int lbm_get_totals(lbm_handle* h, double* mass, double* momentum) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    BIND(h);
    const long long nb = (h->N + kTotBlock - 1) / kTotBlock;
    int rc = ensure_tmp(h, sizeof(double) * (4 * nb + 4));
    if (rc) return rc;
    CodecArgs c = codec_args(h);
    h->ops.totals(c, h->d_tmp, h->d_tmp + 4 * nb, h->stream);
    CUDA_TRY(h, cudaGetLastError());
    double t[4];
    CUDA_TRY(h, cudaMemcpyAsync(t, h->d_tmp + 4 * nb, sizeof(t), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (mass) *mass = t[0];
    if (momentum)
        for (int k = 0; k < 3; ++k) momentum[k] = k < h->dims ? t[1 + k] : 0.0;
    return LBM_OK;
}

int lbm_record_trajectories(lbm_handle* h, int64_t capacity) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    if (capacity < 0) return set_err(h, LBM_ERR_INVALID, "capacity must be non-negative");
    BIND(h);
    return trj_alloc(h, capacity);
}

int lbm_read_trajectories(lbm_handle* h, double* out, int64_t capacity, int64_t* ticks) {
    if (!h || !ticks) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    *ticks = 0;
    if (h->trj_cap == 0 || h->hparts.empty()) return LBM_OK;
    long long nrec = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&nrec, &h->d_parts[0].nrec, sizeof(nrec), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    const long long n = nrec - h->trj_read;
    *ticks = n;
    if (!out) return LBM_OK;
    if (n > h->trj_cap)
        return set_err(h, LBM_ERR_STATE, "trajectory records were overwritten: " + std::to_string(n) +
                                             " ticks since the last read, the ring holds " + std::to_string(h->trj_cap));
    if (n > capacity) return set_err(h, LBM_ERR_INVALID, "output buffer holds fewer ticks than were recorded");
    const size_t per = 9 * h->hparts.size();  // doubles per tick
    for (long long t = h->trj_read; t < nrec;) {  // at most two contiguous pieces of the ring
        const long long slot = t % h->trj_cap;
        const long long len = std::min(nrec - t, h->trj_cap - slot);
        CUDA_TRY(h, cudaMemcpyAsync(out + (t - h->trj_read) * per, h->d_trj + slot * per, sizeof(double) * per * len,
                                    cudaMemcpyDeviceToHost, h->stream));
        t += len;
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->trj_read = nrec;
    return LBM_OK;
}

int lbm_output_flush(lbm_handle* h) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    if (h->writer.joinable()) h->writer.join();
    if (!h->writer_err.empty()) {
        const std::string e = h->writer_err;
        h->writer_err.clear();
        return set_err(h, LBM_ERR_INVALID, e);
    }
    return LBM_OK;
}

// writeTrajectories (src/gpu/aux.jl:271-317): one row per node in column-major
// order with tick, time, the 1-based node indices, coordinates, density,
// velocity and the Q populations, as CSV.jl writes them.  The fields are read
// back here; formatting and writing run on a host thread while the caller
// goes on stepping.
int lbm_write_fluid_csv(lbm_handle* h, const char* path) {
    if (!h || !path) return set_err(h, LBM_ERR_INVALID, "null argument");
    int rc = lbm_output_flush(h);  // one snapshot in flight at a time
    if (rc) return rc;
    BIND(h);
    const long long N = h->N;
    const int d = h->dims, q = h->q;
    auto rho = std::make_shared<std::vector<double>>(N);
    auto u = std::make_shared<std::vector<double>>((size_t)N * d);
    auto f = std::make_shared<std::vector<double>>((size_t)N * q);
    rc = lbm_get_fields(h, rho->data(), u->data());
    if (!rc) rc = lbm_get_distributions(h, f->data());
    if (rc) return rc;
    std::vector<double> X[3] = {h->X[0], h->X[1], h->X[2]};
    const int n[3] = {h->n[0], h->n[1], h->n[2]};
    const long long tick = h->tick;
    const double time = h->time;
    const std::string file(path);
    h->writer = std::thread([h, rho, u, f, X, n, N, d, q, tick, time, file]() {
        FILE* fp = std::fopen(file.c_str(), "w");
        if (!fp) {
            h->writer_err = "cannot open " + file;
            return;
        }
        static const char* ax = "xyz";
        std::string line = "tick,time";
        for (int a = 0; a < d; ++a) line += std::string(",id_") + ax[a];
        for (int a = 0; a < d; ++a) line += std::string(",coordinate_") + ax[a];
        line += ",massDensity";
        for (int a = 0; a < d; ++a) line += std::string(",fluidVelocity_") + ax[a];
        for (int i = 1; i <= q; ++i) line += ",f" + std::to_string(i);
        line += '\n';
        std::string head = std::to_string(tick) + ",";
        julia_float(time, head);
        bool ok = std::fputs(line.c_str(), fp) >= 0;
        std::string buf;
        buf.reserve(1 << 22);
        for (long long c = 0; c < N && ok; ++c) {
            const long long idx[3] = {c % n[0], (c / n[0]) % n[1], c / ((long long)n[0] * n[1])};
            buf += head;
            for (int a = 0; a < d; ++a) buf += "," + std::to_string(idx[a] + 1);
            for (int a = 0; a < d; ++a) {
                buf += ',';
                julia_float(X[a][idx[a]], buf);
            }
            buf += ',';
            julia_float((*rho)[c], buf);
            for (int a = 0; a < d; ++a) {
                buf += ',';
                julia_float((*u)[(size_t)a * N + c], buf);
            }
            for (int i = 0; i < q; ++i) {
                buf += ',';
                julia_float((*f)[(size_t)i * N + c], buf);
            }
            buf += '\n';
            if (buf.size() > (1 << 22) - 4096) {
                ok = std::fwrite(buf.data(), 1, buf.size(), fp) == buf.size();
                buf.clear();
            }
        }
        if (ok && !buf.empty()) ok = std::fwrite(buf.data(), 1, buf.size(), fp) == buf.size();
        if (std::fclose(fp) != 0 || !ok) h->writer_err = "short write to " + file;
    });
    return LBM_OK;
}

int lbm_get_distributions(lbm_handle* h, double* f) {
    if (!h || !f) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    const size_t nb = sizeof(double) * h->N * h->q;
    int rc = ensure_tmp(h, nb);
    if (rc) return rc;
    CodecArgs c = codec_args(h);
    c.f64 = h->d_tmp;
    h->ops.decode(c, h->stream);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaMemcpyAsync(f, c.f64, nb, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

int lbm_set_distributions(lbm_handle* h, const double* f) {
    if (!h || !f) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    const size_t nb = sizeof(double) * h->N * h->q;
    int rc = ensure_tmp(h, nb);
    if (rc) return rc;
    CodecArgs c = codec_args(h);
    c.f64 = h->d_tmp;
    CUDA_TRY(h, cudaMemcpyAsync(c.f64, f, nb, cudaMemcpyHostToDevice, h->stream));
    h->ops.encode(c, h->stream);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

int lbm_get_particles(lbm_handle* h, lbm_particle_state* out, int32_t capacity, int32_t* count) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    BIND(h);
    const int np = (int)h->hparts.size();
    if (count) *count = np;
    if (!out || capacity <= 0 || np == 0) return LBM_OK;
    std::vector<ParticleDev> tmp(np);
    CUDA_TRY(h, cudaMemcpyAsync(tmp.data(), h->d_parts, sizeof(ParticleDev) * np, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (int i = 0; i < np && i < capacity; ++i) {
        const ParticleDev& P = tmp[i];
        lbm_particle_state& s = out[i];
        std::memset(&s, 0, sizeof(s));
        s.id = i + 1;
        s.kind = P.kind;
        s.couple_forces = P.coupleF;
        s.couple_torques = P.coupleT;
        s.radius = P.radius;
        s.inverse_mass = P.inv_mass;
        s.inverse_inertia = P.inv_inertia;
        s.B1 = P.B1;
        s.B2 = P.B2;
        for (int k = 0; k < 3; ++k) {
            s.position[k] = P.R[k];
            s.velocity[k] = P.v[k];
            s.angular_velocity[k] = P.w[k];
            s.swimming_direction[k] = P.e[k];
            s.last_force[k] = P.lastF[k];
            s.last_torque[k] = P.lastT[k];
        }
    }
    return LBM_OK;
}

int lbm_set_particle(lbm_handle* h, int32_t id, const lbm_particle_state* s) {
    if (!h || !s) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    if (id < 1 || id > (int)h->hparts.size()) return set_err(h, LBM_ERR_INVALID, "no such particle");
    ParticleDev P;
    CUDA_TRY(h, cudaMemcpyAsync(&P, h->d_parts + (id - 1), sizeof(P), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (int k = 0; k < 3; ++k) {
        P.R[k] = s->position[k];
        P.v[k] = s->velocity[k];
        P.w[k] = s->angular_velocity[k];
        P.e[k] = s->swimming_direction[k];
    }
    CUDA_TRY(h, cudaMemcpyAsync(h->d_parts + (id - 1), &P, sizeof(P), cudaMemcpyHostToDevice, h->stream));
    h->ops.particles(particle_args(h, 1, id - 1), 1, h->stream);
    CUDA_TRY(h, cudaGetLastError());
    return check_device_error(h);
}

int lbm_set_interactions(lbm_handle* h, const lbm_interaction* list, int32_t n) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    if (n < 0 || (n > 0 && !list)) return set_err(h, LBM_ERR_INVALID, "bad interaction list");
    if (n > (1 << 26)) return set_err(h, LBM_ERR_UNSUPPORTED, "too many interaction items");
    BIND(h);
    if (n > 0 && h->particle_rules != LBM_RULES_GPU_MODULE)
        return set_err(h, LBM_ERR_UNSUPPORTED, "the CPU module has no particle interactions");
    const int np = (int)h->hparts.size();
    for (int t = 0; t < n; ++t) {
        const lbm_interaction& e = list[t];
        if (e.kind < LBM_INTERACTION_LINEAR || e.kind > LBM_INTERACTION_DIPOLE)
            return set_err(h, LBM_ERR_INVALID, "unknown interaction kind");
        const bool three = e.kind == LBM_INTERACTION_POLAR;
        if (e.id1 < 1 || e.id1 > np || e.id2 < 1 || e.id2 > np || (three && (e.id3 < 1 || e.id3 > np)) ||
            e.id1 == e.id2 || (three && (e.id3 == e.id1 || e.id3 == e.id2)))
            return set_err(h, LBM_ERR_INVALID, "interaction " + std::to_string(t + 1) + " names no valid particles");
    }
    h->inter.assign(list, list + n);
    const int rc = upload_interactions(h);
    if (rc) {
        h->inter.clear();
        return rc;
    }
    drop_graphs(h);  // the graphs hold the interaction and particle kernels' arguments
    return LBM_OK;
}

int lbm_record_force(lbm_handle* h, int32_t id, int32_t on) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    BIND(h);
    if (id < 1 || id > (int)h->hparts.size()) return set_err(h, LBM_ERR_INVALID, "no such particle");
    const int v = on ? 1 : 0;
    CUDA_TRY(h, cudaMemcpyAsync(&h->d_parts[id - 1].recordF, &v, sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

int lbm_get_mask(lbm_handle* h, int32_t id, uint8_t* mask) {
    if (!h || !mask) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    if (id < 1 || id > (int)h->hparts.size()) return set_err(h, LBM_ERR_INVALID, "no such particle");
    int rc = ensure_tmp(h, h->N);
    if (rc) return rc;
    MaskArgs m{};
    m.mask = reinterpret_cast<unsigned char*>(h->d_tmp);
    m.part = h->d_parts + (id - 1);
    m.ivl = h->d_ivl;
    for (int k = 0; k < 3; ++k) m.n[k] = h->n[k];
    m.N = h->N;
    h->ops.mask(m, h->stream);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaMemcpyAsync(mask, m.mask, h->N, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

// Boundary links of a particle as the fix-up kernel sees them: the entries
// (fluid cell, direction mask) of its device link list, bit j of the mask set
// where x - c_j is solid (the streamingInvasionRegions of bounceBackPrep,
// src/gpu/aux.jl:187-198), expanded to (cell, direction) pairs sorted by
// (direction, cell).
int lbm_get_links(lbm_handle* h, int32_t id, int64_t* cells, int8_t* dirs, int64_t capacity, int64_t* n) {
    if (!h || !n) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    if (id < 1 || id > (int)h->hparts.size()) return set_err(h, LBM_ERR_INVALID, "no such particle");
    ParticleDev P;
    CUDA_TRY(h, cudaMemcpyAsync(&P, h->d_parts + (id - 1), sizeof(P), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (P.relink) return set_err(h, LBM_ERR_STATE, "the particle's link list awaits its rebuild");
    std::vector<int2> ent(std::max(0, P.nlinks));
    if (!ent.empty())
        CUDA_TRY(h, cudaMemcpyAsync(ent.data(), h->d_links + P.link_off, sizeof(int2) * ent.size(),
                                    cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    std::vector<std::vector<int64_t>> per(h->q);
    for (const int2& e : ent)
        for (int j = 1; j < h->q; ++j)
            if ((unsigned)e.y >> j & 1u) per[j].push_back(e.x);
    int64_t k = 0;
    for (int j = 0; j < h->q; ++j) {
        std::sort(per[j].begin(), per[j].end());
        for (int64_t x : per[j]) {
            if (cells && dirs && k < capacity) {
                cells[k] = x;
                dirs[k] = (int8_t)j;
            }
            ++k;
        }
    }
    *n = k;
    return LBM_OK;
}

int lbm_get_info(lbm_handle* h, lbm_info* info) {
    if (!h || !info) return set_err(h, LBM_ERR_INVALID, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->dims = h->dims;
    info->lattice = h->lattice;
    info->q = h->q;
    info->storage = h->storage;
    for (int a = 0; a < 3; ++a) info->n[a] = h->n[a];
    info->cells = h->N;
    info->tick = h->tick;
    info->time = h->time;
    info->num_particles = (int32_t)h->hparts.size();
    info->bytes_per_population = storage_bytes(h->storage);
    info->device_bytes = (int64_t)h->device_bytes;
    if (use_tma_bulk(h)) {
        info->bulk_kernel = LBM_BULK_TMA;
        info->bulk_threads = h->tma.rows * (h->n[0] / 4);
        info->bulk_stages = h->tma.stages;
    } else {
        info->bulk_kernel = use_vector_bulk(h) ? LBM_BULK_VECTOR : LBM_BULK_SCALAR;
        info->bulk_threads = use_vector_bulk(h) ? h->vblock : h->g.t[0] * h->g.t[1];
        info->bulk_stages = 0;
    }
    return LBM_OK;
}

// checkpoint: magic, header ints, tick/time, raw populations, particle records
int lbm_save_state(lbm_handle* h, const char* path) {
    if (!h || !path) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    const size_t pop_bytes = (size_t)h->N * h->q * storage_bytes(h->storage);
    std::vector<char> buf(pop_bytes);
    CUDA_TRY(h, cudaMemcpyAsync(buf.data(), h->pop[h->cur], pop_bytes, cudaMemcpyDeviceToHost, h->stream));
    const int np = (int)h->hparts.size();
    std::vector<ParticleDev> parts(np);
    if (np) CUDA_TRY(h, cudaMemcpyAsync(parts.data(), h->d_parts, sizeof(ParticleDev) * np, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return set_err(h, LBM_ERR_INVALID, std::string("cannot open ") + path);
    const int32_t hdr[8] = {0x4c424d42, LBM_ABI_VERSION, h->lattice, h->storage, h->n[0], h->n[1], h->n[2], np};
    bool ok = std::fwrite(hdr, sizeof(hdr), 1, fp) == 1;
    ok = ok && std::fwrite(&h->tick, sizeof(h->tick), 1, fp) == 1;
    ok = ok && std::fwrite(&h->time, sizeof(h->time), 1, fp) == 1;
    ok = ok && std::fwrite(buf.data(), 1, pop_bytes, fp) == pop_bytes;
    if (np) ok = ok && std::fwrite(parts.data(), sizeof(ParticleDev), np, fp) == (size_t)np;
    std::fclose(fp);
    return ok ? LBM_OK : set_err(h, LBM_ERR_INVALID, "short write");
}

int lbm_load_state(lbm_handle* h, const char* path) {
    if (!h || !path) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return set_err(h, LBM_ERR_INVALID, std::string("cannot open ") + path);
    int32_t hdr[8];
    bool ok = std::fread(hdr, sizeof(hdr), 1, fp) == 1;
    const int np = (int)h->hparts.size();
    if (!ok || hdr[0] != 0x4c424d42 || hdr[2] != h->lattice || hdr[3] != h->storage || hdr[4] != h->n[0] ||
        hdr[5] != h->n[1] || hdr[6] != h->n[2] || hdr[7] != np) {
        std::fclose(fp);
        return set_err(h, LBM_ERR_INVALID, "checkpoint does not match this model (lattice, storage, grid, particles)");
    }
    long long tick = 0;
    double time = 0;
    const size_t pop_bytes = (size_t)h->N * h->q * storage_bytes(h->storage);
    std::vector<char> buf(pop_bytes);
    std::vector<ParticleDev> parts(np);
    ok = std::fread(&tick, sizeof(tick), 1, fp) == 1 && std::fread(&time, sizeof(time), 1, fp) == 1 &&
         std::fread(buf.data(), 1, pop_bytes, fp) == pop_bytes &&
         (np == 0 || std::fread(parts.data(), sizeof(ParticleDev), np, fp) == (size_t)np);
    std::fclose(fp);
    if (!ok) return set_err(h, LBM_ERR_INVALID, "truncated checkpoint");
    // clear the tile bits of the current geometry, then restore and re-voxelise
    CUDA_TRY(h, cudaMemsetAsync(h->d_tilebits, 0, sizeof(unsigned long long) * h->g.ntiles * h->words, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->pop[h->cur], buf.data(), pop_bytes, cudaMemcpyHostToDevice, h->stream));
    for (int i = 0; i < np; ++i) {
        const ParticleDev& hp = h->hparts[i];
        parts[i].ivl_off = hp.ivl_off;
        parts[i].ivl_cap = hp.ivl_cap;
        parts[i].link_off = hp.link_off;
        parts[i].link_cap = hp.link_cap;
        parts[i].part_off = hp.part_off;
        parts[i].valid = 0;
        for (int k = 0; k < 3; ++k) {
            parts[i].slo[k] = 1;
            parts[i].shi[k] = 0;
        }
    }
    if (np) CUDA_TRY(h, cudaMemcpyAsync(h->d_parts, parts.data(), sizeof(ParticleDev) * np, cudaMemcpyHostToDevice, h->stream));
    for (int i = 0; i < np; ++i) h->ops.particles(particle_args(h, 2, i), 1, h->stream);
    CUDA_TRY(h, cudaGetLastError());
    h->tick = tick;
    h->time = time;
    return check_device_error(h);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free stepping (lbm_step_noalloc)
// ---------------------------------------------------------------------------
namespace {

// Momentum-exchange partials of lbm_step_noalloc, compiled into the library
// image: LBM_NOALLOC_SLOTS slots of kPartialStride doubles (1 MiB) that every
// device loading the library holds until the process exits.  In host code
// this name only stands for the symbol; the kernels get the device address
// that cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) double g_noalloc_partials[LBM_NOALLOC_SLOTS * kPartialStride];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_addr[kNoallocMaxDevices] = {};

// device address of g_noalloc_partials on the handle's device (current after BIND)
int noalloc_scratch(lbm_handle* h, double** out) {
    if (h->device < 0 || h->device >= kNoallocMaxDevices)
        return set_err(h, LBM_ERR_UNSUPPORTED, "lbm_step_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[h->device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return set_err(h, LBM_ERR_CUDA,
                           std::string("lbm_step_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        }
        g_noalloc_addr[h->device] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[h->device];
    return LBM_OK;
}

}  // namespace

extern "C" {

// lbm_step without allocation: direct launches on the handle's stream, the
// fix-up partials in g_noalloc_partials (see include/lbm_b200.h)
int lbm_step_noalloc(lbm_handle* h, int64_t nsteps) {
    if (!h) return set_err(h, LBM_ERR_INVALID, "null handle");
    if (nsteps < 0) return set_err(h, LBM_ERR_INVALID, "ticks must be non-negative");
    BIND(h);
    long long slots = 0;  // partial slots the particles use: max(part_off + chunks)
    for (const ParticleDev& q : h->hparts)
        slots = std::max<long long>(slots, (long long)q.part_off + (q.link_cap + kFixBlock - 1) / kFixBlock);
    if (slots > LBM_NOALLOC_SLOTS) {
        char msg[192];
        std::snprintf(msg, sizeof(msg),
                      "lbm_step_noalloc: the particles need %lld momentum-exchange slots; the fixed array holds %d",
                      slots, LBM_NOALLOC_SLOTS);
        return set_err(h, LBM_ERR_UNSUPPORTED, msg);
    }
    double* scratch = nullptr;
    int rc = noalloc_scratch(h, &scratch);
    if (rc) return rc;
    if (slots > 0)  // slots used by this model start from zero in every call
        CUDA_TRY(h, cudaMemsetAsync(scratch, 0, sizeof(double) * kPartialStride * slots, h->stream));
    ParticleArgs pa = particle_args(h, 0, 0, h->cur);
    pa.partial = scratch;
    const long long nb = fixup_blocks(h);
    const int np = (int)h->hparts.size();
    for (int64_t s = 0; s < nsteps; ++s) {
        const StepArgs a = make_step_args(h, h->cur, scratch);
        pa.nbox_out[0] = h->d_nbox[h->cur];
        launch_bulk(h, a, h->stream);
        if (nb > 0) h->ops.fixup(a, (unsigned)fixup_grid(h), h->stream, false, fixup_walk(h));
        if (np > 0) {
            launch_interactions(h, h->stream);
            h->ops.particles(pa, (unsigned)np, h->stream);
            h->ops.links(pa, np, h->link_bpp, h->d_linkcnt, h->stream);
        }
        h->cur = 1 - h->cur;
    }
    CUDA_TRY(h, cudaGetLastError());
    for (int64_t s = 0; s < nsteps; ++s) h->time += h->dt;
    h->tick += nsteps;
    return check_device_error(h);
}

void lbm_destroy(lbm_handle* h) { destroy_all(h); }

}  // extern "C"

// ===========================================================================
// Batches of independent replicas (lbm_batch_*): the replicas' tick items in
// one work queue (tick.cuh).
// ===========================================================================
struct lbm_batch {
    int device = 0;
    std::vector<lbm_handle*> reps;
    Ops ops{};
    cudaStream_t stream = nullptr, side = nullptr;
    cudaEvent_t ev_fix = nullptr, ev_part = nullptr;
    bool part_pending = false;
    int sms = 0, max_per_sm = 0;
    lbm_batch_tuning tuning{};
    // queue items and per-parity arguments, valid while `ready`
    bool ready = false;
    std::vector<int> base;  // each replica's buffer index when the items were built
    int par = 0;            // ticks since then, mod 2
    int4* d_amap = nullptr;
    int2 *d_bmap = nullptr, *d_cmap = nullptr, *d_dmap = nullptr;
    long long na = 0, nb = 0, nc = 0, nd = 0;
    StepArgs* d_targs = nullptr;      // [2][n]
    ParticleArgs* d_pargs = nullptr;  // [2][n]
    TickCounters* d_tq = nullptr;     // [0] main-stream launches, [1] side-stream launches
    int* d_err = nullptr;             // [n] per replica, plus one for the queue waits
    std::vector<int> diverged;        // [n] replicas whose density sentinel fired (sticky)
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};
    int profiling = 0;
    cudaEvent_t t_begin = nullptr, t_end = nullptr;
    lbm_profile prof{};
    long long cells = 0;
    std::string err;
};

namespace {

int bset_err(lbm_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    else g_global_err = msg;
    return code;
}

#define BCUDA_TRY(b, call)                                                                             \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            return bset_err((b), e_ == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,         \
                            std::string(#call) + ": " + cudaGetErrorString(e_));                        \
        }                                                                                              \
    } while (0)

template <class P>
int bdev_alloc(lbm_batch* b, P** p, size_t bytes) {
    cudaError_t e = block_alloc((void**)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return bset_err(b, LBM_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    return LBM_OK;
}

void batch_drop_graphs(lbm_batch* b) {
    for (auto& g : b->graphs) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

void batch_free_items(lbm_batch* b) {
    dev_free(b->d_amap);
    dev_free(b->d_bmap);
    dev_free(b->d_cmap);
    dev_free(b->d_dmap);
    b->ready = false;
}

// Queue items and arguments of every replica.  Bulk tiles go replica by
// replica, or interleaved (tile k of every replica, then tile k+1, ...).
int batch_prepare(lbm_batch* b) {
    const int n = (int)b->reps.size();
    bool same = b->ready && (int)b->base.size() == n;
    for (int r = 0; same && r < n; ++r) same = (b->reps[r]->cur ^ b->base[r]) == b->par;
    if (same) return LBM_OK;
    batch_drop_graphs(b);
    batch_free_items(b);
    std::vector<int4> am;
    std::vector<int2> bm, cm, dm;
    long long maxt = 0;
    for (int r = 0; r < n; ++r) {
        lbm_handle* h = b->reps[r];
        for (long long t = 0; t < (long long)h->vnear.size(); ++t)
            if (h->vnear[t]) am.push_back(make_int4(r, 0, (int)t, 0));
        const int np = (int)h->hparts.size();
        for (int p = 0; p < np; ++p) {
            const long long len = (long long)std::floor(2.0 * h->hparts[p].radius / h->dx) + 9;
            const long long nys = std::min<long long>(h->vnt1 + 1, (len + h->vrows - 1) / h->vrows + 2);
            const long long nzs = h->dims == 3 ? std::min<long long>(h->n[2], len) : 1;
            if (nys >= 65536 || nzs >= 32768)
                return bset_err(b, LBM_ERR_UNSUPPORTED, "particle too large for the tick kernel's tile slots");
            for (long long dz = 0; dz < nzs; ++dz)
                for (long long dy = 0; dy < nys; ++dy) am.push_back(make_int4(r, 1, p, (int)(dy | (dz << 16))));
        }
        const long long nfb = fixup_blocks(h);
        for (long long k = 0; k < nfb; ++k) bm.push_back(make_int2(r, (int)k));
        for (int p = 0; p < np; ++p) cm.push_back(make_int2(r, p));
        maxt = std::max(maxt, h->vtiles);
    }
    if (b->tuning.tile_order == 1) {
        for (long long t = 0; t < maxt; ++t)
            for (int r = 0; r < n; ++r)
                if (t < b->reps[r]->vtiles) dm.push_back(make_int2(r, (int)t));
    } else {
        for (int r = 0; r < n; ++r)
            for (long long t = 0; t < b->reps[r]->vtiles; ++t) dm.push_back(make_int2(r, (int)t));
    }
    std::vector<StepArgs> ta(2 * (size_t)n);
    std::vector<ParticleArgs> pa(2 * (size_t)n);
    b->base.resize(n);
    for (int r = 0; r < n; ++r) {
        lbm_handle* h = b->reps[r];
        b->base[r] = h->cur;
        for (int s = 0; s < 2; ++s) {
            const int src = h->cur ^ s;
            StepArgs& a = ta[(size_t)s * n + r];
            a = step_args(h, src);
            a.nbox = h->d_nbox[1 - src];
            a.err = b->d_err + r;
            ParticleArgs& q = pa[(size_t)s * n + r];
            q = particle_args(h, 0, 0, src);
            q.inline_links = 1;  // the queue has no separate link kernels
            q.err = b->d_err + r;
        }
    }
    b->par = 0;
    int rc = bdev_alloc(b, &b->d_amap, sizeof(int4) * std::max<size_t>(1, am.size()));
    if (!rc) rc = bdev_alloc(b, &b->d_bmap, sizeof(int2) * std::max<size_t>(1, bm.size()));
    if (!rc) rc = bdev_alloc(b, &b->d_cmap, sizeof(int2) * std::max<size_t>(1, cm.size()));
    if (!rc) rc = bdev_alloc(b, &b->d_dmap, sizeof(int2) * std::max<size_t>(1, dm.size()));
    if (rc) return rc;
    if (!am.empty()) BCUDA_TRY(b, cudaMemcpyAsync(b->d_amap, am.data(), sizeof(int4) * am.size(), cudaMemcpyHostToDevice, b->stream));
    if (!bm.empty()) BCUDA_TRY(b, cudaMemcpyAsync(b->d_bmap, bm.data(), sizeof(int2) * bm.size(), cudaMemcpyHostToDevice, b->stream));
    if (!cm.empty()) BCUDA_TRY(b, cudaMemcpyAsync(b->d_cmap, cm.data(), sizeof(int2) * cm.size(), cudaMemcpyHostToDevice, b->stream));
    if (!dm.empty()) BCUDA_TRY(b, cudaMemcpyAsync(b->d_dmap, dm.data(), sizeof(int2) * dm.size(), cudaMemcpyHostToDevice, b->stream));
    BCUDA_TRY(b, cudaMemcpyAsync(b->d_targs, ta.data(), sizeof(StepArgs) * ta.size(), cudaMemcpyHostToDevice, b->stream));
    BCUDA_TRY(b, cudaMemcpyAsync(b->d_pargs, pa.data(), sizeof(ParticleArgs) * pa.size(), cudaMemcpyHostToDevice, b->stream));
    BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
    b->na = (long long)am.size();
    b->nb = (long long)bm.size();
    b->nc = (long long)cm.size();
    b->nd = (long long)dm.size();
    b->ready = true;
    return LBM_OK;
}

TickItems batch_items(const lbm_batch* b, bool a, bool bb, bool c, bool d, int d_test) {
    TickItems it{};
    it.amap = b->d_amap;
    it.bmap = b->d_bmap;
    it.cmap = b->d_cmap;
    it.dmap = b->d_dmap;
    it.na = a ? b->na : 0;
    it.nb = bb ? b->nb : 0;
    it.nc = c ? b->nc : 0;
    it.nd = d ? b->nd : 0;
    it.d_test = d_test;
    it.spin_limit = kSpinLimit;
    // items past the enabled phases are addressed from the start of their map
    if (!a) it.amap = nullptr;
    return it;
}

void batch_launch(lbm_batch* b, int s, const TickItems& it, int q, cudaStream_t st) {
    const long long items = it.na + it.nb + it.nc + it.nd;
    if (items == 0) return;
    const long long cap = (long long)std::max(1, b->tuning.ctas_per_sm) * b->sms;
    const unsigned grid = (unsigned)std::max<long long>(1, std::min(items, cap));
    const size_t n = b->reps.size();
    b->ops.tick(b->d_targs + (size_t)s * n, b->d_pargs + (size_t)s * n, it, b->d_tq + q,
                b->d_err + n, grid, st, b->reps[0]->rounding == LBM_ROUND_STOCHASTIC);
}

// one tick of every replica with arguments of parity s (capturable)
void batch_enqueue(lbm_batch* b, int s) {
    if (b->tuning.schedule == LBM_SCHEDULE_PERSISTENT) {
        batch_launch(b, s, batch_items(b, true, true, true, true, 1), 0, b->stream);
        return;
    }
    // stream order: all tiles; then the fix-up blocks once the previous
    // particle update is done; the particle update on the side stream
    if (b->tuning.tile_cta)
        b->ops.bulk_batch(b->d_targs + (size_t)s * b->reps.size(), b->d_dmap, b->nd, b->stream,
                          b->reps[0]->rounding == LBM_ROUND_STOCHASTIC, s == 1);
    else
        batch_launch(b, s, batch_items(b, false, false, false, true, 0), 0, b->stream);
    if (b->part_pending) {
        cudaStreamWaitEvent(b->stream, b->ev_part, 0);
        b->part_pending = false;
    }
    if (b->nb > 0) batch_launch(b, s, batch_items(b, false, true, false, false, 0), 0, b->stream);
    if (b->nc > 0) {
        cudaEventRecord(b->ev_fix, b->stream);
        cudaStreamWaitEvent(b->side, b->ev_fix, 0);
        batch_launch(b, s, batch_items(b, false, false, true, false, 0), 1, b->side);
        cudaEventRecord(b->ev_part, b->side);
        b->part_pending = true;
    }
}

void batch_join(lbm_batch* b) {
    if (b->part_pending) {
        cudaStreamWaitEvent(b->stream, b->ev_part, 0);
        b->part_pending = false;
    }
}

int batch_graph(lbm_batch* b, int s0) {
    if (b->graphs[s0]) return LBM_OK;
    cudaGraph_t graph = nullptr;
    BCUDA_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kGraphSteps; ++k) batch_enqueue(b, s0 ^ (k & 1));
    batch_join(b);
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return bset_err(b, LBM_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(e));
    }
    e = cudaGraphInstantiate(&b->graphs[s0], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        b->graphs[s0] = nullptr;
        return bset_err(b, LBM_ERR_CUDA, std::string("graph instantiation failed: ") + cudaGetErrorString(e));
    }
    return LBM_OK;
}

int batch_check(lbm_batch* b) {
    const size_t n = b->reps.size();
    std::vector<int> err(n + 1, 0);
    BCUDA_TRY(b, cudaMemcpyAsync(err.data(), b->d_err, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, b->stream));
    BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
    bool any = false;
    for (size_t r = 0; r <= n; ++r) any = any || err[r] != 0;
    if (any) {  // reported below; the words start from zero again
        BCUDA_TRY(b, cudaMemsetAsync(b->d_err, 0, sizeof(int) * (n + 1), b->stream));
        BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
    }
    b->diverged.resize(n, 0);
    for (size_t r = 0; r < n; ++r)
        if (err[r] & kErrNumeric) b->diverged[r] = 1;  // a sweep goes on; lbm_batch_status reports them
    if (err[n] & kErrSpinTimeout) return bset_err(b, LBM_ERR_TIMEOUT, "a wait inside the tick kernel gave up");
    for (size_t r = 0; r < n; ++r) {
        if (err[r] & kErrLinkOverflow)
            return bset_err(b, LBM_ERR_STATE, "replica " + std::to_string(r) + ": particle links exceeded their capacity");
        if (err[r] & kErrIntervalOverflow)
            return bset_err(b, LBM_ERR_STATE, "replica " + std::to_string(r) + ": particle solid box exceeded its capacity");
    }
    return LBM_OK;
}

// run `ticks` ticks without touching the replicas' tick counters; the caller
// restores the state
int batch_run_raw(lbm_batch* b, int ticks, float* ms) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BCUDA_TRY(b, cudaEventCreate(&e0));
    BCUDA_TRY(b, cudaEventCreate(&e1));
    int s = b->par;
    for (int k = 0; k < 3; ++k, s ^= 1) batch_enqueue(b, s);  // warm-up
    batch_join(b);
    BCUDA_TRY(b, cudaEventRecord(e0, b->stream));
    for (int k = 0; k < ticks; ++k, s ^= 1) batch_enqueue(b, s);
    batch_join(b);
    BCUDA_TRY(b, cudaEventRecord(e1, b->stream));
    BCUDA_TRY(b, cudaEventSynchronize(e1));
    BCUDA_TRY(b, cudaGetLastError());
    BCUDA_TRY(b, cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return LBM_OK;
}

// everything a tick writes, for every replica: into / out of one device buffer
int batch_snapshot(lbm_batch* b, char** buf, size_t* bytes, bool save) {
    auto regions = [](lbm_handle* h, std::vector<std::pair<void*, size_t>>& v) {
        const size_t pop = (size_t)h->N * h->q * storage_bytes(h->storage);
        const size_t np = h->hparts.size();
        v.push_back({h->pop[0], pop});
        v.push_back({h->pop[1], pop});
        v.push_back({h->d_parts, sizeof(ParticleDev) * np});
        v.push_back({h->d_ivl, sizeof(int2) * h->ivl_slots});
        v.push_back({h->d_links, sizeof(int2) * h->link_slots});
        v.push_back({h->d_tilebits, sizeof(unsigned long long) * h->g.ntiles * h->words});
        v.push_back({h->d_nbox[0], sizeof(int) * 6 * np});
        v.push_back({h->d_nbox[1], sizeof(int) * 6 * np});
    };
    std::vector<std::pair<void*, size_t>> v;
    for (lbm_handle* h : b->reps) regions(h, v);
    if (save) {
        size_t total = 0;
        for (auto& r : v) total += (r.first ? r.second : 0);
        int rc = bdev_alloc(b, buf, total);
        if (rc) return rc;
        *bytes = total;
    }
    char* p = *buf;
    for (auto& r : v) {
        if (!r.first || !r.second) continue;
        if (save) BCUDA_TRY(b, cudaMemcpyAsync(p, r.first, r.second, cudaMemcpyDeviceToDevice, b->stream));
        else BCUDA_TRY(b, cudaMemcpyAsync(r.first, p, r.second, cudaMemcpyDeviceToDevice, b->stream));
        p += r.second;
    }
    BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
    return LBM_OK;
}

void batch_destroy_all(lbm_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->side) cudaStreamSynchronize(b->side);
    batch_drop_graphs(b);
    batch_free_items(b);
    dev_free(b->d_targs);
    dev_free(b->d_pargs);
    dev_free(b->d_tq);
    dev_free(b->d_err);
    if (b->t_begin) cudaEventDestroy(b->t_begin);
    if (b->t_end) cudaEventDestroy(b->t_end);
    if (b->ev_fix) cudaEventDestroy(b->ev_fix);
    if (b->ev_part) cudaEventDestroy(b->ev_part);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (lbm_handle* h : b->reps) destroy_all(h);
    delete b;
}

}  // namespace

extern "C" {

int lbm_batch_create(int32_t n, const lbm_config* cfgs, const int32_t* nparticles,
                     const lbm_particle_params* particles, lbm_batch** out) {
    if (!out || !cfgs || n < 1) return bset_err(nullptr, LBM_ERR_INVALID, "a batch needs at least one replica");
    *out = nullptr;
    lbm_batch* b = new lbm_batch();
    b->tuning.schedule = LBM_SCHEDULE_PERSISTENT;
    b->tuning.tile_order = 0;
    long long k = 0;
    for (int r = 0; r < n; ++r) {
        lbm_config c = cfgs[r];
        c.schedule = LBM_SCHEDULE_STREAM;
        lbm_handle* h = nullptr;
        int rc = lbm_create(&c, &h);
        if (rc) {
            const std::string m = "replica " + std::to_string(r) + ": " + g_global_err;
            batch_destroy_all(b);
            return bset_err(nullptr, rc, m);
        }
        h->in_batch = true;
        if (use_vector_bulk(h) && h->n[0] / 4 <= kTickBlock) set_vector_block(h, kTickBlock);  // queue tiles
        b->reps.push_back(h);
        const int np = nparticles ? nparticles[r] : 0;
        for (int p = 0; p < np; ++p, ++k) {
            rc = lbm_add_particle(h, particles + k, nullptr);
            if (rc) {
                const std::string m = "replica " + std::to_string(r) + ", particle " + std::to_string(p) + ": " + h->err;
                batch_destroy_all(b);
                return bset_err(nullptr, rc, m);
            }
        }
        const lbm_handle* h0 = b->reps[0];
        std::string why;
        if (!use_vector_bulk(h) || h->vblock != kTickBlock || !h->ops.tick) why = "needs the vector bulk path with x-rows of at most 256 nodes";
        else if (h->device != h0->device) why = "all replicas must be on one device";
        else if (h->lattice != h0->lattice || h->storage != h0->storage || h->trt != h0->trt ||
                 h->rounding != h0->rounding)
            why = "all replicas must share the velocity set, storage format, rounding and collision model";
        if (!why.empty()) {
            batch_destroy_all(b);
            return bset_err(nullptr, LBM_ERR_UNSUPPORTED, "replica " + std::to_string(r) + ": " + why);
        }
        b->cells += h->N;
    }
    b->device = b->reps[0]->device;
    b->ops = b->reps[0]->ops;
    cudaSetDevice(b->device);
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    int rc = LBM_OK;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithPriority(&b->side, cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fix, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_part, cudaEventDisableTiming) != cudaSuccess)
        rc = bset_err(b, LBM_ERR_CUDA, "stream or event creation failed");
    if (!rc) rc = bdev_alloc(b, &b->d_targs, sizeof(StepArgs) * 2 * n);
    if (!rc) rc = bdev_alloc(b, &b->d_pargs, sizeof(ParticleArgs) * 2 * n);
    if (!rc) rc = bdev_alloc(b, &b->d_tq, sizeof(TickCounters) * 2);
    if (!rc) rc = bdev_alloc(b, &b->d_err, sizeof(int) * (n + 1));
    if (!rc && (cudaMemset(b->d_tq, 0, sizeof(TickCounters) * 2) != cudaSuccess ||
                cudaMemset(b->d_err, 0, sizeof(int) * (n + 1)) != cudaSuccess))
        rc = bset_err(b, LBM_ERR_CUDA, "memset failed");
    if (!rc && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &b->max_per_sm, b->reps[0]->rounding == LBM_ROUND_STOCHASTIC ? b->ops.tick_fn_sr : b->ops.tick_fn,
                    kTickBlock, 0) != cudaSuccess ||
                cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess))
        rc = bset_err(b, LBM_ERR_CUDA, "occupancy query failed");
    if (rc) {
        const std::string m = b->err;
        batch_destroy_all(b);
        return bset_err(nullptr, rc, m);
    }
    b->tuning.ctas_per_sm = std::max(1, b->max_per_sm);
    *out = b;
    return LBM_OK;
}

int32_t lbm_batch_size(const lbm_batch* b) { return b ? (int32_t)b->reps.size() : 0; }

lbm_handle* lbm_batch_replica(lbm_batch* b, int32_t i) {
    if (!b || i < 0 || i >= (int32_t)b->reps.size()) return nullptr;
    return b->reps[i];
}

int lbm_batch_step(lbm_batch* b, int64_t nsteps) {
    if (!b) return bset_err(b, LBM_ERR_INVALID, "null batch");
    if (nsteps < 0) return bset_err(b, LBM_ERR_INVALID, "ticks must be non-negative");
    if (cudaSetDevice(b->device) != cudaSuccess) return bset_err(b, LBM_ERR_CUDA, "cannot select the batch's device");
    for (lbm_handle* h : b->reps) {  // work a replica stepped alone left on its streams
        if (cudaStreamSynchronize(h->stream) != cudaSuccess)
            return bset_err(b, LBM_ERR_CUDA, "replica stream failed");
    }
    for (lbm_handle* h : b->reps)
        if (!h->inter.empty()) return bset_err(b, LBM_ERR_UNSUPPORTED, "batches do not run particle interactions");
    int rc = batch_prepare(b);
    if (rc) return rc;
    if (b->profiling) BCUDA_TRY(b, cudaEventRecord(b->t_begin, b->stream));
    int64_t done = 0;
    while (nsteps - done >= kGraphSteps) {
        rc = batch_graph(b, b->par);
        if (rc) return rc;
        BCUDA_TRY(b, cudaGraphLaunch(b->graphs[b->par], b->stream));
        done += kGraphSteps;  // even: the parity is unchanged
    }
    for (; done < nsteps; ++done) {
        batch_enqueue(b, b->par);
        b->par ^= 1;
    }
    batch_join(b);
    if (b->profiling) BCUDA_TRY(b, cudaEventRecord(b->t_end, b->stream));
    BCUDA_TRY(b, cudaGetLastError());
    for (lbm_handle* h : b->reps) {
        if (nsteps & 1) h->cur ^= 1;
        h->tick += nsteps;
        for (int64_t s = 0; s < nsteps; ++s) h->time += h->dt;
    }
    rc = batch_check(b);
    b->prof = lbm_profile{};
    b->prof.steps = nsteps;
    b->prof.bulk_cells = b->cells;
    b->prof.launches = nsteps * (b->tuning.schedule == LBM_SCHEDULE_PERSISTENT
                                     ? 1 : 1 + (b->nb > 0 ? 1 : 0) + (b->nc > 0 ? 1 : 0));
    if (b->profiling && nsteps > 0) {
        float ms = 0;
        BCUDA_TRY(b, cudaEventElapsedTime(&ms, b->t_begin, b->t_end));
        b->prof.total_ms = ms;
    }
    return rc;
}

int lbm_batch_set_tuning(lbm_batch* b, const lbm_batch_tuning* t) {
    if (!b || !t) return bset_err(b, LBM_ERR_INVALID, "null argument");
    if ((t->schedule != LBM_SCHEDULE_STREAM && t->schedule != LBM_SCHEDULE_PERSISTENT) || t->ctas_per_sm < 1 ||
        t->ctas_per_sm > std::max(1, b->max_per_sm) || t->tile_order < 0 || t->tile_order > 1 || t->tile_cta < 0 ||
        t->tile_cta > 1)
        return bset_err(b, LBM_ERR_INVALID, "invalid tuning");
    if (cudaSetDevice(b->device) != cudaSuccess) return bset_err(b, LBM_ERR_CUDA, "cannot select the batch's device");
    BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
    const bool reorder = t->tile_order != b->tuning.tile_order;
    b->tuning = *t;
    batch_drop_graphs(b);
    if (reorder) batch_free_items(b);
    return LBM_OK;
}

int lbm_batch_get_tuning(const lbm_batch* b, lbm_batch_tuning* t) {
    if (!b || !t) return LBM_ERR_INVALID;
    *t = b->tuning;
    return LBM_OK;
}

int lbm_batch_autotune(lbm_batch* b, int32_t ticks, lbm_batch_tuning* results, int32_t capacity, int32_t* count,
                       lbm_batch_tuning* chosen) {
    if (!b || ticks < 1) return bset_err(b, LBM_ERR_INVALID, "autotune needs a batch and at least one tick");
    if (cudaSetDevice(b->device) != cudaSuccess) return bset_err(b, LBM_ERR_CUDA, "cannot select the batch's device");
    for (lbm_handle* h : b->reps) BCUDA_TRY(b, cudaStreamSynchronize(h->stream));
    int rc = batch_prepare(b);
    if (rc) return rc;
    char* save = nullptr;
    size_t bytes = 0;
    rc = batch_snapshot(b, &save, &bytes, true);
    if (rc) return rc;
    std::vector<lbm_batch_tuning> cand;
    std::vector<int> per_sm;
    for (int c : {2, 4, 6, 8, 12, 16})
        if (c <= b->max_per_sm) per_sm.push_back(c);
    if (per_sm.empty() || per_sm.back() != b->max_per_sm) per_sm.push_back(b->max_per_sm);
    for (int sched : {LBM_SCHEDULE_PERSISTENT, LBM_SCHEDULE_STREAM})
        for (int cta : {0, 1}) {
            if (sched == LBM_SCHEDULE_PERSISTENT && cta) continue;  // everything goes through the queue
            for (int order : {0, 1})
                for (int c : per_sm) {
                    lbm_batch_tuning t{};
                    t.schedule = sched;
                    t.ctas_per_sm = c;
                    t.tile_order = order;
                    t.tile_cta = cta;
                    cand.push_back(t);
                }
        }
    const lbm_batch_tuning keep = b->tuning;
    const std::vector<int> keep_diverged = b->diverged;  // the candidates' ticks are undone
    int best = -1;
    for (size_t i = 0; i < cand.size(); ++i) {
        if (cand[i].tile_order != b->tuning.tile_order) {
            b->tuning.tile_order = cand[i].tile_order;
            batch_free_items(b);
            rc = batch_prepare(b);
            if (rc) break;
        }
        b->tuning = cand[i];
        float ms = 0;
        rc = batch_run_raw(b, ticks, &ms);
        if (!rc) rc = batch_snapshot(b, &save, &bytes, false);  // restore
        if (!rc) rc = batch_check(b);
        if (rc) break;
        cand[i].ms_per_tick = ms / ticks;
        if (best < 0 || cand[i].ms_per_tick < cand[best].ms_per_tick) best = (int)i;
    }
    dev_free(save);
    batch_drop_graphs(b);
    b->diverged = keep_diverged;
    if (rc || best < 0) {
        b->tuning = keep;
        batch_free_items(b);
        return rc ? rc : bset_err(b, LBM_ERR_STATE, "no tuning candidate ran");
    }
    if (cand[best].tile_order != b->tuning.tile_order) batch_free_items(b);
    b->tuning = cand[best];
    if (results && count) {
        const int m = std::min<int>(capacity, (int)cand.size());
        for (int i = 0; i < m; ++i) results[i] = cand[i];
    }
    if (count) *count = (int32_t)cand.size();
    if (chosen) *chosen = cand[best];
    return LBM_OK;
}

int lbm_batch_set_profiling(lbm_batch* b, int32_t level) {
    if (!b) return LBM_ERR_INVALID;
    if (cudaSetDevice(b->device) != cudaSuccess) return bset_err(b, LBM_ERR_CUDA, "cannot select the batch's device");
    if (level > 0 && !b->t_begin) {
        BCUDA_TRY(b, cudaEventCreate(&b->t_begin));
        BCUDA_TRY(b, cudaEventCreate(&b->t_end));
    }
    b->profiling = level > 0 ? 1 : 0;
    return LBM_OK;
}

int lbm_batch_get_profile(const lbm_batch* b, lbm_profile* out) {
    if (!b || !out) return LBM_ERR_INVALID;
    *out = b->prof;
    return LBM_OK;
}

int lbm_batch_status(const lbm_batch* b, int32_t* status) {
    if (!b) return set_err(nullptr, LBM_ERR_INVALID, "null batch");
    int count = 0;
    for (size_t r = 0; r < b->reps.size(); ++r) {
        const bool d = r < b->diverged.size() && b->diverged[r];
        if (status) status[r] = d ? LBM_ERR_NUMERIC : LBM_OK;
        count += d ? 1 : 0;
    }
    return count;
}

const char* lbm_batch_last_error(const lbm_batch* b) { return b ? b->err.c_str() : g_global_err.c_str(); }

void lbm_batch_destroy(lbm_batch* b) { batch_destroy_all(b); }

}  // extern "C"

// ===========================================================================
// Gradients (lbm_adjoint): discrete adjoint of the tick with binomial
// checkpointing.  Device: the field adjoint (adjoint.cuh).  Host: the
// particle update's adjoint (a handful of FP64 values per tick) and the
// checkpoint schedule.
// ===========================================================================
namespace {

// forward-mode dual with one direction, host side
struct HD {
    double v = 0, d = 0;
};
HD operator+(HD a, HD b) { return {a.v + b.v, a.d + b.d}; }
HD operator-(HD a, HD b) { return {a.v - b.v, a.d - b.d}; }
HD operator*(HD a, HD b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
HD operator/(HD a, HD b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
HD operator*(double s, HD a) { return {s * a.v, s * a.d}; }
HD hsqrt(HD a) {
    const double r = std::sqrt(a.v);
    return {r, a.d / (2 * r)};
}
HD hcos(HD a) { return {std::cos(a.v), -std::sin(a.v) * a.d}; }
HD hsin(HD a) { return {std::sin(a.v), std::cos(a.v) * a.d}; }
HD habs(HD a) { return a.v < 0 ? HD{-a.v, -a.d} : a; }

// the swimming-direction update of moveParticles! (particles.jl:48-70:
// Rodrigues rotation by |w| dt about w, then normalised), as the particle
// kernel does it
void rodrigues(const HD* e, const HD* w, double dt, int D, HD* out) {
    for (int k = 0; k < 3; ++k) out[k] = e[k];
    HD theta;
    if (D == 2) theta = habs(w[0]);
    else theta = hsqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    if (theta.v == 0.0) return;
    HD vr[3];
    if (D == 2) {
        const HD k = w[0] / theta;
        const HD th = dt * theta;
        const HD ct = hcos(th), st = hsin(th);
        vr[0] = e[0] * ct + (HD{0, 0} - k * e[1]) * st;
        vr[1] = e[1] * ct + (k * e[0]) * st;
        vr[2] = HD{};
    } else {
        const HD k[3] = {w[0] / theta, w[1] / theta, w[2] / theta};
        const HD th = dt * theta;
        const HD ct = hcos(th), st = hsin(th);
        const HD cr[3] = {k[1] * e[2] - k[2] * e[1], HD{0, 0} - k[0] * e[2] + k[2] * e[0], k[0] * e[1] - k[1] * e[0]};
        const HD kv = k[0] * e[0] + k[1] * e[1] + k[2] * e[2];
        for (int q = 0; q < 3; ++q) vr[q] = e[q] * ct + cr[q] * st + k[q] * kv * (HD{1, 0} - ct);
    }
    HD n2{};
    for (int q = 0; q < D; ++q) n2 = n2 + vr[q] * vr[q];
    const HD nr = hsqrt(n2);
    for (int q = 0; q < D; ++q) out[q] = vr[q] / nr;
}

// adjoint of the particle state carried backwards through the ticks
struct PartAdj {
    double R[3] = {0, 0, 0}, v[3] = {0, 0, 0}, w[3] = {0, 0, 0}, e[3] = {0, 0, 0};
    double S[12] = {0};  // snapshot sR, sV, sW, sE
    double mR[3] = {0, 0, 0};
};

struct Snap {
    char* buf = nullptr;
    long long tick = 0;
    double time = 0;
    int cur = 0;
};

struct AdjointRun {
    lbm_handle* h = nullptr;
    lbm_adjoint_spec spec{};
    std::vector<ParticleDev> rec;  // rec[t]: the particle after t ticks
    std::vector<char> have;        // rec[t] has been recorded
    std::vector<Snap> snaps;       // stored states (a stack)
    size_t snap_bytes = 0;
    int max_used = 0;
    long long forward = 0;
    double* lam[2] = {nullptr, nullptr};
    int lcur = 0;  // lam[lcur]: adjoint of the populations at the current tick
    double* partial = nullptr;
    double* dsum = nullptr;
    long long nblocks = 0;
    PartAdj pa;
    double e0[3] = {0, 0, 0};
    double dB1 = 0, dB2 = 0, dtp = 0, dtm = 0, dF[3] = {0, 0, 0};
};

std::vector<std::pair<void*, size_t>> snap_regions(lbm_handle* h) {
    const size_t np = h->hparts.size();
    return {{h->pop[h->cur], (size_t)h->N * h->q * storage_bytes(h->storage)},
            {h->d_parts, sizeof(ParticleDev) * np},
            {h->d_ivl, sizeof(int2) * h->ivl_slots},
            {h->d_links, sizeof(int2) * h->link_slots},
            {h->d_tilebits, sizeof(unsigned long long) * h->g.ntiles * h->words},
            {h->d_nbox[0], sizeof(int) * 6 * np},
            {h->d_nbox[1], sizeof(int) * 6 * np}};
}

int snap_push(AdjointRun& R) {
    lbm_handle* h = R.h;
    Snap s;
    int rc = dev_alloc(h, &s.buf, R.snap_bytes);
    if (rc) return rc;
    char* p = s.buf;
    for (auto& r : snap_regions(h)) {
        if (r.first && r.second) CUDA_TRY(h, cudaMemcpyAsync(p, r.first, r.second, cudaMemcpyDeviceToDevice, h->stream));
        p += r.second;
    }
    s.tick = h->tick;
    s.time = h->time;
    s.cur = h->cur;
    R.snaps.push_back(s);
    R.max_used = std::max(R.max_used, (int)R.snaps.size());
    return LBM_OK;
}

int snap_restore(AdjointRun& R, const Snap& s) {
    lbm_handle* h = R.h;
    h->cur = s.cur;
    h->tick = s.tick;
    h->time = s.time;
    h->part_pending = false;
    char* p = s.buf;
    for (auto& r : snap_regions(h)) {
        if (r.first && r.second) CUDA_TRY(h, cudaMemcpyAsync(r.first, p, r.second, cudaMemcpyDeviceToDevice, h->stream));
        p += r.second;
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

void snap_pop(AdjointRun& R) {
    dev_free(R.snaps.back().buf);
    R.h->device_bytes -= R.snap_bytes;
    R.snaps.pop_back();
}

// k ticks forward, recording the particle after each
int advance(AdjointRun& R, long long k) {
    lbm_handle* h = R.h;
    for (long long s = 0; s < k; ++s) {
        int rc = lbm_step(h, 1);
        if (rc) return rc;
        CUDA_TRY(h, cudaMemcpy(&R.rec[h->tick], h->d_parts, sizeof(ParticleDev), cudaMemcpyDeviceToHost));
        R.have[h->tick] = 1;
        ++R.forward;
    }
    return LBM_OK;
}

// backward step of tick n; the device holds the state at tick n and
// rec[n + 1] is known
int backward_tick(AdjointRun& R, long long n) {
    lbm_handle* h = R.h;
    const int D = h->dims;
    const ParticleDev& P0 = R.rec[n];
    const ParticleDev& P1 = R.rec[n + 1];
    PartAdj& A = R.pa;
    const double dt = h->dt;
    // the observable reads the velocity after tick n + 1, or the force of tick n + 1
    const bool in_window = n + 1 >= R.spec.window_begin && n + 1 <= R.spec.window_end;
    const double K = (double)(R.spec.window_end - R.spec.window_begin + 1);
    if (in_window && R.spec.observable == LBM_OBSERVABLE_VELOCITY)
        for (int k = 0; k < D; ++k) A.v[k] += R.e0[k] / K;
    // reverse the particle update of tick n (particles.cuh, moveParticles!)
    bool moved = false, alpha = false;
    if (P0.coupleF)
        for (int k = 0; k < D; ++k) moved = moved || P1.v[k] != 0.0;
    if (P0.coupleT)
        for (int k = 0; k < (D == 2 ? 1 : 3); ++k) alpha = alpha || P1.lastT[k] * P0.inv_inertia != 0.0;
    if (moved || alpha) {  // the snapshot after the update is the updated state
        for (int k = 0; k < 3; ++k) {
            A.R[k] += A.S[k];
            A.v[k] += A.S[3 + k];
            A.w[k] += A.S[6 + k];
            A.e[k] += A.S[9 + k];
        }
        for (double& s : A.S) s = 0.0;
    }
    if (moved) {  // the torque arm after the update is the new position
        for (int k = 0; k < 3; ++k) A.R[k] += A.mR[k];
        for (double& s : A.mR) s = 0.0;
    }
    if (P0.coupleT && P0.kind == LBM_SQUIRMER) {  // e' = rot(e, w')
        double le[3] = {0, 0, 0}, lw[3] = {0, 0, 0};
        for (int q = 0; q < 6; ++q) {
            HD e[3], w[3], o[3];
            for (int k = 0; k < 3; ++k) {
                e[k] = HD{P0.e[k], q == k ? 1.0 : 0.0};
                w[k] = HD{P1.w[k], q == 3 + k ? 1.0 : 0.0};
            }
            rodrigues(e, w, dt, D, o);
            double g = 0.0;
            for (int k = 0; k < D; ++k) g += A.e[k] * o[k].d;
            if (q < 3) le[q] = g;
            else lw[q - 3] = g;
        }
        for (int k = 0; k < 3; ++k) {
            A.e[k] = le[k];
            A.w[k] += lw[k];
        }
    }
    AdjArgs a{};
    if (P0.coupleT)
        for (int k = 0; k < (D == 2 ? 1 : 3); ++k) a.lamT[k] = dt * P0.inv_inertia * A.w[k];  // w' = w + dt T / I
    if (P0.coupleF) {
        for (int k = 0; k < D; ++k) A.v[k] += dt * A.R[k];                                    // R' = R + dt v'
        for (int k = 0; k < D; ++k) a.lamF[k] = dt * P0.inv_mass * A.v[k];                   // v' = v + dt F / m
    }
    if (in_window && R.spec.observable == LBM_OBSERVABLE_FORCE)
        for (int k = 0; k < D; ++k) a.lamF[k] += R.e0[k] / K;  // J += e.F / K
    // the field adjoint of tick n on the device
    a.src = h->pop[h->cur];
    a.lam_in = R.lam[R.lcur];
    a.lam_out = R.lam[1 - R.lcur];
    a.g = h->g;
    for (int k = 0; k < 3; ++k) a.coord[k] = h->d_coord[k];
    a.part = h->d_parts;
    a.ivl = h->d_ivl;
    a.wall = h->d_wall;
    a.uw = h->d_uw;
    a.has_part = 1;
    a.rho0 = h->rho0;
    a.inv_scale = 1.0 / h->scale;
    a.dt = h->dt;
    a.tau_p = h->tau;
    a.tau_m = h->trt ? h->tau_minus : h->tau;
    for (int k = 0; k < 3; ++k) a.F[k] = h->F[k];
    a.guo = h->force_mode == LBM_FORCE_UNIFORM ? 1 : 0;
    a.incompressible = h->incompressible;
    a.rho_inc = h->rho_inc;
    a.coeff = std::pow(h->dx, h->dims) / h->dt;
    a.partial = R.partial;
    h->ops.adjoint(a, h->stream);
    k_adjoint_sum<kAdjAcc><<<kAdjAcc, kSumBlock, 0, h->stream>>>(R.partial, R.nblocks, R.dsum);
    double acc[kAdjAcc];
    CUDA_TRY(h, cudaMemcpyAsync(acc, R.dsum, sizeof(acc), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    R.lcur = 1 - R.lcur;
    R.dtp += acc[0];
    R.dtm += acc[1];
    for (int k = 0; k < 3; ++k) R.dF[k] += acc[2 + k];
    for (int k = 0; k < 12; ++k) A.S[k] += acc[5 + k];  // the snapshot tick n used
    R.dB1 += acc[17];
    R.dB2 += acc[18];
    for (int k = 0; k < 3; ++k) A.mR[k] += acc[19 + k];
    return LBM_OK;
}

// binomial coefficient C(s + r, s), saturating
long long beta_sr(long long s, long long r) {
    double b = 1.0;
    for (long long k = 1; k <= r; ++k) {
        b = b * (double)(s + k) / (double)k;
        if (b > 4e18) return (long long)4e18;
    }
    return (long long)(b + 0.5);
}

// Reverse ticks [a, b) with the state at tick a on the device (and on top of
// the snapshot stack) and `free` further snapshot slots.  Binomial
// checkpointing: with r the fewest repetitions for which C(free + r, free)
// covers the segment, the next checkpoint goes where the right part can
// still be reversed with one slot fewer.
int reverse(AdjointRun& R, long long a, long long b, int free) {
    int rc;
    if (b - a == 1) {
        if (!R.have[b]) {  // the particle after the last tick: one tick ahead and back
            if (free > 0) {
                rc = snap_push(R);
                if (!rc) rc = advance(R, 1);
                if (!rc) rc = snap_restore(R, R.snaps.back());
                if (rc) return rc;
                snap_pop(R);
            } else {
                const Snap base = R.snaps.back();
                rc = advance(R, 1);
                if (!rc) rc = snap_restore(R, base);
                if (!rc) rc = advance(R, a - base.tick);
                if (rc) return rc;
            }
        }
        return backward_tick(R, a);
    }
    if (free == 0) {  // no slot left: recompute from a for every tick
        const Snap base = R.snaps.back();
        for (long long t = b - 1; t >= a; --t) {
            rc = LBM_OK;
            if (!R.have[t + 1]) {
                rc = snap_restore(R, base);
                if (!rc) rc = advance(R, t + 1 - a);
            }
            if (!rc) rc = snap_restore(R, base);
            if (!rc) rc = advance(R, t - a);
            if (!rc) rc = backward_tick(R, t);
            if (rc) return rc;
        }
        return LBM_OK;
    }
    const long long n = b - a;
    long long r = 0;
    while (beta_sr(free, r) < n) ++r;
    const long long m = std::max<long long>(1, std::min<long long>(n - 1, n - beta_sr(free - 1, r)));
    rc = advance(R, m);
    if (!rc) rc = snap_push(R);
    if (!rc) rc = reverse(R, a + m, b, free - 1);
    if (rc) return rc;
    snap_pop(R);
    rc = snap_restore(R, R.snaps.back());
    if (!rc) rc = reverse(R, a, a + m, free);
    return rc;
}

}  // namespace

extern "C" {

int lbm_adjoint(lbm_handle* h, const lbm_adjoint_spec* spec, lbm_adjoint_result* out) {
    if (!h || !spec || !out) return set_err(h, LBM_ERR_INVALID, "null argument");
    BIND(h);
    const auto t0 = std::chrono::steady_clock::now();
    if (h->hparts.size() != 1) return set_err(h, LBM_ERR_UNSUPPORTED, "the adjoint supports models with one particle");
    if (h->particle_rules != LBM_RULES_GPU_MODULE)
        return set_err(h, LBM_ERR_UNSUPPORTED, "the adjoint follows the GPU module's particle update");
    if (!h->inter.empty()) return set_err(h, LBM_ERR_UNSUPPORTED, "the adjoint does not support particle interactions");
    if (h->force_mode == LBM_FORCE_FIELD) return set_err(h, LBM_ERR_UNSUPPORTED, "the adjoint does not support force fields");
    if (spec->ticks < 1 || spec->window_begin < 1 || spec->window_end < spec->window_begin ||
        spec->window_end > spec->ticks)
        return set_err(h, LBM_ERR_INVALID, "need 1 <= window_begin <= window_end <= ticks");
    if (spec->snapshots < 2) return set_err(h, LBM_ERR_INVALID, "at least two snapshots");
    if (h->tick != 0) return set_err(h, LBM_ERR_STATE, "the adjoint runs from tick 0 (a freshly built model)");
    AdjointRun R;
    R.h = h;
    R.spec = *spec;
    const long long T = spec->ticks;
    R.rec.resize(T + 1);
    R.have.assign(T + 1, 0);
    R.have[0] = 1;
    join_particles(h);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (spec->observable != LBM_OBSERVABLE_VELOCITY && spec->observable != LBM_OBSERVABLE_FORCE)
        return set_err(h, LBM_ERR_INVALID, "unknown observable");
    const int record = spec->observable == LBM_OBSERVABLE_FORCE ? 1 : 0;
    int record_before = 0;  // the caller's lbm_record_force setting, restored at the end
    CUDA_TRY(h, cudaMemcpy(&record_before, &h->d_parts[0].recordF, sizeof(int), cudaMemcpyDeviceToHost));
    // the force observable needs the momentum exchange even of a held particle
    CUDA_TRY(h, cudaMemcpy(&h->d_parts[0].recordF, &record, sizeof(int), cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(&R.rec[0], h->d_parts, sizeof(ParticleDev), cudaMemcpyDeviceToHost));
    double en = 0.0;
    for (int k = 0; k < 3; ++k) en += spec->direction[k] * spec->direction[k];
    for (int k = 0; k < 3; ++k) R.e0[k] = en > 0 ? spec->direction[k] : R.rec[0].e[k];
    for (auto& r : snap_regions(h)) R.snap_bytes += r.second;
    const size_t lam_bytes = sizeof(double) * (size_t)h->N * h->q;
    R.nblocks = (h->N + kAdjBlock - 1) / kAdjBlock;
    int rc = dev_alloc(h, &R.lam[0], lam_bytes);
    if (!rc) rc = dev_alloc(h, &R.lam[1], lam_bytes);
    if (!rc) rc = dev_alloc(h, &R.partial, sizeof(double) * kAdjAcc * R.nblocks);
    if (!rc) rc = dev_alloc(h, &R.dsum, sizeof(double) * kAdjAcc);
    if (!rc && cudaMemset(R.lam[0], 0, lam_bytes) != cudaSuccess) rc = set_err(h, LBM_ERR_CUDA, "memset failed");
    if (!rc) rc = snap_push(R);  // the initial state
    if (!rc) rc = reverse(R, 0, T, spec->snapshots - 1);
    if (!rc) {  // the initial condition depends on the body force
        rc = snap_restore(R, R.snaps.front());
        if (!rc && h->force_mode == LBM_FORCE_UNIFORM) {
            AdjArgs a{};
            a.src = h->pop[h->cur];
            a.lam_in = R.lam[R.lcur];
            a.g = h->g;
            a.rho0 = h->rho0;
            a.inv_scale = 1.0 / h->scale;
            a.dt = h->dt;
            a.guo = 1;
            a.incompressible = h->incompressible;
            a.rho_inc = h->rho_inc;
            a.partial = R.partial;
            h->ops.adjoint_init(a, h->stream);
            k_adjoint_sum<kAdjAcc><<<kAdjAcc, kSumBlock, 0, h->stream>>>(R.partial, R.nblocks, R.dsum);
            double acc[kAdjAcc];
            // on the handle's stream: a plain cudaMemcpy would not wait for it
            if (cudaMemcpyAsync(acc, R.dsum, sizeof(acc), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
                cudaStreamSynchronize(h->stream) != cudaSuccess)
                rc = set_err(h, LBM_ERR_CUDA, "read-back failed");
            else
                for (int k = 0; k < 3; ++k) R.dF[k] += acc[k];
        }
    }
    while (!R.snaps.empty()) snap_pop(R);
    if (cudaMemcpy(&h->d_parts[0].recordF, &record_before, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess &&
        !rc)
        rc = set_err(h, LBM_ERR_CUDA, "cannot restore the force record flag");
    dev_free(R.lam[0]);
    dev_free(R.lam[1]);
    dev_free(R.partial);
    dev_free(R.dsum);
    h->device_bytes -= 2 * lam_bytes + sizeof(double) * kAdjAcc * (R.nblocks + 1);
    if (rc) return rc;
    std::memset(out, 0, sizeof(*out));
    const double K = (double)(spec->window_end - spec->window_begin + 1);
    double J = 0.0;
    for (long long t = spec->window_begin; t <= spec->window_end; ++t)
        for (int k = 0; k < h->dims; ++k)
            J += (record ? R.rec[t].lastF[k] : R.rec[t].v[k]) * R.e0[k] / K;
    out->value = J;
    out->dB1 = R.dB1;
    out->dB2 = R.dB2;
    out->dtau_plus = R.dtp;
    out->dtau_minus = h->trt ? R.dtm : 0.0;
    out->dtau = R.dtp + (h->trt ? spec->tau_minus_slope * R.dtm : 0.0);
    for (int k = 0; k < 3; ++k) out->dF[k] = k < h->dims ? R.dF[k] : 0.0;
    out->forward_ticks = R.forward;
    out->snapshots_used = R.max_used;
    out->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return LBM_OK;
}

}  // extern "C"
