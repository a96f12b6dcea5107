// Fix-up kernel: boundary links and walls.
//
// CTA kinds (blockIdx.x):
//   [0, nparts*maxchunks)            chunk `c` (kFixBlock entries) of particle p's link list;
//   [.., + ceil(nwlinks/kFixBlock))  static wall-link entries (cell, direction mask);
//   [.., + ceil(nwnodes/kFixBlock))  wall nodes (reset to f = 0).
// A particle's link list (built by the particle update whenever its solid
// intervals change) holds the fluid nodes x of its near box with mask bit j
// set where x - c_j is solid (streamingInvasionRegions, src/gpu/aux.jl:187-198);
// chunks past the list's length return at once.
// The value written to slot (x, j) follows tick! (fluids.jl:143-206) for the
// whole region (walls and every particle):
//     f*_opp(j)(x)  (+ moving wall term)  (+ Ladd terms of the particles, in
//     order, up to the first one without links in direction j, fluids.jl:184)
// so CTAs of different owners that meet the same slot write the same value.
// Particle CTAs also add their particle's momentum exchange
// (fluids.jl:191-205) to a per-chunk FP64 partial, reduced in a fixed order.
//
// Each entry's node is collided once into shared memory; its link slots
// are then processed one per thread (see fixup_body), each a runtime walk
// over the candidate particles, which keeps the kernel body small.
#pragma once
#include "kernels.cuh"

namespace lbm {

constexpr int kFixThreads = 256;  // threads of a k_fixup CTA

// Ladd term and momentum exchange of one link slot (fluids.jl:176-205) for
// particle P; v accumulates the slot value, acc the owner's F and T.
template <int D>
__device__ __forceinline__ void ladd_link(const StepArgs& a, const ParticleDev& P, bool owner, int ci0, int ci1,
                                          int ci2, const double* Tc, const double* Xc, double rhoL, double gi,
                                          double wi, double& v, double* acc) {
    double up[3];
    if (P.rules == 1)  // LBM_RULES_CPU_MODULE: uw = u_p(x) + u_p(x - c), u_p(x) = 0 at the fluid node x
        slip_velocity_cpu<D>(P.sR, P.sV, P.sW, P.sE, P.B1, P.B2, P.kind, P.radius, 2.0 * a.half_dt, Tc[0], Tc[1],
                             Tc[2], up);
    else
        slip_velocity<D>(P.sR, P.sV, P.sW, P.sE, P.B1, P.B2, P.kind, Tc[0], Tc[1], Tc[2], up);
    v += 6.0 * rhoL * (-(ci0 * up[0] + ci1 * up[1] + ci2 * up[2]));
    if (owner && (P.coupleF || P.coupleT || P.recordF)) {
        // f*_i(x) + f_j(x) in f units; F -= coeff*s*c_j = coeff*s*c_i
        const double cs = a.coeff * (wi * (2.0 * a.rho0 + gi + v));
        if (P.coupleF || P.recordF) {
            acc[0] += cs * ci0;
            acc[1] += cs * ci1;
            acc[2] += cs * ci2;
        }
        if (P.coupleT) {  // T -= coeff*cross(s*(x-R), c_j) = coeff*cross(s*(x-R), c_i)
            const double r0 = Xc[0] - P.mR[0], r1 = Xc[1] - P.mR[1], r2 = D == 3 ? Xc[2] - P.mR[2] : 0.0;
            if (D == 2) {
                acc[3] += cs * (r0 * ci1 - r1 * ci0);
            } else {
                acc[3] += cs * (r1 * ci2 - r2 * ci1);
                acc[4] += cs * (-r0 * ci2 + r2 * ci0);
                acc[5] += cs * (r0 * ci1 - r1 * ci0);
            }
        }
    }
}

// One CTA per kFixBlock link entries, NT threads (NT >= kFixBlock).
//   first loads: the particle record, the entry (cell, mask) of threads < kFixBlock
//            ((link_off, link_cap) of the first particles come with the
//            kernel parameters, so the entry load does not wait for the record)
//   second loads: each entry's populations and the coordinates of its node and of
//            the node's +-1 neighbours per axis (every link target x + c_i is
//            among them); the node is collided once into shared memory and
//            the links of all entries are listed (entry, j)
//   links:   the list is spread over all NT threads, one link slot each
//            (the Ladd terms are FP64 chains with a square root and a
//            division; one thread per entry would run its links in series)
//   the momentum exchange of the CTA is reduced in a fixed order.
// Everything before the stores reads only state that the bulk pass of the
// same tick does not write (source populations, particle records, link
// lists), so the values are staged in shared memory and stored after
// grid_dep_wait(): launched with a programmatic edge from the bulk pass, the
// kernel computes during the bulk pass's last wave.
template <class L, int ST, bool TRT, int NT>
__device__ __forceinline__ bool fixup_body(const StepArgs& a, const long long b) {
    static_assert(NT >= kFixBlock && NT % 32 == 0 && kFixBlock == 64, "fix-up CTA shape");
    using SS = Store<ST>;
    using T = typename SS::T;
    using R = typename SS::R;
    constexpr int Q = L::Q;
    constexpr int D = L::D;
    __shared__ int s_first[Q];
    __shared__ int s_lat[4][Q];  // cx, cy, cz, opp
    __shared__ double s_w[Q];
    __shared__ R s_g[Q][kFixBlock];      // post-collision populations of the entries (f/w - rho0)
    __shared__ double s_rho[kFixBlock];  // rho^n of the entries
    __shared__ int s_cell[kFixBlock];
    __shared__ int s_xyz[3][kFixBlock];
    __shared__ double s_C[3][3][kFixBlock];  // coordinate of x-1, x, x+1 per axis
    __shared__ unsigned short s_list[kFixBlock * Q];  // (entry << 5) | j of every link slot
    __shared__ R s_val[kFixBlock * Q];                // the value of each listed slot
    __shared__ int s_wcnt[2];
    __shared__ double s_red[NT / 32][6];
    __shared__ ParticleDev sP;
    __shared__ int s_alone;
    const int tid = threadIdx.x;
    const long long npb = (long long)a.nparts * a.maxchunks;
    const long long nwlb = (a.nwlinks + kFixBlock - 1) / kFixBlock;
    T* __restrict__ dst = static_cast<T*>(a.dst);
    const long long N = a.g.N;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    if (b >= npb + nwlb) {  // wall nodes hold f = 0 (g = -rho0)
        const long long k0 = (b - npb - nwlb) * kFixBlock;
        const int n = (int)min((long long)kFixBlock, (long long)a.nwnodes - k0);
        const T z0 = SS::enc(R(-a.rho0), R(a.scale));
        grid_dep_wait();
        for (int s = tid; s < n * Q; s += NT) dst[(long long)(s % Q) * N + a.wnodes[k0 + s / Q]] = z0;
        return true;
    }
    const bool is_part = b < npb;
    int p = -1, chunk = 0;
    int2 ent = make_int2(0, 0);
    bool valid = false;
    if (is_part) {
        p = (int)(b / a.maxchunks);
        chunk = (int)(b % a.maxchunks);
        const int e = chunk * kFixBlock + tid;
        int loff, lcap;
        if (p < a.nlinkoc) {
            loff = a.linkoc[p][0];
            lcap = a.linkoc[p][1];
        } else {
            loff = a.parts[p].link_off;
            lcap = a.parts[p].link_cap;
        }
        if (tid < kFixBlock && e < lcap) ent = a.links[loff + e];  // in the list's capacity
        const int nl = a.parts[p].nlinks;
        if (chunk * kFixBlock >= nl) return false;  // uniform: chunk past the link list
        valid = tid < kFixBlock && e < nl;
        const unsigned long long* gsrc = reinterpret_cast<const unsigned long long*>(a.parts + p);
        unsigned long long* sdst = reinterpret_cast<unsigned long long*>(&sP);
        for (int k = tid; k < (int)(sizeof(ParticleDev) / 8); k += NT) sdst[k] = gsrc[k];
    } else {
        const long long e = (b - npb) * kFixBlock + tid;
        if (tid < kFixBlock && e < a.nwlinks) {
            ent = a.wlinks[e];
            valid = true;
        }
    }
    for (int j = tid; j < Q; j += NT) {
        s_first[j] = a.nparts;
        s_lat[0][j] = L::cx(j);
        s_lat[1][j] = L::cy(j);
        s_lat[2][j] = L::cz(j);
        s_lat[3][j] = L::opp(j);
        s_w[j] = L::w(j);
    }
    if (tid == 0) s_alone = 1;
    __syncthreads();
    // the second loads first: populations and coordinates of each entry's node
    const unsigned mask = valid ? (unsigned)ent.y : 0u;
    NodeState<L, ST, TRT> st;
    double cc[3][3];
    int xyz[3] = {0, 0, 0};
    if (valid) {
        const int cell = ent.x;
        xyz[0] = cell % nx;
        xyz[1] = (cell / nx) % ny;
        xyz[2] = cell / (nx * ny);
        load_pops<L, ST>(a, cell, true, st.g);
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int o = 0; o < 3; ++o)
                cc[k][o] = k < D ? a.coord[k][wrap_idx(xyz[k] + o - 1, a.g.n[k])] : 0.0;
    }
    // break rule of the Ladd loop (fluids.jl:184): for streaming direction j
    // only particles before the first one without links in j contribute.
    // The owner is "alone" when no other particle's near box meets its own:
    // then no other particle can have a link at the owner's link nodes.
    for (int q = tid; q < a.nparts; q += NT) {
        const ParticleDev& Pq = q == p ? sP : a.parts[q];
        const unsigned none = ~Pq.dirlinks;
        for (int j = 0; j < Q; ++j)
            if ((none >> j) & 1u) atomicMin(&s_first[j], q);
        if (is_part && q != p && !a.wall) {
            bool meet = true;
            for (int k = 0; k < D; ++k) {
                // near boxes [slo-1, shi+1] on a periodic axis of n nodes
                const int n = a.g.n[k];
                const int la = sP.shi[k] - sP.slo[k] + 3, lb = Pq.shi[k] - Pq.slo[k] + 3;
                if (la >= n || lb >= n || Pq.slo[k] > Pq.shi[k]) {
                    meet = meet && Pq.slo[k] <= Pq.shi[k];
                    continue;
                }
                const int d0 = wrap_idx((Pq.slo[k] - 1) - (sP.slo[k] - 1), n);
                meet = meet && (d0 < la || d0 + lb > n);
            }
            if (meet) s_alone = 0;
        }
    }
    if (is_part && a.wall && tid == 0) s_alone = 0;
    // collide each entry's node once
    if (valid) {
        st.rho = collide_node<L, ST, TRT>(a, ent.x, true, st.g);
        s_rho[tid] = (double)st.rho;  // rho^n(x), the density of model.massDensity
        s_cell[tid] = ent.x;
#pragma unroll
        for (int i = 0; i < Q; ++i) s_g[i][tid] = st.g[i] * R(a.inv_scale);  // storage -> f/w - rho0
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            s_xyz[k][tid] = xyz[k];
#pragma unroll
            for (int o = 0; o < 3; ++o) s_C[k][o][tid] = cc[k][o];
        }
    }
    // list the link slots: entries 0..31 and 32..63 scan their counts per warp
    int off = 0;
    if (tid < kFixBlock) {
        const int lane = tid & 31;
        int c = __popc(mask);
        off = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, off, o);
            if (lane >= o) off += v;
        }
        if (lane == 31) s_wcnt[tid >> 5] = off;
        off -= c;  // exclusive
    }
    __syncthreads();
    const int nlist = s_wcnt[0] + s_wcnt[1];
    if (tid < kFixBlock) {
        if (tid >= 32) off += s_wcnt[0];
        for (unsigned m = mask; m; m &= m - 1) s_list[off++] = (unsigned short)((tid << 5) | (__ffs(m) - 1));
    }
    __syncthreads();
    const bool alone = is_part && s_alone;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int l = tid; l < nlist; l += NT) {
        const int item = s_list[l];
        const int el = item >> 5, j = item & 31;
        const int cell = s_cell[el];
        const int i = s_lat[3][j];  // x - c_j = x + c_i is the solid source node
        const int ci0 = s_lat[0][i], ci1 = s_lat[1][i], ci2 = s_lat[2][i];
        R vout;
        if (a.wall && a.wall[cell]) {
            vout = R(-a.rho0);  // wall nodes hold f = 0 (fluids.jl:154)
        } else {
            const int x = s_xyz[0][el], y = s_xyz[1][el], z = s_xyz[2][el];
            const double rhoL = s_rho[el];
            const double gi = (double)s_g[i][el];
            const double wi = s_w[i];
            const double Tc[3] = {s_C[0][1 + ci0][el], s_C[1][1 + ci1][el], D == 3 ? s_C[2][1 + ci2][el] : 0.0};
            const double Xc[3] = {s_C[0][1][el], s_C[1][1][el], D == 3 ? s_C[2][1][el] : 0.0};
            double v = gi;  // halfway bounce-back: f_j(x) = f*_i(x)
            const int tx = wrap_idx(x + ci0, nx), ty = wrap_idx(y + ci1, ny), tz = wrap_idx(z + ci2, nz);
            if (a.uw) {  // moving walls (fluids.jl:168-174)
                const long long t = tx + (long long)nx * (ty + (long long)ny * tz);
                const double dot = -(ci0 * a.uw[t] + ci1 * a.uw[N + t] + (D == 3 ? ci2 * a.uw[2 * N + t] : 0.0));
                v += 6.0 * rhoL * dot;
            }
            // Ladd terms (fluids.jl:176-189) of every particle with link (x, j), in order
            if (alone) {
                if (p < s_first[j]) ladd_link<D>(a, sP, true, ci0, ci1, ci2, Tc, Xc, rhoL, gi, wi, v, acc);
            } else {
                const int tile = x / a.g.t[0] + a.g.nt[0] * (y / a.g.t[1] + a.g.nt[1] * (z / a.g.t[2]));
                int w = 0;
                unsigned long long bits = 0;
                while (true) {  // candidates of the tile, in ascending order
                    while (bits == 0 && w < a.words) bits = a.tilebits[(long long)tile * a.words + w++];
                    if (bits == 0) break;
                    const int q = (w - 1) * 64 + __ffsll((long long)bits) - 1;
                    bits &= bits - 1;
                    if (q >= s_first[j]) break;  // particles are visited in ascending order
                    const ParticleDev& P = q == p ? sP : a.parts[q];
                    if (solid_at(P, a.ivl, tx, ty, tz) && !solid_at(P, a.ivl, x, y, z))
                        ladd_link<D>(a, P, q == p, ci0, ci1, ci2, Tc, Xc, rhoL, gi, wi, v, acc);
                }
            }
            vout = (R)v;
        }
        s_val[l] = vout;
    }
    // the stores, after the bulk pass's stores to the same slots (each thread
    // stores the slots it computed)
    grid_dep_wait();
    for (int l = tid; l < nlist; l += NT) {
        const int item = s_list[l];
        dst[(item & 31) * N + s_cell[item >> 5]] =
            a.stochastic ? SS::enc_sr(s_val[l], R(a.scale), (unsigned)s_cell[item >> 5], item & 31)
                         : SS::enc(s_val[l], R(a.scale));
    }
    if (!is_part) return true;
    // fixed-order reduction: butterfly inside warps, warps summed in order
#pragma unroll
    for (int k = 0; k < 6; ++k)
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if ((tid & 31) == 0)
        for (int k = 0; k < 6; ++k) s_red[tid >> 5][k] = acc[k];
    __syncthreads();
    if (tid < 6) {
        double sum = 0.0;
        for (int w = 0; w < NT / 32; ++w) sum += s_red[w][tid];
        a.partial[(long long)(sP.part_off + chunk) * kPartialStride + tid] = sum;
    }
    return true;
}

template <class L, int ST, bool TRT>
__global__ void __launch_bounds__(kFixThreads) k_fixup(const StepArgs a) {
    fixup_body<L, ST, TRT, kFixThreads>(a, blockIdx.x);
}

// Many particles: k_fixup_walk.  Its CTA g of a particle walks chunks g,
// g + G, ... of the particle's list up to the list's end, so the CTAs past the
// lists' ends number G - chunks per particle rather than the capacity's
// chunks (the capacity is the near box; 64 particles of r = 6 in 192^3 launch
// 2,048 CTAs instead of 8,000).  With one particle k_fixup is faster: the
// walk costs registers, and the CTAs past the list end overlap the others.
constexpr int kFixCtasPerPart = 32;
constexpr long long kFixWalkMin = 1024;  // particle CTAs of k_fixup from which k_fixup_walk is used
__host__ __device__ __forceinline__ int fixup_ctas_per_particle(int maxchunks) {
    return maxchunks < kFixCtasPerPart ? maxchunks : kFixCtasPerPart;
}

// one chunk, as a called function (the parameter block is addressed in place)
template <class L, int ST, bool TRT>
__device__ __noinline__ bool fixup_chunk(const StepArgs& a, const long long b) {
    return fixup_body<L, ST, TRT, kFixThreads>(a, b);
}

// Grid: nparts * fixup_ctas_per_particle(maxchunks) CTAs, chunk-major (the
// first chunks of every particle first), then one per wall-link or
// wall-node block.
template <class L, int ST, bool TRT>
__global__ void __launch_bounds__(kFixThreads, 2) k_fixup_walk(const __grid_constant__ StepArgs a) {
    const long long bi = blockIdx.x;
    const int G = fixup_ctas_per_particle(a.maxchunks);
    const long long pb = (long long)a.nparts * G;
    if (bi >= pb) {
        fixup_chunk<L, ST, TRT>(a, (long long)a.nparts * a.maxchunks + (bi - pb));
        return;
    }
    const int p = (int)(bi % a.nparts);
    for (int c = (int)(bi / a.nparts); c < a.maxchunks; c += G) {
        if (!fixup_chunk<L, ST, TRT>(a, (long long)p * a.maxchunks + c)) break;
        __syncthreads();  // shared memory is reused by the next chunk
    }
}

}  // namespace lbm
