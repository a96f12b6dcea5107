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
// The node's collided populations are kept in shared memory and the link
// directions are visited with a runtime loop over the mask, which keeps the
// kernel body small (instruction fetch limited the fully unrolled form).
#pragma once
#include "kernels.cuh"

namespace lbm {

constexpr int kFixCoord = 64;   // near-box node coordinates staged per axis

template <class L, int ST, bool TRT>
__device__ __forceinline__ void fixup_body(const StepArgs& a, const long long b) {
    using SS = Store<ST>;
    using T = typename SS::T;
    using R = typename SS::R;
    constexpr int Q = L::Q;
    constexpr int D = L::D;
    __shared__ int s_first[Q];
    __shared__ int s_lat[4][Q];  // cx, cy, cz, opp
    __shared__ double s_w[Q];
    __shared__ R s_g[Q][kFixBlock];
    __shared__ double s_red[kFixBlock / 32][6];
    __shared__ ParticleDev sP;
    __shared__ double s_X[3][kFixCoord];
    __shared__ int s_alone;
    const int tid = threadIdx.x;
    const long long npb = (long long)a.nparts * a.maxchunks;
    const long long nwlb = (a.nwlinks + kFixBlock - 1) / kFixBlock;
    T* __restrict__ dst = static_cast<T*>(a.dst);
    const long long N = a.g.N;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    if (b >= npb + nwlb) {  // wall nodes hold f = 0 (g = -rho0)
        const long long k = (b - npb - nwlb) * kFixBlock + tid;
        if (k < a.nwnodes) {
            const int cell = a.wnodes[k];
            const T z0 = SS::enc(R(-a.rho0), R(a.scale));
#pragma unroll
            for (int i = 0; i < Q; ++i) dst[i * N + cell] = z0;
        }
        return;
    }
    const bool is_part = b < npb;
    int p = -1, chunk = 0;
    if (is_part) {
        p = (int)(b / a.maxchunks);
        chunk = (int)(b % a.maxchunks);
        if (chunk * kFixBlock >= a.parts[p].nlinks) return;  // uniform: chunk past the link list
        const unsigned long long* gsrc = reinterpret_cast<const unsigned long long*>(a.parts + p);
        unsigned long long* sdst = reinterpret_cast<unsigned long long*>(&sP);
        for (int k = tid; k < (int)(sizeof(ParticleDev) / 8); k += kFixBlock) sdst[k] = gsrc[k];
    }
    for (int j = tid; j < Q; j += kFixBlock) {
        s_first[j] = a.nparts;
        s_lat[0][j] = L::cx(j);
        s_lat[1][j] = L::cy(j);
        s_lat[2][j] = L::cz(j);
        s_lat[3][j] = L::opp(j);
        s_w[j] = L::w(j);
    }
    if (tid == 0) s_alone = 1;
    __syncthreads();
    // break rule of the Ladd loop (fluids.jl:184): for streaming direction j
    // only particles before the first one without links in j contribute.
    // The owner is "alone" when no other particle's near box meets its own:
    // then no other particle can have a link at the owner's link nodes.
    for (int q = tid; q < a.nparts; q += kFixBlock) {
        const ParticleDev& Pq = a.parts[q];
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
    // the owner's near-box coordinates, and this thread's entry of the link list
    int ext[3] = {1, 1, 1};
    if (is_part)
        for (int k = 0; k < D; ++k) ext[k] = near_extent(sP, a.g, k, D);
    const bool cst = is_part && ext[0] <= kFixCoord && ext[1] <= kFixCoord && ext[2] <= kFixCoord;
    bool valid = false;
    int cell = 0, x = 0, y = 0, z = 0;
    unsigned mask = 0;
    if (is_part) {
        if (cst)
            for (int k = 0; k < D; ++k)
                for (int i = tid; i < ext[k]; i += kFixBlock)
                    s_X[k][i] = a.coord[k][wrap_idx(sP.slo[k] - 1 + i, a.g.n[k])];
        const int e = chunk * kFixBlock + tid;
        if (e < sP.nlinks) {
            const int2 ent = a.links[sP.link_off + e];
            cell = ent.x;
            mask = (unsigned)ent.y;
            x = cell % nx;
            y = (cell / nx) % ny;
            z = cell / (nx * ny);
            valid = true;
        }
    }
    __syncthreads();
    // coordinate of node index i on axis k (staged for the owner's near box)
    auto coordf = [&](int k, int i) -> double {
        return cst ? s_X[k][wrap_idx(i - (sP.slo[k] - 1), a.g.n[k])] : a.coord[k][i];
    };
    if (!is_part) {
        const long long e = (b - npb) * kFixBlock + tid;
        if (e < a.nwlinks) {
            const int2 ent = a.wlinks[e];
            cell = ent.x;
            mask = (unsigned)ent.y;
            x = cell % nx;
            y = (cell / nx) % ny;
            z = cell / (nx * ny);
            valid = true;
        }
    }

    // collide the node once; keep its post-collision populations in shared memory
    double rhoL = 0.0;
    if (valid) {
        NodeState<L, ST, TRT> s;
        load_collide<L, ST, TRT>(a, cell, true, s);
        rhoL = (double)s.rho;  // rho^n(x), the density of model.massDensity
#pragma unroll
        for (int i = 0; i < Q; ++i) s_g[i][tid] = s.g[i] * R(a.inv_scale);  // storage -> f/w - rho0
    }

    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (valid) {
        const bool oW = a.wall && a.wall[cell];
        const int tile = x / a.g.t[0] + a.g.nt[0] * (y / a.g.t[1] + a.g.nt[1] * (z / a.g.t[2]));
        const double X0 = coordf(0, x), X1 = coordf(1, y), X2 = D == 3 ? coordf(2, z) : 0.0;
        const double rho0 = a.rho0;
        const bool alone = is_part && s_alone;
        for (unsigned m = mask; m; m &= m - 1) {
            const int j = __ffs(m) - 1;
            const int i = s_lat[3][j];  // x - c_j = x + c_i is the solid source node
            const int ci0 = s_lat[0][i], ci1 = s_lat[1][i], ci2 = s_lat[2][i];
            const int tx = wrap_idx(x + ci0, nx), ty = wrap_idx(y + ci1, ny), tz = wrap_idx(z + ci2, nz);
            const int t = tx + nx * (ty + ny * tz);
            R vout;
            if (oW) {
                vout = R(-rho0);  // wall nodes hold f = 0 (fluids.jl:154)
            } else {
                const double gi = (double)s_g[i][tid];
                double v = gi;  // halfway bounce-back: f_j(x) = f*_i(x)
                if (a.uw) {     // moving walls (fluids.jl:168-174)
                    const double dot = -(ci0 * a.uw[t] + ci1 * a.uw[N + t] + (D == 3 ? ci2 * a.uw[2 * N + t] : 0.0));
                    v += 6.0 * rhoL * dot;
                }
                // Ladd terms (fluids.jl:176-189) of every particle with link (x, j), in order
                const double T0 = coordf(0, tx), T1 = coordf(1, ty), T2 = D == 3 ? coordf(2, tz) : 0.0;
                const double wi = s_w[i];
                int q = alone ? p : -1;
                const ParticleDev* Pp = alone ? &sP : nullptr;
                int w = 0;
                unsigned long long bits = 0;
                while (true) {
                    if (!alone) {  // next candidate of the tile, in ascending order
                        while (bits == 0 && w < a.words) bits = a.tilebits[(long long)tile * a.words + w++];
                        if (bits == 0) break;
                        q = (w - 1) * 64 + __ffsll((long long)bits) - 1;
                        bits &= bits - 1;
                        Pp = a.parts + q;
                    }
                    if (q >= s_first[j]) break;  // particles are visited in ascending order
                    const ParticleDev& P = *Pp;
                    if (alone || (solid_at(P, a.ivl, tx, ty, tz) && !solid_at(P, a.ivl, x, y, z))) {
                        double up[3];
                        slip_velocity<D>(P.sR, P.sV, P.sW, P.sE, P.B1, P.B2, P.kind, T0, T1, T2, up);
                        v += 6.0 * rhoL * (-(ci0 * up[0] + ci1 * up[1] + ci2 * up[2]));
                        if (q == p && (P.coupleF || P.coupleT)) {
                            // f*_i(x) + f_j(x) in f units; F -= coeff*s*c_j = coeff*s*c_i
                            const double cs = a.coeff * (wi * (2.0 * rho0 + gi + v));
                            if (P.coupleF) {
                                acc[0] += cs * ci0;
                                acc[1] += cs * ci1;
                                acc[2] += cs * ci2;
                            }
                            if (P.coupleT) {  // T -= coeff*cross(s*(x-R), c_j) = coeff*cross(s*(x-R), c_i)
                                const double r0 = X0 - P.mR[0], r1 = X1 - P.mR[1], r2 = D == 3 ? X2 - P.mR[2] : 0.0;
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
                    if (alone) break;
                }
                vout = (R)v;
            }
            dst[j * N + cell] = SS::enc(vout, R(a.scale));
        }
    }
    if (!is_part) return;
    // fixed-order reduction: butterfly inside warps, warps summed in order
#pragma unroll
    for (int k = 0; k < 6; ++k)
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if ((tid & 31) == 0)
        for (int k = 0; k < 6; ++k) s_red[tid >> 5][k] = acc[k];
    __syncthreads();
    if (tid == 0) {
        double* out = a.partial + (long long)(sP.part_off + chunk) * kPartialStride;
        for (int k = 0; k < 6; ++k) {
            double sum = 0.0;
            for (int w = 0; w < kFixBlock / 32; ++w) sum += s_red[w][k];
            out[k] = sum;
        }
    }
}

template <class L, int ST, bool TRT>
__global__ void __launch_bounds__(kFixBlock) k_fixup(const StepArgs a) {
    fixup_body<L, ST, TRT>(a, blockIdx.x);
}

}  // namespace lbm
