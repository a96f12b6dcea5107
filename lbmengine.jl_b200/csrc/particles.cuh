// Particle update on the device: momentum-exchange reduction, Newton-Euler
// integration with Rodrigues rotation, re-voxelisation and boundary-link
// bookkeeping.  Restates moveParticles! (src/gpu/particles.jl:7-92), one
// particle per CTA.
//
// The solid region of a particle (getSphere, src/gpu/aux.jl:206-215) is kept
// as one x-interval per (y, z) row of its index box, each found with the exact
// FP64 sphere test, so every membership query afterwards is two integer
// compares.  The boundary links (bounceBackPrep, src/gpu/aux.jl:187-198) are
// kept as a list of (fluid cell, direction mask) entries that is rebuilt only
// when the intervals change; a sub-node move leaves both untouched.
#pragma once
#include "kernels.cuh"

namespace lbm {

constexpr int kIvlSmem = 512;  // rows of solid intervals staged in shared memory
constexpr int kXSmem = 256;    // x coordinates of the solid box staged in shared memory
constexpr int kLinkSmem = 2048;  // link entries staged in shared memory during a rebuild
constexpr int kPartBlock = 512;  // CTA size of the stand-alone particle kernel (one near-box row
                                 // per thread in a link rebuild of a particle up to r ~ 10)
constexpr int kMaxPartWarps = 32;

struct ParticleArgs {
    ParticleDev* parts;
    int nparts;
    int mode;        // 0: tick update; 1: initial setup of particle `setup_pid`;
                     // 2: re-voxelise `setup_pid` keeping its slip snapshot (checkpoint restore)
    int setup_pid;
    int words;
    const double* partial;
    unsigned long long* tilebits;
    int2* ivl;
    int2* links;
    GridDesc g;
    const double* coord[3];
    double x0[3];
    double dx, dt;
    int* err;
    int inline_links;  // 1: rebuild changed link lists here; 0: flag them (relink) for k_links
    int pad;
    int* nbox_out[2];  // [nparts][6] solid boxes (lo, hi) published for the bulk pass two ticks
                       // later (tick update writes [0]; setup writes both); null to skip
    double* trj;       // trajectory ring: [trj_cap][nparts][9] (position, velocity, angular
                       // velocity after each tick's update), or null
    long long trj_cap;
    const double* fint;  // [nparts][3] forces of the particle interactions (interactions.cuh), or null
};

// publish particle p's solid box for the far/near split of the bulk pass
__device__ __forceinline__ void publish_box(const ParticleArgs& a, int p, const ParticleDev& P) {
    for (int b = 0; b < 2; ++b) {
        if (!a.nbox_out[b]) continue;
        for (int k = 0; k < 3; ++k) {
            a.nbox_out[b][6 * p + k] = P.slo[k];
            a.nbox_out[b][6 * p + 3 + k] = P.shi[k];
        }
    }
}

// index box (clipped, not periodic) that contains every node of the sphere;
// the +-1 margin absorbs the rounding of the affine index estimate
__device__ __forceinline__ void solid_box(const ParticleArgs& a, const double* R, double radius, int D, int* lo, int* hi) {
    for (int k = 0; k < 3; ++k) {
        if (k >= D) {
            lo[k] = 0;
            hi[k] = 0;
            continue;
        }
        const double c = (R[k] - a.x0[k]) / a.dx;
        const double rr = radius / a.dx;
        double l = floor(c - rr) - 1.0, h = ceil(c + rr) + 1.0;
        const int n = a.g.n[k];
        if (!(l <= h) || h < 0.0 || l > (double)(n - 1)) {  // NaN or outside the domain
            lo[k] = 1;
            hi[k] = 0;
            continue;
        }
        lo[k] = l < 0.0 ? 0 : (int)l;
        hi[k] = h > (double)(n - 1) ? n - 1 : (int)h;
    }
}

// tile range covering nodes [s, s+len) of a periodic axis (s may be -1)
__device__ __forceinline__ void tile_range(int s, int len, int n, int t, int nt, int* tlo, int* tn) {
    if (len >= n) {
        *tlo = 0;
        *tn = nt;
        return;
    }
    const int s0 = wrap_idx(s, n);
    const int e = s0 + len - 1;  // unwrapped last node, < 2n
    const int t0 = s0 / t;
    const int t1 = e < n ? e / t : nt + (e - n) / t;
    int c = t1 - t0 + 1;
    *tlo = t0;
    *tn = c > nt ? nt : c;
}

__device__ __forceinline__ void tile_bits_update(const ParticleArgs& a, const int* tlo, const int* tn, int p, bool set) {
    const int total = tn[0] * tn[1] * tn[2];
    const unsigned long long bit = 1ull << (p & 63);
    const int word = p >> 6;
    for (int l = threadIdx.x; l < total; l += blockDim.x) {
        const int dx = l % tn[0], dy = (l / tn[0]) % tn[1], dz = l / (tn[0] * tn[1]);
        const long long tx = (tlo[0] + dx) % a.g.nt[0];
        const long long ty = (tlo[1] + dy) % a.g.nt[1];
        const long long tz = (tlo[2] + dz) % a.g.nt[2];
        const long long tile = tx + a.g.nt[0] * (ty + a.g.nt[1] * tz);
        unsigned long long* wp = a.tilebits + tile * a.words + word;
        if (set) atomicOr(wp, bit);
        else atomicAnd(wp, ~bit);
    }
}

// interval of row (y, z) of P's solid box (rows y-fastest from `rows`), or empty
__device__ __forceinline__ int2 box_row_ivl(const ParticleDev& P, const int2* rows, int y, int z) {
    if (y < P.slo[1] || y > P.shi[1] || z < P.slo[2] || z > P.shi[2]) return make_int2(1, 0);
    return rows[(y - P.slo[1]) + (P.shi[1] - P.slo[1] + 1) * (z - P.slo[2])];
}

// The link entries of near-box row rr of P (near box ex x ey x .., x' = x - s0),
// counted, and written to `out` unless it is null.  In x' coordinates every
// row interval lies in [1, ex - 2] (the caller checks ex + 2 <= nx), so node
// x' has a solid source x + c_i exactly when x' + c_i,x lies in the interval
// of row (y + c_i,y, z + c_i,z); the candidates are the span of those shifted
// intervals outside the row's own one.  A free function with its values in
// registers: a lambda's captures or an indexed array could sit in local
// memory, whose L1 lines the bulk pass running beside this kernel evicts.
template <class L>
__device__ __forceinline__ int near_row_links(const ParticleDev& P, const int2* rows, const GridDesc& g, int ex,
                                              int ey, int s0, int rr, int2* out) {
    constexpr int D = L::D;
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const int y = wrap_idx(P.slo[1] - 1 + rr % ey, ny);
    const int z = D == 3 ? wrap_idx(P.slo[2] - 1 + rr / ey, nz) : 0;
    auto nbr = [&](int dy, int dz) -> int2 {
        if (D == 2 && dz != 0) return make_int2(1, 0);
        const int2 iv = box_row_ivl(P, rows, wrap_idx(y + dy, ny), D == 3 ? wrap_idx(z + dz, nz) : 0);
        return iv.x <= iv.y ? make_int2(iv.x - s0, iv.y - s0) : make_int2(1, 0);
    };
    const int2 r00 = nbr(-1, -1), r10 = nbr(0, -1), r20 = nbr(1, -1);
    const int2 r01 = nbr(-1, 0), r11 = nbr(0, 0), r21 = nbr(1, 0);
    const int2 r02 = nbr(-1, 1), r12 = nbr(0, 1), r22 = nbr(1, 1);
    auto iv_of = [&](int cy, int cz) -> int2 {  // cy, cz are constants after unrolling
        switch ((cy + 1) * 3 + (cz + 1)) {
            case 0: return r00;
            case 1: return r01;
            case 2: return r02;
            case 3: return r10;
            case 4: return r11;
            case 5: return r12;
            case 6: return r20;
            case 7: return r21;
            default: return r22;
        }
    };
    int cl = ex, ch = -1;
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        const int2 iv = iv_of(L::cy(i), L::cz(i));
        if (iv.x <= iv.y) {
            cl = min(cl, iv.x - L::cx(i));
            ch = max(ch, iv.y - L::cx(i));
        }
    }
    cl = max(cl, 0);
    ch = min(ch, ex - 1);
    const int o0 = r11.x, o1 = r11.y;  // the row's own solid interval
    int cnt = 0;
    for (int xr = cl; xr <= ch; ++xr) {
        if (xr >= o0 && xr <= o1) {
            xr = o1;
            continue;
        }
        unsigned mask = 0;
#pragma unroll
        for (int j = 1; j < L::Q; ++j) {
            const int i = L::opp(j);  // source x - c_j = x + c_i
            const int2 iv = iv_of(L::cy(i), L::cz(i));
            const int t = xr + L::cx(i);
            if (t >= iv.x && t <= iv.y) mask |= 1u << j;
        }
        if (!mask) continue;
        if (out) out[cnt] = make_int2(wrap_idx(s0 + xr, nx) + nx * (y + ny * z), (int)mask);
        ++cnt;
    }
    return cnt;
}

// LK: link entries staged in shared memory during a rebuild (kLinkSmem for
// the particle kernel; less inside the persistent tick kernel, whose CTAs
// also hold the bulk and fix-up items' shared memory)
template <class L, int LK = kLinkSmem>
__device__ __forceinline__ void particles_body(const ParticleArgs& a, const int p) {
    constexpr int D = L::D;
    const int tid = threadIdx.x;
    __shared__ double s_red[kMaxPartWarps][6];
    __shared__ int s_moved, s_oldbox[6], s_newbox[6], s_changed, s_rows, s_bad, s_nonempty, s_keep;
    __shared__ unsigned long long s_slack;  // bit pattern of a non-negative double
    __shared__ unsigned s_links;
    __shared__ int s_warp[kMaxPartWarps + 1];
    __shared__ int2 s_ivl[kIvlSmem];  // the particle's solid intervals during a link rebuild
    __shared__ double s_xc[kXSmem];   // x coordinates of the solid box (interval rebuild)
    // A rebuild's new intervals (s_ivl) and link entries (s_lk) are written to
    // global memory at the end, coalesced: scattered stores issued in between
    // drain slowly beside the bulk pass and hold up the shared-memory accesses
    // queued behind them.
    __shared__ int2 s_lk[LK];
    __shared__ int s_lkn;  // entries [0, s_lkn) of the new list are in s_lk
    // the particle record is staged in shared memory: the update below is a
    // serial chain of reads and writes that must not go to global memory
    __shared__ ParticleDev sP;
    static_assert(sizeof(ParticleDev) % 8 == 0, "ParticleDev is copied in 8-byte words");
    {
        const unsigned long long* gsrc = reinterpret_cast<const unsigned long long*>(a.parts + p);
        unsigned long long* sdst = reinterpret_cast<unsigned long long*>(&sP);
        for (int k = tid; k < (int)(sizeof(ParticleDev) / 8); k += blockDim.x) sdst[k] = gsrc[k];
    }
    __syncthreads();
    ParticleDev& P = sP;
    if (tid == 0) P.relink = 0;  // set again below when this update changes the intervals

    // 1. momentum exchange: fixed-order reduction of the per-chunk partials
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (a.mode == 0) {
        const int nch = (P.nlinks + kFixBlock - 1) / kFixBlock;  // chunks of the link list the fix-up ran over
        for (int l = tid; l < nch; l += blockDim.x) {
            const double* q = a.partial + (long long)(P.part_off + l) * kPartialStride;
            for (int k = 0; k < 6; ++k) acc[k] += q[k];
        }
    }
    for (int k = 0; k < 6; ++k)
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if ((tid & 31) == 0)
        for (int k = 0; k < 6; ++k) s_red[tid >> 5][k] = acc[k];
    __syncthreads();

    // 2. Newton-Euler update in FP64: translation (thread 0) and rotation
    //    (thread 32) are independent chains and run on different warps
    __shared__ int s_alpha;
    if (tid == 0 || tid == 32) {
        double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
        const int nw = blockDim.x >> 5;
        for (int k = 0; k < 3; ++k) {
            for (int w = 0; w < nw; ++w) {
                F[k] += s_red[w][k];
                T[k] += s_red[w][3 + k];
            }
        }
        const double dt = a.dt;
        if (a.mode == 0 && a.fint)  // molecularDynamicsTick!: the interactions' share of the force input
            for (int k = 0; k < 3; ++k) F[k] += a.fint[3 * p + k];
        const bool cpu = P.rules == 1;  // LBM_RULES_CPU_MODULE
        if (tid == 0) {
            bool moved = a.mode != 0;
            if (a.mode == 0 && cpu) {
                // src/cpu/particles.jl:55-60: v += m^-1 dP (dP = dt F, the momentum
                // input of the tick), then an Euler step whenever v != 0
                bool vnz = false;
                for (int k = 0; k < D; ++k) {
                    P.v[k] = P.v[k] + P.inv_mass * (dt * F[k]);
                    vnz = vnz || P.v[k] != 0.0;
                }
                if (vnz) {
                    for (int k = 0; k < D; ++k) P.R[k] = P.R[k] + dt * P.v[k];
                    moved = true;
                }
            } else if (a.mode == 0 && P.coupleF) {
                for (int k = 0; k < D; ++k) P.v[k] = P.v[k] + dt * (F[k] * P.inv_mass);
                for (int k = 0; k < D; ++k) P.R[k] = P.R[k] + dt * P.v[k];
                for (int k = 0; k < D; ++k)
                    if (P.v[k] != 0.0) moved = true;
            }
            s_moved = moved ? 1 : 0;
            if (a.mode != 2)
                for (int k = 0; k < 3; ++k) {  // CPU rules report the momentum inputs dP, dL
                    P.lastF[k] = cpu ? dt * F[k] : F[k];
                    P.lastT[k] = cpu ? dt * T[k] : T[k];
                }
        } else if (cpu) {  // w += I^-1 dL; the swimming direction never rotates (:7-18)
            bool alpha = false;
            if (a.mode == 0) {
                const int nw2 = D == 2 ? 1 : 3;
                for (int k = 0; k < nw2; ++k) {
                    const double dL = dt * T[k];
                    P.w[k] = P.w[k] + P.inv_inertia * dL;
                    alpha = alpha || dL != 0.0;
                }
            }
            s_alpha = alpha ? 1 : 0;
        } else {
            bool alpha = false;
            if (a.mode == 0 && P.coupleT) {
                const int nw2 = D == 2 ? 1 : 3;
                double Al[3] = {0, 0, 0};
                for (int k = 0; k < nw2; ++k) Al[k] = T[k] * P.inv_inertia;
                for (int k = 0; k < nw2; ++k) P.w[k] = P.w[k] + dt * Al[k];
                if (P.kind == 1) {
                    double theta = D == 2 ? fabs(P.w[0]) : sqrt(P.w[0] * P.w[0] + P.w[1] * P.w[1] + P.w[2] * P.w[2]);
                    if (theta != 0.0) {  // Rodrigues' rotation of the swimming direction
                        const double* v = P.e;
                        double vr[3] = {0, 0, 0};
                        if (D == 2) {
                            const double k = P.w[0] / theta;
                            theta *= dt;
                            const double ct = cos(theta), st = sin(theta);
                            vr[0] = v[0] * ct + (-k * v[1]) * st;
                            vr[1] = v[1] * ct + (k * v[0]) * st;
                        } else {
                            const double k[3] = {P.w[0] / theta, P.w[1] / theta, P.w[2] / theta};
                            theta *= dt;
                            const double ct = cos(theta), st = sin(theta);
                            const double cr[3] = {k[1] * v[2] - k[2] * v[1], -k[0] * v[2] + k[2] * v[0],
                                                  k[0] * v[1] - k[1] * v[0]};
                            const double kv = k[0] * v[0] + k[1] * v[1] + k[2] * v[2];
                            for (int q = 0; q < 3; ++q) vr[q] = v[q] * ct + cr[q] * st + k[q] * kv * (1.0 - ct);
                        }
                        double nr = 0.0;
                        for (int q = 0; q < D; ++q) nr += vr[q] * vr[q];
                        nr = sqrt(nr);
                        for (int q = 0; q < D; ++q) P.e[q] = vr[q] / nr;
                    }
                }
                for (int k = 0; k < nw2; ++k)
                    if (Al[k] != 0.0) alpha = true;
            }
            s_alpha = alpha ? 1 : 0;
        }
    }
    __syncthreads();
    if (tid == 0) {
        const bool moved = s_moved != 0;
        const bool need_nv = a.mode == 1 || (a.mode == 0 && (moved || s_alpha));
        if (need_nv)
            for (int k = 0; k < 3; ++k) {
                P.sR[k] = P.R[k];
                P.sV[k] = P.v[k];
                P.sW[k] = P.w[k];
                P.sE[k] = P.e[k];
            }
        s_moved = moved ? 1 : 0;
        if (a.mode == 0 && a.trj) {  // the state writeParticleTrajectory writes after each tick
            double* r = a.trj + ((P.nrec % a.trj_cap) * a.nparts + p) * 9;
            for (int k = 0; k < 3; ++k) {
                r[k] = P.R[k];
                r[3 + k] = P.v[k];
                r[6 + k] = P.w[k];
            }
            P.nrec += 1;
        }
        s_changed = (a.mode != 0 || !P.valid) ? 1 : 0;
        s_bad = 0;
        s_nonempty = 0;
        s_slack = (unsigned long long)__double_as_longlong(1e300);
        for (int k = 0; k < 3; ++k) {
            s_oldbox[k] = P.tlo[k];
            s_oldbox[3 + k] = P.valid ? P.tn[k] : 0;
        }
        s_keep = 0;
        if (moved) {
            for (int k = 0; k < 3; ++k) P.mR[k] = P.R[k];
            int lo[3], hi[3];
            solid_box(a, P.R, P.radius, D, lo, hi);
            // Keep the stored intervals when no node of the (unchanged) solid box
            // can change sides: |d^2(R) - d^2(vR)| <= 2 dmax |R - vR| + |R - vR|^2
            // for every node, dmax its largest distance from vR, and the stored
            // slack exceeds that bound by far more than the FP64 rounding of d^2.
            if (a.mode == 0 && P.valid && P.slack > 0.0) {
                bool same = true;
                double dlt2 = 0.0, dmax2 = 0.0;
                for (int k = 0; k < D; ++k) {
                    same = same && lo[k] == P.slo[k] && hi[k] == P.shi[k];
                    const double dk = P.R[k] - P.vR[k];
                    dlt2 += dk * dk;
                    if (lo[k] <= hi[k]) {
                        const double e0 = fabs(a.coord[k][lo[k]] - P.vR[k]), e1 = fabs(a.coord[k][hi[k]] - P.vR[k]);
                        const double e = e0 > e1 ? e0 : e1;
                        dmax2 += e * e;
                    }
                }
                const double dlt = sqrt(dlt2), dmax = sqrt(dmax2);
                const double bound = 2.0 * dmax * dlt + dlt2;
                if (same && bound < P.slack - 1e-9 * (P.r2 + dmax2)) s_keep = 1;
            }
        }
        if (moved && !s_keep) {
            for (int k = 0; k < 3; ++k) P.vR[k] = P.R[k];
            P.slack = 0.0;
            int lo[3], hi[3];
            solid_box(a, P.R, P.radius, D, lo, hi);
            bool empty = false;
            for (int k = 0; k < 3; ++k) {
                if (lo[k] != P.slo[k] || hi[k] != P.shi[k]) s_changed = 1;
                P.slo[k] = lo[k];
                P.shi[k] = hi[k];
                empty = empty || lo[k] > hi[k];
            }
            int rows = empty ? 0 : (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
            if (rows > P.ivl_cap) {
                atomicOr(a.err, kErrIntervalOverflow);
                rows = 0;
                empty = true;
            }
            s_rows = rows;
            int tlo[3] = {0, 0, 0}, tn[3] = {0, 0, 0};
            if (!empty)
                for (int k = 0; k < 3; ++k)
                    tile_range(lo[k] - 1, hi[k] - lo[k] + 3, a.g.n[k], a.g.t[k], a.g.nt[k], &tlo[k], &tn[k]);
            for (int k = 0; k < 3; ++k) {
                P.tlo[k] = tlo[k];
                P.tn[k] = tn[k];
                s_newbox[k] = tlo[k];
                s_newbox[3 + k] = tn[k];
            }
        }
        P.valid = 1;
    }
    __syncthreads();
    if (!s_moved || s_keep) {
        // nothing geometric changed; write the record back
        const unsigned long long* ssrc = reinterpret_cast<const unsigned long long*>(&sP);
        unsigned long long* gdst = reinterpret_cast<unsigned long long*>(a.parts + p);
        for (int k = tid; k < (int)(sizeof(ParticleDev) / 8); k += blockDim.x) gdst[k] = ssrc[k];
        if (tid == 0) publish_box(a, p, P);
        return;
    }

    // 3. solid intervals of the new position, compared with the stored ones
    {
        const int lx0 = P.slo[0], lx1 = P.shi[0];
        const int ly = P.shi[1] - P.slo[1] + 1;
        // the row loop below reads every x coordinate of the box once per row:
        // from shared memory (global loads there would each wait out the
        // memory latency of the bulk pass running beside this kernel)
        const bool xs = lx1 - lx0 + 1 <= kXSmem;
        if (xs)
            for (int i = tid; i <= lx1 - lx0; i += blockDim.x) s_xc[i] = a.coord[0][lx0 + i];
        __syncthreads();
        int changed = 0;
        for (int r = tid; r < s_rows; r += blockDim.x) {
            const int y = P.slo[1] + r % ly;
            const int z = P.slo[2] + r / ly;
            // the row's global loads first, so that their latencies overlap
            int2* slot = a.ivl + P.ivl_off + r;
            const int2 old = *slot;
            const double Y = a.coord[1][y], Z = D == 3 ? a.coord[2][z] : 0.0;
            int xlo = 1, xhi = 0;
            double slack = 1e300;
            for (int x = lx0; x <= lx1; ++x) {
                const double d2 = sphere_d2<D>(xs ? s_xc[x - lx0] : a.coord[0][x], Y, Z, P.vR);
                if (d2 < P.r2) {
                    if (xlo > xhi) xlo = x;
                    xhi = x;
                }
                slack = fmin(slack, fabs(d2 - P.r2));
            }
            // non-negative doubles order like their bit patterns
            atomicMin(&s_slack, (unsigned long long)__double_as_longlong(slack));
            if (old.x != xlo || old.y != xhi) changed = 1;
            if (s_rows > kIvlSmem) *slot = make_int2(xlo, xhi);  // else written at the end
            if (r < kIvlSmem) s_ivl[r] = make_int2(xlo, xhi);
            if (xlo <= xhi) s_nonempty = 1;
        }
        if (changed) atomicOr(&s_changed, 1);
    }
    __syncthreads();
    if (tid == 0) P.slack = __longlong_as_double((long long)s_slack);

    // 4. boundary-link entries over the near box (solid box + 1, periodic)
    const bool ivl_smem = s_rows <= kIvlSmem;
    auto inS = [&](int x, int y, int z) -> bool {
        if (!ivl_smem) return solid_at(P, a.ivl, x, y, z);
        if (y < P.slo[1] || y > P.shi[1] || z < P.slo[2] || z > P.shi[2]) return false;
        const int2 iv = s_ivl[(y - P.slo[1]) + (P.shi[1] - P.slo[1] + 1) * (z - P.slo[2])];
        return x >= iv.x && x <= iv.y;
    };
    // Directions with at least one link (the break rule of fluids.jl:184).  A
    // non-empty solid region that spans no periodic axis has a link in every
    // moving direction (its extreme node along c_j always has a fluid
    // neighbour); otherwise the links are counted exactly over the solid box.
    if (s_changed) {
        bool spans = false;
        for (int k = 0; k < D; ++k) spans = spans || (P.shi[k] - P.slo[k] + 1 >= a.g.n[k]);
        if (!s_nonempty) {
            if (tid == 0) P.dirlinks = 0u;
        } else if (!spans) {
            if (tid == 0) {
                unsigned m = 0;
                for (int j = 1; j < L::Q; ++j) m |= 1u << j;
                P.dirlinks = m;
            }
        } else {
            if (tid == 0) s_links = 0u;
            __syncthreads();
            const int l0 = P.shi[0] - P.slo[0] + 1, l1 = P.shi[1] - P.slo[1] + 1, l2 = P.shi[2] - P.slo[2] + 1;
            const long long vol = (long long)l0 * l1 * l2;
            unsigned m = 0;
            for (long long q = tid; q < vol; q += blockDim.x) {
                const int x = P.slo[0] + (int)(q % l0);
                const int y = P.slo[1] + (int)((q / l0) % l1);
                const int z = P.slo[2] + (int)(q / ((long long)l0 * l1));
                if (!inS(x, y, z)) continue;
#pragma unroll
                for (int j = 1; j < L::Q; ++j) {  // link (y + c_j, j): source y solid, target fluid
                    const int tx = wrap_idx(x + L::cx(j), a.g.n[0]);
                    const int ty = wrap_idx(y + L::cy(j), a.g.n[1]);
                    const int tz = wrap_idx(z + L::cz(j), a.g.n[2]);
                    if (!inS(tx, ty, tz)) m |= 1u << j;
                }
            }
            if (m) atomicOr(&s_links, m);
            __syncthreads();
            if (tid == 0) P.dirlinks = s_links;
        }
    }
    __syncthreads();

    // 4b. the boundary-link list the next fix-up runs over: fluid nodes x of
    //     the near box with mask bit j set where x - c_j is solid.  Rebuilt
    //     only when the intervals changed: here, one near-box row per thread
    //     from the rows' intervals (the stream schedule and the persistent
    //     tick kernel), or flagged for k_links_count and k_links_write (a grid
    //     over the near box).
    if (s_changed && !a.inline_links && tid == 0) P.relink = 1;
    if (s_changed && a.inline_links) {
        const int ex = near_extent(P, a.g, 0, D), ey = near_extent(P, a.g, 1, D), ez = near_extent(P, a.g, 2, D);
        const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
        const int nrows = (P.slo[0] > P.shi[0] || P.slo[1] > P.shi[1] || P.slo[2] > P.shi[2]) ? 0 : ey * ez;
        // interval of row (y, z) of the solid box, or empty
        auto row_ivl = [&](int y, int z) -> int2 {
            if (y < P.slo[1] || y > P.shi[1] || z < P.slo[2] || z > P.shi[2]) return make_int2(1, 0);
            const int r = (y - P.slo[1]) + (P.shi[1] - P.slo[1] + 1) * (z - P.slo[2]);
            return ivl_smem ? s_ivl[r] : a.ivl[P.ivl_off + r];
        };
        // the links of near-box row rr, counted or written from `out`
        auto scan_row = [&](int rr, int2* out) -> int {
            const int y = wrap_idx(P.slo[1] - 1 + rr % ey, ny);
            const int z = D == 3 ? wrap_idx(P.slo[2] - 1 + rr / ey, nz) : 0;
            int2 nb[9];
            int nn = 0;
            for (int dz = (D == 3 ? -1 : 0); dz <= (D == 3 ? 1 : 0); ++dz)
                for (int dy = -1; dy <= 1; ++dy) {
                    const int2 iv = row_ivl(wrap_idx(y + dy, ny), D == 3 ? wrap_idx(z + dz, nz) : 0);
                    if (iv.x <= iv.y) nb[nn++] = iv;
                }
            if (nn == 0) return 0;
            int cnt = 0;
#pragma unroll 1
            for (int rx = 0; rx < ex; ++rx) {
                const int x = wrap_idx(P.slo[0] - 1 + rx, nx);
                const int xm = wrap_idx(x - 1, nx), xp = wrap_idx(x + 1, nx);
                bool cand = false;
                for (int k = 0; k < nn; ++k)
                    cand = cand || (x >= nb[k].x && x <= nb[k].y) || (xm >= nb[k].x && xm <= nb[k].y) ||
                           (xp >= nb[k].x && xp <= nb[k].y);
                if (!cand || inS(x, y, z)) continue;
                unsigned mask = 0;
                for (int j = 1; j < L::Q; ++j) {
                    const int i = L::opp(j);  // source x - c_j = x + c_i
                    if (inS(wrap_idx(x + L::cx(i), nx), wrap_idx(y + L::cy(i), ny), wrap_idx(z + L::cz(i), nz)))
                        mask |= 1u << j;
                }
                if (!mask) continue;
                if (out) out[cnt] = make_int2(x + nx * (y + ny * z), (int)mask);
                ++cnt;
            }
            return cnt;
        };
        // fast form (near_row_links) where the near box is narrower than the x
        // axis by two; the node-by-node scan above otherwise
        const int s0 = P.slo[0] - 1;
        const bool fast = ex + 2 <= nx;
        const int2* ivl_rows = ivl_smem ? s_ivl : a.ivl + P.ivl_off;
        auto row_links = [&](int rr, int2* out) -> int {
            return near_row_links<L>(P, ivl_rows, a.g, ex, ey, s0, rr, out);
        };
        int base = 0;
        if (tid == 0) s_lkn = LK;
        __syncthreads();
        for (int r0 = 0; r0 < nrows; r0 += blockDim.x) {
            const int rr = r0 + tid;
            const int c = rr < nrows ? (fast ? row_links(rr, nullptr) : scan_row(rr, nullptr)) : 0;
            // exclusive prefix of the counts over the CTA
            const int lane = tid & 31, warp = tid >> 5;
            int v = c;
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += t;
            }
            if (lane == 31) s_warp[warp] = v;
            __syncthreads();
            if (tid == 0) {
                int run = 0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
                    const int t = s_warp[w];
                    s_warp[w] = run;
                    run += t;
                }
                s_warp[kMaxPartWarps] = run;
            }
            __syncthreads();
            const int off = base + s_warp[warp] + v - c;
            if (c > 0) {
                if (off + c <= P.link_cap) {
                    // rows that fit go to shared memory; they form a prefix of the list
                    int2* out = off + c <= LK ? s_lk + off : a.links + P.link_off + off;
                    if (off + c > LK) atomicMin(&s_lkn, off);
                    if (fast) row_links(rr, out);
                    else scan_row(rr, out);
                }
                else atomicOr(a.err, kErrLinkOverflow);
            }
            base += s_warp[kMaxPartWarps];
            __syncthreads();
        }
        if (tid == 0) {
            P.nlinks = base < P.link_cap ? base : P.link_cap;
            s_lkn = min(s_lkn, (int)P.nlinks);
        }
    }
    __syncthreads();

    // 5. candidate bits of the tiles around the particle
    bool same = true;
    for (int k = 0; k < 6; ++k) same = same && s_oldbox[k] == s_newbox[k];
    if (!same) {
        if (s_oldbox[3] * s_oldbox[4] * s_oldbox[5] > 0) tile_bits_update(a, s_oldbox, s_oldbox + 3, p, false);
        __syncthreads();
        if (s_newbox[3] * s_newbox[4] * s_newbox[5] > 0) tile_bits_update(a, s_newbox, s_newbox + 3, p, true);
    }
    __syncthreads();
    // the staged intervals and link entries, coalesced
    if (s_changed && s_rows <= kIvlSmem)
        for (int r = tid; r < s_rows; r += blockDim.x) a.ivl[P.ivl_off + r] = s_ivl[r];
    if (s_changed && a.inline_links)
        for (int e = tid; e < s_lkn; e += blockDim.x) a.links[P.link_off + e] = s_lk[e];
    {
        const unsigned long long* ssrc = reinterpret_cast<const unsigned long long*>(&sP);
        unsigned long long* gdst = reinterpret_cast<unsigned long long*>(a.parts + p);
        for (int k = tid; k < (int)(sizeof(ParticleDev) / 8); k += blockDim.x) gdst[k] = ssrc[k];
        if (tid == 0) publish_box(a, p, P);
    }
}

template <class L>
__global__ void __launch_bounds__(kPartBlock) k_particles(const ParticleArgs a) {
    particles_body<L>(a, a.mode != 0 ? a.setup_pid : (int)blockIdx.x);
}

// ---------------------------------------------------------------------------
// Link-list rebuild for particles flagged by the particle update, in two
// passes over the near box (one thread per node, blocks_per_particle CTAs per
// particle): k_links_count stores each CTA's number of link nodes, then
// k_links_write places each CTA's link nodes, in node order, after those of
// the CTAs before it.  The list comes out in near-box order whatever the
// scheduling, so the fix-up's chunks and FP64 partial sums are reproducible.
// ---------------------------------------------------------------------------
constexpr int kLinkBlock = 256;

// the mask of near-box node v of particle P (0: not a link node)
template <class L>
__device__ __forceinline__ unsigned near_node_mask(const ParticleArgs& a, const ParticleDev& P, int v, int* cell) {
    constexpr int Q = L::Q, D = L::D;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int e0 = near_extent(P, a.g, 0, D), e1 = near_extent(P, a.g, 1, D);
    const int x = wrap_idx(P.slo[0] - 1 + v % e0, nx);
    const int y = wrap_idx(P.slo[1] - 1 + (v / e0) % e1, ny);
    const int z = D == 3 ? wrap_idx(P.slo[2] - 1 + v / (e0 * e1), nz) : 0;
    *cell = x + nx * (y + ny * z);
    if (solid_at(P, a.ivl, x, y, z)) return 0u;
    unsigned mask = 0;
#pragma unroll
    for (int j = 1; j < Q; ++j) {
        const int i = L::opp(j);  // source x - c_j = x + c_i
        if (solid_at(P, a.ivl, wrap_idx(x + L::cx(i), nx), wrap_idx(y + L::cy(i), ny), wrap_idx(z + L::cz(i), nz)))
            mask |= 1u << j;
    }
    return mask;
}

template <class L>
__global__ void __launch_bounds__(kLinkBlock) k_links_count(const ParticleArgs a, int bpp, int* counts) {
    __shared__ int s_w[kLinkBlock / 32];
    const int p = blockIdx.x / bpp, chunk = blockIdx.x % bpp;
    const ParticleDev& P = a.parts[p];
    if (!P.relink) return;
    const int v = chunk * kLinkBlock + threadIdx.x;
    int cell = 0;
    const bool link = v < near_volume(P, a.g, L::D) && near_node_mask<L>(a, P, v, &cell) != 0u;
    const unsigned bal = __ballot_sync(0xffffffffu, link);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        int c = 0;
        for (int w = 0; w < kLinkBlock / 32; ++w) c += s_w[w];
        counts[blockIdx.x] = c;
    }
}

template <class L>
__global__ void __launch_bounds__(kLinkBlock) k_links_write(const ParticleArgs a, int bpp, const int* counts) {
    __shared__ int s_w[kLinkBlock / 32];
    __shared__ int s_base;
    const int p = blockIdx.x / bpp, chunk = blockIdx.x % bpp;
    ParticleDev* G = a.parts + p;
    const ParticleDev& P = *G;
    if (!P.relink) return;
    if (threadIdx.x == 0) {
        int base = 0, total = 0;
        for (int c = 0; c < bpp; ++c) {
            if (c == chunk) base = total;
            total += counts[p * bpp + c];
        }
        s_base = base;
        if (chunk == 0) G->nlinks = total < P.link_cap ? total : P.link_cap;
        if (total > P.link_cap) atomicOr(a.err, kErrLinkOverflow);
    }
    const int v = chunk * kLinkBlock + threadIdx.x;
    int cell = 0;
    const unsigned mask = v < near_volume(P, a.g, L::D) ? near_node_mask<L>(a, P, v, &cell) : 0u;
    const bool link = mask != 0u;
    const unsigned bal = __ballot_sync(0xffffffffu, link);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_w[warp] = __popc(bal);
    __syncthreads();
    int off = s_base;
    for (int w = 0; w < warp; ++w) off += s_w[w];
    off += __popc(bal & ((1u << lane) - 1u));
    if (link && off < P.link_cap) a.links[P.link_off + off] = make_int2(cell, (int)mask);
}

}  // namespace lbm
