// Device kernels of one lattice-Boltzmann tick (B200, sm_100a).
//
// One tick of the reference (tick!, src/gpu/fluids.jl:132-226) is
//     collide -> pull-stream -> bounce-back / moving walls / Ladd -> hydro -> particles.
// Here it is fused into a push ("collide then stream") pass over the stored
// pre-collision populations f^n, which are exactly the reference's
// model.distributions between ticks:
//   * every node loads its own Q populations (aligned, coalesced), forms
//     rho^n, u^n (= hydroVariablesUpdate! of the previous tick), collides and
//     pushes f*_i to x + c_i;
//   * halfway bounce-back, moving walls and the Ladd momentum term are
//     evaluated by the fluid node itself, which owns every quantity the
//     reference uses there (f*_i(x), rho^n(x), the solid node x + c_i);
//   * tiles whose halo touches a wall or a particle are processed by a
//     separate "boundary" kernel (k_boundary) so that the bulk kernel
//     (k_bulk) carries no boundary code at all;
//   * particle force/torque partials are reduced per tile in FP64 in a fixed
//     order and finished by k_particles (one CTA per particle), which also
//     performs the Newton-Euler update and re-voxelisation
//     (moveParticles!, src/gpu/particles.jl:7-92).
#pragma once
#include <cstdint>
#include "lattice.cuh"
#include "storage.cuh"

namespace lbm {

constexpr int kBlock = 256;       // threads per CTA (tile size)
constexpr int kMaxCand = 16;      // particles whose halo may meet one tile
constexpr int kPartialStride = 8; // doubles per partial-sum slot (F[3], T[3], pad)

// device error word bits
constexpr int kErrTooManyCandidates = 1;
constexpr int kErrPartialOverflow = 2;

struct GridDesc {
    int n[3];        // nodes per axis
    int t[3];        // tile (CTA) extent per axis
    int nt[3];       // tiles per axis
    int pad;
    long long N;     // cells
    long long ntiles;
};

// FP64 particle state on the device.  The first block is the LBMparticle
// state of the reference; the second block is what the stream kernels need.
struct ParticleDev {
    double R[3], v[3], w[3], e[3];          // position, velocity, angular velocity, swimming direction
    double radius, r2, B1, B2, inv_mass, inv_inertia;
    double lastF[3], lastT[3];              // forceInput / torqueInput of the last tick
    int kind, coupleF, coupleT, valid;
    // slip-velocity snapshot: state seen by the last getNodeVelocity call
    double sR[3], sV[3], sW[3], sE[3];
    // mask geometry (solidRegion of the last re-voxelisation, centred at mR)
    double mR[3];
    int slo[3], shi[3];      // index box that contains every solid node (slo > shi: empty)
    int tlo[3], tn[3];       // tile box: first tile and tile count per axis (periodic)
    unsigned dirlinks;       // bit i set: the particle has >= 1 boundary link in direction i
    int part_off, part_cap;  // partial-sum slots owned by the particle
    int pad;
};

struct StepArgs {
    const void* src;
    void* dst;
    GridDesc g;
    const double* coord[3];
    const unsigned long long* tilebits;   // [ntiles][words]: particles whose halo meets the tile
    const unsigned char* tileflags;       // [ntiles]: bit0 = wall in the tile's halo
    const int* walltiles;                 // list of wall tiles
    int nwalltiles;
    int words;
    const unsigned char* wall;            // [N] wall mask or null
    const double* uw;                     // [d][N] moving-wall velocity or null
    const double* ffield;                 // [d][N] force field or null
    const ParticleDev* parts;
    int nparts;
    int maxtl;                            // max tile-box size over particles
    double* partial;
    int* err;
    double rho0;                          // shift density of the stored populations
    double scale, inv_scale;              // storage scale (F16/BF16)
    double omega, omega_p, omega_m;       // dt/tau (BGK), dt/tau+, dt/tau- (TRT)
    double guo_k, guo_kp, guo_km;         // dt(1-dt/2tau), dt(1-dt/2tau+), dt(1-dt/2tau-)
    double F[3];                          // uniform force density
    double half_dt;                       // dt/2 (momentum correction of the Guo scheme)
    double coeff;                         // dx^d/dt (momentum-exchange prefactor)
    int force_mode;                       // 0 none, 1 uniform, 2 field
    int incompressible;
    double rho_inc;                       // rho0 of the incompressible equilibrium
};

__device__ __forceinline__ int wrap_idx(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// getSphere test (src/gpu/kernels.jl:335-353): ((X1-R1)^2 + (X2-R2)^2 [+ (X3-R3)^2]) < r^2,
// evaluated left to right in FP64 without contraction so that masks are
// bit-identical to the reference's.
template <int D>
__device__ __forceinline__ bool sphere_test(double X0, double X1, double X2, const double* c, double r2) {
    double a = __dsub_rn(X0, c[0]);
    double b = __dsub_rn(X1, c[1]);
    double s = __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b));
    if (D == 3) {
        double q = __dsub_rn(X2, c[2]);
        s = __dadd_rn(s, __dmul_rn(q, q));
    }
    return s < r2;
}

// getNodeVelocity at one solid node (src/gpu/aux.jl:229-263, kernels.jl:376-415)
template <int D>
__device__ __forceinline__ void slip_velocity(const double* sR, const double* sV, const double* sW, const double* sE,
                                              double B1, double B2, int kind, double X0, double X1, double X2,
                                              double* out) {
    double xr[3] = {X0 - sR[0], X1 - sR[1], D == 3 ? X2 - sR[2] : 0.0};
    double bulk[3];
    if (D == 2) {
        bulk[0] = sV[0] - sW[0] * xr[1];
        bulk[1] = sV[1] + sW[0] * xr[0];
        bulk[2] = 0.0;
    } else {
        bulk[0] = sV[0] + sW[1] * xr[2] - sW[2] * xr[1];
        bulk[1] = sV[1] - sW[0] * xr[2] + sW[2] * xr[0];
        bulk[2] = sV[2] + sW[0] * xr[1] - sW[1] * xr[0];
    }
    if (kind == 0) {  // bead
        out[0] = bulk[0];
        out[1] = bulk[1];
        out[2] = bulk[2];
        return;
    }
    double nrm = sqrt(xr[0] * xr[0] + xr[1] * xr[1] + xr[2] * xr[2]);
    if (nrm == 0.0) nrm = 1.0;
    double inv = 1.0 / nrm;
    double ur[3] = {inv * xr[0], inv * xr[1], inv * xr[2]};
    double edr = ur[0] * sE[0] + ur[1] * sE[1] + (D == 3 ? ur[2] * sE[2] : 0.0);
    double first = B1 + B2 * edr;
    for (int k = 0; k < 3; ++k) out[k] = first * (edr * ur[k] - (k < D ? sE[k] : 0.0)) + bulk[k];
}

// ---------------------------------------------------------------------------
// Collision of one node (collisionStep + guoForcingTerm, src/gpu/fluids.jl:58-127)
// on the shifted, weight-normalised populations g_i = f_i/w_i - rho0.
// ---------------------------------------------------------------------------
template <class L, int ST, bool TRT>
struct NodeState {
    using R = typename Store<ST>::R;
    R g[L::Q];   // post-collision populations after collide()
    R rho;       // rho^n: the density the reference holds in model.massDensity
};

template <class L, int ST, bool TRT>
__device__ __forceinline__ void load_collide(const StepArgs& a, int cell, bool valid, NodeState<L, ST, TRT>& s) {
    using SS = Store<ST>;
    using T = typename SS::T;
    using R = typename SS::R;
    constexpr int Q = L::Q;
    const T* __restrict__ src = static_cast<const T*>(a.src);
    const long long N = a.g.N;
    const R inv_scale = R(a.inv_scale);
#pragma unroll
    for (int i = 0; i < Q; ++i) s.g[i] = valid ? SS::dec(__ldcs(src + i * N + cell), inv_scale) : R(0);

    // moments: rho = rho0 + sum w g ; j = sum w g c (+ dt/2 F)
    R drho = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const R wg = R(L::w(i)) * s.g[i];
        drho += wg;
        if (L::cx(i) == 1) jx += wg; else if (L::cx(i) == -1) jx -= wg;
        if (L::cy(i) == 1) jy += wg; else if (L::cy(i) == -1) jy -= wg;
        if (L::cz(i) == 1) jz += wg; else if (L::cz(i) == -1) jz -= wg;
    }
    R Fx = 0, Fy = 0, Fz = 0;
    if (a.force_mode == 1) {
        Fx = R(a.F[0]);
        Fy = R(a.F[1]);
        Fz = R(a.F[2]);
    } else if (a.force_mode == 2 && valid) {
        Fx = R(a.ffield[cell]);
        Fy = R(a.ffield[N + cell]);
        if (L::D == 3) Fz = R(a.ffield[2 * N + cell]);
    }
    const R rho = R(a.rho0) + drho;
    s.rho = rho;
    const R hdt = R(a.half_dt);
    jx += hdt * Fx;
    jy += hdt * Fy;
    jz += hdt * Fz;
    R ux = 0, uy = 0, uz = 0;
    if (rho != R(0)) {  // findFluidVelocity: u = 0 where rho == 0
        ux = jx / rho;
        uy = jy / rho;
        uz = jz / rho;
    }
    const R usq = ux * ux + uy * uy + uz * uz;
    const R uF = ux * Fx + uy * Fy + uz * Fz;
    const bool inc = a.incompressible != 0;
    const R rq = inc ? R(a.rho_inc) : rho;   // density multiplying the velocity terms of f_eq
    if (!TRT) {
        const R om = R(a.omega);
        const R gk = R(a.guo_k);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const R cu = R(L::cx(i)) * ux + R(L::cy(i)) * uy + R(L::cz(i)) * uz;
            const R geq = drho + rq * (R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq);
            R gi = s.g[i] - om * (s.g[i] - geq);
            if (a.force_mode != 0) {
                const R cF = R(L::cx(i)) * Fx + R(L::cy(i)) * Fy + R(L::cz(i)) * Fz;
                gi += gk * (R(3) * (cF - uF) + R(9) * cu * cF);
            }
            s.g[i] = gi;
        }
    } else {
        const R omp = R(a.omega_p), omm = R(a.omega_m);
        const R gkp = R(a.guo_kp), gkm = R(a.guo_km);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int ib = L::opp(i);
            if (ib < i) continue;  // handled together with its partner
            const R cu = R(L::cx(i)) * ux + R(L::cy(i)) * uy + R(L::cz(i)) * uz;
            const R ep = drho + rq * (R(4.5) * cu * cu - R(1.5) * usq);  // symmetric part of g_eq
            const R em = rq * (R(3) * cu);                               // antisymmetric part
            const R gp = R(0.5) * (s.g[i] + s.g[ib]);
            const R gm = R(0.5) * (s.g[i] - s.g[ib]);
            const R dp = omp * (gp - ep);
            const R dm = omm * (gm - em);
            R Gi = 0, Gb = 0;
            if (a.force_mode != 0) {
                const R cF = R(L::cx(i)) * Fx + R(L::cy(i)) * Fy + R(L::cz(i)) * Fz;
                const R plus = gkp * (R(-3) * uF + R(9) * cu * cF);  // even in c
                const R minus = gkm * (R(3) * cF);                    // odd in c
                Gi = plus + minus;
                Gb = plus - minus;
            }
            if (ib == i) {
                s.g[i] = s.g[i] - dp + Gi;
            } else {
                const R gi = s.g[i] - dp - dm + Gi;
                const R gb = s.g[ib] - dp + dm + Gb;
                s.g[i] = gi;
                s.g[ib] = gb;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Bulk kernel: tiles with no wall and no particle in their halo.
// ---------------------------------------------------------------------------
template <class L, int ST, bool TRT>
__global__ void __launch_bounds__(kBlock) k_bulk(const StepArgs a) {
    using SS = Store<ST>;
    using T = typename SS::T;
    using R = typename SS::R;
    constexpr int Q = L::Q;
    const long long tile = blockIdx.x;
    if (a.tileflags[tile]) return;
    for (int k = 0; k < a.words; ++k)
        if (a.tilebits[tile * a.words + k]) return;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int bx = (int)(tile % a.g.nt[0]);
    const int rr = (int)(tile / a.g.nt[0]);
    const int by = rr % a.g.nt[1], bz = rr / a.g.nt[1];
    const int x = bx * a.g.t[0] + threadIdx.x;
    const int y = by * a.g.t[1] + threadIdx.y;
    const int z = bz * a.g.t[2] + threadIdx.z;
    const bool valid = x < nx && y < ny && z < nz;
    const int cell = valid ? x + nx * (y + ny * z) : 0;
    NodeState<L, ST, TRT> s;
    load_collide<L, ST, TRT>(a, cell, valid, s);
    if (!valid) return;
    const int xs[3] = {x == 0 ? nx - 1 : x - 1, x, x == nx - 1 ? 0 : x + 1};
    const int ys[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
    const int zs[3] = {z == 0 ? nz - 1 : z - 1, z, z == nz - 1 ? 0 : z + 1};
    T* __restrict__ dst = static_cast<T*>(a.dst);
    const long long N = a.g.N;
    const R scale = R(a.scale);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int t = xs[L::cx(i) + 1] + nx * (ys[L::cy(i) + 1] + ny * zs[L::cz(i) + 1]);
        dst[i * N + t] = SS::enc(s.g[i], scale);
    }
}

// ---------------------------------------------------------------------------
// Boundary kernel: tiles whose halo meets a wall or a particle.
// ---------------------------------------------------------------------------
struct Cand {
    double mR[3];
    double r2;
    double sR[3], sV[3], sW[3], sE[3];
    double B1, B2;
    int lo[3], len[3];   // near box: wrapped first index and length per axis
    int kind, coupleF, coupleT, pid;
    int slot;            // partial-sum slot of this (particle, tile)
    int pad;
};

// maps a CTA of the boundary grid to a tile; returns -1 if the CTA has no work
__device__ __forceinline__ long long boundary_tile(const StepArgs& a) {
    const long long b = blockIdx.x;
    const long long np = (long long)a.nparts * a.maxtl;
    if (b < np) {
        const int p = (int)(b / a.maxtl);
        const int l = (int)(b % a.maxtl);
        const ParticleDev& P = a.parts[p];
        const int tn0 = P.tn[0], tn1 = P.tn[1], tn2 = P.tn[2];
        if (l >= tn0 * tn1 * tn2) return -1;
        const int dx = l % tn0, dy = (l / tn0) % tn1, dz = l / (tn0 * tn1);
        const int tx = (P.tlo[0] + dx) % a.g.nt[0];
        const int ty = (P.tlo[1] + dy) % a.g.nt[1];
        const int tz = (P.tlo[2] + dz) % a.g.nt[2];
        const long long tile = tx + (long long)a.g.nt[0] * (ty + (long long)a.g.nt[1] * tz);
        if (a.tileflags[tile]) return -1;  // wall tiles are processed from the wall list
        // owner: the lowest particle whose halo meets the tile
        for (int k = 0; k < a.words; ++k) {
            const unsigned long long wbits = a.tilebits[tile * a.words + k];
            if (wbits) return (k * 64 + __ffsll((long long)wbits) - 1) == p ? tile : -1;
        }
        return -1;
    }
    const long long wi = b - np;
    return wi < a.nwalltiles ? a.walltiles[wi] : -1;
}

template <class L>
__device__ __forceinline__ void reduce6(double* acc, double (*red)[6], double* out, bool write) {
    // deterministic: fixed butterfly inside each warp, then warps summed in order
#pragma unroll
    for (int k = 0; k < 6; ++k)
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int warp = tid >> 5, lane = tid & 31;
    if (lane == 0)
        for (int k = 0; k < 6; ++k) red[warp][k] = acc[k];
    __syncthreads();
    if (tid == 0 && write) {
        const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
        for (int k = 0; k < 6; ++k) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += red[w][k];
            out[k] = s;
        }
        out[6] = 0.0;
        out[7] = 0.0;
    }
    __syncthreads();
}

template <class L, int ST, bool TRT>
__global__ void __launch_bounds__(kBlock) k_boundary(const StepArgs a) {
    using SS = Store<ST>;
    using T = typename SS::T;
    using R = typename SS::R;
    constexpr int Q = L::Q;
    constexpr int D = L::D;
    __shared__ Cand s_c[kMaxCand];
    __shared__ int s_pid[kMaxCand];
    __shared__ int s_nc;
    __shared__ int s_first[Q];
    __shared__ double s_red[kBlock / 32][6];

    const long long tile = boundary_tile(a);
    if (tile < 0) return;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int bx = (int)(tile % a.g.nt[0]);
    const int rr = (int)(tile / a.g.nt[0]);
    const int by = rr % a.g.nt[1], bz = rr / a.g.nt[1];
    if (tid == 0) {
        int nc = 0;
        for (int k = 0; k < a.words; ++k) {
            unsigned long long b = a.tilebits[tile * a.words + k];
            while (b) {
                const int bit = __ffsll((long long)b) - 1;
                b &= b - 1;
                if (nc < kMaxCand) s_pid[nc] = k * 64 + bit;
                ++nc;
            }
        }
        if (nc > kMaxCand) {
            atomicOr(a.err, kErrTooManyCandidates);
            nc = kMaxCand;
        }
        s_nc = nc;
    }
    // break rule of the Ladd loop (fluids.jl:184): for streaming direction j
    // only particles before the first one without links in j contribute
    if (tid < Q) {
        int f = a.nparts;
        for (int p = 0; p < a.nparts; ++p)
            if (!((a.parts[p].dirlinks >> tid) & 1u)) {
                f = p;
                break;
            }
        s_first[tid] = f;
    }
    __syncthreads();
    if (tid < s_nc) {
        const int p = s_pid[tid];
        const ParticleDev& P = a.parts[p];
        Cand& c = s_c[tid];
        for (int k = 0; k < 3; ++k) {
            c.mR[k] = P.mR[k];
            c.sR[k] = P.sR[k];
            c.sV[k] = P.sV[k];
            c.sW[k] = P.sW[k];
            c.sE[k] = P.sE[k];
            const int n = a.g.n[k];
            const int len = P.shi[k] - P.slo[k] + 3;
            c.lo[k] = wrap_idx(P.slo[k] - 1, n);
            c.len[k] = len >= n ? n : len;
        }
        c.r2 = P.r2;
        c.B1 = P.B1;
        c.B2 = P.B2;
        c.kind = P.kind;
        c.coupleF = P.coupleF;
        c.coupleT = P.coupleT;
        c.pid = p;
        const int dx = (bx - P.tlo[0] + a.g.nt[0]) % a.g.nt[0];
        const int dy = (by - P.tlo[1] + a.g.nt[1]) % a.g.nt[1];
        const int dz = (bz - P.tlo[2] + a.g.nt[2]) % a.g.nt[2];
        const int l = dx + P.tn[0] * (dy + P.tn[1] * dz);
        if (l >= P.part_cap) {
            atomicOr(a.err, kErrPartialOverflow);
            c.slot = -1;
        } else {
            c.slot = P.part_off + l;
        }
    }
    __syncthreads();

    const int x = bx * a.g.t[0] + threadIdx.x;
    const int y = by * a.g.t[1] + threadIdx.y;
    const int z = bz * a.g.t[2] + threadIdx.z;
    const bool valid = x < nx && y < ny && z < nz;
    const int cell = valid ? x + nx * (y + ny * z) : 0;
    NodeState<L, ST, TRT> s;
    load_collide<L, ST, TRT>(a, cell, valid, s);

    const int nc = s_nc;
    unsigned near = 0;
    if (valid)
        for (int k = 0; k < nc; ++k) {
            const Cand& c = s_c[k];
            const bool in = ((x - c.lo[0] + nx) % nx) < c.len[0] && ((y - c.lo[1] + ny) % ny) < c.len[1] &&
                            ((z - c.lo[2] + nz) % nz) < c.len[2];
            if (in) near |= 1u << k;
        }
    const bool walls = a.wall != nullptr;
    const bool special = valid && (near != 0 || walls);
    const int xs[3] = {x == 0 ? nx - 1 : x - 1, x, x == nx - 1 ? 0 : x + 1};
    const int ys[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
    const int zs[3] = {z == 0 ? nz - 1 : z - 1, z, z == nz - 1 ? 0 : z + 1};
    double Xo[3] = {0, 0, 0};
    unsigned ob = 0;
    bool oW = false;
    if (special) {
        Xo[0] = a.coord[0][x];
        Xo[1] = a.coord[1][y];
        Xo[2] = D == 3 ? a.coord[2][z] : 0.0;
        for (unsigned m = near; m; m &= m - 1) {
            const int k = __ffs(m) - 1;
            if (sphere_test<D>(Xo[0], Xo[1], Xo[2], s_c[k].mR, s_c[k].r2)) ob |= 1u << k;
        }
        if (walls) oW = a.wall[cell] != 0;
    }
    const double rhoL = (double)s.rho;  // rho^n(x), the density of model.massDensity
    T* __restrict__ dst = static_cast<T*>(a.dst);
    const long long N = a.g.N;
    const R scale = R(a.scale);
    unsigned linkb[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int j = L::opp(i);
        const int tx = xs[L::cx(i) + 1], ty = ys[L::cy(i) + 1], tz = zs[L::cz(i) + 1];
        const int t = tx + nx * (ty + ny * tz);
        bool push = valid;
        bool own = false;
        R vown = 0;
        unsigned lb = 0;
        if (special) {
            unsigned tb = 0;
            if (near) {
                const double X0 = a.coord[0][tx], X1 = a.coord[1][ty], X2 = D == 3 ? a.coord[2][tz] : 0.0;
                for (unsigned m = near; m; m &= m - 1) {
                    const int k = __ffs(m) - 1;
                    if (sphere_test<D>(X0, X1, X2, s_c[k].mR, s_c[k].r2)) tb |= 1u << k;
                }
            }
            const bool tW = walls && a.wall[t] != 0;
            lb = tb & ~ob;  // particles with x fluid and x + c_i solid: link (x, j)
            push = !tW && !oW && !(ob & ~tb);
            const bool region = (tW && !oW) || lb != 0;
            if (oW) {
                own = true;  // wall nodes hold f = 0 (fluids.jl:154)
                vown = R(-a.rho0);
            } else if (region) {
                own = true;
                double v = (double)s.g[i];  // halfway bounce-back: f_j(x) = f*_i(x)
                if (a.uw) {                  // moving walls (fluids.jl:168-174)
                    double dot = 0.0;
                    dot -= L::cx(i) * a.uw[t];
                    dot -= L::cy(i) * a.uw[N + t];
                    if (D == 3) dot -= L::cz(i) * a.uw[2 * N + t];
                    v += 6.0 * rhoL * dot;
                }
                if (lb) {  // Ladd momentum term (fluids.jl:176-189)
                    const double X0 = a.coord[0][tx], X1 = a.coord[1][ty], X2 = D == 3 ? a.coord[2][tz] : 0.0;
                    for (unsigned m = lb; m; m &= m - 1) {
                        const int k = __ffs(m) - 1;
                        const Cand& c = s_c[k];
                        if (c.pid >= s_first[j]) continue;
                        double up[3];
                        slip_velocity<D>(c.sR, c.sV, c.sW, c.sE, c.B1, c.B2, c.kind, X0, X1, X2, up);
                        const double dot = -(L::cx(i) * up[0] + L::cy(i) * up[1] + L::cz(i) * up[2]);
                        v += 6.0 * rhoL * dot;
                    }
                }
                vown = (R)v;
            }
        }
        linkb[i] = (special && !oW) ? lb : 0u;
        if (push) dst[i * N + t] = SS::enc(s.g[i], scale);
        if (own) dst[j * N + cell] = SS::enc(vown, scale);
    }

    // momentum exchange (fluids.jl:191-205), one candidate at a time
    const double rho0 = a.rho0;
    for (int k = 0; k < nc; ++k) {
        const Cand& c = s_c[k];
        double acc[6] = {0, 0, 0, 0, 0, 0};
        if (special && ((near >> k) & 1u) && (c.coupleF || c.coupleT)) {
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const int j = L::opp(i);
                if (!((linkb[i] >> k) & 1u) || c.pid >= s_first[j]) continue;
                const int tx = xs[L::cx(i) + 1], ty = ys[L::cy(i) + 1], tz = zs[L::cz(i) + 1];
                const int t = tx + nx * (ty + ny * tz);
                // f_j(x) as it stood when particle k was processed: bounce-back,
                // moving walls and the Ladd terms of particles up to k
                double v = (double)s.g[i];
                if (a.uw) {
                    double dot = 0.0;
                    dot -= L::cx(i) * a.uw[t];
                    dot -= L::cy(i) * a.uw[N + t];
                    if (D == 3) dot -= L::cz(i) * a.uw[2 * N + t];
                    v += 6.0 * rhoL * dot;
                }
                const double X0 = a.coord[0][tx], X1 = a.coord[1][ty], X2 = D == 3 ? a.coord[2][tz] : 0.0;
                for (unsigned m = linkb[i] & ((2u << k) - 1u); m; m &= m - 1) {
                    const int kk = __ffs(m) - 1;
                    const Cand& ck = s_c[kk];
                    if (ck.pid >= s_first[j]) continue;
                    double up[3];
                    slip_velocity<D>(ck.sR, ck.sV, ck.sW, ck.sE, ck.B1, ck.B2, ck.kind, X0, X1, X2, up);
                    v += 6.0 * rhoL * (-(L::cx(i) * up[0] + L::cy(i) * up[1] + L::cz(i) * up[2]));
                }
                // f*_i(x) + f_j(x) in f units; F -= coeff*s*c_j = coeff*s*c_i
                const double sterm = L::w(i) * (2.0 * rho0 + (double)s.g[i] + v);
                const double cs = a.coeff * sterm;
                if (c.coupleF) {
                    acc[0] += cs * L::cx(i);
                    acc[1] += cs * L::cy(i);
                    acc[2] += cs * L::cz(i);
                }
                if (c.coupleT) {
                    // T -= coeff*cross(s*(x-R), c_j) = coeff*cross(s*(x-R), c_i)
                    const double r0 = Xo[0] - c.mR[0], r1 = Xo[1] - c.mR[1], r2 = D == 3 ? Xo[2] - c.mR[2] : 0.0;
                    if (D == 2) {
                        acc[3] += cs * (r0 * L::cy(i) - r1 * L::cx(i));
                    } else {
                        acc[3] += cs * (r1 * L::cz(i) - r2 * L::cy(i));
                        acc[4] += cs * (-r0 * L::cz(i) + r2 * L::cx(i));
                        acc[5] += cs * (r0 * L::cy(i) - r1 * L::cx(i));
                    }
                }
            }
        }
        double* out = c.slot >= 0 ? a.partial + (long long)c.slot * kPartialStride : nullptr;
        reduce6<L>(acc, s_red, out, out != nullptr);
    }
}

}  // namespace lbm
