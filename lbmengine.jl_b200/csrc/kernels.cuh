// Device kernels of one lattice-Boltzmann tick (B200, sm_100a).
//
// One tick of the reference (tick!, src/gpu/fluids.jl:132-226) is
//     collide -> pull-stream -> bounce-back / moving walls / Ladd -> hydro -> particles.
// Here it runs as three kernels over the stored pre-collision populations
// f^n (exactly the reference's model.distributions between ticks):
//   1. k_bulk_v4 / k_bulk: every node loads its own Q populations (aligned,
//      vectorised), forms rho^n and u^n (= hydroVariablesUpdate! of the
//      previous tick), collides and pushes f*_i to x + c_i.  No wall or
//      particle logic: the whole lattice streams at memory speed.
//   2. k_fixup: only the fluid nodes that own a boundary link are revisited.
//      A node x re-collides from the (unchanged) source populations and
//      overwrites its link slots (x, j), x - c_j solid, with halfway
//      bounce-back f*_opp(j)(x) + moving-wall and Ladd terms; it accumulates
//      the momentum exchange per particle (FP64, fixed-order reduction).
//      Wall nodes are reset to f = 0 (fluids.jl:154).
//   3. k_particles (particles.cuh): force/torque reduction, Newton-Euler with
//      Rodrigues rotation, re-voxelisation and link-list rebuild
//      (moveParticles!, src/gpu/particles.jl:7-92).
// Nodes inside a particle stream like fluid, as in the reference (its
// particle interiors are not reset).  The three run either as separate
// kernels in stream order or as the items of one persistent kernel per tick
// (k_tick, tick.cuh), which overlaps the boundary work with the bulk pass.
#pragma once
#include <cstdint>
#include "lattice.cuh"
#include "storage.cuh"

namespace lbm {

constexpr int kBlock = 256;        // threads per CTA of the scalar kernels
constexpr int kFixBlock = 64;      // link entries per fix-up CTA
constexpr int kPartialStride = 8;  // doubles per partial-sum slot (F[3], T[3], pad)
constexpr int kLinkOcParams = 8;   // particles whose (link_off, link_cap) the fix-up gets as parameters

// device error word bits
constexpr int kErrLinkOverflow = 1;
constexpr int kErrIntervalOverflow = 2;
constexpr int kErrSpinTimeout = 4;  // a bounded wait gave up (tick kernel, TMA ring)
constexpr int kErrNumeric = 8;

// Density sentinel of the bulk pass: rho^n is not finite or below -1e-3.  Wall
// nodes hold zero density (their populations are reset to f = 0, fluids.jl:154),
// so the test cannot stop at zero.
template <class R>
__device__ __forceinline__ bool bad_density(R rho) {
    return !(rho >= R(-1e-3) && rho <= R(1e30));
}

// raise kErrNumeric once per warp if any of its threads saw a bad density
// (every thread of the warp must call it)
__device__ __forceinline__ void report_density(bool bad, int* err) {
    const unsigned any = __ballot_sync(0xffffffffu, bad);
    if (any && (threadIdx.x & 31) == __ffs(any) - 1) atomicOr(err, kErrNumeric);
}

struct GridDesc {
    int n[3];        // nodes per axis
    int t[3];        // tile (CTA) extent per axis
    int nt[3];       // tiles per axis
    int pad;
    long long N;     // cells
    long long ntiles;
};

// FP64 particle state on the device.  The first block is the LBMparticle
// state of the reference; the rest is what the fix-up kernel needs.
struct ParticleDev {
    double R[3], v[3], w[3], e[3];          // position, velocity, angular velocity, swimming direction
    double radius, r2, B1, B2, inv_mass, inv_inertia;
    double lastF[3], lastT[3];              // forceInput / torqueInput of the last tick
    int kind, coupleF, coupleT, valid;
    // slip-velocity snapshot: state seen by the last getNodeVelocity call
    double sR[3], sV[3], sW[3], sE[3];
    // mR: position at the last move (torque arm of the momentum exchange);
    // vR: centre of the stored solid intervals, slack: min |d^2 - r^2| over the
    // nodes of the solid box at that centre (<= 0: intervals must be rebuilt)
    double mR[3];
    double vR[3], slack;
    int slo[3], shi[3];      // index box that contains every solid node (slo > shi: empty)
    int tlo[3], tn[3];       // tile box of the near box (periodic), for candidate bits
    unsigned dirlinks;       // bit j set: the particle has >= 1 boundary link in streaming direction j
    int ivl_off, ivl_cap;    // solid x-interval per (y, z) row of the solid box
    int link_off, link_cap;  // boundary-link entries (cell, direction mask)
    int nlinks;              // entries in use
    int part_off;            // partial-sum slots: one per chunk of kFixBlock entries
    int relink;              // the link list must be rebuilt (k_links, k_links_sort) before the next fix-up
    int rules;               // LBM_RULES_* of the model: which module's particle update and node velocity
    int recordF;             // accumulate the momentum-exchange force even when coupleF is off (the
                             // adjoint's force observable; the force is reported, never applied)
    int pad2;
    long long nrec;          // ticks recorded into the trajectory ring (ParticleArgs::trj)
};

// Collision constants in one precision (see collide()), derived on the host
// from the FP64 fields of StepArgs by fill_collide_consts(), so that no kernel
// converts them per node.
template <class R>
struct CollideK {
    R S, invS, rho0, hdt, rho_inc;
    R rest;      // rest population: a* = rest a + e0 (1 - omega+ or 1 - omega)
    R hsum;      // BGK pairs: a* = hsum a + E + O (1 - omega)
    R le, lo;    // TRT pairs: a* = le (a + b) + lo (a - b) + E + O ((1 - omega+)/2, (1 - omega-)/2)
    R omE;       // omega+ (TRT) or omega (BGK): weight of the equilibrium's even part
    R c45, c3;   // 4.5 omega+ and 3 omega- (TRT), 4.5 omega and 3 omega (BGK)
    R gK0, gkA, gkB;
    R F[3];
    R gA[27], gB[27];
};

struct StepArgs {
    const void* src;
    void* dst;
    GridDesc g;
    const double* coord[3];
    const unsigned long long* tilebits;   // [ntiles][words]: particles whose near box meets the tile
    int words;
    int nparts;
    const unsigned char* wall;            // [N] wall mask or null
    const double* uw;                     // [d][N] moving-wall velocity or null
    const double* ffield;                 // [d][N] force field or null
    const ParticleDev* parts;
    const int2* ivl;                      // solid intervals of all particles
    const int2* links;                    // (cell, mask) link entries of all particles
    const int2* wlinks;                   // (cell, mask) wall-link entries (static)
    const int* wnodes;                    // wall nodes (static)
    int nwlinks, nwnodes;
    int maxchunks;                        // fix-up CTAs reserved per particle
    int nlinkoc;                          // particles [0, nlinkoc) have linkoc filled (0: read the records)
    int linkoc[kLinkOcParams][2];         // (link_off, link_cap) of the first particles (static)
    int vrows;                            // x-rows per tile of the vector bulk pass
    long long vtiles;                     // tiles of the vector bulk pass
    int vnt1;                             // vector tiles per z-slice
    int pad;
    const int* nbox;                      // [nparts][6] solid boxes (lo, hi) the fix-up of this tick uses
    const unsigned char* vnear;           // [vtiles] tiles next to wall links (static) or null
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
    // Guo term per direction for a uniform force (see collide()): A_i, B_i, and
    // the coefficients used when the force is a per-node field
    double gA[27], gB[27];
    double gK0, gkA, gkB;
    int trt;                              // collision model of the constants below (0 BGK, 1 TRT)
    int stochastic;                       // 2-byte storage: 1 stochastic rounding of the stores, 0 nearest
    int reverse;                          // the vector bulk pass walks its tiles last to first (see k_bulk_v4)
    CollideK<float> kf;                   // the constants in FP32 and FP64 (fill_collide_consts)
    CollideK<double> kd;
    // per-direction population planes of src / dst (vector bulk kernel)
    const void* srcq[27];
    void* dstq[27];
};

template <class R>
inline void fill_collide_k(const StepArgs& a, CollideK<R>& k) {
    k.S = R(a.scale);
    k.invS = R(a.inv_scale);
    k.rho0 = R(a.rho0);
    k.hdt = R(a.half_dt);
    k.rho_inc = R(a.rho_inc);
    const double omE = a.trt ? a.omega_p : a.omega;
    const double omO = a.trt ? a.omega_m : a.omega;
    k.rest = R(1.0 - omE);
    k.hsum = R(1.0 - a.omega);
    k.le = R(0.5 * (1.0 - omE));
    k.lo = R(0.5 * (1.0 - omO));
    k.omE = R(omE);
    k.c45 = R(4.5 * omE);
    k.c3 = R(3.0 * omO);
    k.gK0 = R(a.gK0);
    k.gkA = R(a.gkA);
    k.gkB = R(a.gkB);
    for (int i = 0; i < 3; ++i) k.F[i] = R(a.F[i]);
    for (int i = 0; i < 27; ++i) {
        k.gA[i] = R(a.gA[i]);
        k.gB[i] = R(a.gB[i]);
    }
}

// derive kf / kd from the FP64 fields (after they are set)
inline void fill_collide_consts(StepArgs& a) {
    fill_collide_k(a, a.kf);
    fill_collide_k(a, a.kd);
}

template <class R>
__device__ __forceinline__ const CollideK<R>& collide_k(const StepArgs& a);
template <>
__device__ __forceinline__ const CollideK<float>& collide_k<float>(const StepArgs& a) { return a.kf; }
template <>
__device__ __forceinline__ const CollideK<double>& collide_k<double>(const StepArgs& a) { return a.kd; }

__device__ __forceinline__ float recip(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double recip(double x) { return 1.0 / x; }

__host__ __device__ __forceinline__ int wrap_idx(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Programmatic dependent launch.  grid_dep_trigger(): once every CTA of this
// grid has issued it (or exited), a kernel that depends on this one through a
// programmatic edge may start.  grid_dep_wait(): blocks until the grids this
// kernel depends on through such an edge have completed and their writes are
// visible.  Both are no-ops for kernels launched without that dependency.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// getSphere test (src/gpu/kernels.jl:335-353): ((X1-R1)^2 + (X2-R2)^2 [+ (X3-R3)^2]) < r^2,
// evaluated left to right in FP64 without contraction so that masks are
// bit-identical to the reference's.  For a fixed (y, z) row the test is
// monotone in |X1 - R1| (every rounding step is monotone), so the solid nodes
// of a row form one contiguous x-interval.
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

// the squared distance of sphere_test, same operations and rounding
template <int D>
__device__ __forceinline__ double sphere_d2(double X0, double X1, double X2, const double* c) {
    double a = __dsub_rn(X0, c[0]);
    double b = __dsub_rn(X1, c[1]);
    double s = __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b));
    if (D == 3) {
        double q = __dsub_rn(X2, c[2]);
        s = __dadd_rn(s, __dmul_rn(q, q));
    }
    return s;
}

// the near box of a particle: its solid box grown by one node (periodic, at
// most the whole axis).  Every boundary-link node lies in it.
__host__ __device__ __forceinline__ int near_extent(const ParticleDev& P, const GridDesc& g, int k, int D) {
    if (k >= D) return 1;
    const int l = P.shi[k] - P.slo[k] + 3;
    return l > g.n[k] ? g.n[k] : l;
}
__host__ __device__ __forceinline__ int near_volume(const ParticleDev& P, const GridDesc& g, int D) {
    for (int k = 0; k < D; ++k)
        if (P.slo[k] > P.shi[k]) return 0;
    return near_extent(P, g, 0, D) * near_extent(P, g, 1, D) * near_extent(P, g, 2, D);
}

// membership of node (x, y, z) in a particle's solid region, from its row intervals
__device__ __forceinline__ bool solid_at(const ParticleDev& P, const int2* ivl, int x, int y, int z) {
    if (y < P.slo[1] || y > P.shi[1] || z < P.slo[2] || z > P.shi[2]) return false;
    const int ly = P.shi[1] - P.slo[1] + 1;
    const int2 iv = ivl[P.ivl_off + (y - P.slo[1]) + ly * (z - P.slo[2])];
    return x >= iv.x && x <= iv.y;
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

// bulkVelocity of the reference's CPU module at one solid node
// (src/cpu/particles.jl:21-46): v + cross(w, x - R) with the CPU module's cross
// (src/cpu/aux.jl:19-28; in 2D the scalar w acts as (0, 0, w)), plus the slip
// (B1 + B2 e.r)((e.r) r - e) with r = (x - R)/|x - R|, the unit vector by a
// division.  Nodes farther than 2 dx from the surface get zero (:25); a solid
// node next to a fluid node lies within sqrt(d) dx of it, so no link does.
template <int D>
__device__ __forceinline__ void slip_velocity_cpu(const double* sR, const double* sV, const double* sW,
                                                  const double* sE, double B1, double B2, int kind, double radius,
                                                  double dx, double X0, double X1, double X2, double* out) {
    const double xr[3] = {X0 - sR[0], X1 - sR[1], D == 3 ? X2 - sR[2] : 0.0};
    const double mx = fmax(fabs(xr[0]), fmax(fabs(xr[1]), fabs(xr[2])));
    double nrm = 0.0;
    if (mx != 0.0) {
        double s2 = xr[0] * xr[0];
        s2 += xr[1] * xr[1];
        if (D == 3) s2 += xr[2] * xr[2];
        nrm = sqrt(s2);
    }
    out[0] = out[1] = out[2] = 0.0;
    if (fabs(nrm - radius) > 2.0 * dx) return;
    double bulk[3];
    if (D == 2) {
        bulk[0] = sV[0] + (0.0 - sW[0] * xr[1]);
        bulk[1] = sV[1] + (sW[0] * xr[0]);
        bulk[2] = 0.0;
    } else {
        bulk[0] = sV[0] + (sW[1] * xr[2] - sW[2] * xr[1]);
        bulk[1] = sV[1] + (-sW[0] * xr[2] + sW[2] * xr[0]);
        bulk[2] = sV[2] + (sW[0] * xr[1] - sW[1] * xr[0]);
    }
    if (kind == 0 || nrm == 0.0) {
        out[0] = bulk[0];
        out[1] = bulk[1];
        out[2] = bulk[2];
        return;
    }
    double fr[3] = {xr[0] / nrm, xr[1] / nrm, D == 3 ? xr[2] / nrm : 0.0};
    double edr = sE[0] * fr[0];
    edr += sE[1] * fr[1];
    if (D == 3) edr += sE[2] * fr[2];
    const double first = B1 + B2 * edr;
    for (int k = 0; k < D; ++k) out[k] = first * (edr * fr[k] - sE[k]) + bulk[k];
}

// ---------------------------------------------------------------------------
// Collision of one node (collisionStep + guoForcingTerm, src/gpu/fluids.jl:58-127)
// on the shifted, weight-normalised populations, in place.  The values are in
// storage units g'_i = S (f_i/w_i - rho0), S = a.scale (1 for FP32/FP64, a
// power of two for FP16/BF16), so no per-value rescaling is needed.
// Returns rho^n (the density the reference holds in model.massDensity).
//
// With m = rho (rho_inc for the incompressible equilibrium) and cu = c_i.u:
//   g_eq_i/S = (rho - rho0) - 1.5 m u.u + 4.5 m cu^2 + 3 m cu
//   Guo/(w_i S): BGK  A_i + K0 + B_i cu   (A_i = 3k c.F, B_i = 9k c.F, K0 = -3k u.F)
//                TRT  even K0 + B_i cu (k = k+), odd A_i (k = k-)
// A_i, B_i (and the K0 coefficient) arrive pre-multiplied by S.  For a pair
// (i, opp(i)) = (a, b) the update is
//   TRT: a* = le (a+b) + lo (a-b) + E + O,  b* = le (a+b) - lo (a-b) + E - O
//   BGK: a* = (1-w) a + E + O,              b* = (1-w) b + E - O
// with E the even part (relaxed symmetric equilibrium + even Guo term), O
// the odd part and le = (1 - omega+)/2, lo = (1 - omega-)/2; the moments are
// summed from the same pair sums and differences.
//
// collide_sd takes the pair sums s_i = a + b and differences d_i = a - b
// (i < opp(i)) from the caller, and g with the rest population (and, for BGK,
// every population); collide forms them from g.
// ---------------------------------------------------------------------------
template <class L, class R, bool TRT>
__device__ __forceinline__ R collide_sd(const StepArgs& a, R* g, const R* s, const R* d, R Fx, R Fy, R Fz,
                                        bool field) {
    constexpr int Q = L::Q;
    const CollideK<R>& k = collide_k<R>(a);
    R drho = 0, jx = 0, jy = 0, jz = 0;  // S (rho - rho0), S (j - dt/2 F)
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int ib = L::opp(i);
        if (ib < i) continue;
        if (ib == i) {
            drho = fma(R(L::w(i)), g[i], drho);
            continue;
        }
        drho = fma(R(L::w(i)), s[i], drho);
        if (L::cx(i) != 0) jx = fma(R(L::w(i) * L::cx(i)), d[i], jx);
        if (L::cy(i) != 0) jy = fma(R(L::w(i) * L::cy(i)), d[i], jy);
        if (L::cz(i) != 0) jz = fma(R(L::w(i) * L::cz(i)), d[i], jz);
    }
    const R rho = fma(drho, k.invS, k.rho0);
    jx = fma(jx, k.invS, k.hdt * Fx);
    jy = fma(jy, k.invS, k.hdt * Fy);
    jz = fma(jz, k.invS, k.hdt * Fz);
    R ux = 0, uy = 0, uz = 0;
    if (rho != R(0)) {  // findFluidVelocity: u = 0 where rho == 0
        const R inv = recip(rho);
        ux = jx * inv;
        uy = jy * inv;
        uz = jz * inv;
    }
    const R usq = ux * ux + uy * uy + uz * uz;
    const R uF = ux * Fx + uy * Fy + uz * Fz;
    const R Srq = k.S * (a.incompressible ? k.rho_inc : rho);
    const R E0 = fma(R(-1.5) * Srq, usq, drho);  // S (g_eq even part at cu = 0)
    const R e0 = fma(k.omE, E0, k.gK0 * uF);
    const R k45 = k.c45 * Srq, k3 = k.c3 * Srq;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int ib = L::opp(i);
        if (ib < i) continue;
        if (ib == i) {  // rest direction: a* = (1 - omega+) a + e0
            g[i] = fma(k.rest, g[i], e0);
            continue;
        }
        const R cu = R(L::cx(i)) * ux + R(L::cy(i)) * uy + R(L::cz(i)) * uz;
        R A = k.gA[i], B = k.gB[i];
        if (field) {
            const R cF = R(L::cx(i)) * Fx + R(L::cy(i)) * Fy + R(L::cz(i)) * Fz;
            A = k.gkA * cF;
            B = k.gkB * cF;
        }
        const R E = fma(fma(k45, cu, B), cu, e0);
        const R O = fma(k3, cu, A);
        if (TRT) {
            const R es = fma(k.le, s[i], E), od = fma(k.lo, d[i], O);
            g[i] = es + od;
            g[ib] = es - od;
        } else {
            const R ga = g[i], gb = g[ib];
            g[i] = fma(k.hsum, ga, E + O);
            g[ib] = fma(k.hsum, gb, E - O);
        }
    }
    return rho;
}

template <class L, class R, bool TRT>
__device__ __forceinline__ R collide(const StepArgs& a, R* g, R Fx, R Fy, R Fz, bool field) {
    constexpr int Q = L::Q;
    R s[Q], d[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int ib = L::opp(i);
        if (ib <= i) continue;
        s[i] = g[i] + g[ib];
        d[i] = g[i] - g[ib];
    }
    return collide_sd<L, R, TRT>(a, g, s, d, Fx, Fy, Fz, field);
}

template <class L, int ST, bool TRT>
struct NodeState {
    using R = typename Store<ST>::R;
    R g[L::Q];   // post-collision populations after load_collide()
    R rho;       // rho^n
};

// the stored populations of one node, in storage units
template <class L, int ST>
__device__ __forceinline__ void load_pops(const StepArgs& a, int cell, bool valid, typename Store<ST>::R* g) {
    using SS = Store<ST>;
    using T = typename SS::T;
    using R = typename SS::R;
    const T* __restrict__ src = static_cast<const T*>(a.src);
    const long long N = a.g.N;
#pragma unroll
    for (int i = 0; i < L::Q; ++i) g[i] = valid ? SS::dec(src[i * N + cell], R(1)) : R(0);
}

// collide loaded populations with the node's force; returns rho^n
template <class L, int ST, bool TRT>
__device__ __forceinline__ typename Store<ST>::R collide_node(const StepArgs& a, int cell, bool valid,
                                                            typename Store<ST>::R* g) {
    using R = typename Store<ST>::R;
    const long long N = a.g.N;
    R Fx = 0, Fy = 0, Fz = 0;
    if (a.force_mode == 1) {
        const CollideK<R>& k = collide_k<R>(a);
        Fx = k.F[0];
        Fy = k.F[1];
        Fz = k.F[2];
    } else if (a.force_mode == 2 && valid) {
        Fx = R(a.ffield[cell]);
        Fy = R(a.ffield[N + cell]);
        if (L::D == 3) Fz = R(a.ffield[2 * N + cell]);
    }
    return collide<L, R, TRT>(a, g, Fx, Fy, Fz, a.force_mode == 2);
}

template <class L, int ST, bool TRT>
__device__ __forceinline__ void load_collide(const StepArgs& a, int cell, bool valid, NodeState<L, ST, TRT>& s) {
    load_pops<L, ST>(a, cell, valid, s.g);
    s.rho = collide_node<L, ST, TRT>(a, cell, valid, s.g);
}

// ---------------------------------------------------------------------------
// Bulk kernel, one node per thread (FP64 storage, rows wider than a tile,
// per-node force fields).
// ---------------------------------------------------------------------------
template <class L, int ST, bool TRT>
__global__ void __launch_bounds__(kBlock) k_bulk(const StepArgs a) {
    using SS = Store<ST>;
    using T = typename SS::T;
    using R = typename SS::R;
    constexpr int Q = L::Q;
    // every other tick the tiles run last to first, as in k_bulk_v4 (L2 reuse)
    const long long tile = a.reverse ? a.g.ntiles - 1 - (long long)blockIdx.x : (long long)blockIdx.x;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int bx = (int)(tile % a.g.nt[0]);
    const int rr = (int)(tile / a.g.nt[0]);
    const int by = rr % a.g.nt[1], bz = rr / a.g.nt[1];
    const int x = bx * a.g.t[0] + threadIdx.x;
    const int y = by * a.g.t[1] + threadIdx.y;
    const int z = bz * a.g.t[2] + threadIdx.z;
    const bool valid = x < nx && y < ny && z < nz;
    const int cell = valid ? x + nx * (y + ny * z) : 0;
    grid_dep_trigger();  // the fix-up may start its stores-free part during the last wave
    NodeState<L, ST, TRT> s;
    load_collide<L, ST, TRT>(a, cell, valid, s);
    report_density(valid && bad_density(s.rho), a.err);
    if (!valid) return;
    const int xs[3] = {x == 0 ? nx - 1 : x - 1, x, x == nx - 1 ? 0 : x + 1};
    const int ys[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
    const int zs[3] = {z == 0 ? nz - 1 : z - 1, z, z == nz - 1 ? 0 : z + 1};
    T* __restrict__ dst = static_cast<T*>(a.dst);
    const long long N = a.g.N;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int t = xs[L::cx(i) + 1] + nx * (ys[L::cy(i) + 1] + ny * zs[L::cz(i) + 1]);
        dst[i * N + t] = a.stochastic ? SS::enc_sr(s.g[i], R(1), (unsigned)t, i) : SS::enc(s.g[i], R(1));
    }
}

// ---------------------------------------------------------------------------
// Bulk kernel, four consecutive x-nodes per thread with 128-bit (FP32) or
// 64-bit (FP16/BF16) loads and stores.  A CTA owns whole x-rows of its tile,
// so the periodic x-wrap stays inside the CTA: pushes along +-x are realigned
// in registers, the one value per row segment that crosses into the
// neighbouring thread goes through shared memory, and every global store is
// an aligned vector store.
// ---------------------------------------------------------------------------
template <int ST> struct Vec4;
template <> struct Vec4<ST_F32> {
    using raw = float4;  // the four values as stored
    static __device__ __forceinline__ void unpack(const raw& q, float* v) {
        v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    }
    static __device__ __forceinline__ void load(const void* base, int cell0, float* v) {
        unpack(__ldcs(reinterpret_cast<const float4*>(static_cast<const float*>(base) + cell0)), v);
    }
    // values of direction `dir` for cells cell0 .. cell0+3 (cell0 a multiple of 4)
    static __device__ __forceinline__ void store(void* base, int cell0, int, float a0, float a1, float a2, float a3,
                                                 const unsigned*, bool keep = false) {
        // streaming (evict-first) store: most lines are read again only a tick
        // later; the last tiles of a pass (keep) store with the default policy
        // instead, and the next pass reads those lines first (k_bulk_v4's
        // alternating tile order)
        float4* p = reinterpret_cast<float4*>(static_cast<float*>(base) + cell0);
        if (keep) *p = make_float4(a0, a1, a2, a3);  // a pass's last tiles: plain stores, kept in L2
        else __stcs(p, make_float4(a0, a1, a2, a3));
    }
};
template <> struct Vec4<ST_F16> {
    using raw = uint2;
    static __device__ __forceinline__ void unpack(const raw& q, float* v) {
        const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&q.x));
        const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&q.y));
        v[0] = lo.x; v[1] = lo.y; v[2] = hi.x; v[3] = hi.y;
    }
    static __device__ __forceinline__ void load(const void* base, int cell0, float* v) {
        unpack(load_raw(base, cell0), v);
    }
    static __device__ __forceinline__ raw load_raw(const void* base, int cell0) {
        return __ldcs(reinterpret_cast<const uint2*>(static_cast<const __half*>(base) + cell0));
    }
    // value `hi` (0: low half, 1: high half) of a packed pair
    static __device__ __forceinline__ float lane(unsigned w, int hi) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w));
        return hi ? f.y : f.x;
    }
    // s = a + b and d = a - b, a the value `hi` of the packed pair w, by the
    // mixed-precision add/sub (f16 + f32 -> f32): the same single rounding as
    // converting a first, one instruction fewer
    static __device__ __forceinline__ void sum_diff(unsigned w, int hi, float b, float& s, float& d) {
        if (hi)
            asm("{.reg .f16 l, h;\n\tmov.b32 {l, h}, %2;\n\tadd.rn.f32.f16 %0, h, %3;\n\tsub.rn.f32.f16 %1, h, %3;}"
                : "=f"(s), "=f"(d) : "r"(w), "f"(b));
        else
            asm("{.reg .f16 l, h;\n\tmov.b32 {l, h}, %2;\n\tadd.rn.f32.f16 %0, l, %3;\n\tsub.rn.f32.f16 %1, l, %3;}"
                : "=f"(s), "=f"(d) : "r"(w), "f"(b));
    }
    // rounding to nearest (dither null) or stochastic with the group's random
    // words (storage.cuh): cells (2p, 2p+1) of direction dir take word (dir + 2p) mod 4
    static __device__ __forceinline__ void store(void* base, int cell0, int dir, float a0, float a1, float a2,
                                                 float a3, const unsigned* dither, bool keep = false) {
        uint2 q;
        if (dither) {
            q.x = pack_half2_rs(a0, a1, dither[dir & 3]);
            q.y = pack_half2_rs(a2, a3, dither[(dir + 2) & 3]);
        } else {
            const __half2 lo = __floats2half2_rn(a0, a1);
            const __half2 hi = __floats2half2_rn(a2, a3);
            q.x = *reinterpret_cast<const unsigned*>(&lo);
            q.y = *reinterpret_cast<const unsigned*>(&hi);
        }
        uint2* p = reinterpret_cast<uint2*>(static_cast<__half*>(base) + cell0);
        if (keep) *p = q;  // as above
        else __stcs(p, q);
    }
};
template <> struct Vec4<ST_BF16> {
    using raw = uint2;
    static __device__ __forceinline__ void unpack(const raw& q, float* v) {
        const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&q.x));
        const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&q.y));
        v[0] = lo.x; v[1] = lo.y; v[2] = hi.x; v[3] = hi.y;
    }
    static __device__ __forceinline__ void load(const void* base, int cell0, float* v) {
        unpack(load_raw(base, cell0), v);
    }
    static __device__ __forceinline__ raw load_raw(const void* base, int cell0) {
        return __ldcs(reinterpret_cast<const uint2*>(static_cast<const __nv_bfloat16*>(base) + cell0));
    }
    static __device__ __forceinline__ float lane(unsigned w, int hi) {
        const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w));
        return hi ? f.y : f.x;
    }
    // as for FP16 (bf16 + f32 -> f32)
    static __device__ __forceinline__ void sum_diff(unsigned w, int hi, float b, float& s, float& d) {
        if (hi)
            asm("{.reg .b16 l, h;\n\tmov.b32 {l, h}, %2;\n\tadd.rn.f32.bf16 %0, h, %3;\n\tsub.rn.f32.bf16 %1, h, %3;}"
                : "=f"(s), "=f"(d) : "r"(w), "f"(b));
        else
            asm("{.reg .b16 l, h;\n\tmov.b32 {l, h}, %2;\n\tadd.rn.f32.bf16 %0, l, %3;\n\tsub.rn.f32.bf16 %1, l, %3;}"
                : "=f"(s), "=f"(d) : "r"(w), "f"(b));
    }
    static __device__ __forceinline__ void store(void* base, int cell0, int dir, float a0, float a1, float a2,
                                                 float a3, const unsigned* dither, bool keep = false) {
        uint2 q;
        if (dither) {
            q.x = pack_bf162_rs(a0, a1, dither[dir & 3]);
            q.y = pack_bf162_rs(a2, a3, dither[(dir + 2) & 3]);
        } else {
            const __nv_bfloat162 lo = __floats2bfloat162_rn(a0, a1);
            const __nv_bfloat162 hi = __floats2bfloat162_rn(a2, a3);
            q.x = *reinterpret_cast<const unsigned*>(&lo);
            q.y = *reinterpret_cast<const unsigned*>(&hi);
        }
        uint2* p = reinterpret_cast<uint2*>(static_cast<__nv_bfloat16*>(base) + cell0);
        if (keep) *p = q;  // as above
        else __stcs(p, q);
    }
};

template <class L>
constexpr int x_moving_dirs() {
    int n = 0;
    for (int i = 0; i < L::Q; ++i) n += L::cx(i) != 0 ? 1 : 0;
    return n;
}
template <class L>
constexpr int x_slot(int i) {  // exchange slot of direction i (cx != 0)
    int n = 0;
    for (int k = 0; k < i; ++k) n += L::cx(k) != 0 ? 1 : 0;
    return n;
}


// The pushes of one thread's four x-nodes (x0 .. x0+3 of row (y, z)) after
// their collision: direction i goes to x + c_i with aligned vector stores.
// from_left(i) / from_right(i) give the value of the +x / -x moving direction
// i that the neighbouring segment pushes into this one (read next to the
// store that needs it, so that the exchanged values are not all live at once).
template <class L, int ST, class FromLeft, class FromRight>
__device__ __forceinline__ void bulk_v4_push(const StepArgs& a, const float (&g)[4][L::Q], FromLeft from_left,
                                             FromRight from_right, int x0, int y, int z, const unsigned* dither,
                                             bool keep = false) {
    constexpr int Q = L::Q;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int ys[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
    const int zs[3] = {z == 0 ? nz - 1 : z - 1, z, z == nz - 1 ? 0 : z + 1};
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int t0 = x0 + nx * (ys[L::cy(i) + 1] + ny * zs[L::cz(i) + 1]);
        if (L::cx(i) == 0) {
            Vec4<ST>::store(a.dstq[i], t0, i, g[0][i], g[1][i], g[2][i], g[3][i], dither, keep);
        } else if (L::cx(i) == 1) {
            Vec4<ST>::store(a.dstq[i], t0, i, from_left(i), g[0][i], g[1][i], g[2][i], dither, keep);
        } else {
            Vec4<ST>::store(a.dstq[i], t0, i, g[1][i], g[2][i], g[3][i], from_right(i), dither, keep);
        }
    }
}

// One tile of the vector bulk pass: `a.vrows` full x-rows of one z-slice, four
// consecutive x-nodes per thread with 128-bit (FP32) or 64-bit (FP16/BF16)
// loads and stores.  Because a CTA owns whole x-rows, the periodic x-wrap
// stays inside the CTA: pushes along +-x are realigned in registers, the one
// value per row segment that crosses into the neighbouring thread goes
// through shared memory, and every global store is an aligned vector store.
// Threads past the tile's rows only take part in the barrier.
// SR: the 2-byte stores round stochastically (a separate instantiation, so
// that the nearest-rounding kernels keep their register allocation)
template <class L, int ST, bool TRT, int B, bool SR = false>
__device__ __forceinline__ void bulk_v4_tile(const StepArgs& a, long long tile, float (*s_ex)[B],
                                             bool keep = false) {
    using R = float;
    constexpr int Q = L::Q;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int RT = nx >> 2;  // threads per x-row
    const int tid = threadIdx.x;
    const int row = tid / RT, j = tid - row * RT;
    const int by = (int)(tile % a.vnt1);
    const int bz = (int)(tile / a.vnt1);
    const int y = by * a.vrows + row;
    const int z = bz;
    const bool valid = row < a.vrows && y < ny;
    const int x0 = 4 * j;
    const int cell0 = valid ? x0 + nx * (y + ny * z) : 0;
    R g[4][Q];
    const R Fx = a.kf.F[0], Fy = a.kf.F[1], Fz = a.kf.F[2];
    bool bad = false;
    if constexpr (TRT && Store<ST>::bytes == 2) {
        // 2-byte TRT: the pair sums and differences take the first value of
        // each pair straight from its 16-bit form (Vec4::sum_diff).  The
        // threads past the tile's rows load cells 0..3 (cell0 = 0, in bounds)
        // and store nothing.  128^3 FP16 pass: 6.6 % fewer instructions than
        // converting every value first, bit-identical results.
        typename Vec4<ST>::raw q[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) q[i] = Vec4<ST>::load_raw(a.srcq[i], cell0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            R s[Q], d[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const int ib = L::opp(i);
                if (ib < i) continue;
                const unsigned wa = k < 2 ? q[i].x : q[i].y;  // cells (0, 1) | (2, 3)
                if (ib == i) {
                    g[k][i] = Vec4<ST>::lane(wa, k & 1);
                    continue;
                }
                const R b = Vec4<ST>::lane(k < 2 ? q[ib].x : q[ib].y, k & 1);
                Vec4<ST>::sum_diff(wa, k & 1, b, s[i], d[i]);
            }
            bad |= bad_density(collide_sd<L, R, TRT>(a, g[k], s, d, Fx, Fy, Fz, false));
        }
    } else {
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            R v[4] = {0, 0, 0, 0};
            if (valid) Vec4<ST>::load(a.srcq[i], cell0, v);
            g[0][i] = v[0];
            g[1][i] = v[1];
            g[2][i] = v[2];
            g[3][i] = v[3];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) bad |= bad_density(collide<L, R, TRT>(a, g[k], Fx, Fy, Fz, false));
    }
    report_density(valid && bad, a.err);
    constexpr bool sr = SR && Store<ST>::bytes == 2;
    unsigned dw[4];
    if (sr) rs_words(group_dither(cell0, g[0][1], g[0][2], g[0][3]), dw);
    const unsigned* dither = sr ? dw : nullptr;
    // the value of each +-x direction that leaves this thread's 4-node segment
    if (row < a.vrows) {
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            if (L::cx(i) == 1) s_ex[x_slot<L>(i)][tid] = g[3][i];
            if (L::cx(i) == -1) s_ex[x_slot<L>(i)][tid] = g[0][i];
        }
    }
    __syncthreads();
    if (!valid) return;
    const int left = row * RT + (j == 0 ? RT - 1 : j - 1);
    const int right = row * RT + (j == RT - 1 ? 0 : j + 1);
    bulk_v4_push<L, ST>(
        a, g, [&](int i) { return s_ex[x_slot<L>(i)][left]; }, [&](int i) { return s_ex[x_slot<L>(i)][right]; }, x0,
        y, z, dither, keep);
}

// Resident threads per SM the vector bulk kernels are compiled for: a D2Q9
// thread holds 36 populations and fits 64 registers (32 warps per SM); the
// 3D sets take up to 128 (16 warps per SM) with FP32/FP64 storage, which is
// memory-bound, and up to 96 (20 warps per SM) with 2-byte storage, whose
// conversions make it issue-bound as well: the extra warps took its 128^3
// pass from 28.4 to 26.9 us, with no change for FP32.
// Stochastic rounding (one conversion per two values with the group's
// random words) fits the same 96 registers.  A D3Q27 thread holds 108
// populations: 12 warps per SM (168 registers) with FP32/FP64 storage, 14
// (144) with 2-byte storage, so that neither spills.
template <class L, int ST = ST_F32, bool SR = false>
constexpr int bulk_threads_per_sm() {
    return L::Q <= 9 ? 1024
                     : (L::Q > 19 ? (Store<ST>::bytes == 2 ? 448 : 384) : (Store<ST>::bytes == 2 ? 640 : 512));
}

// the vector bulk pass over all tiles, one CTA of B threads per tile
// CTAs start in blockIdx order.  Every other tick (a.reverse) the pass walks
// its tiles last to first, so that it first reads the populations the
// previous tick stored last, which are still in L2 (126 MB, two fifths of a
// 128^3 FP32 population buffer): a share of each tick's reads comes from L2
// instead of HBM (the 128^3 FP32 tick 55.2 -> 51.3 us).  The result does not
// depend on the order.
template <class L, int ST, bool TRT, int B, bool SR>
__global__ void __launch_bounds__(B, bulk_threads_per_sm<L, ST, SR>() / B) k_bulk_v4(const StepArgs a) {
    __shared__ float s_ex[x_moving_dirs<L>()][B];
    grid_dep_trigger();  // the fix-up may start its stores-free part during the last wave
    const long long tiles = (long long)a.vnt1 * a.g.n[2];
    // FP32: the last three fifths of the pass store with the default policy,
    // so that L2 keeps those lines for the next pass (128^3 tick: 51.3 us with
    // none, 50.5 with two fifths, 49.4 with three, 50.2 with four, 51.6 with
    // all); the issue-bound 2-byte passes measured slower with it
    const bool keep = Store<ST>::bytes == 4 && (long long)blockIdx.x * 5 >= tiles * 2;
    bulk_v4_tile<L, ST, TRT, B, SR>(a, a.reverse ? tiles - 1 - (long long)blockIdx.x : (long long)blockIdx.x, s_ex,
                                    keep);
}

// periodic intervals [a0, a0+la) and [b0, b0+lb) of an axis of n nodes meet
__device__ __forceinline__ bool ranges_meet(int a0, int la, int b0, int lb, int n) {
    if (la >= n || lb >= n) return true;
    const int d = ((b0 - a0) % n + n) % n;  // start of b relative to a
    return d < la || d + lb > n;
}

// does vector tile `tile` come within two nodes of particle p's solid box?
template <int D>
__device__ __forceinline__ bool tile_meets_box(const StepArgs& a, long long tile, int p) {
    const int by = (int)(tile % a.vnt1), bz = (int)(tile / a.vnt1);
    const int ny = a.g.n[1], nz = a.g.n[2];
    const int y0 = by * a.vrows, ly = min(a.vrows, ny - y0);
    const int* b = a.nbox + 6 * p;
    if (b[0] > b[3] || b[1] > b[4] || b[2] > b[5]) return false;  // no solid node
    if (!ranges_meet(y0, ly, b[1] - 2, b[4] - b[1] + 5, ny)) return false;
    return D == 2 || ranges_meet(bz, 1, b[2] - 2, b[5] - b[2] + 5, nz);
}

}  // namespace lbm
