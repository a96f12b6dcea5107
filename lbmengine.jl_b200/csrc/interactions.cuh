// Particle-particle interactions: molecularDynamicsTick! (src/gpu/particles.jl:
// 100-197) before the particle update.  One CTA: every thread evaluates some
// items (a bond, a bond angle, or one pair of a pair potential) from the
// particles' positions before this tick's move; then every particle sums the
// forces of its items in the order the reference adds them to its force
// input (interactions in order, pairs in order), in FP64.  The particle update
// adds the sum to the momentum exchange (particles.cuh).
#pragma once
#include "kernels.cuh"

namespace lbm {

constexpr int kInterThreads = 256;

// one item as the host passes it (lbm_interaction with 0-based particle ids)
struct InterItem {
    int kind, id1, id2, id3;
    double p[4];
};

struct InterArgs {
    const InterItem* items;
    int nitems;
    int nparts;
    int dims;
    int pad;
    const ParticleDev* parts;
    const int* coff;  // [nparts + 1]: the contributions to particle p are cent[coff[p] .. coff[p+1])
    const int* cent;  // item << 2 | vector (0: first force, 1: second, 2: their sum) << 1 | subtract
    double* pf;       // [nitems][3][3] forces of the items
    double* fint;     // [nparts][3] interaction force of each particle
};

// |v| as LinearAlgebra.norm: 0 for the zero vector, else the root of the
// squares summed in component order
__device__ __forceinline__ double inorm(const double* v, int d) {
    double m = 0.0;
    for (int k = 0; k < d; ++k) m = fmax(m, fabs(v[k]));
    if (m == 0.0) return 0.0;
    double s = v[0] * v[0];
    for (int k = 1; k < d; ++k) s += v[k] * v[k];
    return sqrt(s);
}

// cross of the reference (src/gpu/aux.jl:139-157): 3D vectors, or in 2D the z
// component of two plane vectors (a scalar in out[0])
__device__ __forceinline__ void icross(const double* a, const double* b, int d, double* out) {
    if (d == 2) {
        out[0] = a[0] * b[1] - a[1] * b[0];
        out[1] = out[2] = 0.0;
    } else {
        out[0] = a[1] * b[2] - a[2] * b[1];
        out[1] = -a[0] * b[2] + a[2] * b[0];
        out[2] = a[0] * b[1] - a[1] * b[0];
    }
}

// cross(w, v) with w a 2D scalar (the z axis): (0, 0, w) x (v, 0) restricted to the plane
__device__ __forceinline__ void icross_scalar(double w, const double* v, double* out) {
    out[0] = 0.0 * 0.0 - w * v[1];
    out[1] = -0.0 * 0.0 + w * v[0];
    out[2] = 0.0;
}

__device__ void interaction_forces(const InterArgs& a, int t) {
    const InterItem it = a.items[t];
    const int d = a.dims;
    double* out = a.pf + (size_t)t * 9;
    for (int k = 0; k < 9; ++k) out[k] = 0.0;
    const double* R1 = a.parts[it.id1].R;
    const double* R2 = a.parts[it.id2].R;
    if (it.kind == 2) {  // applyInteraction!(::PolarInteraction), particles.jl:140-162
        const double* R3 = a.parts[it.id3].R;
        double d12[3] = {0, 0, 0}, d32[3] = {0, 0, 0}, u12[3] = {0, 0, 0}, u32[3] = {0, 0, 0};
        for (int k = 0; k < d; ++k) {
            d12[k] = R1[k] - R2[k];
            d32[k] = R3[k] - R2[k];
        }
        const double n12 = inorm(d12, d), n32 = inorm(d32, d);
        for (int k = 0; k < d; ++k) {
            u12[k] = d12[k] / n12;
            u32[k] = d32[k] / n32;
        }
        double x = u12[0] * u32[0];
        for (int k = 1; k < d; ++k) x += u12[k] * u32[k];
        if (fabs(x) > 1.0) x = x > 0 ? 1.0 : -1.0;
        const double ang = acos(x);
        double td[3];
        icross(u32, u12, d, td);
        const double an = d == 2 ? fabs(td[0]) : inorm(td, 3);
        if (an > 0)
            for (int k = 0; k < 3; ++k) td[k] /= an;
        const double s = it.p[1] * (ang - it.p[0]);
        double f321[3], f123[3];
        if (d == 2) {
            icross_scalar(s * td[0], u12, f321);
            icross_scalar(s * td[0], u32, f123);
        } else {
            const double tq[3] = {s * td[0], s * td[1], s * td[2]};
            icross(tq, u12, 3, f321);
            icross(tq, u32, 3, f123);
        }
        for (int k = 0; k < d; ++k) {
            out[k] = -f321[k] / n12;      // on id1
            out[3 + k] = f123[k] / n32;   // on id3
            out[6 + k] = out[k] + out[3 + k];  // subtracted from id2
        }
        return;
    }
    double dv[3] = {0, 0, 0}, u[3] = {0, 0, 0};
    for (int k = 0; k < d; ++k) dv[k] = R2[k] - R1[k];  // disp21
    const double dist = inorm(dv, d);
    for (int k = 0; k < d; ++k) u[k] = dv[k] / dist;
    double f = 0.0;
    if (it.kind == 0) {  // LinearInteraction: k (d - d_eq) r^
        f = it.p[1] * (dist - it.p[0]);
    } else if (it.kind == 1) {  // BistableInteraction: (a (d - R)^3 - b (d - R)) r^
        const double x = dist - it.p[0];
        f = it.p[1] * (x * x * x) - it.p[2] * x;
    } else if (it.kind == 3) {  // LennardJonesInteraction inside its cutoff
        if (!(dist < it.p[2])) return;
        const double sd = it.p[1] / dist;
        const double s2 = sd * sd, s6 = s2 * s2 * s2;
        f = -4.0 * it.p[0] / dist * (12.0 * (s6 * s6) - 6.0 * s6);
    } else {  // DipoleDipoleInteraction, when the field is not zero
        const double B[3] = {it.p[1], it.p[2], it.p[3]};
        if (inorm(B, d) == 0.0) return;
        double cb[3], ccb[3];
        icross(u, B, d, cb);
        double sq;
        if (d == 2) {
            icross_scalar(cb[0], B, ccb);
            sq = cb[0] * cb[0];
        } else {
            icross(cb, B, 3, ccb);
            sq = cb[0] * cb[0] + cb[1] * cb[1] + cb[2] * cb[2];
        }
        double bb = B[0] * B[0];
        for (int k = 1; k < d; ++k) bb += B[k] * B[k];
        const double d2 = dist * dist;
        const double pre = -it.p[0] / (d2 * d2);
        for (int k = 0; k < d; ++k) out[k] = pre * (2.0 * ccb[k] - 2.0 * bb * u[k] + 5.0 * u[k] * sq);
        return;
    }
    for (int k = 0; k < d; ++k) out[k] = f * u[k];
}

__global__ void __launch_bounds__(kInterThreads) k_interactions(const InterArgs a) {
    for (int t = threadIdx.x; t < a.nitems; t += blockDim.x) interaction_forces(a, t);
    __syncthreads();
    for (int p = threadIdx.x; p < a.nparts; p += blockDim.x) {
        double F[3] = {0.0, 0.0, 0.0};
        for (int e = a.coff[p]; e < a.coff[p + 1]; ++e) {
            const int c = a.cent[e];
            const double* v = a.pf + (size_t)(c >> 3) * 9 + 3 * ((c >> 1) & 3);
            for (int k = 0; k < 3; ++k) F[k] = (c & 1) ? F[k] - v[k] : F[k] + v[k];
        }
        for (int k = 0; k < 3; ++k) a.fint[3 * p + k] = F[k];
    }
}

}  // namespace lbm
