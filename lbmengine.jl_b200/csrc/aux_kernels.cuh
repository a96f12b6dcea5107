// Set-up and read-back kernels (not on the per-tick path).
#pragma once
#include "kernels.cuh"

namespace lbm {

struct CodecArgs {
    void* pop;            // stored populations
    double* f64;          // [Q][N] FP64 populations (f units)
    double* rho;          // [N] or null
    double* u;            // [d][N] or null
    const unsigned char* wall;
    const double* ffield;
    long long N;
    double rho0, scale, inv_scale, half_dt;
    double F[3];
    int force_mode;
    double* stress;       // [d][d][N] viscous stress tensor (k_stress) or null
    double stress_coeff;  // 1 - dt/(2 tau)
    int incompressible;
    double rho_inc;       // rho0 of the incompressible equilibrium
};

// f (FP64, reference units) -> stored g = (f/w - rho0)*scale
template <class L, int ST>
__global__ void k_encode(const CodecArgs a) {
    using SS = Store<ST>;
    using T = typename SS::T;
    using R = typename SS::R;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= a.N) return;
    T* pop = static_cast<T*>(a.pop);
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        const double g = a.f64[i * a.N + c] * (1.0 / L::w(i)) - a.rho0;
        pop[i * a.N + c] = SS::enc((R)g, (R)a.scale);
    }
}

// stored g -> f (FP64); wall nodes hold f = 0 exactly
template <class L, int ST>
__global__ void k_decode(const CodecArgs a) {
    using SS = Store<ST>;
    using T = typename SS::T;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= a.N) return;
    const T* pop = static_cast<const T*>(a.pop);
    const bool w = a.wall && a.wall[c];
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        const double g = (double)SS::dec(pop[i * a.N + c], (typename SS::R)a.inv_scale);
        a.f64[i * a.N + c] = w ? 0.0 : L::w(i) * (a.rho0 + g);
    }
}

// hydroVariablesUpdate! (src/gpu/fluids.jl:7-37) from the stored populations, in FP64
template <class L, int ST>
__global__ void k_macro(const CodecArgs a) {
    using SS = Store<ST>;
    using T = typename SS::T;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= a.N) return;
    const T* pop = static_cast<const T*>(a.pop);
    if (a.wall && a.wall[c]) {
        if (a.rho) a.rho[c] = 0.0;
        if (a.u)
            for (int k = 0; k < L::D; ++k) a.u[k * a.N + c] = 0.0;
        return;
    }
    double drho = 0, j[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        const double wg = L::w(i) * (double)SS::dec(pop[i * a.N + c], (typename SS::R)a.inv_scale);
        drho += wg;
        j[0] += L::cx(i) * wg;
        j[1] += L::cy(i) * wg;
        j[2] += L::cz(i) * wg;
    }
    const double rho = a.rho0 + drho;
    double F[3] = {0, 0, 0};
    if (a.force_mode == 1) {
        F[0] = a.F[0];
        F[1] = a.F[1];
        F[2] = a.F[2];
    } else if (a.force_mode == 2) {
        for (int k = 0; k < L::D; ++k) F[k] = a.ffield[k * a.N + c];
    }
    if (a.rho) a.rho[c] = rho;
    if (a.u)
        for (int k = 0; k < L::D; ++k) a.u[k * a.N + c] = rho == 0.0 ? 0.0 : (j[k] + a.half_dt * F[k]) / rho;
}


// viscousStressTensor (src/cpu/fluids.jl:507-520; commented out in the GPU
// module, src/gpu/fluids.jl:272-285) from the stored populations, in FP64:
//   sigma_ab = -(1 - dt/(2 tau)) sum_i c_ia c_ib (f_i - f_eq_i(rho, u))
// with rho and u of hydroVariablesUpdate! (u with the Guo half force) and the
// equilibrium of equilibriumDistribution (src/gpu/fluids.jl:39-52).  Wall
// nodes hold f = 0, rho = u = 0, hence sigma = 0.
template <class L, int ST>
__global__ void k_stress(const CodecArgs a) {
    using SS = Store<ST>;
    using T = typename SS::T;
    constexpr int D = L::D;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= a.N) return;
    const T* pop = static_cast<const T*>(a.pop);
    const bool wall = a.wall && a.wall[c];
    double f[L::Q];
    double rho = 0.0, j[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        f[i] = wall ? 0.0 : L::w(i) * (a.rho0 + (double)SS::dec(pop[i * a.N + c], (typename SS::R)a.inv_scale));
        rho += f[i];
        j[0] += L::cx(i) * f[i];
        j[1] += L::cy(i) * f[i];
        j[2] += L::cz(i) * f[i];
    }
    double F[3] = {0, 0, 0};
    if (!wall) {
        if (a.force_mode == 1) {
            F[0] = a.F[0];
            F[1] = a.F[1];
            F[2] = a.F[2];
        } else if (a.force_mode == 2) {
            for (int k = 0; k < D; ++k) F[k] = a.ffield[k * a.N + c];
        }
    }
    double u[3] = {0, 0, 0};
    if (rho != 0.0)
        for (int k = 0; k < D; ++k) u[k] = (j[k] + a.half_dt * F[k]) / rho;
    const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    double s[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        const double uc = u[0] * L::cx(i) + u[1] * L::cy(i) + u[2] * L::cz(i);
        const double second = uc * 3.0 + uc * uc * 4.5 - uu * 1.5;
        const double feq = a.incompressible ? L::w(i) * rho + L::w(i) * (a.rho_inc * second)
                                            : L::w(i) * ((second + 1.0) * rho);
        const double fneq = f[i] - feq;
        const int ci[3] = {L::cx(i), L::cy(i), L::cz(i)};
        for (int p = 0; p < D; ++p)
            for (int q = 0; q < D; ++q) s[p][q] += ci[p] * ci[q] * fneq;
    }
    for (int p = 0; p < D; ++p)
        for (int q = 0; q < D; ++q) a.stress[(p + D * q) * a.N + c] = -a.stress_coeff * s[p][q];
}

// Global FP64 sums of the density and the momentum density (rho, rho u with
// the Guo half force, as hydroVariablesUpdate! forms them; wall nodes hold
// zero), in a fixed order: every CTA sums its kTotBlock cells by a tree into
// part[cta][4]; k_totals_final sums the CTA parts in CTA order.
constexpr int kTotBlock = 256;

template <class L, int ST>
__global__ void __launch_bounds__(kTotBlock) k_totals(const CodecArgs a, double* part) {
    using SS = Store<ST>;
    using T = typename SS::T;
    __shared__ double s[4][kTotBlock];
    const long long c = blockIdx.x * (long long)kTotBlock + threadIdx.x;
    double v[4] = {0, 0, 0, 0};
    if (c < a.N && !(a.wall && a.wall[c])) {
        const T* pop = static_cast<const T*>(a.pop);
        double drho = 0, j[3] = {0, 0, 0};
#pragma unroll
        for (int i = 0; i < L::Q; ++i) {
            const double wg = L::w(i) * (double)SS::dec(pop[i * a.N + c], (typename SS::R)a.inv_scale);
            drho += wg;
            j[0] += L::cx(i) * wg;
            j[1] += L::cy(i) * wg;
            j[2] += L::cz(i) * wg;
        }
        v[0] = a.rho0 + drho;
        for (int k = 0; k < L::D; ++k) {
            const double F = a.force_mode == 1 ? a.F[k] : (a.force_mode == 2 ? a.ffield[k * a.N + c] : 0.0);
            v[1 + k] = j[k] + a.half_dt * F;
        }
    }
    for (int k = 0; k < 4; ++k) s[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int w = kTotBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < 4; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 4) part[blockIdx.x * 4 + threadIdx.x] = s[threadIdx.x][0];
}

static __global__ void __launch_bounds__(kTotBlock) k_totals_final(const double* part, long long nblocks, double* out) {
    __shared__ double s[4][kTotBlock];
    double v[4] = {0, 0, 0, 0};
    for (long long b = threadIdx.x; b < nblocks; b += kTotBlock)
        for (int k = 0; k < 4; ++k) v[k] += part[b * 4 + k];
    for (int k = 0; k < 4; ++k) s[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int w = kTotBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < 4; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 4) out[threadIdx.x] = s[threadIdx.x][0];
}

struct InitArgs {
    void* pop;
    long long N;
    const double* rho;      // [N] or null -> rho_uniform
    const double* u;        // [d][N] or null -> u_uniform
    const unsigned char* wall;
    const double* ffield;   // [d][N] (already zero on walls) or null
    double rho_uniform;
    double u_uniform[3];
    double F[3];
    double dt, rho0, scale;
    int zero_walls;         // rho = u = 0 on wall nodes (initMethods.jl:622-624)
    int force_mode;
};

// findInitialConditions (src/gpu/initMethods.jl:417-438):
//   u' = u - dt/2 F/rho (F/rho = 0 where rho == 0), f_i = f_eq(rho, u')
// evaluated in FP64 in the reference's operation order, then encoded.
template <class L, int ST>
__global__ void k_init(const InitArgs a) {
    using SS = Store<ST>;
    using T = typename SS::T;
    using R = typename SS::R;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= a.N) return;
    constexpr int D = L::D;
    double rho = a.rho ? a.rho[c] : a.rho_uniform;
    double u[3] = {0, 0, 0};
    for (int k = 0; k < D; ++k) u[k] = a.u ? a.u[k * a.N + c] : a.u_uniform[k];
    const bool w = a.wall && a.wall[c];
    if (a.zero_walls && w) {
        rho = 0.0;
        u[0] = u[1] = u[2] = 0.0;
    }
    if (a.force_mode != 0) {
        for (int k = 0; k < D; ++k) {
            const double Fk = a.force_mode == 1 ? (w ? 0.0 : a.F[k]) : a.ffield[k * a.N + c];
            const double cons = rho == 0.0 ? 0.0 : __ddiv_rn(Fk, rho);
            u[k] = __dsub_rn(u[k], __dmul_rn(__dmul_rn(0.5, a.dt), cons));
        }
    }
    double uu = 0.0;
    for (int k = 0; k < D; ++k) uu = __dadd_rn(uu, __dmul_rn(u[k], u[k]));
    T* pop = static_cast<T*>(a.pop);
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        double uc = 0.0;
        uc = __dadd_rn(uc, __dmul_rn(u[0], (double)L::cx(i)));
        uc = __dadd_rn(uc, __dmul_rn(u[1], (double)L::cy(i)));
        if (D == 3) uc = __dadd_rn(uc, __dmul_rn(u[2], (double)L::cz(i)));
        const double first = __dadd_rn(__dmul_rn(uc, 3.0), __dmul_rn(__dmul_rn(uc, uc), 4.5));
        const double second = __dadd_rn(__dsub_rn(first, __dmul_rn(uu, 1.5)), 1.0);
        const double f = __dmul_rn(second, __dmul_rn(L::w(i), rho));
        const double g = f * (1.0 / L::w(i)) - a.rho0;
        pop[i * a.N + c] = SS::enc((R)g, (R)a.scale);
    }
}

struct MaskArgs {
    unsigned char* mask;
    const ParticleDev* part;
    const int2* ivl;
    int n[3];
    long long N;
};

// solidRegion of one particle over the whole grid (getSphere, src/gpu/aux.jl:206-215),
// read from the row intervals that the fix-up kernel uses
template <int D>
__global__ void k_mask(const MaskArgs a) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= a.N) return;
    const int x = (int)(q % a.n[0]);
    const int y = (int)((q / a.n[0]) % a.n[1]);
    const int z = (int)(q / ((long long)a.n[0] * a.n[1]));
    a.mask[q] = solid_at(*a.part, a.ivl, x, y, z) ? 1 : 0;
}

}  // namespace lbm
