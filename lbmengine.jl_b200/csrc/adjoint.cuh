// Discrete adjoint of one tick (reverse mode), for gradients of a particle
// observable with respect to the squirmer modes B1, B2, the relaxation times
// and the uniform body force.  No counterpart in the reference (it has no
// differentiation); the forward map differentiated is the tick of
// tick!/moveParticles! (src/gpu/fluids.jl:132-226, src/gpu/particles.jl:7-92)
// as this library runs it:
//   f*(x)        = collide(f^n(x); tau+, tau-, F)                (fluids.jl:58-127)
//   f^{n+1}_i(x+c_i) = f*_i(x)                                   (push streaming)
//   f^{n+1}_j(x) = f*_i(x) + 6 w_j rho^n(x) c_j.u_p(x-c_j),  i = opp(j),
//                  for the particle's boundary links (x fluid, x - c_j solid)
//   F = sum_links coeff (f*_i + f^{n+1}_j) c_i,  T = sum_links coeff (f*_i + f^{n+1}_j) (x - R) x c_i
// Walls (static, fluids.jl:147-174): wall nodes hold f = 0 after streaming,
// and a fluid node x whose source x - c_j is a wall node gets
//   f^{n+1}_j(x) = f*_i(x) + 6 w_j rho^n(x) c_j.u_w(x - c_j)  (+ the particles' Ladd terms),
// which the momentum exchange of a particle with the same link also sees.
// The solid masks are held as the forward run computed them (their
// derivative is zero almost everywhere).  Adjoint populations are FP64 and
// in f units; the forward populations are read in their storage format and
// the local linearisation is evaluated in FP64.
//
// One thread per node x, gathering ("pull" form of the transposed push):
//   lam*_i(x) = lam^{n+1}_i(x + c_i)   unless (x + c_i, i) is a link slot
//             + sum over links (x, j) with opp(j) = i of the link terms;
//   lam^n(x)  = (d collide / d f)^T lam*(x) + (d rho / d f)^T mu_rho(x).
// Parameter and particle adjoints are reduced per CTA in a fixed order.
#pragma once
#include "kernels.cuh"

namespace lbm {

// accumulators reduced per CTA: dtau+, dtau-, dF (3), particle snapshot
// sR, sV, sW, sE (12), dB1, dB2, torque arm mR (3)
constexpr int kAdjAcc = 22;
constexpr int kAdjBlock = 128;

// forward-mode dual number with one direction
struct DD1 {
    double v, d;
};
__device__ __forceinline__ DD1 dd(double v, double d = 0.0) { return DD1{v, d}; }
__device__ __forceinline__ DD1 operator+(DD1 a, DD1 b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ DD1 operator-(DD1 a, DD1 b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ DD1 operator-(DD1 a) { return {-a.v, -a.d}; }
__device__ __forceinline__ DD1 operator*(DD1 a, DD1 b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ DD1 operator/(DD1 a, DD1 b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ DD1 operator+(DD1 a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ DD1 operator+(double b, DD1 a) { return {b + a.v, a.d}; }
__device__ __forceinline__ DD1 operator-(DD1 a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ DD1 operator-(double b, DD1 a) { return {b - a.v, -a.d}; }
__device__ __forceinline__ DD1 operator*(DD1 a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ DD1 operator*(double b, DD1 a) { return {b * a.v, b * a.d}; }
__device__ __forceinline__ DD1 operator/(DD1 a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ DD1 operator/(double b, DD1 a) { return dd(b) / a; }
__device__ __forceinline__ DD1 dsqrt(DD1 a) {
    const double r = ::sqrt(a.v);
    return {r, a.d / (2.0 * r)};
}
__device__ __forceinline__ double dsqrt(double a) { return ::sqrt(a); }
__device__ __forceinline__ double value(double a) { return a; }
__device__ __forceinline__ double value(DD1 a) { return a.v; }
template <class T> __device__ __forceinline__ T lift(double x) { return T(x); }
template <> __device__ __forceinline__ DD1 lift<DD1>(double x) { return dd(x); }

// the forward state of one tick the linearisation needs
struct AdjArgs {
    const void* src;         // f^n in its storage format
    const double* lam_in;    // lam^{n+1} [Q][N], f units
    double* lam_out;         // lam^n [Q][N]
    GridDesc g;
    const double* coord[3];
    const ParticleDev* part;  // the particle at tick n (one particle)
    const int2* ivl;
    const unsigned char* wall;  // wall nodes (null: no walls)
    const double* uw;           // wall velocity [d][N] (null: static walls)
    int has_part;
    int pad;
    double rho0, inv_scale;  // stored g' = S (f/w - rho0)
    double dt, tau_p, tau_m;  // tau_m unused for BGK
    double F[3];
    int guo, incompressible;
    double rho_inc;
    double coeff;             // dx^d / dt
    double lamF[3], lamT[3];  // adjoints of this tick's particle force and torque
    double* partial;          // [gridDim.x][kAdjAcc]
};

// collisionStep + guoForcingTerm (fluids.jl:58-127) of one node in f units,
// as a function of (rho, u, tau+, tau-, F) at fixed f
template <class L, bool TRT, class T>
__device__ __forceinline__ void ref_collide(const double* f, T rho, const T* u, T taup, T taum, const T* Fv,
                                            const AdjArgs& a, T* out) {
    constexpr int Q = L::Q, D = L::D;
    const double dt = a.dt;
    T uu = lift<T>(0.0);
    for (int k = 0; k < D; ++k) uu = uu + u[k] * u[k];
    T eq[L::Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int c[3] = {L::cx(i), L::cy(i), L::cz(i)};
        T uc = lift<T>(0.0);
        for (int k = 0; k < D; ++k) uc = uc + u[k] * (double)c[k];
        const T second = uc * 3.0 + (uc * uc) * 4.5 - uu * 1.5;
        eq[i] = a.incompressible ? rho * L::w(i) + (second * a.rho_inc) * L::w(i) : ((second + 1.0) * rho) * L::w(i);
    }
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int c[3] = {L::cx(i), L::cy(i), L::cz(i)};
        const int ib = L::opp(i);
        T om;
        if (!TRT) {
            om = (-dt / taup) * (f[i] - eq[i]);
        } else {
            const double fp = 0.5 * (f[i] + f[ib]), fm = 0.5 * (f[i] - f[ib]);
            const T ep = (eq[i] + eq[ib]) * 0.5, em = (eq[i] - eq[ib]) * 0.5;
            om = (-dt / taup) * (fp - ep) + (-dt / taum) * (fm - em);
        }
        if (a.guo) {
            T uc = lift<T>(0.0);
            for (int k = 0; k < D; ++k) uc = uc + u[k] * (double)c[k];
            T G;
            if (!TRT) {
                T inter = lift<T>(0.0);
                for (int k = 0; k < D; ++k)
                    inter = inter + ((((-u[k]) + (double)c[k]) * 3.0) + (uc * (double)c[k]) * 9.0) * Fv[k];
                G = (1.0 - dt / (taup * 2.0)) * inter * (L::w(i) * dt);
            } else {
                T inter = lift<T>(0.0), inter2 = lift<T>(0.0);
                for (int k = 0; k < D; ++k) {
                    inter = inter + ((-u[k]) * 3.0 + (uc * (double)c[k]) * 9.0) * Fv[k];
                    inter2 = inter2 + Fv[k] * ((double)c[k] * 3.0);
                }
                G = ((1.0 - dt / (taup * 2.0)) * inter + (1.0 - dt / (taum * 2.0)) * inter2) * (L::w(i) * dt);
            }
            om = om + G;
        }
        out[i] = om + f[i];
    }
}

// getNodeVelocity (aux.jl:229-263) over any scalar type
template <int D, class T>
__device__ __forceinline__ void slip_velocity_t(const T* sR, const T* sV, const T* sW, const T* sE, T B1, T B2,
                                                int kind, double X0, double X1, double X2, T* out) {
    const T xr[3] = {X0 - sR[0], X1 - sR[1], D == 3 ? X2 - sR[2] : lift<T>(0.0)};
    T bulk[3];
    if (D == 2) {
        bulk[0] = sV[0] - sW[0] * xr[1];
        bulk[1] = sV[1] + sW[0] * xr[0];
        bulk[2] = lift<T>(0.0);
    } else {
        bulk[0] = sV[0] + sW[1] * xr[2] - sW[2] * xr[1];
        bulk[1] = sV[1] - sW[0] * xr[2] + sW[2] * xr[0];
        bulk[2] = sV[2] + sW[0] * xr[1] - sW[1] * xr[0];
    }
    if (kind == 0) {
        for (int k = 0; k < 3; ++k) out[k] = bulk[k];
        return;
    }
    T nrm = dsqrt(xr[0] * xr[0] + xr[1] * xr[1] + xr[2] * xr[2]);
    if (value(nrm) == 0.0) nrm = lift<T>(1.0);
    const T inv = 1.0 / nrm;
    const T ur[3] = {inv * xr[0], inv * xr[1], inv * xr[2]};
    const T edr = ur[0] * sE[0] + ur[1] * sE[1] + (D == 3 ? ur[2] * sE[2] : lift<T>(0.0));
    const T first = B1 + B2 * edr;
    for (int k = 0; k < 3; ++k) out[k] = first * (edr * ur[k] - (k < D ? sE[k] : lift<T>(0.0))) + bulk[k];
}

// The transposed derivatives of the collision at fixed f, contracted with
// lam*: with feq_i(rho, u), the Guo term G_i(u, F, tau+-) and
//   TRT  f*_i = f_i - w+ (f+_i - feq+_i) - w- (f-_i - feq-_i) + G_i,  w+- = dt / tau+-
//   BGK  f*_i = f_i - w (f_i - feq_i) + G_i
// sum_i lam*_i d f*_i / d theta = sum_i mu_i d feq_i / d theta + sum_i lam*_i d G_i / d theta
// (+ the tau terms of w+-), where mu_i = w+ (lam*_i + lam*_opp)/2 + w- (lam*_i - lam*_opp)/2.
// Outputs: d/drho, d/du_k, d/dtau+, d/dtau-, d/dF_k (u held fixed).
template <class L, bool TRT>
__device__ __forceinline__ void collide_vjp(const double* f, const double* ls, double rho, const double* u,
                                            const AdjArgs& a, double& g_rho, double* g_u, double& g_tp,
                                            double& g_tm, double* g_F) {
    constexpr int Q = L::Q, D = L::D;
    const double dt = a.dt;
    const double wp = dt / a.tau_p, wm = TRT ? dt / a.tau_m : wp;
    const double ap = 1.0 - dt / (2.0 * a.tau_p), am = TRT ? 1.0 - dt / (2.0 * a.tau_m) : ap;
    const double dap = dt / (2.0 * a.tau_p * a.tau_p), dam = TRT ? dt / (2.0 * a.tau_m * a.tau_m) : 0.0;
    double uu = 0.0, uF = 0.0;
    for (int k = 0; k < D; ++k) {
        uu += u[k] * u[k];
        uF += u[k] * a.F[k];
    }
    g_rho = 0.0;
    g_tp = g_tm = 0.0;
    for (int k = 0; k < 3; ++k) g_u[k] = g_F[k] = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int ib = L::opp(i);
        const double c[3] = {(double)L::cx(i), (double)L::cy(i), (double)L::cz(i)};
        const double w = L::w(i);
        double uc = 0.0, cF = 0.0;
        for (int k = 0; k < D; ++k) {
            uc += u[k] * c[k];
            cF += c[k] * a.F[k];
        }
        const double second = 3.0 * uc + 4.5 * uc * uc - 1.5 * uu;
        const double scale = a.incompressible ? a.rho_inc : rho;  // the factor of the velocity terms
        const double eq = a.incompressible ? w * rho + w * a.rho_inc * second : w * rho * (1.0 + second);
        const double mu = TRT ? 0.5 * wp * (ls[i] + ls[ib]) + 0.5 * wm * (ls[i] - ls[ib]) : wp * ls[i];
        g_rho += mu * (a.incompressible ? w : w * (1.0 + second));
        for (int k = 0; k < D; ++k) g_u[k] += mu * w * scale * (3.0 * c[k] + 9.0 * uc * c[k] - 3.0 * u[k]);
        // relaxation rates: d w+-/d tau+- = -dt / tau+-^2 times -(f+- - feq+-)
        if (TRT) {
            const double eqb = a.incompressible ? w * rho + w * a.rho_inc * (3.0 * (-uc) + 4.5 * uc * uc - 1.5 * uu)
                                                : w * rho * (1.0 + (3.0 * (-uc) + 4.5 * uc * uc - 1.5 * uu));
            const double fp = 0.5 * (f[i] + f[ib]) - 0.5 * (eq + eqb), fm = 0.5 * (f[i] - f[ib]) - 0.5 * (eq - eqb);
            g_tp += ls[i] * (wp / a.tau_p) * fp;
            g_tm += ls[i] * (wm / a.tau_m) * fm;
        } else {
            g_tp += ls[i] * (wp / a.tau_p) * (f[i] - eq);
        }
        if (a.guo) {
            const double lw = ls[i] * w * dt;
            if (TRT) {
                // G = w dt [a+ (-3 u.F + 9 uc cF) + a- 3 cF]
                for (int k = 0; k < D; ++k) {
                    g_u[k] += lw * ap * (-3.0 * a.F[k] + 9.0 * c[k] * cF);
                    g_F[k] += lw * (ap * (-3.0 * u[k] + 9.0 * uc * c[k]) + am * 3.0 * c[k]);
                }
                g_tp += lw * dap * (-3.0 * uF + 9.0 * uc * cF);
                g_tm += lw * dam * 3.0 * cF;
            } else {
                // G = w dt a (3 (c - u).F + 9 uc cF)
                for (int k = 0; k < D; ++k) {
                    g_u[k] += lw * ap * (-3.0 * a.F[k] + 9.0 * c[k] * cF);
                    g_F[k] += lw * ap * (3.0 * (c[k] - u[k]) + 9.0 * uc * c[k]);
                }
                g_tp += lw * dap * (3.0 * (cF - uF) + 9.0 * uc * cF);
            }
        }
    }
}

template <class L, int ST, bool TRT>
__global__ void __launch_bounds__(kAdjBlock) k_adjoint(const AdjArgs a) {
    using SS = Store<ST>;
    using T = typename SS::T;
    constexpr int Q = L::Q, D = L::D;
    __shared__ double s_red[kAdjBlock / 32][kAdjAcc];
    const long long N = a.g.N;
    const long long cell = (long long)blockIdx.x * kAdjBlock + threadIdx.x;
    const bool active = cell < N;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    double acc[kAdjAcc];
    for (int k = 0; k < kAdjAcc; ++k) acc[k] = 0.0;
    if (active) {
        const int x = (int)(cell % nx), y = (int)((cell / nx) % ny), z = (int)(cell / ((long long)nx * ny));
        const T* __restrict__ src = static_cast<const T*>(a.src);
        double f[L::Q];
        double rho = 0.0, J[3] = {0, 0, 0};
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            f[i] = L::w(i) * ((double)SS::dec(src[i * N + cell], typename SS::R(1)) * a.inv_scale + a.rho0);
            rho += f[i];
            J[0] += f[i] * L::cx(i);
            J[1] += f[i] * L::cy(i);
            J[2] += f[i] * L::cz(i);
        }
        double u[3] = {0, 0, 0};
        const bool live = rho != 0.0;  // findFluidVelocity: u = 0 where rho == 0
        if (live)
            for (int k = 0; k < D; ++k) u[k] = (J[k] + (a.guo ? 0.5 * a.dt * a.F[k] : 0.0)) / rho;
        double fs[L::Q];
        ref_collide<L, TRT, double>(f, rho, u, a.tau_p, a.tau_m, a.F, a, fs);

        // 1. adjoint of the post-collision populations: transposed streaming
        const ParticleDev& P = *a.part;
        const bool wx = a.wall && a.wall[cell];  // a wall node: everything it streams is discarded
        const bool sx = a.has_part && solid_at(P, a.ivl, x, y, z);
        double ls[L::Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int tx = wrap_idx(x + L::cx(i), nx), ty = wrap_idx(y + L::cy(i), ny), tz = wrap_idx(z + L::cz(i), nz);
            const long long t = tx + (long long)nx * (ty + (long long)ny * tz);
            // (x + c_i, i) was overwritten by the fix-up (a particle's or a wall's link slot), or zeroed (a wall node)
            const bool slot = wx || (sx && !solid_at(P, a.ivl, tx, ty, tz)) || (a.wall && a.wall[t]);
            ls[i] = slot ? 0.0 : a.lam_in[i * N + t];
        }
        // 2. link terms of a fluid node: bounce-back, moving walls, Ladd and momentum exchange
        double mu_rho = 0.0;
        if (!wx && !sx && (a.has_part || a.wall)) {
            const double X[3] = {a.coord[0][x], a.coord[1][y], D == 3 ? a.coord[2][z] : 0.0};
            for (int j = 1; j < Q; ++j) {
                const int i = L::opp(j);
                const int sxx = wrap_idx(x + L::cx(i), nx), syy = wrap_idx(y + L::cy(i), ny),
                          szz = wrap_idx(z + L::cz(i), nz);
                const long long sc = sxx + (long long)nx * (syy + (long long)ny * szz);  // source x - c_j = x + c_i
                const bool wlink = a.wall && a.wall[sc];
                const bool plink = a.has_part && solid_at(P, a.ivl, sxx, syy, szz);
                if (!wlink && !plink) continue;
                const double cj[3] = {(double)L::cx(j), (double)L::cy(j), (double)L::cz(j)};
                const double w6 = 6.0 * L::w(j);
                const double lj = a.lam_in[j * N + cell];
                // moving wall term 6 w_j rho c_j.u_w(x - c_j) (fluids.jl:167-174)
                double cw = 0.0;
                if (wlink && a.uw)
                    for (int k = 0; k < D; ++k) cw += cj[k] * a.uw[(long long)k * N + sc];
                if (!plink) {  // a wall link only: bounce-back copy and the wall term
                    ls[i] += lj;
                    mu_rho += lj * w6 * cw;
                    continue;
                }
                const double ci[3] = {-cj[0], -cj[1], -cj[2]};
                const double Y[3] = {a.coord[0][sxx], a.coord[1][syy], D == 3 ? a.coord[2][szz] : 0.0};
                double up[3];
                slip_velocity_t<D, double>(P.sR, P.sV, P.sW, P.sE, P.B1, P.B2, P.kind, Y[0], Y[1], Y[2], up);
                const double cu = cj[0] * up[0] + cj[1] * up[1] + cj[2] * up[2] + cw;  // Ladd and wall terms
                const double s = 2.0 * fs[i] + w6 * rho * cu;  // f*_i + f^{n+1}_j
                double lsi = lj, gmu = lj * w6 * cu, gup = lj * w6 * rho;  // lam_up = gup * c_j
                if (P.coupleF || P.recordF) {
                    const double t = a.coeff * (a.lamF[0] * ci[0] + a.lamF[1] * ci[1] + a.lamF[2] * ci[2]);
                    lsi += 2.0 * t;
                    gmu += t * w6 * cu;
                    gup += t * w6 * rho;
                }
                if (P.coupleT) {
                    const double r[3] = {X[0] - P.mR[0], X[1] - P.mR[1], D == 3 ? X[2] - P.mR[2] : 0.0};
                    double tq;
                    if (D == 2) {
                        tq = a.lamT[0] * (r[0] * ci[1] - r[1] * ci[0]);
                        // d/dr (r0 c1 - r1 c0) = (c1, -c0); the arm is x - mR
                        acc[19] -= a.coeff * s * a.lamT[0] * ci[1];
                        acc[20] += a.coeff * s * a.lamT[0] * ci[0];
                    } else {
                        const double rc[3] = {r[1] * ci[2] - r[2] * ci[1], r[2] * ci[0] - r[0] * ci[2],
                                              r[0] * ci[1] - r[1] * ci[0]};
                        tq = a.lamT[0] * rc[0] + a.lamT[1] * rc[1] + a.lamT[2] * rc[2];
                        // d/dr lamT.(r x c) = c x lamT
                        const double cl[3] = {ci[1] * a.lamT[2] - ci[2] * a.lamT[1],
                                              ci[2] * a.lamT[0] - ci[0] * a.lamT[2],
                                              ci[0] * a.lamT[1] - ci[1] * a.lamT[0]};
                        for (int k = 0; k < 3; ++k) acc[19 + k] -= a.coeff * s * cl[k];
                    }
                    const double t = a.coeff * tq;
                    lsi += 2.0 * t;
                    gmu += t * w6 * cu;
                    gup += t * w6 * rho;
                }
                ls[i] += lsi;
                mu_rho += gmu;
                // slip velocity: its dependence on the snapshot (sR, sV, sW, sE) and on B1, B2
                const double lup[3] = {gup * cj[0], gup * cj[1], gup * cj[2]};
                for (int q = 0; q < 14; ++q) {
                    DD1 R_[3], V_[3], W_[3], E_[3];
                    for (int k = 0; k < 3; ++k) {
                        R_[k] = dd(P.sR[k], q == k ? 1.0 : 0.0);
                        V_[k] = dd(P.sV[k], q == 3 + k ? 1.0 : 0.0);
                        W_[k] = dd(P.sW[k], q == 6 + k ? 1.0 : 0.0);
                        E_[k] = dd(P.sE[k], q == 9 + k ? 1.0 : 0.0);
                    }
                    DD1 o[3];
                    slip_velocity_t<D, DD1>(R_, V_, W_, E_, dd(P.B1, q == 12 ? 1.0 : 0.0),
                                            dd(P.B2, q == 13 ? 1.0 : 0.0), P.kind, Y[0], Y[1], Y[2], o);
                    acc[5 + q] += lup[0] * o[0].d + lup[1] * o[1].d + lup[2] * o[2].d;
                }
            }
        }
        // 3. transposed collision at fixed f, then the chain through rho(f), u(f)
        double mu_u[3] = {0, 0, 0};
        {
            double g_rho, g_tp, g_tm, g_F[3];
            collide_vjp<L, TRT>(f, ls, rho, u, a, g_rho, mu_u, g_tp, g_tm, g_F);
            if (live) mu_rho += g_rho;
            else mu_u[0] = mu_u[1] = mu_u[2] = 0.0;
            acc[0] += g_tp;
            acc[1] += TRT ? g_tm : 0.0;
            for (int k = 0; k < D; ++k) acc[2 + k] += g_F[k];
        }
        if (live && a.guo)
            for (int k = 0; k < D; ++k) acc[2 + k] += mu_u[k] * 0.5 * a.dt / rho;  // u = (J + dt F / 2) / rho
        const double op = a.dt / a.tau_p, om = TRT ? a.dt / a.tau_m : op;
        const double hs = 1.0 - 0.5 * (op + om), hd = 0.5 * (om - op);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            double v = hs * ls[i] + hd * ls[L::opp(i)] + mu_rho;
            if (live) {
                const int c[3] = {L::cx(i), L::cy(i), L::cz(i)};
                for (int k = 0; k < D; ++k) v += mu_u[k] * ((double)c[k] - u[k]) / rho;
            }
            a.lam_out[i * N + cell] = v;
        }
    }
    // fixed-order reduction of the accumulators of this CTA
    for (int k = 0; k < kAdjAcc; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < kAdjAcc) {
        double v = 0.0;
        for (int w = 0; w < kAdjBlock / 32; ++w) v += s_red[w][threadIdx.x];
        a.partial[(long long)blockIdx.x * kAdjAcc + threadIdx.x] = v;
    }
}

// d/dF of the initial populations f^0 = feq(rho, u0 - dt F / (2 rho))
// (findInitialConditions, initMethods.jl:417-438), contracted with lam^0
template <class L, int ST>
__global__ void __launch_bounds__(kAdjBlock) k_adjoint_init(const AdjArgs a) {
    using SS = Store<ST>;
    using T = typename SS::T;
    constexpr int Q = L::Q, D = L::D;
    __shared__ double s_red[kAdjBlock / 32][3];
    const long long N = a.g.N;
    const long long cell = (long long)blockIdx.x * kAdjBlock + threadIdx.x;
    double acc[3] = {0, 0, 0};
    if (cell < N && a.guo) {
        const T* __restrict__ src = static_cast<const T*>(a.src);
        double rho = 0.0, J[3] = {0, 0, 0};
        for (int i = 0; i < Q; ++i) {
            const double fi = L::w(i) * ((double)SS::dec(src[i * N + cell], typename SS::R(1)) * a.inv_scale + a.rho0);
            rho += fi;
            J[0] += fi * L::cx(i);
            J[1] += fi * L::cy(i);
            J[2] += fi * L::cz(i);
        }
        if (rho != 0.0) {
            for (int k = 0; k < D; ++k) {
                double g = 0.0;
                for (int i = 0; i < Q; ++i) {  // d feq_i / d u_k at (rho, J / rho)
                    const int c[3] = {L::cx(i), L::cy(i), L::cz(i)};
                    double uc = 0.0;
                    for (int q = 0; q < D; ++q) uc += (J[q] / rho) * c[q];
                    const double dsec = 3.0 * c[k] + 9.0 * uc * c[k] - 3.0 * (J[k] / rho);
                    const double dfeq = a.incompressible ? L::w(i) * a.rho_inc * dsec : L::w(i) * rho * dsec;
                    g += a.lam_in[i * N + cell] * dfeq;
                }
                acc[k] = g * (-0.5 * a.dt / rho);
            }
        }
    }
    for (int k = 0; k < 3; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < kAdjAcc) {
        double v = 0.0;
        if (threadIdx.x < 3)
            for (int w = 0; w < kAdjBlock / 32; ++w) v += s_red[w][threadIdx.x];
        a.partial[(long long)blockIdx.x * kAdjAcc + threadIdx.x] = v;
    }
}

// Sum of the per-CTA accumulators, one CTA per accumulator: thread t adds
// the CTAs t, t + 256, ... in order, then a fixed tree over the threads, so
// the result does not depend on scheduling.
constexpr int kSumBlock = 256;
template <int NA>
__global__ void __launch_bounds__(kSumBlock) k_adjoint_sum(const double* __restrict__ partial, long long nblocks,
                                                          double* out) {
    __shared__ double s[kSumBlock];
    const int k = blockIdx.x;
    double v = 0.0;
    for (long long b = threadIdx.x; b < nblocks; b += kSumBlock) v += partial[b * NA + k];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int w = kSumBlock / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[k] = s[0];
}

}  // namespace lbm
