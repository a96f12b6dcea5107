/*
 * lbm_oracle.cpp — FP64 CPU restatement of LBMengine.jl's GPU-module time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  It is never part of the product path.
 *
 * Parity status: UNPINNED by the reference itself.  The reference ships no
 * tests, golden vectors or fixtures (test/runtests.jl:1 is a println) and its
 * toolchain (Julia + CUDA.jl) is not available here, so this restatement is
 * pinned instead by known-answer tests of the physics (velocity-set moments,
 * equilibrium moments, conservation, analytic shear-wave decay, Poiseuille
 * profile) and by the direction tables read from the reference source text.
 *
 * Semantics followed, function by function (paths inside the reference):
 *   modelInit                 src/gpu/initMethods.jl:440-702
 *   findInitialConditions     src/gpu/initMethods.jl:417-438
 *   addBead! / addSquirmer!   src/gpu/initMethods.jl:7-89 / :91-222
 *   hydroVariablesUpdate!     src/gpu/fluids.jl:7-37, findFluidVelocity src/gpu/aux.jl:169-179
 *   equilibriumDistribution   src/gpu/fluids.jl:39-52
 *   collisionStep             src/gpu/fluids.jl:58-101
 *   guoForcingTerm            src/gpu/fluids.jl:103-127
 *   tick!                     src/gpu/fluids.jl:132-226 (stream, bounce-back, moving walls, Ladd)
 *   bounceBackPrep            src/gpu/aux.jl:187-198
 *   getSphere                 src/gpu/aux.jl:206-215, kernels src/gpu/kernels.jl:335-353
 *   getNodeVelocity           src/gpu/aux.jl:229-263, kernels src/gpu/kernels.jl:376-415
 *   moveParticles!            src/gpu/particles.jl:7-92
 *   cross (2D/3D)             src/gpu/aux.jl:139-157
 *   viscousStressTensor       src/cpu/fluids.jl:507-520 (nonEquilibriumDistribution :65-67)
 *   molecularDynamicsTick!    src/gpu/particles.jl:100-197 (applyInteraction!, per interaction kind)
 * CPU-module particle rules (lbm_config.particle_rules == LBM_RULES_CPU_MODULE):
 *   moveParticles! / eulerStep!  src/cpu/particles.jl:7-18, :48-100
 *   bulkVelocity              src/cpu/particles.jl:21-46, cross src/cpu/aux.jl:19-28
 *   Ladd momentum inputs      src/cpu/fluids.jl:423-438 (per-direction inputs, summed)
 * Floating-point operations are written in the reference's evaluation order
 * (left to right, no fused multiply-add: build with -ffp-contract=off).
 * Reductions the reference does with CUDA.jl parallel sums are done here
 * sequentially in column-major cell order.
 *
 * The model is a template on its scalar type.  With `double` it is the FP64
 * oracle (orc_* entry points).  With Dual<kDirs> (forward-mode dual numbers,
 * value + kDirs directional derivatives) it carries the derivatives of the
 * whole trajectory with respect to seeded parameters (ord_* entry points):
 * the value parts follow exactly the operations of the FP64 run, every
 * comparison (masks, zero tests) looks at the value part only, so the
 * derivatives are those of the reference's tick with its solid masks held as
 * computed.  The reference's CPU module is hard-typed Float64
 * (src/cpu/structs.jl:14-37), so dual numbers cannot flow through the Julia
 * code itself; they flow through this restatement.
 */
#include "lbm_b200.h"
#include "lattice_tables.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace lbm_oracle;

namespace {

thread_local std::string g_err;

// ---- forward-mode dual numbers ---------------------------------------------
constexpr int kDirs = 6;  // derivative directions carried by the dual oracle

template <int K>
struct Dual {
    double v = 0.0;
    double d[K] = {};
    Dual() = default;
    Dual(double x) : v(x) {}  // NOLINT: constants enter as duals with zero derivatives
    Dual& operator+=(const Dual& o) { v += o.v; for (int k = 0; k < K; ++k) d[k] += o.d[k]; return *this; }
    Dual& operator-=(const Dual& o) { v -= o.v; for (int k = 0; k < K; ++k) d[k] -= o.d[k]; return *this; }
};
template <int K> Dual<K> operator+(Dual<K> a, const Dual<K>& b) { a += b; return a; }
template <int K> Dual<K> operator-(Dual<K> a, const Dual<K>& b) { a -= b; return a; }
template <int K> Dual<K> operator-(const Dual<K>& a) { Dual<K> r; r.v = -a.v; for (int k = 0; k < K; ++k) r.d[k] = -a.d[k]; return r; }
template <int K> Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r; r.v = a.v * b.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int K> Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r; r.v = a.v / b.v;
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
    return r;
}
template <int K> Dual<K> operator+(Dual<K> a, double b) { a.v += b; return a; }
template <int K> Dual<K> operator+(double b, Dual<K> a) { a.v = b + a.v; return a; }
template <int K> Dual<K> operator-(Dual<K> a, double b) { a.v -= b; return a; }
template <int K> Dual<K> operator-(double b, const Dual<K>& a) { return Dual<K>(b) - a; }
template <int K> Dual<K> operator*(Dual<K> a, double b) { a.v *= b; for (int k = 0; k < K; ++k) a.d[k] *= b; return a; }
template <int K> Dual<K> operator*(double b, Dual<K> a) { a.v = b * a.v; for (int k = 0; k < K; ++k) a.d[k] = b * a.d[k]; return a; }
template <int K> Dual<K> operator/(Dual<K> a, double b) { a.v /= b; for (int k = 0; k < K; ++k) a.d[k] /= b; return a; }
template <int K> Dual<K> operator/(double b, const Dual<K>& a) { return Dual<K>(b) / a; }
template <int K> bool operator==(const Dual<K>& a, double b) { return a.v == b; }
template <int K> bool operator!=(const Dual<K>& a, double b) { return a.v != b; }
template <int K> Dual<K> sqrt(const Dual<K>& a) {
    Dual<K> r; r.v = std::sqrt(a.v);
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] / (2.0 * r.v);
    return r;
}
template <int K> Dual<K> fabs(const Dual<K>& a) { return a.v < 0 ? -a : a; }
template <int K> Dual<K> sin(const Dual<K>& a) {
    Dual<K> r; r.v = std::sin(a.v); const double c = std::cos(a.v);
    for (int k = 0; k < K; ++k) r.d[k] = c * a.d[k];
    return r;
}
template <int K> Dual<K> cos(const Dual<K>& a) {
    Dual<K> r; r.v = std::cos(a.v); const double sn = std::sin(a.v);
    for (int k = 0; k < K; ++k) r.d[k] = -sn * a.d[k];
    return r;
}
inline double val(double x) { return x; }
inline double acos_(double x) { return std::acos(x); }
template <int K> Dual<K> acos_(const Dual<K>& a) {
    Dual<K> r;
    r.v = std::acos(a.v);
    const double g = -1.0 / std::sqrt(1.0 - a.v * a.v);
    for (int k = 0; k < K; ++k) r.d[k] = g * a.d[k];
    return r;
}
template <int K> double val(const Dual<K>& x) { return x.v; }
using std::cos;
using std::fabs;
using std::sin;
using std::sqrt;
using D6 = Dual<kDirs>;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

template <class Real>
struct Particle {
    int id = 0;
    int kind = LBM_SQUIRMER;
    bool couple_f = false, couple_t = false;
    bool record_f = false;  // accumulate the momentum-exchange force without applying it (force observable)
    double radius = 0;
    Real B1 = 0, B2 = 0;
    double inv_mass = 0, inv_inertia = 0;
    Real R[3] = {0, 0, 0}, v[3] = {0, 0, 0}, w[3] = {0, 0, 0}, e[3] = {0, 0, 0};
    Real F[3] = {0, 0, 0}, T[3] = {0, 0, 0};  // forceInput / torqueInput
    Real lastF[3] = {0, 0, 0}, lastT[3] = {0, 0, 0};
    std::vector<uint8_t> S;  // solidRegion
    std::vector<int64_t> solid;  // cells with S set, ascending
    // CPU-module rules: momentumInput / angularMomentumInput, one slot per
    // streaming direction (src/cpu/fluids.jl:434-437), summed at the move
    std::vector<std::array<Real, 3>> dP, dL;
    // state captured by the last getNodeVelocity call (nodeVelocity is a
    // function of it, evaluated on demand)
    Real nvR[3] = {0, 0, 0}, nvV[3] = {0, 0, 0}, nvW[3] = {0, 0, 0}, nvE[3] = {0, 0, 0};
};

template <class Real>
struct Model {
    int dims = 0;
    VelocitySet vs;
    int64_t n[3] = {1, 1, 1};
    int64_t N = 0;
    std::vector<double> X[3];
    double dx = 1, dt = 1;
    Real tau = 1, tau_plus = 1, tau_minus = 1;
    double invC2 = 3, invC4 = 9;
    bool trt = false, compressible = true;
    bool bounce_back = false, moving_walls = false, guo = false, ladd = false;
    std::vector<Real> f, rho, u, F, rho0;
    std::vector<double> uw;
    std::vector<uint8_t> W;
    std::vector<Particle<Real>> parts;
    int64_t tick = 0;
    double time = 0;
    int rules = LBM_RULES_GPU_MODULE;
    std::vector<lbm_interaction> inter;  // particleInteractions, pairs flattened in order
    // bit id of wmark[c]: c is fluid and c - c_id a wall node (the walls'
    // streamingInvasionRegions of the opposite direction); mark[c] adds the
    // particles' regions for the current tick
    std::vector<uint32_t> wmark, mark;
    // wrapped index of i + s along axis a: wrap[a][s + 1][i], s in {-1, 0, 1}
    std::vector<int64_t> wrap[3][3];

    void build_wrap() {
        for (int a = 0; a < 3; ++a)
            for (int s = -1; s <= 1; ++s) {
                auto& t = wrap[a][s + 1];
                t.resize(n[a]);
                for (int64_t i = 0; i < n[a]; ++i) t[i] = ((i + s) % n[a] + n[a]) % n[a];
            }
    }

    int64_t cell(int64_t x, int64_t y, int64_t z) const { return x + n[0] * (y + n[1] * z); }
    void coords(int64_t c, int64_t& x, int64_t& y, int64_t& z) const {
        x = c % n[0];
        y = (c / n[0]) % n[1];
        z = c / (n[0] * n[1]);
    }
    // index of the node at c + s (periodic, mod1 semantics of circshift)
    int64_t shifted(int64_t c, int sx, int sy, int sz) const {
        int64_t x, y, z;
        coords(c, x, y, z);
        x = ((x + sx) % n[0] + n[0]) % n[0];
        y = ((y + sy) % n[1] + n[1]) % n[1];
        z = ((z + sz) % n[2] + n[2]) % n[2];
        return cell(x, y, z);
    }
    double coord(int a, int64_t c) const {
        int64_t x, y, z;
        coords(c, x, y, z);
        int64_t idx = a == 0 ? x : (a == 1 ? y : z);
        return X[a][idx];
    }
};

// getSphere: ((X1-R1)^2 + (X2-R2)^2 [+ (X3-R3)^2]) < r^2, kernels.jl:335-353.
// X + (-R) equals X - R exactly in IEEE arithmetic.  The test is a comparison:
// it uses the value part of the position.
template <class Real>
inline bool in_sphere(const Model<Real>& m, int64_t x, int64_t y, int64_t z, const Real* R, double r2) {
    double a = m.X[0][x] - val(R[0]);
    double b = m.X[1][y] - val(R[1]);
    double s = a * a + b * b;
    if (m.dims == 3) {
        double c = m.X[2][z] - val(R[2]);
        s = s + c * c;
    }
    return s < r2;
}

// per-axis index range that can satisfy the sphere test (conservative and
// exact: fl(a*a) <= the full rounded sum, so nodes outside fail the test too)
template <class Real>
void axis_range(const Model<Real>& m, int a, double Ra, double r2, int64_t& lo, int64_t& hi) {
    lo = m.n[a];
    hi = -1;
    for (int64_t i = 0; i < m.n[a]; ++i) {
        double d = m.X[a][i] - Ra;
        if (d * d < r2) {
            lo = std::min(lo, i);
            hi = std::max(hi, i);
        }
    }
}

template <class Real>
void get_sphere(const Model<Real>& m, double radius, const Real* R, std::vector<uint8_t>& S,
                std::vector<int64_t>* solid = nullptr) {
    S.assign(m.N, 0);
    if (solid) solid->clear();
    double r2 = radius * radius;
    int64_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int a = 0; a < m.dims; ++a) axis_range(m, a, val(R[a]), r2, lo[a], hi[a]);
    if (m.dims == 2) { lo[2] = 0; hi[2] = 0; }
    for (int64_t z = lo[2]; z <= hi[2]; ++z)
        for (int64_t y = lo[1]; y <= hi[1]; ++y)
            for (int64_t x = lo[0]; x <= hi[0]; ++x)
                if (in_sphere(m, x, y, z, R, r2)) {
                    S[m.cell(x, y, z)] = 1;
                    if (solid) solid->push_back(m.cell(x, y, z));
                }
}

// dot of a vector with a lattice vector, vectorFieldDotVector (kernels.jl:198-224):
// sumTerm = 0 then += v_k * c_k in component order
template <class V>
inline V dot_c(const V* v, const std::array<int, 3>& c, int dims) {
    V s = 0.0;
    for (int k = 0; k < dims; ++k) s += v[k] * (double)c[k];
    return s;
}

// getNodeVelocity evaluated at node y (aux.jl:229-263, kernels.jl:376-415)
template <class Real>
void node_velocity(const Model<Real>& m, const Particle<Real>& p, int64_t y, Real* out) {
    int d = m.dims;
    Real xr[3] = {0, 0, 0};
    for (int k = 0; k < d; ++k) xr[k] = m.coord(k, y) + (-p.nvR[k]);
    Real nrm2 = 0.0;
    for (int k = 0; k < d; ++k) nrm2 += xr[k] * xr[k];
    Real nrm = sqrt(nrm2);
    if (nrm == 0) nrm = 1;
    Real bulk[3];
    if (d == 2) {
        bulk[0] = p.nvV[0] - p.nvW[0] * xr[1];
        bulk[1] = p.nvV[1] + p.nvW[0] * xr[0];
    } else {
        bulk[0] = p.nvV[0] + p.nvW[1] * xr[2] - p.nvW[2] * xr[1];
        bulk[1] = p.nvV[1] - p.nvW[0] * xr[2] + p.nvW[2] * xr[0];
        bulk[2] = p.nvV[2] + p.nvW[0] * xr[1] - p.nvW[1] * xr[0];
    }
    if (p.kind == LBM_BEAD) {
        for (int k = 0; k < d; ++k) out[k] = bulk[k];
        return;
    }
    Real inv = 1.0 / nrm;
    Real ur[3];
    for (int k = 0; k < d; ++k) ur[k] = inv * xr[k];
    Real edr = 0.0;
    for (int k = 0; k < d; ++k) edr += ur[k] * p.nvE[k];
    Real first = p.B1 + p.B2 * edr;
    for (int k = 0; k < d; ++k) {
        Real second = edr * ur[k] + (-p.nvE[k]);
        out[k] = first * second + bulk[k];
    }
}

template <class Real>
void capture_node_velocity(Particle<Real>& p) {
    for (int k = 0; k < 3; ++k) {
        p.nvR[k] = p.R[k];
        p.nvV[k] = p.v[k];
        p.nvW[k] = p.w[k];
        p.nvE[k] = p.e[k];
    }
}

// hydroVariablesUpdate! (fluids.jl:7-37): rho = sum_i f_i ; rho*u = sum_i f_i c_i
// (+ dt/2 F with Guo) ; u = rho*u / rho unless rho == 0 (isapprox with atol 0)
template <class Real>
void hydro(Model<Real>& m) {
    const int64_t N = m.N;
    const int d = m.dims, Q = m.vs.q;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        Real r = 0.0;
        for (int i = 0; i < Q; ++i) r = (i == 0) ? m.f[c] : r + m.f[(int64_t)i * N + c];
        m.rho[c] = r;
        for (int k = 0; k < d; ++k) {
            Real j = 0.0;
            for (int i = 0; i < Q; ++i) {
                Real t = m.f[(int64_t)i * N + c] * (double)m.vs.c[i][k];
                j = (i == 0) ? t : j + t;
            }
            if (m.guo) j = j + (0.5 * m.dt) * m.F[(int64_t)k * N + c];
            m.u[(int64_t)k * N + c] = (r == 0.0) ? Real(0.0) : j / r;
        }
    }
}

// Relaxation and Guo prefactors of one tick.  The reference evaluates them
// inside its per-node expressions; each is the same rounded value at every
// node, so computing it once gives the same results.
template <class Real>
struct CollideConsts {
    Real om, om_p, om_m;      // -dt/tau, -dt/tau+, -dt/tau-
    Real kb, kp, km;          // 1 - dt/(2 tau), 1 - dt/(2 tau+), 1 - dt/(2 tau-)
};

template <class Real>
CollideConsts<Real> collide_consts(const Model<Real>& m) {
    CollideConsts<Real> k;
    k.om = -m.dt / m.tau;
    k.om_p = -m.dt / m.tau_plus;
    k.om_m = -m.dt / m.tau_minus;
    k.kb = 1 - m.dt / (2 * m.tau);
    k.kp = 1 - m.dt / (2 * m.tau_plus);
    k.km = 1 - m.dt / (2 * m.tau_minus);
    return k;
}

// collisionStep (fluids.jl:58-101) with equilibriumDistribution (:39-52) and
// guoForcingTerm (:103-127) at one cell: fs_i = f_i + Omega_i (+ G_i).
// Per direction, with uc = u.c_i and uu = u.u (sums from 0 in component order):
//   f_eq = w ((uc/cs2 + uc^2/(2 cs4) - uu/(2 cs2) + 1) rho)            compressible
//        = w rho + w (rho0 (uc/cs2 + uc^2/(2 cs4) - uu/(2 cs2)))       incompressible
//   BGK  Omega = (-dt/tau)(f - f_eq),
//        G = w dt (1 - dt/2tau) sum_k ((c_k - u_k)/cs2 + uc c_k/cs4) F_k
//   TRT  Omega = (-dt/tau+)(f+ - f_eq+) + (-dt/tau-)(f- - f_eq-),
//        G = w dt ((1 - dt/2tau+) sum_k (-u_k/cs2 + uc c_k/cs4) F_k
//                 + (1 - dt/2tau-) sum_k F_k c_k/cs2)
// The products u.c_i and u.u are the same values in the equilibrium and in
// the Guo term; each is computed once per cell.
template <class Real>
inline void collide_cell(const Model<Real>& m, const CollideConsts<Real>& K, int64_t c, Real* out) {
    const int64_t N = m.N;
    const int d = m.dims, Q = m.vs.q;
    Real U[3] = {0, 0, 0}, Fv[3] = {0, 0, 0}, f[27], eq[27], uc[27];
    for (int k = 0; k < d; ++k) U[k] = m.u[(int64_t)k * N + c];
    if (m.guo)
        for (int k = 0; k < d; ++k) Fv[k] = m.F[(int64_t)k * N + c];
    Real uu = 0.0;
    for (int k = 0; k < d; ++k) uu += U[k] * U[k];
    const Real rho = m.rho[c];
    for (int i = 0; i < Q; ++i) {
        f[i] = m.f[(int64_t)i * N + c];
        Real x = 0.0;
        for (int k = 0; k < d; ++k) x += U[k] * (double)m.vs.c[i][k];
        uc[i] = x;
        Real first = x * m.invC2 + (x * x) * (0.5 * m.invC4);
        Real second = first - uu * (0.5 * m.invC2);
        const double wi = m.vs.w[i];
        eq[i] = m.compressible ? wi * ((second + 1) * rho) : wi * rho + wi * (m.rho0[c] * second);
    }
    for (int i = 0; i < Q; ++i) {
        const Real fi = f[i];
        Real om;
        if (!m.trt) {
            om = K.om * (fi - eq[i]);
        } else {
            const int ib = m.vs.opp[i];
            const Real fb = f[ib];
            Real fp = 0.5 * (fi + fb), fm = 0.5 * (fi - fb);
            Real ep = 0.5 * (eq[i] + eq[ib]), em = 0.5 * (eq[i] - eq[ib]);
            om = K.om_p * (fp - ep) + K.om_m * (fm - em);
        }
        if (m.guo) {
            const auto& ci = m.vs.c[i];
            const double wi = m.vs.w[i];
            Real G;
            if (!m.trt) {
                Real inter = 0.0;
                for (int k = 0; k < d; ++k) {
                    Real second = (uc[i] * (double)ci[k]) * m.invC4;
                    Real first = ((-U[k]) + (double)ci[k]) * m.invC2;
                    inter += (first + second) * Fv[k];
                }
                G = wi * m.dt * K.kb * inter;
            } else {
                Real inter = 0.0;
                for (int k = 0; k < d; ++k) {
                    Real second = (uc[i] * (double)ci[k]) * m.invC4;
                    inter += ((-U[k]) * m.invC2 + second) * Fv[k];
                }
                Real plus = K.kp * inter;
                Real inter2 = 0.0;
                for (int k = 0; k < d; ++k) inter2 += Fv[k] * ((double)ci[k] * m.invC2);
                Real minus = K.km * inter2;
                G = wi * m.dt * (plus + minus);
            }
            om = om + G;
        }
        out[i] = om + fi;
    }
}

template <class Real>
void collision(const Model<Real>& m, std::vector<Real>& fs) {
    const int64_t N = m.N;
    const int Q = m.vs.q;
    const CollideConsts<Real> K = collide_consts(m);
    fs.resize((size_t)N * Q);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        Real out[27];
        collide_cell(m, K, c, out);
        for (int i = 0; i < Q; ++i) fs[(int64_t)i * N + c] = out[i];
    }
}

// streamingInvasionRegions[j](x) = S(x + c_j) && !S(x)   (aux.jl:190)
template <class Real>
inline bool invasion(const Model<Real>& m, const std::vector<uint8_t>& S, int j, int64_t c) {
    if (S[c]) return false;
    const auto& cj = m.vs.c[j];
    return S[m.shifted(c, cj[0], cj[1], cj[2])] != 0;
}

// 2D/3D cross product of the reference (aux.jl:139-145)
template <class A, class B, class C>
void cross_ref(int d, const A* v, const B* w, C* out) {
    if (d == 2) {
        out[0] = v[0] * w[1] - v[1] * w[0];
    } else {
        out[0] = v[1] * w[2] - v[2] * w[1];
        out[1] = -v[0] * w[2] + v[2] * w[0];
        out[2] = v[0] * w[1] - v[1] * w[0];
    }
}

// sorted fluid cells x with x - c_id in S and x not in S (conjugate boundary nodes),
// from the particle's solid cells (the same set as a scan of the whole grid)
template <class Real>
void particle_links(const Model<Real>& m, const Particle<Real>& p, int id, std::vector<int64_t>& out) {
    out.clear();
    const auto& ci = m.vs.c[id];
    if (ci[0] == 0 && ci[1] == 0 && ci[2] == 0) return;
    for (int64_t y : p.solid) {
        const int64_t x = m.shifted(y, ci[0], ci[1], ci[2]);
        if (!p.S[x]) out.push_back(x);
    }
    std::sort(out.begin(), out.end());
}

// bulkVelocity of the CPU module at node y (src/cpu/particles.jl:21-46), with
// the state captured at the last node-velocity update: v + cross(w, x - R)
// (cross of src/cpu/aux.jl:19-28; in 2D the scalar w acts as (0, 0, w)), plus
// the squirmer slip (B1 + B2 e.r)((e.r) r - e) with r = (x - R)/|x - R|.
// `norm` is LinearAlgebra's generic 2-norm (0 for a zero vector); `dot` is
// summed in component order.  Nodes farther than 2 dx from the surface get
// zero (:25), which no boundary link reaches: a solid node next to a fluid
// node lies within sqrt(d) dx of the surface.
template <class Real>
void node_velocity_cpu(const Model<Real>& m, const Particle<Real>& p, int64_t y, Real* out) {
    const int d = m.dims;
    Real xr[3] = {0, 0, 0};
    for (int k = 0; k < d; ++k) xr[k] = m.coord(k, y) - p.nvR[k];
    double mx = 0.0;
    for (int k = 0; k < d; ++k) mx = std::max(mx, std::fabs(val(xr[k])));
    Real nrm = 0.0;
    if (mx != 0.0) {
        Real s2 = xr[0] * xr[0];
        for (int k = 1; k < d; ++k) s2 += xr[k] * xr[k];
        nrm = sqrt(s2);
    }
    if (std::fabs(val(nrm) - p.radius) > 2 * m.dx) {
        for (int k = 0; k < d; ++k) out[k] = 0.0;
        return;
    }
    Real bulk[3];
    if (d == 2) {
        Real c0 = 0.0 * 0.0 - p.nvW[0] * xr[1];
        Real c1 = (-0.0) * 0.0 + p.nvW[0] * xr[0];
        bulk[0] = p.nvV[0] + c0;
        bulk[1] = p.nvV[1] + c1;
    } else {
        Real c0 = p.nvW[1] * xr[2] - p.nvW[2] * xr[1];
        Real c1 = (-p.nvW[0]) * xr[2] + p.nvW[2] * xr[0];
        Real c2 = p.nvW[0] * xr[1] - p.nvW[1] * xr[0];
        bulk[0] = p.nvV[0] + c0;
        bulk[1] = p.nvV[1] + c1;
        bulk[2] = p.nvV[2] + c2;
    }
    if (p.kind == LBM_BEAD || nrm == 0.0) {
        for (int k = 0; k < d; ++k) out[k] = bulk[k];
        return;
    }
    Real fr[3];
    for (int k = 0; k < d; ++k) fr[k] = xr[k] / nrm;
    Real edr = p.nvE[0] * fr[0];
    for (int k = 1; k < d; ++k) edr += p.nvE[k] * fr[k];
    Real first = p.B1 + p.B2 * edr;
    for (int k = 0; k < d; ++k) {
        Real second = edr * fr[k] - p.nvE[k];
        out[k] = first * second + bulk[k];
    }
}

// moveParticles! (particles.jl:7-92)
template <class Real>
void move_particle(Model<Real>& m, Particle<Real>& p, bool initial) {
    const int d = m.dims;
    bool moved = initial, need_nv = initial;
    if (!initial) {
        if (p.couple_f) {
            Real A[3];
            for (int k = 0; k < d; ++k) A[k] = p.F[k] * p.inv_mass;
            // the tick == 0 half step (particles.jl:19) is unreachable: tick! has
            // already incremented model.tick when it calls moveParticles!
            for (int k = 0; k < d; ++k) p.v[k] = p.v[k] + m.dt * A[k];
            for (int k = 0; k < d; ++k) p.R[k] = p.R[k] + m.dt * p.v[k];
            for (int k = 0; k < d; ++k)
                if (p.v[k] != 0.0) moved = true;
        }
        if (p.couple_t) {
            int nw = d == 2 ? 1 : 3;
            Real Al[3];
            for (int k = 0; k < nw; ++k) Al[k] = p.T[k] * p.inv_inertia;
            for (int k = 0; k < nw; ++k) p.w[k] = p.w[k] + m.dt * Al[k];
            if (p.kind == LBM_SQUIRMER) {
                Real theta;
                if (d == 2) {
                    theta = fabs(p.w[0]);
                } else {
                    Real s = 0.0;
                    for (int k = 0; k < 3; ++k) s += p.w[k] * p.w[k];
                    theta = sqrt(s);
                }
                if (theta != 0.0) {  // !(theta ≈ 0) with atol 0
                    Real vr[3] = {0, 0, 0};
                    const Real* v = p.e;
                    if (d == 2) {
                        Real k = p.w[0] / theta;
                        theta = theta * m.dt;
                        Real cr[2] = {-k * v[1], k * v[0]};
                        Real ct = cos(theta), st = sin(theta);
                        for (int q = 0; q < 2; ++q) vr[q] = v[q] * ct + cr[q] * st;
                    } else {
                        Real k[3];
                        for (int q = 0; q < 3; ++q) k[q] = p.w[q] / theta;
                        theta = theta * m.dt;
                        Real cr[3];
                        cross_ref(3, k, v, cr);
                        Real ct = cos(theta), st = sin(theta);
                        for (int q = 0; q < 3; ++q) vr[q] = v[q] * ct + cr[q] * st;
                        Real kv = 0.0;
                        for (int q = 0; q < 3; ++q) kv += k[q] * v[q];
                        for (int q = 0; q < 3; ++q) vr[q] = vr[q] + k[q] * kv * (1 - ct);
                    }
                    Real s = 0.0;
                    for (int q = 0; q < d; ++q) s += vr[q] * vr[q];
                    Real nr = sqrt(s);
                    for (int q = 0; q < d; ++q) p.e[q] = vr[q] / nr;
                }
            }
            for (int k = 0; k < nw; ++k)
                if (Al[k] != 0.0) need_nv = true;
        }
        need_nv = moved || need_nv;
    }
    for (int k = 0; k < 3; ++k) {
        p.lastF[k] = p.F[k];
        p.lastT[k] = p.T[k];
        p.F[k] = 0;
        p.T[k] = 0;
    }
    if (moved) get_sphere(m, p.radius, p.R, p.S, &p.solid);
    if (need_nv) capture_node_velocity(p);
}

// moveParticles! of the CPU module (src/cpu/particles.jl:48-100): the inputs
// of all directions summed in direction order, v += m^-1 dP, w += I^-1 dL, an
// Euler step R += dt v whenever v != 0 (eulerStep!, :7-18: spherical
// particles never rotate), node velocities refreshed when dL != 0 or the
// particle moved.  last force/torque report dP and dL.
template <class Real>
void move_particle_cpu(Model<Real>& m, Particle<Real>& p, bool initial) {
    const int d = m.dims, nw = d == 2 ? 1 : 3, Q = m.vs.q;
    bool moved = initial, need_nv = initial;
    Real dP[3] = {0, 0, 0}, dL[3] = {0, 0, 0};
    if (!p.dP.empty()) {
        for (int k = 0; k < 3; ++k) {
            dP[k] = p.dP[0][k] + p.dP[1][k];
            dL[k] = p.dL[0][k] + p.dL[1][k];
            for (int id = 2; id < Q; ++id) {
                dP[k] += p.dP[id][k];
                dL[k] += p.dL[id][k];
            }
        }
    }
    if (!initial) {
        for (int k = 0; k < d; ++k) p.v[k] = p.v[k] + p.inv_mass * dP[k];
        for (int k = 0; k < nw; ++k) p.w[k] = p.w[k] + p.inv_inertia * dL[k];
        bool vnz = false;
        for (int k = 0; k < d; ++k) vnz = vnz || (p.v[k] != 0.0);
        if (vnz) {
            for (int k = 0; k < d; ++k) p.R[k] = p.R[k] + m.dt * p.v[k];
            moved = true;
        }
        for (int k = 0; k < nw; ++k)
            if (dL[k] != 0.0) need_nv = true;
        need_nv = need_nv || moved;
    }
    for (int k = 0; k < 3; ++k) {
        p.lastF[k] = dP[k];
        p.lastT[k] = dL[k];
        p.F[k] = 0;
        p.T[k] = 0;
    }
    p.dP.assign(Q, {Real(0.0), Real(0.0), Real(0.0)});
    p.dL.assign(Q, {Real(0.0), Real(0.0), Real(0.0)});
    if (moved) get_sphere(m, p.radius, p.R, p.S, &p.solid);
    if (need_nv) capture_node_velocity(p);
}

template <class Real>
void move(Model<Real>& m, Particle<Real>& p, bool initial) {
    if (m.rules == LBM_RULES_CPU_MODULE) move_particle_cpu(m, p, initial);
    else move_particle(m, p, initial);
}

// marks of the current tick: the walls' (static) plus every particle's
// streamingInvasionRegions; bit id of mark[c] set when f_id(c) takes the
// bounce-back value (c fluid for that solid, c - c_id solid)
template <class Real>
void build_marks(Model<Real>& m) {
    m.mark = m.wmark;
    if (!m.ladd) return;
    const int Q = m.vs.q;
    for (const auto& p : m.parts)
        for (int64_t y : p.solid)
            for (int id = 1; id < Q; ++id) {
                const auto& ci = m.vs.c[id];
                const int64_t x = m.shifted(y, ci[0], ci[1], ci[2]);
                if (!p.S[x]) m.mark[x] |= 1u << id;
            }
}

// LinearAlgebra.norm of a d-vector: 0 for the zero vector, else sqrt of the
// squares summed in component order
template <class V>
V vnorm(const V* v, int d) {
    double mx = 0.0;
    for (int k = 0; k < d; ++k) mx = std::max(mx, std::fabs(val(v[k])));
    if (mx == 0.0) return V(0.0);
    V s = v[0] * v[0];
    for (int k = 1; k < d; ++k) s += v[k] * v[k];
    return sqrt(s);
}

// applyInteraction! (src/gpu/particles.jl:111-197) of one item into the
// particles' force inputs, from their current positions
template <class Real>
void apply_interaction(Model<Real>& m, const lbm_interaction& it) {
    const int d = m.dims;
    auto& P1 = m.parts[it.id1 - 1];
    auto& P2 = m.parts[it.id2 - 1];
    if (it.kind == LBM_INTERACTION_POLAR) {
        auto& P3 = m.parts[it.id3 - 1];
        Real d12[3] = {0, 0, 0}, d32[3] = {0, 0, 0}, u12[3] = {0, 0, 0}, u32[3] = {0, 0, 0};
        for (int k = 0; k < d; ++k) {
            d12[k] = P1.R[k] - P2.R[k];
            d32[k] = P3.R[k] - P2.R[k];
        }
        const Real n12 = vnorm(d12, d), n32 = vnorm(d32, d);
        for (int k = 0; k < d; ++k) {
            u12[k] = d12[k] / n12;
            u32[k] = d32[k] / n32;
        }
        Real x = u12[0] * u32[0];
        for (int k = 1; k < d; ++k) x += u12[k] * u32[k];
        if (std::fabs(val(x)) > 1.0) x = val(x) > 0 ? Real(1.0) : Real(-1.0);
        const Real ang = acos_(x);
        Real td[3] = {0, 0, 0};
        cross_ref(d, u32, u12, td);
        const Real an = d == 2 ? fabs(td[0]) : vnorm(td, 3);
        if (val(an) > 0)
            for (int k = 0; k < 3; ++k) td[k] = td[k] / an;
        const Real s = it.p[1] * (ang - it.p[0]);
        Real f321[3] = {0, 0, 0}, f123[3] = {0, 0, 0};
        if (d == 2) {  // cross(omega::Real, V) = cross([0; 0; omega], [V; 0])[1:2]
            const Real w = s * td[0];
            f321[0] = 0.0 * 0.0 - w * u12[1];
            f321[1] = -0.0 * 0.0 + w * u12[0];
            f123[0] = 0.0 * 0.0 - w * u32[1];
            f123[1] = -0.0 * 0.0 + w * u32[0];
        } else {
            const Real tq[3] = {s * td[0], s * td[1], s * td[2]};
            cross_ref(3, tq, u12, f321);
            cross_ref(3, tq, u32, f123);
        }
        Real a[3], b[3];
        for (int k = 0; k < d; ++k) {
            a[k] = -f321[k] / n12;
            b[k] = f123[k] / n32;
        }
        for (int k = 0; k < d; ++k) P1.F[k] += a[k];
        for (int k = 0; k < d; ++k) P3.F[k] += b[k];
        for (int k = 0; k < d; ++k) P2.F[k] -= a[k] + b[k];
        return;
    }
    Real dv[3] = {0, 0, 0}, u[3] = {0, 0, 0};
    for (int k = 0; k < d; ++k) dv[k] = P2.R[k] - P1.R[k];  // disp21
    const Real dist = vnorm(dv, d);
    for (int k = 0; k < d; ++k) u[k] = dv[k] / dist;
    Real f[3] = {0, 0, 0};
    if (it.kind == LBM_INTERACTION_LINEAR) {
        for (int k = 0; k < d; ++k) f[k] = it.p[1] * (dist - it.p[0]) * u[k];
    } else if (it.kind == LBM_INTERACTION_BISTABLE) {
        const Real x = dist - it.p[0];
        for (int k = 0; k < d; ++k) f[k] = (it.p[1] * (x * x * x) - it.p[2] * x) * u[k];
    } else if (it.kind == LBM_INTERACTION_LENNARD_JONES) {
        if (!(val(dist) < it.p[2])) return;
        const Real sd = it.p[1] / dist;
        const Real s2 = sd * sd, s6 = s2 * s2 * s2;
        for (int k = 0; k < d; ++k) f[k] = -4.0 * it.p[0] / dist * (12.0 * (s6 * s6) - 6.0 * s6) * u[k];
    } else {  // dipoles, unless the field is zero (!(norm(B) ~ 0) with atol 0)
        const double B[3] = {it.p[1], it.p[2], it.p[3]};
        if (vnorm(B, d) == 0.0) return;
        Real cb[3] = {0, 0, 0}, ccb[3] = {0, 0, 0};
        cross_ref(d, u, B, cb);
        Real sq;
        if (d == 2) {
            ccb[0] = 0.0 * 0.0 - cb[0] * B[1];
            ccb[1] = -0.0 * 0.0 + cb[0] * B[0];
            sq = cb[0] * cb[0];
        } else {
            cross_ref(3, cb, B, ccb);
            sq = cb[0] * cb[0] + cb[1] * cb[1] + cb[2] * cb[2];
        }
        double bb = B[0] * B[0];
        for (int k = 1; k < d; ++k) bb += B[k] * B[k];
        const Real d2 = dist * dist;
        const Real pre = -it.p[0] / (d2 * d2);
        for (int k = 0; k < d; ++k) f[k] = pre * (2.0 * ccb[k] - 2.0 * bb * u[k] + 5.0 * u[k] * sq);
    }
    for (int k = 0; k < d; ++k) P1.F[k] += f[k];
    for (int k = 0; k < d; ++k) P2.F[k] -= f[k];
}

template <class Real>
void tick(Model<Real>& m, std::vector<Real>& fs, std::vector<Real>& fn) {
    const int64_t N = m.N;
    const int Q = m.vs.q, d = m.dims;
    const int64_t n0 = m.n[0], n1 = m.n[1], rows = m.n[1] * m.n[2];
    const bool cpu = m.rules == LBM_RULES_CPU_MODULE;
    collision(m, fs);
    fn.resize((size_t)N * Q);
    const double coeff = std::pow(m.dx, d) / m.dt;
    if (m.bounce_back) build_marks(m);
    std::vector<int64_t> nodes;
    for (int id = 0; id < Q; ++id) {
        const auto& ci = m.vs.c[id];
        const int ib = m.vs.opp[id];
        const double wi = m.vs.w[id];
        Real* s = &fn[(size_t)id * N];
        const Real* fsi = &fs[(size_t)id * N];
        const Real* fsb = &fs[(size_t)ib * N];
        const int64_t* wx = m.wrap[0][1 - ci[0]].data();
        const int64_t* wy = m.wrap[1][1 - ci[1]].data();
        const int64_t* wz = m.wrap[2][1 - ci[2]].data();
        const uint32_t bit = 1u << id;
#pragma omp parallel for schedule(static)
        for (int64_t row = 0; row < rows; ++row) {
            const int64_t y = row % n1, z = row / n1;
            const int64_t srow = n0 * (wy[y] + n1 * wz[z]);
            for (int64_t x = 0; x < n0; ++x) {
                const int64_t c = x + n0 * row;
                const int64_t src = wx[x] + srow;
                // circshift (pull): out(x) = in(x - c)
                Real v = fsi[src];
                if (m.bounce_back) {
                    if (m.W[c]) v = 0;
                    if (m.mark[c] & bit) {  // streaming invasion exchange (walls and particles)
                        v = fsb[c];
                        if (m.moving_walls) {
                            double uwv[3];
                            for (int k = 0; k < d; ++k) uwv[k] = m.uw[(int64_t)k * N + src];
                            v += (2 * wi * m.invC2) * m.rho[c] * dot_c(uwv, ci, d);
                        }
                    }
                }
                s[c] = v;
            }
        }
        if (m.bounce_back && m.ladd) {
            for (auto& p : m.parts) {
                particle_links(m, p, id, nodes);
                if (nodes.empty()) break;  // fluids.jl:184 exits the particle loop
                for (int64_t x : nodes) {
                    int64_t src = m.shifted(x, -ci[0], -ci[1], -ci[2]);
                    Real up[3];
                    if (cpu) {
                        // uw = u_p(x) + u_p(x - c) (src/cpu/fluids.jl:429); x is fluid, u_p(x) = 0
                        node_velocity_cpu(m, p, src, up);
                        for (int k = 0; k < d; ++k) up[k] = 0.0 + up[k];
                    } else {
                        node_velocity(m, p, src, up);
                    }
                    s[x] += (2 * wi * m.invC2) * m.rho[x] * dot_c(up, ci, d);
                }
                if (p.couple_f || p.couple_t || p.record_f) {
                    if (p.couple_f || p.record_f) {
                        Real S = 0.0;
                        for (int64_t x : nodes) S += fsb[x] + s[x];
                        if (cpu) {  // momentumInput[id] -= dx^d sum(sumTerm) c (dx/dt)
                            const Real t = std::pow(m.dx, d) * S;
                            for (int k = 0; k < d; ++k) p.dP[id][k] -= t * ((double)ci[k] * (m.dx / m.dt));
                        } else {
                            for (int k = 0; k < d; ++k) p.F[k] -= coeff * S * (double)ci[k];
                        }
                    }
                    if (p.couple_t) {
                        Real aux[3] = {0, 0, 0};
                        for (int64_t x : nodes) {
                            Real st = fsb[x] + s[x];
                            for (int k = 0; k < d; ++k) aux[k] += st * (m.coord(k, x) + (-p.R[k]));
                        }
                        double cd[3] = {(double)ci[0], (double)ci[1], (double)ci[2]};
                        Real cr[3] = {0, 0, 0};
                        int nt = d == 2 ? 1 : 3;
                        if (cpu) {
                            for (int k = 0; k < 3; ++k) cd[k] = cd[k] * (m.dx / m.dt);
                            cross_ref(d, aux, cd, cr);
                            const double ld = std::pow(m.dx, d);
                            for (int k = 0; k < nt; ++k) p.dL[id][k] -= ld * cr[k];
                        } else {
                            cross_ref(d, aux, cd, cr);
                            for (int k = 0; k < nt; ++k) p.T[k] -= coeff * cr[k];
                        }
                    }
                }
            }
        }
    }
    m.f.swap(fn);
    m.time += m.dt;
    m.tick += 1;
    hydro(m);
    if (m.ladd) {  // molecularDynamicsTick! (src/gpu/particles.jl:100-107)
        for (const auto& it : m.inter) apply_interaction(m, it);
        for (auto& p : m.parts) move(m, p, false);
    }
}

template <class Real>
struct HandleT {
    Model<Real> m;
    std::vector<Real> fs, fn;
};
using Handle = HandleT<double>;
using DualHandle = HandleT<D6>;

// seed: value `x` with derivatives `dx[kDirs]` (null: none); plain for double
inline double seeded(double x, const double*) { return x; }
inline D6 seeded_d(double x, const double* dx) {
    D6 r(x);
    if (dx)
        for (int k = 0; k < kDirs; ++k) r.d[k] = dx[k];
    return r;
}
template <class Real> Real seed_as(double x, const double* dx);
template <> double seed_as<double>(double x, const double* dx) { return seeded(x, dx); }
template <> D6 seed_as<D6>(double x, const double* dx) { return seeded_d(x, dx); }

// modelInit + findInitialConditions into m.  seeds (dual model only):
// derivatives of tau+ (and the BGK tau), tau- and of each uniform force
// component along the kDirs directions.
template <class Real>
int create_model(const lbm_config* cfg, Model<Real>& m, const double* seed_tau_plus, const double* seed_tau_minus,
                 const double* seed_force) {
    if (cfg->dims != 2 && cfg->dims != 3) return fail(LBM_ERR_INVALID, "dims must be 2 or 3");
    m.dims = cfg->dims;
    m.vs = make_velocity_set(cfg->lattice);
    if (m.vs.q == 0) return fail(LBM_ERR_INVALID, "unknown velocity set");
    if (m.vs.dims != m.dims) return fail(LBM_ERR_INVALID, "The chosen velocity must be " + std::to_string(m.dims) + "-dimensional!");
    for (int a = 0; a < 3; ++a) m.n[a] = (a < m.dims) ? cfg->n[a] : 1;
    for (int a = 0; a < m.dims; ++a)
        if (m.n[a] < 1) return fail(LBM_ERR_INVALID, "grid sizes must be positive");
    m.N = m.n[0] * m.n[1] * m.n[2];
    if (!(cfg->dx > 0)) return fail(LBM_ERR_INVALID, "latticeParameter must be positive");
    m.dx = cfg->dx;
    m.dt = cfg->dx;
    for (int a = 0; a < 3; ++a) {
        m.X[a].resize(m.n[a]);
        for (int64_t i = 0; i < m.n[a]; ++i)
            m.X[a][i] = (a < m.dims && cfg->coords[a]) ? cfg->coords[a][i] : cfg->x0[a] + (double)i * m.dx;
    }
    if (cfg->collision != LBM_BGK && cfg->collision != LBM_TRT)
        return fail(LBM_ERR_INVALID, "Collision model is not implemented!");
    m.trt = cfg->collision == LBM_TRT;
    m.tau = seed_as<Real>(cfg->tau, seed_tau_plus);
    m.tau_plus = seed_as<Real>(cfg->tau, seed_tau_plus);
    m.tau_minus = seed_as<Real>(cfg->tau_minus, seed_tau_minus);
    if (!(cfg->tau > 0) || (m.trt && !(cfg->tau_minus > 0))) return fail(LBM_ERR_INVALID, "relaxation times must be positive");
    m.compressible = cfg->compressible != 0;
    const int64_t N = m.N;
    const int d = m.dims, Q = m.vs.q;
    m.rho.assign(N, cfg->rho_uniform);
    if (cfg->rho_init) std::copy(cfg->rho_init, cfg->rho_init + N, m.rho.begin());
    m.u.assign((size_t)N * d, 0.0);
    for (int k = 0; k < d; ++k)
        for (int64_t c = 0; c < N; ++c)
            m.u[(int64_t)k * N + c] = cfg->u_init ? cfg->u_init[(int64_t)k * N + c] : cfg->u_uniform[k];
    // walls (initMethods.jl:568-628)
    m.W.assign(N, 0);
    if (cfg->wall_mask) {
        for (int64_t c = 0; c < N; ++c) m.W[c] = cfg->wall_mask[c] ? 1 : 0;
        m.bounce_back = true;
    }
    if (cfg->wall_velocity) {
        m.uw.assign(cfg->wall_velocity, cfg->wall_velocity + (size_t)N * d);
        for (int64_t c = 0; c < N; ++c) {
            bool nz = false;
            for (int k = 0; k < d; ++k) nz = nz || (m.uw[(int64_t)k * N + c] != 0.0);
            if (nz) m.W[c] = 1;
        }
        m.moving_walls = true;
        m.bounce_back = true;
    }
    if (m.bounce_back || m.trt) {
        for (int64_t c = 0; c < N; ++c)
            if (m.W[c]) {
                m.rho[c] = 0;
                for (int k = 0; k < d; ++k) m.u[(int64_t)k * N + c] = 0;
            }
    }
    // forcing (initMethods.jl:631-654)
    m.F.assign((size_t)N * d, 0.0);
    if (cfg->force_mode == LBM_FORCE_UNIFORM || cfg->force_mode == LBM_FORCE_FIELD) {
        if (cfg->force_mode == LBM_FORCE_FIELD && !cfg->force_field)
            return fail(LBM_ERR_INVALID, "force density does not have consistent dimensions!");
        for (int k = 0; k < d; ++k) {
            const Real Fk = seed_as<Real>(cfg->force_mode == LBM_FORCE_UNIFORM ? cfg->force[k] : 0.0,
                                          seed_force ? seed_force + (size_t)k * kDirs : nullptr);
            for (int64_t c = 0; c < N; ++c)
                m.F[(int64_t)k * N + c] = m.W[c] ? Real(0.0)
                    : (cfg->force_mode == LBM_FORCE_UNIFORM ? Fk : Real(cfg->force_field[(int64_t)k * N + c]));
        }
        m.guo = true;
    } else if (cfg->force_mode != LBM_FORCE_NONE) {
        return fail(LBM_ERR_INVALID, "unknown force mode");
    }
    m.rho0 = m.rho;
    if (cfg->particle_rules != LBM_RULES_GPU_MODULE && cfg->particle_rules != LBM_RULES_CPU_MODULE)
        return fail(LBM_ERR_INVALID, "unknown particle rules");
    m.rules = cfg->particle_rules;
    m.build_wrap();
    m.wmark.assign(N, 0u);
    if (m.bounce_back)
        for (int64_t c = 0; c < N; ++c)
            for (int id = 1; id < Q; ++id)
                if (invasion(m, m.W, m.vs.opp[id], c)) m.wmark[c] |= 1u << id;
    // findInitialConditions (initMethods.jl:417-438)
    m.f.assign((size_t)N * Q, 0.0);
    for (int64_t c = 0; c < N; ++c) {
        Real uu_[3] = {0, 0, 0};
        for (int k = 0; k < d; ++k) {
            Real uk = m.u[(int64_t)k * N + c];
            if (m.guo) {
                Real cons = (m.rho[c] == 0.0) ? Real(0.0) : m.F[(int64_t)k * N + c] / m.rho[c];
                uk = uk - 0.5 * m.dt * cons;
            }
            uu_[k] = uk;
        }
        for (int i = 0; i < Q; ++i) {
            Real uc = dot_c(uu_, m.vs.c[i], d);
            Real first = uc * m.invC2 + (uc * uc) * (0.5 * m.invC4);
            Real uu = 0.0;
            for (int k = 0; k < d; ++k) uu += uu_[k] * uu_[k];
            Real second = first - uu * (0.5 * m.invC2) + 1;
            m.f[(int64_t)i * N + c] = second * (m.vs.w[i] * m.rho[c]);
        }
    }
    hydro(m);
    return LBM_OK;
}

// addBead!/addSquirmer! into m (seeds: derivatives of B1 and B2, dual model only)
template <class Real>
int add_particle(Model<Real>& m, const lbm_particle_params* pp, const double* seed_B1, const double* seed_B2,
                 int32_t* id_out) {
    if (pp->kind != LBM_BEAD && pp->kind != LBM_SQUIRMER) return fail(LBM_ERR_INVALID, "unknown particle kind");
    if (m.parts.size() >= 255) return fail(LBM_ERR_INVALID, "particle ids are UInt8: at most 255 particles");
    if (!(pp->radius > 0)) return fail(LBM_ERR_INVALID, "radius must be positive");
    const int d = m.dims;
    Particle<Real> p;
    p.id = (int)m.parts.size() + 1;
    p.kind = pp->kind;
    p.couple_f = pp->couple_forces != 0;
    p.couple_t = pp->couple_torques != 0;
    p.radius = pp->radius;
    // mass: origin-centred sphere node count (initMethods.jl:108)
    std::vector<uint8_t> S0;
    Real zero[3] = {0, 0, 0};
    get_sphere(m, pp->radius, zero, S0);
    int64_t count = 0;
    for (uint8_t s : S0) count += s;
    double mass = pp->mass_density * (double)count * std::pow(m.dx, d);
    double r2 = pp->radius * pp->radius;
    double inertia = d == 2 ? 0.5 * mass * r2 : 0.4 * mass * r2;
    p.inv_mass = 1 / mass;
    p.inv_inertia = 1 / inertia;
    for (int k = 0; k < d; ++k) {
        p.R[k] = pp->position[k];
        p.v[k] = pp->velocity[k];
    }
    if (d == 2) p.w[0] = pp->angular_velocity[0];
    else for (int k = 0; k < 3; ++k) p.w[k] = pp->angular_velocity[k];
    if (p.kind == LBM_SQUIRMER) {
        p.B1 = seed_as<Real>(pp->B1, seed_B1);
        p.B2 = seed_as<Real>(pp->B2, seed_B2);
        for (int k = 0; k < d; ++k) p.e[k] = pp->swimming_direction[k];
    }
    m.parts.push_back(p);
    m.ladd = true;
    m.bounce_back = true;  // addSquirmer!/addBead! install an empty wall if needed (:210-214)
    move(m, m.parts.back(), true);
    if (id_out) *id_out = m.parts.back().id;
    return LBM_OK;
}

}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int orc_create(const lbm_config* cfg, void** out) {
    if (!cfg || !out) return fail(LBM_ERR_INVALID, "null argument");
    auto h = std::make_unique<Handle>();
    const int rc = create_model(cfg, h->m, nullptr, nullptr, nullptr);
    if (rc) return rc;
    *out = h.release();
    return LBM_OK;
}

int orc_add_particle(void* hp, const lbm_particle_params* pp, int32_t* id_out) {
    if (!hp || !pp) return fail(LBM_ERR_INVALID, "null argument");
    return add_particle(static_cast<Handle*>(hp)->m, pp, nullptr, nullptr, id_out);
}

int orc_step(void* hp, int64_t n) {
    if (!hp) return fail(LBM_ERR_INVALID, "null handle");
    if (n < 0) return fail(LBM_ERR_INVALID, "ticks must be non-negative");
    auto* h = static_cast<Handle*>(hp);
    for (int64_t t = 0; t < n; ++t) tick(h->m, h->fs, h->fn);
    return LBM_OK;
}

int orc_get_fields(void* hp, double* rho, double* u) {
    if (!hp) return fail(LBM_ERR_INVALID, "null handle");
    Model<double>& m = static_cast<Handle*>(hp)->m;
    if (rho) std::copy(m.rho.begin(), m.rho.end(), rho);
    if (u) std::copy(m.u.begin(), m.u.end(), u);
    return LBM_OK;
}

int orc_get_distributions(void* hp, double* f) {
    if (!hp || !f) return fail(LBM_ERR_INVALID, "null argument");
    Model<double>& m = static_cast<Handle*>(hp)->m;
    std::copy(m.f.begin(), m.f.end(), f);
    return LBM_OK;
}

int orc_set_distributions(void* hp, const double* f) {
    if (!hp || !f) return fail(LBM_ERR_INVALID, "null argument");
    Model<double>& m = static_cast<Handle*>(hp)->m;
    std::copy(f, f + m.f.size(), m.f.begin());
    hydro(m);
    return LBM_OK;
}

int orc_get_particles(void* hp, lbm_particle_state* out, int32_t cap, int32_t* count) {
    if (!hp) return fail(LBM_ERR_INVALID, "null handle");
    Model<double>& m = static_cast<Handle*>(hp)->m;
    if (count) *count = (int32_t)m.parts.size();
    for (int32_t i = 0; i < cap && i < (int32_t)m.parts.size(); ++i) {
        const Particle<double>& p = m.parts[i];
        lbm_particle_state& s = out[i];
        std::memset(&s, 0, sizeof(s));
        s.id = p.id;
        s.kind = p.kind;
        s.couple_forces = p.couple_f;
        s.couple_torques = p.couple_t;
        s.radius = p.radius;
        s.inverse_mass = p.inv_mass;
        s.inverse_inertia = p.inv_inertia;
        s.B1 = p.B1;
        s.B2 = p.B2;
        for (int k = 0; k < 3; ++k) {
            s.position[k] = p.R[k];
            s.velocity[k] = p.v[k];
            s.angular_velocity[k] = p.w[k];
            s.swimming_direction[k] = p.e[k];
            s.last_force[k] = p.lastF[k];
            s.last_torque[k] = p.lastT[k];
        }
    }
    return LBM_OK;
}

// Overwrite the position, velocity, angular velocity and swimming direction
// of particle `id` (1-based) and re-voxelise it: its solid region and node
// velocities are recomputed from the new state (the initial-setup branch of
// moveParticles!, src/gpu/particles.jl:62-91), the momentum inputs are kept.
int orc_set_particle(void* hp, int32_t id, const lbm_particle_state* st) {
    if (!hp || !st) return fail(LBM_ERR_INVALID, "null argument");
    Model<double>& m = static_cast<Handle*>(hp)->m;
    if (id < 1 || id > (int32_t)m.parts.size()) return fail(LBM_ERR_INVALID, "no such particle");
    Particle<double>& p = m.parts[id - 1];
    for (int k = 0; k < 3; ++k) {
        p.R[k] = st->position[k];
        p.v[k] = st->velocity[k];
        p.w[k] = st->angular_velocity[k];
        p.e[k] = st->swimming_direction[k];
    }
    get_sphere(m, p.radius, p.R, p.S, &p.solid);
    capture_node_velocity(p);
    return LBM_OK;
}

// particleInteractions: the items of lbm_set_interactions (pairs flattened,
// 1-based ids), applied every tick before the particles move
int orc_set_interactions(void* hp, const lbm_interaction* list, int32_t n) {
    if (!hp || n < 0 || (n > 0 && !list)) return fail(LBM_ERR_INVALID, "bad interaction list");
    Model<double>& m = static_cast<Handle*>(hp)->m;
    const int np = (int)m.parts.size();
    for (int t = 0; t < n; ++t)
        if (list[t].id1 < 1 || list[t].id1 > np || list[t].id2 < 1 || list[t].id2 > np ||
            (list[t].kind == LBM_INTERACTION_POLAR && (list[t].id3 < 1 || list[t].id3 > np)))
            return fail(LBM_ERR_INVALID, "interaction names no valid particles");
    m.inter.assign(list, list + n);
    return LBM_OK;
}

// Accumulate particle `id`'s momentum-exchange force even when coupleForces
// is off (`on` != 0), reporting it as last_force without applying it: the
// drag of a held particle.  The reference accumulates no force for such a
// particle; this switch exists for the force observable of the gradients.
int orc_record_force(void* hp, int32_t id, int32_t on) {
    if (!hp) return fail(LBM_ERR_INVALID, "null handle");
    Model<double>& m = static_cast<Handle*>(hp)->m;
    if (id < 1 || id > (int32_t)m.parts.size()) return fail(LBM_ERR_INVALID, "no such particle");
    m.parts[id - 1].record_f = on != 0;
    return LBM_OK;
}

int orc_get_mask(void* hp, int32_t id, uint8_t* mask) {
    if (!hp || !mask) return fail(LBM_ERR_INVALID, "null argument");
    Model<double>& m = static_cast<Handle*>(hp)->m;
    if (id < 1 || id > (int32_t)m.parts.size()) return fail(LBM_ERR_INVALID, "no such particle");
    std::copy(m.parts[id - 1].S.begin(), m.parts[id - 1].S.end(), mask);
    return LBM_OK;
}

int orc_get_links(void* hp, int32_t id, int64_t* cells, int8_t* dirs, int64_t cap, int64_t* n) {
    if (!hp || !n) return fail(LBM_ERR_INVALID, "null argument");
    Model<double>& m = static_cast<Handle*>(hp)->m;
    if (id < 1 || id > (int32_t)m.parts.size()) return fail(LBM_ERR_INVALID, "no such particle");
    std::vector<int64_t> nodes;
    int64_t k = 0;
    for (int dir = 0; dir < m.vs.q; ++dir) {
        particle_links(m, m.parts[id - 1], dir, nodes);
        for (int64_t x : nodes) {
            if (cells && k < cap) {
                cells[k] = x;
                dirs[k] = (int8_t)dir;
            }
            ++k;
        }
    }
    *n = k;
    return LBM_OK;
}

int orc_get_info(void* hp, lbm_info* info) {
    if (!hp || !info) return fail(LBM_ERR_INVALID, "null argument");
    Model<double>& m = static_cast<Handle*>(hp)->m;
    std::memset(info, 0, sizeof(*info));
    info->dims = m.dims;
    info->lattice = m.vs.q;
    info->q = m.vs.q;
    info->storage = LBM_STORE_F64;
    for (int a = 0; a < 3; ++a) info->n[a] = m.n[a];
    info->cells = m.N;
    info->tick = m.tick;
    info->time = m.time;
    info->num_particles = (int32_t)m.parts.size();
    info->bytes_per_population = 8;
    return LBM_OK;
}

// viscousStressTensor (src/cpu/fluids.jl:507-520): sigma_ab = -(1 - dt/(2 tau))
// sum_i c_ia c_ib (f_i - f_eq_i), f_eq of equilibriumDistribution
// (src/gpu/fluids.jl:39-52) at the model's rho and u, the sum over i a left
// fold; out (N..., d, d) column-major
int orc_get_stress(void* hp, double* out) {
    if (!hp || !out) return fail(LBM_ERR_INVALID, "null argument");
    const Model<double>& m = static_cast<Handle*>(hp)->m;
    const int64_t N = m.N;
    const int d = m.dims, Q = m.vs.q;
    const double coeff = 1 - 0.5 * m.dt / m.tau;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        double neq[27];
        double uu = 0.0;
        for (int k = 0; k < d; ++k) uu += m.u[(int64_t)k * N + c] * m.u[(int64_t)k * N + c];
        for (int i = 0; i < Q; ++i) {
            double uc = 0.0;
            for (int k = 0; k < d; ++k) uc += m.u[(int64_t)k * N + c] * (double)m.vs.c[i][k];
            const double first = uc * m.invC2 + (uc * uc) * (0.5 * m.invC4);
            const double second = first - uu * (0.5 * m.invC2);
            const double wi = m.vs.w[i];
            const double feq = m.compressible ? wi * ((second + 1) * m.rho[c]) : wi * m.rho[c] + wi * (m.rho0[c] * second);
            neq[i] = m.f[(int64_t)i * N + c] - feq;
        }
        for (int b = 0; b < d; ++b)
            for (int a = 0; a < d; ++a) {
                double sum = 0.0;
                for (int i = 0; i < Q; ++i) {
                    const double t = (double)(m.vs.c[i][a] * m.vs.c[i][b]) * neq[i];
                    sum = i == 0 ? t : sum + t;
                }
                out[c + N * (a + (int64_t)d * b)] = -coeff * sum;
            }
    }
    return LBM_OK;
}

// the velocity set as the oracle builds it (c as int8 triples, w, opposite index)
int orc_velocity_set(int32_t q, int8_t* c, double* w, int32_t* opp) {
    VelocitySet s = make_velocity_set(q);
    if (s.q == 0) return fail(LBM_ERR_INVALID, "unknown velocity set");
    for (int i = 0; i < s.q; ++i) {
        for (int a = 0; a < 3; ++a) c[3 * i + a] = (int8_t)s.c[i][a];
        w[i] = s.w[i];
        opp[i] = s.opp[i];
    }
    return LBM_OK;
}

void orc_destroy(void* hp) { delete static_cast<Handle*>(hp); }

// ---- dual-number oracle: derivatives along kDirs seeded directions ---------
int ord_directions(void) { return kDirs; }

// seed_tau_plus / seed_tau_minus: [kDirs]; seed_force: [3][kDirs] (uniform force); any may be null
int ord_create(const lbm_config* cfg, const double* seed_tau_plus, const double* seed_tau_minus,
               const double* seed_force, void** out) {
    if (!cfg || !out) return fail(LBM_ERR_INVALID, "null argument");
    auto h = std::make_unique<DualHandle>();
    const int rc = create_model(cfg, h->m, seed_tau_plus, seed_tau_minus, seed_force);
    if (rc) return rc;
    *out = h.release();
    return LBM_OK;
}

int ord_add_particle(void* hp, const lbm_particle_params* pp, const double* seed_B1, const double* seed_B2,
                     int32_t* id_out) {
    if (!hp || !pp) return fail(LBM_ERR_INVALID, "null argument");
    return add_particle(static_cast<DualHandle*>(hp)->m, pp, seed_B1, seed_B2, id_out);
}

int ord_step(void* hp, int64_t n) {
    if (!hp) return fail(LBM_ERR_INVALID, "null handle");
    if (n < 0) return fail(LBM_ERR_INVALID, "ticks must be non-negative");
    auto* h = static_cast<DualHandle*>(hp);
    for (int64_t t = 0; t < n; ++t) tick(h->m, h->fs, h->fn);
    return LBM_OK;
}

// particle `id` (1-based): values [12] = position, velocity, angular velocity,
// swimming direction (3 each); derivatives [12][kDirs] in the same order
int ord_particle(void* hp, int32_t id, double* values, double* derivs) {
    if (!hp || !values || !derivs) return fail(LBM_ERR_INVALID, "null argument");
    const Model<D6>& m = static_cast<DualHandle*>(hp)->m;
    if (id < 1 || id > (int32_t)m.parts.size()) return fail(LBM_ERR_INVALID, "no such particle");
    const Particle<D6>& p = m.parts[id - 1];
    const D6* groups[4] = {p.R, p.v, p.w, p.e};
    for (int g = 0; g < 4; ++g)
        for (int k = 0; k < 3; ++k) {
            const D6& x = groups[g][k];
            values[3 * g + k] = x.v;
            for (int q = 0; q < kDirs; ++q) derivs[(size_t)(3 * g + k) * kDirs + q] = x.d[q];
        }
    return LBM_OK;
}

int ord_record_force(void* hp, int32_t id, int32_t on) {
    if (!hp) return fail(LBM_ERR_INVALID, "null handle");
    Model<D6>& m = static_cast<DualHandle*>(hp)->m;
    if (id < 1 || id > (int32_t)m.parts.size()) return fail(LBM_ERR_INVALID, "no such particle");
    m.parts[id - 1].record_f = on != 0;
    return LBM_OK;
}

// momentum-exchange force of the last tick of particle `id`: values [3],
// derivatives [3][kDirs]
int ord_particle_force(void* hp, int32_t id, double* values, double* derivs) {
    if (!hp || !values || !derivs) return fail(LBM_ERR_INVALID, "null argument");
    const Model<D6>& m = static_cast<DualHandle*>(hp)->m;
    if (id < 1 || id > (int32_t)m.parts.size()) return fail(LBM_ERR_INVALID, "no such particle");
    const Particle<D6>& p = m.parts[id - 1];
    for (int k = 0; k < 3; ++k) {
        values[k] = p.lastF[k].v;
        for (int q = 0; q < kDirs; ++q) derivs[(size_t)k * kDirs + q] = p.lastF[k].d[q];
    }
    return LBM_OK;
}

// density and velocity values (as orc_get_fields)
int ord_get_fields(void* hp, double* rho, double* u) {
    if (!hp) return fail(LBM_ERR_INVALID, "null handle");
    const Model<D6>& m = static_cast<DualHandle*>(hp)->m;
    for (size_t c = 0; rho && c < m.rho.size(); ++c) rho[c] = m.rho[c].v;
    for (size_t c = 0; u && c < m.u.size(); ++c) u[c] = m.u[c].v;
    return LBM_OK;
}

void ord_destroy(void* hp) { delete static_cast<DualHandle*>(hp); }

}  // extern "C"
