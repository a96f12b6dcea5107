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
 * Floating-point operations are written in the reference's evaluation order
 * (left to right, no fused multiply-add: build with -ffp-contract=off).
 * Reductions the reference does with CUDA.jl parallel sums are done here
 * sequentially in column-major cell order.
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

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

struct Particle {
    int id = 0;
    int kind = LBM_SQUIRMER;
    bool couple_f = false, couple_t = false;
    double radius = 0, B1 = 0, B2 = 0;
    double inv_mass = 0, inv_inertia = 0;
    double R[3] = {0, 0, 0}, v[3] = {0, 0, 0}, w[3] = {0, 0, 0}, e[3] = {0, 0, 0};
    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};  // forceInput / torqueInput
    double lastF[3] = {0, 0, 0}, lastT[3] = {0, 0, 0};
    std::vector<uint8_t> S;  // solidRegion
    // state captured by the last getNodeVelocity call (nodeVelocity is a
    // function of it, evaluated on demand)
    double nvR[3] = {0, 0, 0}, nvV[3] = {0, 0, 0}, nvW[3] = {0, 0, 0}, nvE[3] = {0, 0, 0};
};

struct Model {
    int dims = 0;
    VelocitySet vs;
    int64_t n[3] = {1, 1, 1};
    int64_t N = 0;
    std::vector<double> X[3];
    double dx = 1, dt = 1, tau = 1, tau_plus = 1, tau_minus = 1;
    double invC2 = 3, invC4 = 9;
    bool trt = false, compressible = true;
    bool bounce_back = false, moving_walls = false, guo = false, ladd = false;
    std::vector<double> f, rho, u, F, rho0, uw;
    std::vector<uint8_t> W;
    std::vector<Particle> parts;
    int64_t tick = 0;
    double time = 0;

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
// X + (-R) equals X - R exactly in IEEE arithmetic.
inline bool in_sphere(const Model& m, int64_t x, int64_t y, int64_t z, const double* R, double r2) {
    double a = m.X[0][x] - R[0];
    double b = m.X[1][y] - R[1];
    double s = a * a + b * b;
    if (m.dims == 3) {
        double c = m.X[2][z] - R[2];
        s = s + c * c;
    }
    return s < r2;
}

// per-axis index range that can satisfy the sphere test (conservative and
// exact: fl(a*a) <= the full rounded sum, so nodes outside fail the test too)
void axis_range(const Model& m, int a, double Ra, double r2, int64_t& lo, int64_t& hi) {
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

void get_sphere(const Model& m, double radius, const double* R, std::vector<uint8_t>& S) {
    S.assign(m.N, 0);
    double r2 = radius * radius;
    int64_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int a = 0; a < m.dims; ++a) axis_range(m, a, R[a], r2, lo[a], hi[a]);
    if (m.dims == 2) { lo[2] = 0; hi[2] = 0; }
    for (int64_t z = lo[2]; z <= hi[2]; ++z)
        for (int64_t y = lo[1]; y <= hi[1]; ++y)
            for (int64_t x = lo[0]; x <= hi[0]; ++x)
                if (in_sphere(m, x, y, z, R, r2)) S[m.cell(x, y, z)] = 1;
}

// dot of a vector with a lattice vector, vectorFieldDotVector (kernels.jl:198-224):
// sumTerm = 0 then += v_k * c_k in component order
inline double dot_c(const double* v, const std::array<int, 3>& c, int dims) {
    double s = 0.0;
    for (int k = 0; k < dims; ++k) s += v[k] * (double)c[k];
    return s;
}

// getNodeVelocity evaluated at node y (aux.jl:229-263, kernels.jl:376-415)
void node_velocity(const Model& m, const Particle& p, int64_t y, double* out) {
    int d = m.dims;
    double xr[3] = {0, 0, 0};
    for (int k = 0; k < d; ++k) xr[k] = m.coord(k, y) + (-p.nvR[k]);
    double nrm2 = 0.0;
    for (int k = 0; k < d; ++k) nrm2 += xr[k] * xr[k];
    double nrm = std::sqrt(nrm2);
    if (nrm == 0) nrm = 1;
    double bulk[3];
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
    double inv = 1.0 / nrm;
    double ur[3];
    for (int k = 0; k < d; ++k) ur[k] = inv * xr[k];
    double edr = 0.0;
    for (int k = 0; k < d; ++k) edr += ur[k] * p.nvE[k];
    double first = p.B1 + p.B2 * edr;
    for (int k = 0; k < d; ++k) {
        double second = edr * ur[k] + (-p.nvE[k]);
        out[k] = first * second + bulk[k];
    }
}

void capture_node_velocity(Particle& p) {
    for (int k = 0; k < 3; ++k) {
        p.nvR[k] = p.R[k];
        p.nvV[k] = p.v[k];
        p.nvW[k] = p.w[k];
        p.nvE[k] = p.e[k];
    }
}

// hydroVariablesUpdate! (fluids.jl:7-37): rho = sum_i f_i ; rho*u = sum_i f_i c_i
// (+ dt/2 F with Guo) ; u = rho*u / rho unless rho == 0 (isapprox with atol 0)
void hydro(Model& m) {
    const int64_t N = m.N;
    const int d = m.dims, Q = m.vs.q;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        double r = 0.0;
        for (int i = 0; i < Q; ++i) r = (i == 0) ? m.f[c] : r + m.f[(int64_t)i * N + c];
        m.rho[c] = r;
        for (int k = 0; k < d; ++k) {
            double j = 0.0;
            for (int i = 0; i < Q; ++i) {
                double t = m.f[(int64_t)i * N + c] * (double)m.vs.c[i][k];
                j = (i == 0) ? t : j + t;
            }
            if (m.guo) j = j + (0.5 * m.dt) * m.F[(int64_t)k * N + c];
            m.u[(int64_t)k * N + c] = (r == 0.0) ? 0.0 : j / r;
        }
    }
}

// equilibriumDistribution (fluids.jl:39-52) at one cell
inline double feq(const Model& m, int i, int64_t c) {
    const int d = m.dims;
    double uc = 0.0, uu = 0.0;
    for (int k = 0; k < d; ++k) uc += m.u[(int64_t)k * m.N + c] * (double)m.vs.c[i][k];
    for (int k = 0; k < d; ++k) uu += m.u[(int64_t)k * m.N + c] * m.u[(int64_t)k * m.N + c];
    double first = uc * m.invC2 + (uc * uc) * (0.5 * m.invC4);
    double second = first - uu * (0.5 * m.invC2);
    double wi = m.vs.w[i];
    if (m.compressible) return wi * ((second + 1) * m.rho[c]);
    return wi * m.rho[c] + wi * (m.rho0[c] * second);
}

// guoForcingTerm (fluids.jl:103-127) at one cell
inline double guo(const Model& m, int i, int64_t c) {
    const int d = m.dims;
    const auto& ci = m.vs.c[i];
    double U[3] = {0, 0, 0}, Fv[3] = {0, 0, 0};
    for (int k = 0; k < d; ++k) {
        U[k] = m.u[(int64_t)k * m.N + c];
        Fv[k] = m.F[(int64_t)k * m.N + c];
    }
    double uc = 0.0;
    for (int k = 0; k < d; ++k) uc += U[k] * (double)ci[k];
    double wi = m.vs.w[i];
    if (!m.trt) {
        double inter = 0.0;
        for (int k = 0; k < d; ++k) {
            double second = (uc * (double)ci[k]) * m.invC4;
            double first = ((-U[k]) + (double)ci[k]) * m.invC2;
            inter += (first + second) * Fv[k];
        }
        return wi * m.dt * (1 - m.dt / (2 * m.tau)) * inter;
    }
    double inter = 0.0;
    for (int k = 0; k < d; ++k) {
        double second = (uc * (double)ci[k]) * m.invC4;
        inter += ((-U[k]) * m.invC2 + second) * Fv[k];
    }
    double plus = (1 - m.dt / (2 * m.tau_plus)) * inter;
    double inter2 = 0.0;
    for (int k = 0; k < d; ++k) inter2 += Fv[k] * ((double)ci[k] * m.invC2);
    double minus = (1 - m.dt / (2 * m.tau_minus)) * inter2;
    return wi * m.dt * (plus + minus);
}

// collisionStep (fluids.jl:58-101): returns f + Omega
void collision(const Model& m, std::vector<double>& fs) {
    const int64_t N = m.N;
    const int Q = m.vs.q;
    fs.resize((size_t)N * Q);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        double eq[27];
        for (int i = 0; i < Q; ++i) eq[i] = feq(m, i, c);
        for (int i = 0; i < Q; ++i) {
            double fi = m.f[(int64_t)i * N + c];
            double om;
            if (!m.trt) {
                om = (-m.dt / m.tau) * (fi - eq[i]);
            } else {
                int ib = m.vs.opp[i];
                double fb = m.f[(int64_t)ib * N + c];
                double fp = 0.5 * (fi + fb), fm = 0.5 * (fi - fb);
                double ep = 0.5 * (eq[i] + eq[ib]), em = 0.5 * (eq[i] - eq[ib]);
                om = (-m.dt / m.tau_plus) * (fp - ep) + (-m.dt / m.tau_minus) * (fm - em);
            }
            if (m.guo) om = om + guo(m, i, c);
            fs[(int64_t)i * N + c] = om + fi;
        }
    }
}

// streamingInvasionRegions[j](x) = S(x + c_j) && !S(x)   (aux.jl:190)
inline bool invasion(const Model& m, const std::vector<uint8_t>& S, int j, int64_t c) {
    if (S[c]) return false;
    const auto& cj = m.vs.c[j];
    return S[m.shifted(c, cj[0], cj[1], cj[2])] != 0;
}

// 2D/3D cross product of the reference (aux.jl:139-145)
void cross_ref(int d, const double* v, const double* w, double* out) {
    if (d == 2) {
        out[0] = v[0] * w[1] - v[1] * w[0];
    } else {
        out[0] = v[1] * w[2] - v[2] * w[1];
        out[1] = -v[0] * w[2] + v[2] * w[0];
        out[2] = v[0] * w[1] - v[1] * w[0];
    }
}

// sorted fluid cells x with x - c_id in S and x not in S (conjugate boundary nodes)
void particle_links(const Model& m, const Particle& p, int id, std::vector<int64_t>& out) {
    out.clear();
    const auto& ci = m.vs.c[id];
    if (ci[0] == 0 && ci[1] == 0 && ci[2] == 0) return;
    for (int64_t y = 0; y < m.N; ++y) {
        if (!p.S[y]) continue;
        int64_t x = m.shifted(y, ci[0], ci[1], ci[2]);
        if (!p.S[x]) out.push_back(x);
    }
    std::sort(out.begin(), out.end());
}

// moveParticles! (particles.jl:7-92)
void move_particle(Model& m, Particle& p, bool initial) {
    const int d = m.dims;
    bool moved = initial, need_nv = initial;
    if (!initial) {
        if (p.couple_f) {
            double A[3];
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
            double Al[3];
            for (int k = 0; k < nw; ++k) Al[k] = p.T[k] * p.inv_inertia;
            for (int k = 0; k < nw; ++k) p.w[k] = p.w[k] + m.dt * Al[k];
            if (p.kind == LBM_SQUIRMER) {
                double theta;
                if (d == 2) {
                    theta = std::fabs(p.w[0]);
                } else {
                    double s = 0.0;
                    for (int k = 0; k < 3; ++k) s += p.w[k] * p.w[k];
                    theta = std::sqrt(s);
                }
                if (theta != 0.0) {  // !(theta ≈ 0) with atol 0
                    double vr[3] = {0, 0, 0};
                    const double* v = p.e;
                    if (d == 2) {
                        double k = p.w[0] / theta;
                        theta = theta * m.dt;
                        double cr[2] = {-k * v[1], k * v[0]};
                        double ct = std::cos(theta), st = std::sin(theta);
                        for (int q = 0; q < 2; ++q) vr[q] = v[q] * ct + cr[q] * st;
                    } else {
                        double k[3];
                        for (int q = 0; q < 3; ++q) k[q] = p.w[q] / theta;
                        theta = theta * m.dt;
                        double cr[3];
                        cross_ref(3, k, v, cr);
                        double ct = std::cos(theta), st = std::sin(theta);
                        for (int q = 0; q < 3; ++q) vr[q] = v[q] * ct + cr[q] * st;
                        double kv = 0.0;
                        for (int q = 0; q < 3; ++q) kv += k[q] * v[q];
                        for (int q = 0; q < 3; ++q) vr[q] = vr[q] + k[q] * kv * (1 - ct);
                    }
                    double s = 0.0;
                    for (int q = 0; q < d; ++q) s += vr[q] * vr[q];
                    double nr = std::sqrt(s);
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
    if (moved) get_sphere(m, p.radius, p.R, p.S);
    if (need_nv) capture_node_velocity(p);
}

void tick(Model& m, std::vector<double>& fs, std::vector<double>& fn) {
    const int64_t N = m.N;
    const int Q = m.vs.q, d = m.dims;
    collision(m, fs);
    fn.resize((size_t)N * Q);
    const double coeff = std::pow(m.dx, d) / m.dt;
    std::vector<int64_t> nodes;
    for (int id = 0; id < Q; ++id) {
        const auto& ci = m.vs.c[id];
        const int ib = m.vs.opp[id];
        const double wi = m.vs.w[id];
        double* s = &fn[(size_t)id * N];
        const double* fsi = &fs[(size_t)id * N];
        const double* fsb = &fs[(size_t)ib * N];
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < N; ++c) {
            // circshift (pull): out(x) = in(x - c)
            double v = fsi[m.shifted(c, -ci[0], -ci[1], -ci[2])];
            if (m.bounce_back) {
                if (m.W[c]) v = 0;
                bool region = invasion(m, m.W, ib, c);
                if (m.ladd)
                    for (const auto& p : m.parts) region = region || invasion(m, p.S, ib, c);
                if (region) {
                    v = fsb[c];
                    if (m.moving_walls) {
                        int64_t src = m.shifted(c, -ci[0], -ci[1], -ci[2]);
                        double uwv[3];
                        for (int k = 0; k < d; ++k) uwv[k] = m.uw[(int64_t)k * N + src];
                        v += (2 * wi * m.invC2) * m.rho[c] * dot_c(uwv, ci, d);
                    }
                }
            }
            s[c] = v;
        }
        if (m.bounce_back && m.ladd) {
            for (auto& p : m.parts) {
                particle_links(m, p, id, nodes);
                if (nodes.empty()) break;  // fluids.jl:184 exits the particle loop
                for (int64_t x : nodes) {
                    int64_t src = m.shifted(x, -ci[0], -ci[1], -ci[2]);
                    double up[3];
                    node_velocity(m, p, src, up);
                    s[x] += (2 * wi * m.invC2) * m.rho[x] * dot_c(up, ci, d);
                }
                if (p.couple_f || p.couple_t) {
                    if (p.couple_f) {
                        double S = 0.0;
                        for (int64_t x : nodes) S += fsb[x] + s[x];
                        for (int k = 0; k < d; ++k) p.F[k] -= coeff * S * (double)ci[k];
                    }
                    if (p.couple_t) {
                        double aux[3] = {0, 0, 0};
                        for (int64_t x : nodes) {
                            double st = fsb[x] + s[x];
                            for (int k = 0; k < d; ++k) aux[k] += st * (m.coord(k, x) + (-p.R[k]));
                        }
                        double cd[3] = {(double)ci[0], (double)ci[1], (double)ci[2]};
                        double cr[3] = {0, 0, 0};
                        cross_ref(d, aux, cd, cr);
                        int nt = d == 2 ? 1 : 3;
                        for (int k = 0; k < nt; ++k) p.T[k] -= coeff * cr[k];
                    }
                }
            }
        }
    }
    m.f.swap(fn);
    m.time += m.dt;
    m.tick += 1;
    hydro(m);
    if (m.ladd)
        for (auto& p : m.parts) move_particle(m, p, false);
}

struct Handle {
    Model m;
    std::vector<double> fs, fn;
};

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
    Model& m = h->m;
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
    m.tau = cfg->tau;
    m.tau_plus = cfg->tau;
    m.tau_minus = cfg->tau_minus;
    if (!(m.tau > 0) || (m.trt && !(m.tau_minus > 0))) return fail(LBM_ERR_INVALID, "relaxation times must be positive");
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
        for (int k = 0; k < d; ++k)
            for (int64_t c = 0; c < N; ++c)
                m.F[(int64_t)k * N + c] = m.W[c] ? 0.0
                    : (cfg->force_mode == LBM_FORCE_UNIFORM ? cfg->force[k] : cfg->force_field[(int64_t)k * N + c]);
        m.guo = true;
    } else if (cfg->force_mode != LBM_FORCE_NONE) {
        return fail(LBM_ERR_INVALID, "unknown force mode");
    }
    m.rho0 = m.rho;
    // findInitialConditions (initMethods.jl:417-438)
    m.f.assign((size_t)N * Q, 0.0);
    for (int64_t c = 0; c < N; ++c) {
        double uu_[3] = {0, 0, 0};
        for (int k = 0; k < d; ++k) {
            double uk = m.u[(int64_t)k * N + c];
            if (m.guo) {
                double cons = (m.rho[c] == 0.0) ? 0.0 : m.F[(int64_t)k * N + c] / m.rho[c];
                uk = uk - 0.5 * m.dt * cons;
            }
            uu_[k] = uk;
        }
        for (int i = 0; i < Q; ++i) {
            double uc = dot_c(uu_, m.vs.c[i], d);
            double first = uc * m.invC2 + (uc * uc) * (0.5 * m.invC4);
            double uu = 0.0;
            for (int k = 0; k < d; ++k) uu += uu_[k] * uu_[k];
            double second = first - uu * (0.5 * m.invC2) + 1;
            m.f[(int64_t)i * N + c] = second * (m.vs.w[i] * m.rho[c]);
        }
    }
    hydro(m);
    *out = h.release();
    return LBM_OK;
}

int orc_add_particle(void* hp, const lbm_particle_params* pp, int32_t* id_out) {
    if (!hp || !pp) return fail(LBM_ERR_INVALID, "null argument");
    Model& m = static_cast<Handle*>(hp)->m;
    if (pp->kind != LBM_BEAD && pp->kind != LBM_SQUIRMER) return fail(LBM_ERR_INVALID, "unknown particle kind");
    if (m.parts.size() >= 255) return fail(LBM_ERR_INVALID, "particle ids are UInt8: at most 255 particles");
    if (!(pp->radius > 0)) return fail(LBM_ERR_INVALID, "radius must be positive");
    const int d = m.dims;
    Particle p;
    p.id = (int)m.parts.size() + 1;
    p.kind = pp->kind;
    p.couple_f = pp->couple_forces != 0;
    p.couple_t = pp->couple_torques != 0;
    p.radius = pp->radius;
    // mass: origin-centred sphere node count (initMethods.jl:108)
    std::vector<uint8_t> S0;
    double zero[3] = {0, 0, 0};
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
        p.B1 = pp->B1;
        p.B2 = pp->B2;
        for (int k = 0; k < d; ++k) p.e[k] = pp->swimming_direction[k];
    }
    m.parts.push_back(p);
    m.ladd = true;
    m.bounce_back = true;  // addSquirmer!/addBead! install an empty wall if needed (:210-214)
    move_particle(m, m.parts.back(), true);
    if (id_out) *id_out = m.parts.back().id;
    return LBM_OK;
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
    Model& m = static_cast<Handle*>(hp)->m;
    if (rho) std::copy(m.rho.begin(), m.rho.end(), rho);
    if (u) std::copy(m.u.begin(), m.u.end(), u);
    return LBM_OK;
}

int orc_get_distributions(void* hp, double* f) {
    if (!hp || !f) return fail(LBM_ERR_INVALID, "null argument");
    Model& m = static_cast<Handle*>(hp)->m;
    std::copy(m.f.begin(), m.f.end(), f);
    return LBM_OK;
}

int orc_set_distributions(void* hp, const double* f) {
    if (!hp || !f) return fail(LBM_ERR_INVALID, "null argument");
    Model& m = static_cast<Handle*>(hp)->m;
    std::copy(f, f + m.f.size(), m.f.begin());
    hydro(m);
    return LBM_OK;
}

int orc_get_particles(void* hp, lbm_particle_state* out, int32_t cap, int32_t* count) {
    if (!hp) return fail(LBM_ERR_INVALID, "null handle");
    Model& m = static_cast<Handle*>(hp)->m;
    if (count) *count = (int32_t)m.parts.size();
    for (int32_t i = 0; i < cap && i < (int32_t)m.parts.size(); ++i) {
        const Particle& p = m.parts[i];
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

int orc_get_mask(void* hp, int32_t id, uint8_t* mask) {
    if (!hp || !mask) return fail(LBM_ERR_INVALID, "null argument");
    Model& m = static_cast<Handle*>(hp)->m;
    if (id < 1 || id > (int32_t)m.parts.size()) return fail(LBM_ERR_INVALID, "no such particle");
    std::copy(m.parts[id - 1].S.begin(), m.parts[id - 1].S.end(), mask);
    return LBM_OK;
}

int orc_get_links(void* hp, int32_t id, int64_t* cells, int8_t* dirs, int64_t cap, int64_t* n) {
    if (!hp || !n) return fail(LBM_ERR_INVALID, "null argument");
    Model& m = static_cast<Handle*>(hp)->m;
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
    Model& m = static_cast<Handle*>(hp)->m;
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

}  // extern "C"
