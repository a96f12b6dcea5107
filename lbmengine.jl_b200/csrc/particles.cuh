// Particle update on the device: momentum-exchange reduction, Newton-Euler
// integration with Rodrigues rotation, re-voxelisation bookkeeping.
// Restates moveParticles! (src/gpu/particles.jl:7-92) for one particle per CTA.
#pragma once
#include "kernels.cuh"

namespace lbm {

struct ParticleArgs {
    ParticleDev* parts;
    int nparts;
    int mode;        // 0: tick update; 1: initial setup of particle `setup_pid`;
                     // 2: re-voxelise `setup_pid` keeping its slip snapshot (checkpoint restore)
    int setup_pid;
    int pad;
    const double* partial;
    unsigned long long* tilebits;
    int words;
    int pad2;
    GridDesc g;
    const double* coord[3];
    double x0[3];
    double dx, dt;
    int* err;
};

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
    const int nthreads = blockDim.x;
    for (int l = threadIdx.x; l < total; l += nthreads) {
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

template <class L>
__global__ void __launch_bounds__(256) k_particles(const ParticleArgs a) {
    constexpr int D = L::D;
    const int p = a.mode != 0 ? a.setup_pid : (int)blockIdx.x;
    ParticleDev& P = a.parts[p];
    const int tid = threadIdx.x;
    __shared__ double s_red[8][6];
    __shared__ int s_moved, s_oldbox[6], s_newbox[6], s_cert;
    __shared__ unsigned s_links;

    // 1. momentum exchange: fixed-order reduction of the per-tile partials
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (a.mode == 0) {
        const int ntl = P.tn[0] * P.tn[1] * P.tn[2];
        for (int l = tid; l < ntl; l += blockDim.x) {
            const double* q = a.partial + (long long)(P.part_off + l) * kPartialStride;
            for (int k = 0; k < 6; ++k) acc[k] += q[k];
        }
    }
    for (int k = 0; k < 6; ++k)
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if ((tid & 31) == 0)
        for (int k = 0; k < 6; ++k) s_red[tid >> 5][k] = acc[k];
    __syncthreads();

    // 2. Newton-Euler update (one thread, FP64)
    if (tid == 0) {
        double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
        const int nw = blockDim.x >> 5;
        for (int k = 0; k < 3; ++k) {
            for (int w = 0; w < nw; ++w) {
                F[k] += s_red[w][k];
                T[k] += s_red[w][3 + k];
            }
        }
        bool moved = a.mode != 0, need_nv = a.mode == 1;
        if (a.mode == 0) {
            const double dt = a.dt;
            if (P.coupleF) {
                for (int k = 0; k < D; ++k) P.v[k] = P.v[k] + dt * (F[k] * P.inv_mass);
                for (int k = 0; k < D; ++k) P.R[k] = P.R[k] + dt * P.v[k];
                for (int k = 0; k < D; ++k)
                    if (P.v[k] != 0.0) moved = true;
            }
            if (P.coupleT) {
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
                    if (Al[k] != 0.0) need_nv = true;
            }
            need_nv = need_nv || moved;
        }
        if (a.mode != 2)
            for (int k = 0; k < 3; ++k) {
                P.lastF[k] = F[k];
                P.lastT[k] = T[k];
            }
        if (need_nv)
            for (int k = 0; k < 3; ++k) {
                P.sR[k] = P.R[k];
                P.sV[k] = P.v[k];
                P.sW[k] = P.w[k];
                P.sE[k] = P.e[k];
            }
        s_moved = moved ? 1 : 0;
        for (int k = 0; k < 3; ++k) {
            s_oldbox[k] = P.tlo[k];
            s_oldbox[3 + k] = (a.mode != 0 && !P.valid) ? 0 : P.tn[k];
        }
        if (moved) {
            for (int k = 0; k < 3; ++k) P.mR[k] = P.R[k];
            int lo[3], hi[3];
            solid_box(a, P.R, P.radius, D, lo, hi);
            bool empty = false;
            for (int k = 0; k < 3; ++k) {
                P.slo[k] = lo[k];
                P.shi[k] = hi[k];
                empty = empty || lo[k] > hi[k];
            }
            int tlo[3] = {0, 0, 0}, tn[3] = {0, 0, 0};
            if (!empty)
                for (int k = 0; k < 3; ++k)
                    tile_range(lo[k] - 1, hi[k] - lo[k] + 3, a.g.n[k], a.g.t[k], a.g.nt[k], &tlo[k], &tn[k]);
            if (tn[0] * tn[1] * tn[2] > P.part_cap) {
                atomicOr(a.err, kErrPartialOverflow);
                tn[0] = tn[1] = tn[2] = 0;
                empty = true;
            }
            for (int k = 0; k < 3; ++k) {
                P.tlo[k] = tlo[k];
                P.tn[k] = tn[k];
                s_newbox[k] = tlo[k];
                s_newbox[3 + k] = tn[k];
            }
            // boundary links exist in every moving direction when the sphere has
            // a node and does not span a whole periodic axis; otherwise count
            int cert = 0;
            if (!empty) {
                int nearest[3];
                for (int k = 0; k < 3; ++k) {
                    if (k >= D) {
                        nearest[k] = 0;
                        continue;
                    }
                    double c = rint((P.R[k] - a.x0[k]) / a.dx);
                    c = c < 0.0 ? 0.0 : (c > (double)(a.g.n[k] - 1) ? (double)(a.g.n[k] - 1) : c);
                    nearest[k] = (int)c;
                }
                const bool nonempty = sphere_test<D>(a.coord[0][nearest[0]], a.coord[1][nearest[1]],
                                                     D == 3 ? a.coord[2][nearest[2]] : 0.0, P.R, P.r2);
                bool spans = false;
                for (int k = 0; k < D; ++k) spans = spans || (hi[k] - lo[k] + 1 >= a.g.n[k]);
                cert = (nonempty && !spans) ? 1 : 0;
            }
            s_cert = empty ? 2 : cert;
        }
        P.valid = 1;
    }
    __syncthreads();

    // 3. tile bits of the candidate lists and exact link directions
    if (s_moved) {
        if (s_oldbox[3] * s_oldbox[4] * s_oldbox[5] > 0) tile_bits_update(a, s_oldbox, s_oldbox + 3, p, false);
        __syncthreads();
        if (s_newbox[3] * s_newbox[4] * s_newbox[5] > 0) tile_bits_update(a, s_newbox, s_newbox + 3, p, true);
        if (tid == 0) {
            if (s_cert == 1) {
                unsigned m = 0;
                for (int i = 1; i < L::Q; ++i) m |= 1u << i;
                P.dirlinks = m;
            } else if (s_cert == 2) {
                P.dirlinks = 0u;
            }
            s_links = 0u;
        }
        __syncthreads();
        if (s_cert == 0) {
            // exact enumeration over the solid box (rare: tiny or domain-spanning spheres)
            const int l0 = P.shi[0] - P.slo[0] + 1, l1 = P.shi[1] - P.slo[1] + 1, l2 = P.shi[2] - P.slo[2] + 1;
            const long long vol = (long long)l0 * l1 * l2;
            unsigned m = 0;
            for (long long q = tid; q < vol; q += blockDim.x) {
                const int x = P.slo[0] + (int)(q % l0);
                const int y = P.slo[1] + (int)((q / l0) % l1);
                const int z = P.slo[2] + (int)(q / ((long long)l0 * l1));
                if (!sphere_test<D>(a.coord[0][x], a.coord[1][y], D == 3 ? a.coord[2][z] : 0.0, P.mR, P.r2))
                    continue;
#pragma unroll
                for (int i = 1; i < L::Q; ++i) {
                    const int tx = wrap_idx(x + L::cx(i), a.g.n[0]);
                    const int ty = wrap_idx(y + L::cy(i), a.g.n[1]);
                    const int tz = wrap_idx(z + L::cz(i), a.g.n[2]);
                    if (!sphere_test<D>(a.coord[0][tx], a.coord[1][ty], D == 3 ? a.coord[2][tz] : 0.0, P.mR, P.r2))
                        m |= 1u << i;
                }
            }
            if (m) atomicOr(&s_links, m);
            __syncthreads();
            if (tid == 0) P.dirlinks = s_links;
        }
    }
}

}  // namespace lbm
