// Compile-time velocity sets.
//
// The direction order is an interface (populations cross the C ABI as
// (N..., Q) arrays), so it is the reference's order, src/gpu/misc.jl:195-272:
// rest vector, axis vectors (-1 then +1 per axis), then the diagonal groups
// with the first listed component varying fastest.  Opposites follow
// src/gpu/aux.jl:195 (first j with c_j == -c_i).  Weights are given as exact
// reciprocals: 1/w_i is a small dyadic number for every set (3, 18, 36, 2.25,
// 9, 4.5, 72, 3.375, 13.5, 54, 216), which the shifted storage format uses.
#pragma once

namespace lbm {

struct D2Q9 {
    static constexpr int D = 2, Q = 9;
    static constexpr __host__ __device__ int cx(int i) {
        constexpr int t[Q] = {0, -1, 1, 0, 0, -1, 1, -1, 1};
        return t[i];
    }
    static constexpr __host__ __device__ int cy(int i) {
        constexpr int t[Q] = {0, 0, 0, -1, 1, -1, -1, 1, 1};
        return t[i];
    }
    static constexpr __host__ __device__ int cz(int i) {
        constexpr int t[Q] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        return t[i];
    }
    static constexpr __host__ __device__ int opp(int i) {
        constexpr int t[Q] = {0, 2, 1, 4, 3, 8, 7, 6, 5};
        return t[i];
    }
    static constexpr __host__ __device__ double w(int i) {
        constexpr double t[Q] = {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9,
                                    1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
        return t[i];
    }
};

struct D3Q15 {
    static constexpr int D = 3, Q = 15;
    static constexpr __host__ __device__ int cx(int i) {
        constexpr int t[Q] = {0, -1, 1, 0, 0, 0, 0, -1, 1, -1, 1, -1, 1, -1, 1};
        return t[i];
    }
    static constexpr __host__ __device__ int cy(int i) {
        constexpr int t[Q] = {0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, -1, -1, 1, 1};
        return t[i];
    }
    static constexpr __host__ __device__ int cz(int i) {
        constexpr int t[Q] = {0, 0, 0, 0, 0, -1, 1, -1, -1, -1, -1, 1, 1, 1, 1};
        return t[i];
    }
    static constexpr __host__ __device__ int opp(int i) {
        constexpr int t[Q] = {0, 2, 1, 4, 3, 6, 5, 14, 13, 12, 11, 10, 9, 8, 7};
        return t[i];
    }
    static constexpr __host__ __device__ double w(int i) {
        constexpr double t[Q] = {2.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9,
                                    1.0 / 72, 1.0 / 72, 1.0 / 72, 1.0 / 72, 1.0 / 72, 1.0 / 72, 1.0 / 72, 1.0 / 72};
        return t[i];
    }
};

struct D3Q19 {
    static constexpr int D = 3, Q = 19;
    static constexpr __host__ __device__ int cx(int i) {
        constexpr int t[Q] = {0, -1, 1, 0, 0, 0, 0, 0, 0, 0, 0, -1, 1, -1, 1, -1, 1, -1, 1};
        return t[i];
    }
    static constexpr __host__ __device__ int cy(int i) {
        constexpr int t[Q] = {0, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 0, 0, 0, 0, -1, -1, 1, 1};
        return t[i];
    }
    static constexpr __host__ __device__ int cz(int i) {
        constexpr int t[Q] = {0, 0, 0, 0, 0, -1, 1, -1, -1, 1, 1, -1, -1, 1, 1, 0, 0, 0, 0};
        return t[i];
    }
    static constexpr __host__ __device__ int opp(int i) {
        constexpr int t[Q] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
        return t[i];
    }
    static constexpr __host__ __device__ double w(int i) {
        constexpr double t[Q] = {1.0 / 3, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18,
                                    1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36,
                                    1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
        return t[i];
    }
};

struct D3Q27 {
    static constexpr int D = 3, Q = 27;
    static constexpr __host__ __device__ int cx(int i) {
        constexpr int t[Q] = {0, -1, 1, 0, 0, 0, 0, 0, 0, 0, 0, -1, 1, -1, 1, -1, 1, -1, 1,
                                  -1, 1, -1, 1, -1, 1, -1, 1};
        return t[i];
    }
    static constexpr __host__ __device__ int cy(int i) {
        constexpr int t[Q] = {0, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 0, 0, 0, 0, -1, -1, 1, 1,
                                  -1, -1, 1, 1, -1, -1, 1, 1};
        return t[i];
    }
    static constexpr __host__ __device__ int cz(int i) {
        constexpr int t[Q] = {0, 0, 0, 0, 0, -1, 1, -1, -1, 1, 1, -1, -1, 1, 1, 0, 0, 0, 0,
                                  -1, -1, -1, -1, 1, 1, 1, 1};
        return t[i];
    }
    static constexpr __host__ __device__ int opp(int i) {
        constexpr int t[Q] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15,
                                   26, 25, 24, 23, 22, 21, 20, 19};
        return t[i];
    }
    static constexpr __host__ __device__ double w(int i) {
        constexpr double t[Q] = {8.0 / 27, 2.0 / 27, 2.0 / 27, 2.0 / 27, 2.0 / 27, 2.0 / 27, 2.0 / 27,
                                    1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54,
                                    1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54,
                                    1.0 / 216, 1.0 / 216, 1.0 / 216, 1.0 / 216,
                                    1.0 / 216, 1.0 / 216, 1.0 / 216, 1.0 / 216};
        return t[i];
    }
};

}  // namespace lbm
