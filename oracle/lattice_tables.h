/*
 * Velocity sets in the reference's exact direction order (TEST ORACLE DATA).
 *
 * The order of the directions is part of the interface: populations are
 * exchanged as (N..., Q) arrays whose last index follows it.  The tables
 * restate src/gpu/misc.jl:195-272 (identical to src/cpu/misc.jl:265-342):
 *   - rest vector first;
 *   - then the axis vectors, axis by axis, each as (-1, +1);
 *   - then the diagonal groups, each enumerated with the FIRST listed
 *     component varying fastest (Julia comprehension + vec, column-major).
 * The opposite-direction table is derived, as in src/gpu/aux.jl:195, as the
 * first index j with c_j == -c_i.
 */
#ifndef LBM_ORACLE_LATTICE_TABLES_H
#define LBM_ORACLE_LATTICE_TABLES_H

#include <vector>
#include <array>
#include <cstdint>

namespace lbm_oracle {

struct VelocitySet {
    int dims = 0;
    int q = 0;
    std::vector<std::array<int, 3>> c;  // c[i][a], a < dims (padded with 0)
    std::vector<double> w;
    std::vector<int> opp;
};

inline void finish_opposites(VelocitySet& s) {
    s.opp.assign(s.q, -1);
    for (int i = 0; i < s.q; ++i)
        for (int j = 0; j < s.q; ++j)
            if (s.c[j][0] == -s.c[i][0] && s.c[j][1] == -s.c[i][1] && s.c[j][2] == -s.c[i][2]) {
                s.opp[i] = j;
                break;  // findfirst
            }
}

inline VelocitySet make_velocity_set(int q) {
    VelocitySet s;
    auto axes = [&](int dims) {
        for (int a = 0; a < dims; ++a)
            for (int p : {-1, 1}) {
                std::array<int, 3> v{0, 0, 0};
                v[a] = p;
                s.c.push_back(v);
            }
    };
    // plane diagonal groups: (0,p,q), (p,0,q), (p,q,0) with p fastest
    auto plane = [&](int zero_axis) {
        for (int qq : {-1, 1})
            for (int p : {-1, 1}) {
                std::array<int, 3> v{0, 0, 0};
                int a1 = zero_axis == 0 ? 1 : 0;
                int a2 = zero_axis == 2 ? 1 : 2;
                v[a1] = p;
                v[a2] = qq;
                s.c.push_back(v);
            }
    };
    auto cube = [&]() {  // (p,q,r), p fastest, then q, then r
        for (int r : {-1, 1})
            for (int qq : {-1, 1})
                for (int p : {-1, 1}) s.c.push_back({p, qq, r});
    };
    if (q == 9) {
        s.dims = 2;
        s.c.push_back({0, 0, 0});
        axes(2);
        for (int qq : {-1, 1})
            for (int p : {-1, 1}) s.c.push_back({p, qq, 0});
        s.w = {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
    } else if (q == 15) {
        s.dims = 3;
        s.c.push_back({0, 0, 0});
        axes(3);
        cube();
        s.w.push_back(2.0 / 9);
        for (int i = 0; i < 6; ++i) s.w.push_back(1.0 / 9);
        for (int i = 0; i < 8; ++i) s.w.push_back(1.0 / 72);
    } else if (q == 19 || q == 27) {
        s.dims = 3;
        s.c.push_back({0, 0, 0});
        axes(3);
        plane(0);
        plane(1);
        plane(2);
        if (q == 27) cube();
        if (q == 19) {
            s.w.push_back(1.0 / 3);
            for (int i = 0; i < 6; ++i) s.w.push_back(1.0 / 18);
            for (int i = 0; i < 12; ++i) s.w.push_back(1.0 / 36);
        } else {
            s.w.push_back(8.0 / 27);
            for (int i = 0; i < 6; ++i) s.w.push_back(2.0 / 27);
            for (int i = 0; i < 12; ++i) s.w.push_back(1.0 / 54);
            for (int i = 0; i < 8; ++i) s.w.push_back(1.0 / 216);
        }
    } else {
        return s;  // q == 0 marks an unknown set
    }
    s.q = (int)s.c.size();
    finish_opposites(s);
    return s;
}

}  // namespace lbm_oracle
#endif
