// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own setup generators (initialize.h) and its only
// native force kernel (core/force_lj.cpp, compiled as a separate object from
// the reference tree) into oracle/_ref/libtinymd_refsetup.so, so the tests can
// pin (a) the product's lattice / velocity generators and (b) the oracle's
// full-list LJ force against code the reference itself ships.  Nothing from
// the reference is copied into this repository: the recipe in oracle/Makefile
// compiles the files where they lie.
//
// md_initialize_grid is the one symbol of anydsl_includes.h that the setup
// generators call; here it only records what the reference would hand to its
// runtime, so the captured arrays are exactly the reference's inputs.

#include <functional>
#include <iostream>
#include <vector>

#include "initialize.h"

namespace {
std::vector<double> cap_m;
std::vector<Vector3D> cap_x, cap_v;
double cap_aabb[6], cap_rank[6];
double cap_spacing = 0.0;
int cap_cell_cap = 0, cap_nb_cap = 0;
}  // namespace

extern "C" int md_initialize_grid(double const* m, Vector3D const* x, Vector3D const* v, int n,
                                  double const* aabb, double const* rank, double spacing, int cell_cap,
                                  int nb_cap) {
    cap_m.assign(m, m + n);
    cap_x.assign(x, x + n);
    cap_v.assign(v, v + n);
    for (int d = 0; d < 6; ++d) {
        cap_aabb[d] = aabb[d];
        cap_rank[d] = rank[d];
    }
    cap_spacing = spacing;
    cap_cell_cap = cell_cap;
    cap_nb_cap = nb_cap;
    return n;
}

// Calls the reference generator the way main.cpp:664-674 does for the given
// benchmark, with world/rank boxes supplied by the caller.
// kind: 0 = default/half rectangular grid, 1 = granular_gas, 2 = body_collision.
extern "C" int ref_generate(int kind, double* world, double* rank, double* aabb1, double* aabb2, int half,
                            double lattice_spacing, double cell_spacing) {
    using namespace std::placeholders;
    auto within = std::bind(is_within_aabb, _1, _2, _3, rank);
    if (kind == 0)
        return init_rectangular_grid(world, rank, half != 0, lattice_spacing, cell_spacing, 60, 100, within);
    if (kind == 1) return init_granular_gas(world, rank, cell_spacing, 60, 100, within);
    return init_body_collision(world, aabb1, aabb2, rank, cell_spacing, 60, 100, within);
}

extern "C" int ref_captured(double* m, double* x, double* v, double* aabb, double* rank, double* spacing,
                            int* caps) {
    int n = (int)cap_m.size();
    for (int i = 0; i < n; ++i) {
        m[i] = cap_m[i];
        x[3 * i + 0] = cap_x[i].x; x[3 * i + 1] = cap_x[i].y; x[3 * i + 2] = cap_x[i].z;
        v[3 * i + 0] = cap_v[i].x; v[3 * i + 1] = cap_v[i].y; v[3 * i + 2] = cap_v[i].z;
    }
    for (int d = 0; d < 6; ++d) {
        aabb[d] = cap_aabb[d];
        rank[d] = cap_rank[d];
    }
    *spacing = cap_spacing;
    caps[0] = cap_cell_cap;
    caps[1] = cap_nb_cap;
    return n;
}

extern "C" int ref_captured_count(void) { return (int)cap_m.size(); }

// The reference's Park-Miller generator (initialize.h:38-49), exposed so the
// product's restatement can be checked value by value.
extern "C" double ref_random(int* idum) { return random(idum); }
