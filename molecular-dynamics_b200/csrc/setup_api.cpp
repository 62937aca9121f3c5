// setup_api.cpp -- tmd_setup_* C entry points: the md driver's benchmark
// setups (main.cpp:491-521, initialize.h) exported for non-C++ callers.

#include <vector>

#include "setups.h"
#include "tinymd_b200.h"

namespace {
tmd::Particles g_setup;
}

extern "C" {

int tmd_setup_world(int benchmark, int const* gridsize, double potmin, double* world, double* aabb1,
                    double* aabb2) {
    return tmd::world_box(benchmark, gridsize, potmin, world, aabb1, aabb2);
}

void tmd_setup_rank_box(double const* world, double* rank) { tmd::node_bounding_box(world, rank); }

int tmd_setup_generate(int benchmark, double const* world, double const* rank, double const* aabb1,
                       double const* aabb2, double potmin) {
    return tmd::generate(benchmark, world, rank, aabb1, aabb2, potmin, g_setup);
}

int tmd_setup_fetch(double* masses, Vector3D* positions, Vector3D* velocities) {
    const int n = (int)g_setup.mass.size();
    for (int i = 0; i < n; ++i) {
        if (masses) masses[i] = g_setup.mass[i];
        if (positions) positions[i] = g_setup.pos[i];
        if (velocities) velocities[i] = g_setup.vel[i];
    }
    return n;
}

int tmd_setup_initialize(double const* world, double const* rank, double cell_spacing, int cell_capacity,
                         int neighborlist_capacity) {
    return md_initialize_grid(g_setup.mass.data(), g_setup.pos.data(), g_setup.vel.data(), (int)g_setup.mass.size(),
                              world, rank, cell_spacing, cell_capacity, neighborlist_capacity);
}

}  // extern "C"
