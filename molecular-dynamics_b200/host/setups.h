// setups.h -- tinyMD benchmark setups (world boxes and particle generators).
//
// Host code of the md driver surface.  Restates the reference's setup logic:
// world boxes from main.cpp:491-521 and the generators of initialize.h
// (miniMD's Park-Miller velocity seeding, FCC lattice walk, granular gas,
// body collision).  The same functions are exported from libtinymd_b200.so
// through the tmd_setup_* C entry points declared in include/tinymd_b200.h.
#pragma once

#include <vector>

#include "tinymd_b200.h"

namespace tmd {

enum Benchmark {
    BENCH_DEFAULT = 0,         // FCC lattice filling the box
    BENCH_HALF = 1,            // FCC lattice, lower half in y
    BENCH_GRANULAR_GAS = 2,    // simple-cubic lattice cut by a plane through the centre, v = 0
    BENCH_BODY_COLLISION = 3,  // two simple-cubic blocks moving towards each other
    BENCH_GRANULAR_GAS_FCC = 4 // FCC lattice kept where x/Lx + y/Ly < 1, v = 0 (DEM diagonal split)
};

struct Particles {
    std::vector<double> mass;
    std::vector<Vector3D> pos, vel;
};

// Park-Miller minimal-standard generator with Schrage's factorisation, as
// used by miniMD and tinyMD (initialize.h:28-49).  Advances *state and
// returns a uniform draw in [0, 1).
double park_miller(int* state);

// World box (and the two body boxes for body collision), main.cpp:491-521.
// Returns 0 on success, -1 for an unknown benchmark.
int world_box(int benchmark, const int gridsize[3], double potmin, double world[6], double aabb1[6],
              double aabb2[6]);

// Rank box of a single process, comm/comm.impala:254-331 with one rank.
void node_bounding_box(const double world[6], double rank[6]);

// Generates the particles of `benchmark` inside `rank` (a point is kept when
// rank.min <= p < rank.max - 1e-5 per axis, initialize.h:51-57).
// Returns the number of particles, or -1 on an invalid configuration.
int generate(int benchmark, const double world[6], const double rank[6], const double aabb1[6],
             const double aabb2[6], double potmin, Particles& out);

}  // namespace tmd
