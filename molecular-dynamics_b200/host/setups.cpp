// setups.cpp -- tinyMD benchmark setups (host side of the md driver surface).
// See setups.h.  Every generator walks lattice sites in the reference's order
// so that particle i here is particle i of the reference run.

#include "setups.h"

#include <algorithm>
#include <cstdio>

namespace tmd {

namespace {

// Park & Miller (1988) "minimal standard" multiplier 16807 modulo 2^31-1,
// evaluated with Schrage's decomposition m = a*q + r (q = 127773, r = 2836)
// so no intermediate overflows 32 bits.
constexpr int kPmA = 16807;
constexpr int kPmM = 2147483647;
constexpr int kPmQ = 127773;
constexpr int kPmR = 2836;

// rank.min <= p < rank.max - 1e-5 on every axis (initialize.h:51-57)
bool inside_rank(const double r[6], double x, double y, double z) {
    return x >= r[0] && x < r[1] - 0.00001 && y >= r[2] && y < r[3] - 0.00001 && z >= r[4] &&
           z < r[5] - 0.00001;
}

// FCC sites on the half-spacing grid whose index sum is even, visited in
// blocks of 8x8x8 sites (block z, y, x outer; site z, y, x inner), as in
// initialize.h:91-201.  `keep` filters sites; when `seeded` the velocity of a
// site is drawn from the site-indexed Park-Miller stream, otherwise it is 0.
template <class Keep>
void fcc_walk(const double box[6], double spacing, bool seeded, Keep keep, Particles& out) {
    const int sub = 8;
    int nvert[3], nhalf[3];
    for (int d = 0; d < 3; ++d) {
        nvert[d] = (int)((box[2 * d + 1] - box[2 * d]) / spacing);
        nhalf[d] = nvert[d] / 2;
    }
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = std::max((int)(box[2 * d] / spacing - 1), 0);
        hi[d] = std::min((int)(box[2 * d + 1] / spacing + 1), nvert[d] - 1);
    }
    for (int bz = 0; bz * sub <= hi[2]; ++bz)
        for (int by = 0; by * sub <= hi[1]; ++by)
            for (int bx = 0; bx * sub <= hi[0]; ++bx)
                for (int sz = 0; sz < sub; ++sz)
                    for (int sy = 0; sy < sub; ++sy)
                        for (int sx = 0; sx < sub; ++sx) {
                            int i = bx * sub + sx, j = by * sub + sy, k = bz * sub + sz;
                            if ((i + j + k) % 2 != 0) continue;
                            if (i < lo[0] || i > hi[0] || j < lo[1] || j > hi[1] || k < lo[2] || k > hi[2])
                                continue;
                            Vector3D p{box[0] + i * spacing, box[2] + j * spacing, box[4] + k * spacing};
                            if (!keep(p, lo, hi)) continue;
                            Vector3D v{0.0, 0.0, 0.0};
                            if (seeded) {
                                int state = k * (2 * nhalf[1]) * (2 * nhalf[0]) + j * (2 * nhalf[0]) + i + 1;
                                double draw[3];
                                for (int d = 0; d < 3; ++d) {
                                    for (int skip = 0; skip < 5; ++skip) park_miller(&state);
                                    draw[d] = park_miller(&state);
                                }
                                v = Vector3D{draw[0], draw[1], draw[2]};
                            }
                            out.mass.push_back(1.0);
                            out.pos.push_back(p);
                            out.vel.push_back(v);
                        }
}

}  // namespace

double park_miller(int* state) {
    int q = *state / kPmQ;
    *state = kPmA * (*state - q * kPmQ) - kPmR * q;
    if (*state < 0) *state += kPmM;
    return (1.0 / kPmM) * (*state);
}

int world_box(int benchmark, const int gridsize[3], double potmin, double world[6], double aabb1[6],
              double aabb2[6]) {
    if (benchmark == BENCH_BODY_COLLISION) {
        double shift = 2.0 * (gridsize[1] + 1);
        for (int d = 0; d < 3; ++d) {
            aabb1[2 * d] = 0;
            aabb1[2 * d + 1] = gridsize[d] * potmin;
            aabb2[2 * d] = 0;
            aabb2[2 * d + 1] = gridsize[d] * potmin;
        }
        aabb2[2] -= shift;
        aabb2[3] -= shift;
        for (int d = 0; d < 3; ++d) {
            world[2 * d] = std::min(aabb1[2 * d], aabb2[2 * d]) - 20;
            world[2 * d + 1] = std::max(aabb1[2 * d + 1], aabb2[2 * d + 1]) + 20;
        }
        return 0;
    }
    if (benchmark < 0 || benchmark > BENCH_GRANULAR_GAS_FCC) return -1;
    for (int d = 0; d < 3; ++d) {
        world[2 * d] = 0;
        world[2 * d + 1] = gridsize[d] * potmin;
        aabb1[2 * d] = aabb2[2 * d] = 0;
        aabb1[2 * d + 1] = aabb2[2 * d + 1] = 0;
    }
    return 0;
}

void node_bounding_box(const double world[6], double rank[6]) {
    // one rank: gx = gy = gz = 1, cartesian location 0
    for (int d = 0; d < 3; ++d) {
        double len = (world[2 * d + 1] - world[2 * d]) / 1.0;
        double lo = world[2 * d] + len * 0.0;
        rank[2 * d] = lo;
        rank[2 * d + 1] = lo + len;
    }
}

int generate(int benchmark, const double world[6], const double rank[6], const double aabb1[6],
             const double aabb2[6], double potmin, Particles& out) {
    out = Particles();
    switch (benchmark) {
        case BENCH_DEFAULT:
        case BENCH_HALF: {
            const bool half = benchmark == BENCH_HALF;
            const double spacing = potmin * 0.5;
            fcc_walk(world, spacing, true,
                     [&](const Vector3D& p, const int* lo, const int* hi) {
                         if (!inside_rank(rank, p.x, p.y, p.z)) return false;
                         // initialize.h:148 -- integer half of the y site range
                         return !half || p.y < world[2] + ((hi[1] - lo[1]) / 2) * spacing + 0.00001;
                     },
                     out);
            break;
        }
        case BENCH_GRANULAR_GAS_FCC: {
            const double spacing = potmin * 0.5;
            const double lx = world[1] - world[0], ly = world[3] - world[2];
            fcc_walk(world, spacing, false,
                     [&](const Vector3D& p, const int*, const int*) {
                         if (!inside_rank(rank, p.x, p.y, p.z)) return false;
                         // strictly below the diagonal; the tolerance keeps sites that lie
                         // on it (i + j = sites per edge) out regardless of rounding
                         return (p.x - world[0]) / lx + (p.y - world[2]) / ly < 1.0 - 1e-9;
                     },
                     out);
            break;
        }
        case BENCH_GRANULAR_GAS: {
            // initialize.h:226-295: unit simple-cubic lattice offset by half a
            // site plus 0.01, kept on the negative side of the plane through the
            // box centre with normal (1,1,1)
            const double spacing = 1.0;
            const double shift = 0.01;
            double centre[3];
            int n[3];
            for (int d = 0; d < 3; ++d) {
                centre[d] = world[2 * d] + (world[2 * d + 1] - world[2 * d]) * 0.5;
                n[d] = (int)((world[2 * d + 1] - world[2 * d]) / spacing);
            }
            for (int x = 0; x < n[0]; ++x)
                for (int y = 0; y < n[1]; ++y)
                    for (int z = 0; z < n[2]; ++z) {
                        Vector3D p{world[0] + (double)x * spacing + spacing * 0.5 + shift,
                                   world[2] + (double)y * spacing + spacing * 0.5 + shift,
                                   world[4] + (double)z * spacing + spacing * 0.5 + shift};
                        double side = (p.x - centre[0]) * 1.0 + (p.y - centre[1]) * 1.0 + (p.z - centre[2]) * 1.0;
                        if (inside_rank(rank, p.x, p.y, p.z) && side < 0.0) {
                            out.mass.push_back(1.0);
                            out.pos.push_back(p);
                            out.vel.push_back(Vector3D{0.0, 0.0, 0.0});
                        }
                    }
            break;
        }
        case BENCH_BODY_COLLISION: {
            // initialize.h:297-362; the site counts keep the reference's
            // operator precedence, aabb1[max] - (aabb1[min] / spacing)
            const double spacing = 1.0;
            const double speed = 5.0;
            if (aabb1[2] < aabb2[3]) {
                std::fprintf(stderr, "The first bounding box must be located on top of the second!\n");
                return -1;
            }
            int n[3];
            for (int d = 0; d < 3; ++d) n[d] = (int)(aabb1[2 * d + 1] - aabb1[2 * d] / spacing);
            for (int x = 0; x < n[0]; ++x)
                for (int y = 0; y < n[1]; ++y)
                    for (int z = 0; z < n[2]; ++z) {
                        const double* boxes[2] = {aabb1, aabb2};
                        for (int b = 0; b < 2; ++b) {
                            const double* a = boxes[b];
                            Vector3D p{a[0] + (double)x * spacing + spacing * 0.5,
                                       a[2] + (double)y * spacing + spacing * 0.5,
                                       a[4] + (double)z * spacing + spacing * 0.5};
                            if (inside_rank(rank, p.x, p.y, p.z)) {
                                out.mass.push_back(1.0);
                                out.pos.push_back(p);
                                out.vel.push_back(Vector3D{0.0, b == 0 ? -speed : speed, 0.0});
                            }
                        }
                    }
            break;
        }
        default:
            return -1;
    }
    return (int)out.mass.size();
}

}  // namespace tmd
