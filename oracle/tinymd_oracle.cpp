// tinymd_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A sequential FP64 restatement of tinyMD's `cpu` backend (vector width 1,
// backend/backend_cpu.impala:1) for the single-domain short-range MD timestep.
// It exports the same `md_*` C-ABI as the CUDA library so the same host
// driver and the same Python test code can run against either, plus
// `oracle_*` introspection entry points used only by the parity tests.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
// load this library.  The product (molecular-dynamics_b200/) never links it.
//
// Floating point: built with -ffp-contract=off and no -ffast-math, so every
// expression below is evaluated exactly in the written operand order; the
// CUDA FP64 kernels use the same order with round-to-nearest intrinsics, which
// makes the two bit-identical wherever the summation order is also the same.
//
// Each function cites the reference file:line it restates.  Parity status:
//   * lattice / velocity generation is not in here (it is host driver code);
//     it is pinned against the reference's own initialize.h (oracle/_ref).
//   * the full-list LJ kernel is pinned bit-exactly against the reference's
//     own core/force_lj.cpp (oracle/_ref) in tests/test_oracle_pins.py.
//   * known answers (FCC lattice energy, neighbour counts) pin the rest.
//
// Extensions beyond the reference (all off by default, so defaults reproduce
// the reference): an "exact" ghost mode (ghost = root local + total periodic
// shift, no lag), a contact-fixed DEM model, potential energy / virial
// reductions (the reference has none, core/thermo.impala:18-27 is dead code)
// and OpenMP over atoms for the full-list paths (results are identical for
// any thread count there because every atom is computed independently).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
struct Vector3D { double x, y, z; };
}

namespace {

struct AABB { double xmin, xmax, ymin, ymax, zmin, zmax; };

// core/grid.impala:1-35 (only the fields the cpu backend path uses)
struct Grid {
    AABB aabb{}, world{};
    int nx = 0, ny = 0, nz = 0;
    int ncells_capacity = 0, particle_capacity = 0, cell_capacity = 0, nb_capacity = 0;
    int ncells = 0, nparticles = 0, nghost = 0;
    double xlength = 0, ylength = 0, zlength = 0, spacing = 0;
    std::vector<double> pos, vel, force, mass;          // [cap*3] / [cap]
    std::vector<int> cell_particles, cell_sizes, particles_cell;
    std::vector<int> nb_sizes, nb_lists;                 // row-major [cap][nb_cap]
};

// comm/comm.impala:1-21
struct Comm {
    int local_start = 0, send_capacity = 0, send_noffsets = 0, recv_noffsets = 0;
    std::vector<double> send_buffer;   // [send_capacity*7]
    std::vector<int> send_offsets;     // [send_capacity]
    std::vector<int8_t> send_pbc;      // [send_capacity*3]
    // extension for the exact ghost mode: root local and total shift per ghost
    std::vector<int> root;
    std::vector<int8_t> tshift;
};

Grid g;
Comm c;
bool g_alive = false;
int64_t force_iters = 0, rsq_iters = 0, integration_iters = 0;
int ghost_exact = 0;        // 0 = reference two-phase (lagged) ghost update
int dem_contact_fixed = 0;  // 0 = reference DEM closure (contact branch unreachable)
int half_ghost = 0;         // 1 = corrected half lists: local-ghost pairs kept by root order
double dem_radius = 1.0;    // core/runtime.impala:210 hard-codes 1.0

// thermo extension: last LJ potential energy sum / virial sum over list pairs
double last_epot = 0.0, last_virial = 0.0;

inline double* P(std::vector<double>& a, int i) { return &a[(size_t)i * 3]; }

// utils/utilities.impala:27-36 -- recursive integer power
double ipow(double x, int n) {
    if (n == 1) return x;
    if (n % 2 == 0) { double y = ipow(x, n / 2); return y * y; }
    return x * ipow(x, n - 1);
}

// core/grid.impala:94-150
void allocate_grid(const AABB& world, const AABB& aabb, double spacing, int cell_cap, int nb_cap) {
    g = Grid();
    g.aabb = aabb;
    g.world = world;
    g.nx = (int)std::floor((aabb.xmax - aabb.xmin + (spacing / 2.0)) / spacing) + 1;
    g.ny = (int)std::floor((aabb.ymax - aabb.ymin + (spacing / 2.0)) / spacing) + 1;
    g.nz = (int)std::floor((aabb.zmax - aabb.zmin + (spacing / 2.0)) / spacing) + 1;
    g.ncells = g.nx * g.ny * g.nz;
    g.ncells_capacity = g.ncells * 4;
    g.particle_capacity = g.ncells_capacity * 8;
    g.cell_capacity = cell_cap;
    g.nb_capacity = nb_cap;
    g.xlength = world.xmax - world.xmin;
    g.ylength = world.ymax - world.ymin;
    g.zlength = world.zmax - world.zmin;
    g.spacing = spacing;
    size_t pc = (size_t)g.particle_capacity;
    g.pos.assign(pc * 3, 0.0);
    g.vel.assign(pc * 3, 0.0);
    g.force.assign(pc * 3, 0.0);
    g.mass.assign(pc, 0.0);
    g.cell_particles.assign((size_t)g.ncells_capacity * cell_cap, 0);
    g.cell_sizes.assign(g.ncells_capacity, 0);
    g.particles_cell.assign(pc, 0);
    g.nb_sizes.assign(pc, 0);
    g.nb_lists.assign(pc * (size_t)nb_cap, 0);
}

// core/grid.impala:180-192 (preserving growth of per-particle arrays)
void reallocate_particle_capacity(int capacity) {
    std::printf("0> reallocate_particle_capacity(): %d\n", capacity);
    size_t pc = (size_t)capacity;
    g.pos.resize(pc * 3, 0.0);
    g.vel.resize(pc * 3, 0.0);
    g.force.resize(pc * 3, 0.0);
    g.mass.resize(pc, 0.0);
    g.particles_cell.resize(pc, 0);
    g.nb_sizes.resize(pc, 0);
    g.nb_lists.assign(pc * (size_t)g.nb_capacity, 0);
    g.particle_capacity = capacity;
}

// core/grid.impala:194-198
void reallocate_cell_capacity(int capacity) {
    std::printf("0> reallocate_cell_capacity(): %d\n", capacity);
    g.cell_particles.assign((size_t)g.ncells_capacity * capacity, 0);
    g.cell_capacity = capacity;
}

// core/grid.impala:200-204
void reallocate_neighborlist_capacity(int capacity) {
    std::printf("0> reallocate_neighborlist_capacity(): %d\n", capacity);
    g.nb_lists.assign((size_t)g.particle_capacity * capacity, 0);
    g.nb_capacity = capacity;
}

// comm/comm.impala:165-198 (send buffer sizing)
void alloc_comm() {
    c = Comm();
    long max_neighs = 6;
    long max_faces = std::max(std::max((long)g.nx * g.ny, (long)g.nx * g.nz), (long)g.ny * g.nz);
    c.send_capacity = (int)(max_neighs * max_faces) * 20;
    c.send_buffer.assign((size_t)c.send_capacity * 7, 0.0);
    c.send_offsets.assign(c.send_capacity, 0);
    c.send_pbc.assign((size_t)c.send_capacity * 3, 0);
    c.root.assign(c.send_capacity, 0);
    c.tshift.assign((size_t)c.send_capacity * 3, 0);
}

// comm/comm.impala:234-240
void resize_send_capacity(int capacity) {
    std::printf("0> resize_send_capacity(): %d\n", capacity);
    c.send_buffer.resize((size_t)capacity * 7, 0.0);
    c.send_offsets.resize(capacity, 0);
    c.send_pbc.resize((size_t)capacity * 3, 0);
    c.root.resize(capacity, 0);
    c.tshift.resize((size_t)capacity * 3, 0);
    c.send_capacity = capacity;
}

// core/grid.impala:265-277
int add_ghost_slots(int slots) {
    int first = g.nparticles + g.nghost;
    if (first + slots > g.particle_capacity) {
        int cap = g.particle_capacity + g.particle_capacity / 10 + slots;
        reallocate_particle_capacity(cap);
    }
    g.nghost += slots;
    return first;
}

// core/grid.impala:406-411 and 419-426 (dense cell list)
int cell_index_of(const double* p) {
    int i = (int)std::floor((p[0] - g.aabb.xmin) / g.spacing);
    int j = (int)std::floor((p[1] - g.aabb.ymin) / g.spacing);
    int k = (int)std::floor((p[2] - g.aabb.zmin) / g.spacing);
    return (k * g.ny + j) * g.nx + i;
}

// comm/comm.impala:152-162
void pbc_correct(double* p) {
    double cx = p[0], cy = p[1], cz = p[2];
    if (p[0] < g.world.xmin) cx += g.xlength;
    if (p[0] > g.world.xmax) cx -= g.xlength;
    if (p[1] < g.world.ymin) cy += g.ylength;
    if (p[1] > g.world.ymax) cy -= g.ylength;
    if (p[2] < g.world.zmin) cz += g.zlength;
    if (p[2] > g.world.zmax) cz -= g.zlength;
    p[0] = cx; p[1] = cy; p[2] = cz;
}

// comm/lb.impala:88-100
void pbc_flags_from_position(const double* p, int px, int py, int pz, int8_t* f) {
    f[0] = f[1] = f[2] = 0;
    bool all = px == 0 && py == 0 && pz == 0;
    if ((all || px > 0) && p[0] < g.world.xmin + g.spacing) f[0] = 1;
    if ((all || px < 0) && p[0] > g.world.xmax - g.spacing) f[0] = -1;
    if ((all || py > 0) && p[1] < g.world.ymin + g.spacing) f[1] = 1;
    if ((all || py < 0) && p[1] > g.world.ymax - g.spacing) f[1] = -1;
    if ((all || pz > 0) && p[2] < g.world.zmin + g.spacing) f[2] = 1;
    if ((all || pz < 0) && p[2] > g.world.zmax - g.spacing) f[2] = -1;
}

// comm/comm.impala:105-127 -- the no-walberla 6-direction pattern, in order
// x+, x-, y+, y-, z+, z-.  Returns true and the shifted position / flags when
// the particle must be sent in direction `dir`.
bool border_position(int dir, const double* p, double* adj, int8_t* flags) {
    double dsp = g.spacing * 2.0;
    bool cond = false;
    int px = 0, py = 0, pz = 0;
    switch (dir) {
        case 0: cond = p[0] > g.aabb.xmax - dsp; px = -1; break;
        case 1: cond = p[0] < g.aabb.xmin + dsp; px = 1; break;
        case 2: cond = p[1] > g.aabb.ymax - dsp; py = -1; break;
        case 3: cond = p[1] < g.aabb.ymin + dsp; py = 1; break;
        case 4: cond = p[2] > g.aabb.zmax - dsp; pz = -1; break;
        default: cond = p[2] < g.aabb.zmin + dsp; pz = 1; break;
    }
    if (!cond) return false;
    pbc_flags_from_position(p, px, py, pz, flags);
    adj[0] = p[0] + g.xlength * (double)flags[0];
    adj[1] = p[1] + g.ylength * (double)flags[1];
    adj[2] = p[2] + g.zlength * (double)flags[2];
    return true;
}

// comm/comm.impala:528-642 (single process: every pass is "local") together
// with unpack_local_particles, comm/comm.impala:723-734.
void borders() {
    int isend = 0, ilocal = 0;
    g.nghost = 0;
    for (int neigh = 0; neigh < 6; ++neigh) {
        int resize = 1;
        int counter = isend;
        while (resize > 0) {
            counter = isend;
            resize = 0;
            int n = g.nparticles + g.nghost;
            for (int i = 0; i < n; ++i) {
                double adj[3];
                int8_t fl[3];
                if (!border_position(neigh, P(g.pos, i), adj, fl)) continue;
                int slot = counter++;
                if (slot >= c.send_capacity) {
                    if (resize < slot) resize = slot;
                    continue;
                }
                c.send_buffer[(size_t)slot * 4 + 0] = g.mass[i];
                c.send_buffer[(size_t)slot * 4 + 1] = adj[0];
                c.send_buffer[(size_t)slot * 4 + 2] = adj[1];
                c.send_buffer[(size_t)slot * 4 + 3] = adj[2];
                c.send_pbc[(size_t)slot * 3 + 0] = fl[0];
                c.send_pbc[(size_t)slot * 3 + 1] = fl[1];
                c.send_pbc[(size_t)slot * 3 + 2] = fl[2];
                c.send_offsets[slot] = i;
                // exact-mode bookkeeping (extension): chain root and total shift
                if (i < g.nparticles) {
                    c.root[slot] = i;
                    for (int d = 0; d < 3; ++d) c.tshift[(size_t)slot * 3 + d] = fl[d];
                } else {
                    int sg = i - g.nparticles;
                    c.root[slot] = c.root[sg];
                    for (int d = 0; d < 3; ++d)
                        c.tshift[(size_t)slot * 3 + d] = (int8_t)(c.tshift[(size_t)sg * 3 + d] + fl[d]);
                }
            }
            if (resize > 0) resize_send_capacity(resize * 2);
        }
        isend = counter;
        if (neigh % 2 != 0) {
            add_ghost_slots(isend - ilocal);
            int recv_offset = g.nparticles + ilocal;
            for (int i = 0; i < isend - ilocal; ++i) {
                size_t idx = (size_t)(ilocal + i) * 4;
                int off = recv_offset + i;
                g.mass[off] = c.send_buffer[idx];
                P(g.pos, off)[0] = c.send_buffer[idx + 1];
                P(g.pos, off)[1] = c.send_buffer[idx + 2];
                P(g.pos, off)[2] = c.send_buffer[idx + 3];
            }
            ilocal = isend;
        }
    }
    c.local_start = 0;
    c.send_noffsets = isend;
    c.recv_noffsets = 0;
    if (dem_contact_fixed) {
        for (int s = 0; s < isend; ++s) {
            int r = c.root[s];
            for (int d = 0; d < 3; ++d) P(g.vel, g.nparticles + s)[d] = P(g.vel, r)[d];
        }
    }
}

// comm/comm.impala:334-388: pack every ghost's source position first, then
// unpack (two phases), which is what makes chained edge/corner ghosts lag.
void synchronize_ghost_layer() {
    int n = c.send_noffsets;
    std::vector<double> buf((size_t)n * 3);
    if (!ghost_exact) {
        for (int i = 0; i < n; ++i) {
            const double* p = P(g.pos, c.send_offsets[i]);
            buf[(size_t)i * 3 + 0] = p[0] + g.xlength * (double)c.send_pbc[(size_t)i * 3 + 0];
            buf[(size_t)i * 3 + 1] = p[1] + g.ylength * (double)c.send_pbc[(size_t)i * 3 + 1];
            buf[(size_t)i * 3 + 2] = p[2] + g.zlength * (double)c.send_pbc[(size_t)i * 3 + 2];
        }
    } else {
        for (int i = 0; i < n; ++i) {
            const double* p = P(g.pos, c.root[i]);
            buf[(size_t)i * 3 + 0] = p[0] + g.xlength * (double)c.tshift[(size_t)i * 3 + 0];
            buf[(size_t)i * 3 + 1] = p[1] + g.ylength * (double)c.tshift[(size_t)i * 3 + 1];
            buf[(size_t)i * 3 + 2] = p[2] + g.zlength * (double)c.tshift[(size_t)i * 3 + 2];
        }
    }
    for (int i = 0; i < n; ++i) {
        double* q = P(g.pos, g.nparticles + c.recv_noffsets + i);
        q[0] = buf[(size_t)(c.local_start + i) * 3 + 0];
        q[1] = buf[(size_t)(c.local_start + i) * 3 + 1];
        q[2] = buf[(size_t)(c.local_start + i) * 3 + 2];
    }
    if (dem_contact_fixed) {
        for (int i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d) P(g.vel, g.nparticles + i)[d] = P(g.vel, c.root[i])[d];
    }
}

// core/grid.impala:280-321 (fill_cells with ghost = true)
void fill_cells() {
    int resize = 1;
    while (resize > 0) {
        resize = 0;
        std::fill(g.cell_sizes.begin(), g.cell_sizes.begin() + g.ncells, 0);
        int n = g.nparticles + g.nghost;
        for (int i = 0; i < n; ++i) {
            int ci = cell_index_of(P(g.pos, i));
            if (ci >= 0 && ci < g.ncells) {
                int slot = g.cell_sizes[ci]++;
                if (slot >= g.cell_capacity) {
                    if (resize < slot) resize = slot;
                } else {
                    g.cell_particles[(size_t)ci * g.cell_capacity + slot] = i;
                    g.particles_cell[i] = ci;
                }
            }
        }
        if (resize > 0) reallocate_cell_capacity(resize * 2);
    }
}

// core/neighborlist.impala:1-78
void assemble_neighborlists(int half, double cutoff) {
    int resize = 1;
    while (resize > 0) {
        resize = 0;
        const double cut2 = cutoff * cutoff;
        const int nbcap = g.nb_capacity;
#pragma omp parallel for schedule(static) reduction(max : resize)
        for (int i = 0; i < g.nparticles; ++i) {
            const double* pi = P(g.pos, i);
            int cell = g.particles_cell[i];
            int cnt = 0;
            for (int oz = -1; oz < 2; ++oz)
                for (int oy = -1; oy < 2; ++oy)
                    for (int ox = -1; ox < 2; ++ox) {
                        int nbc = cell + oz * g.nx * g.ny + oy * g.nx + ox;
                        if (nbc < 0 || nbc >= g.ncells) continue;
                        bool chk = (nbc == cell);
                        int size = g.cell_sizes[nbc];
                        const int* cp = &g.cell_particles[(size_t)nbc * g.cell_capacity];
                        for (int k = 0; k < size; ++k) {
                            int j = cp[k];
                            if (chk && i == j) continue;
                            // core/neighborlist.impala:34; the corrected mode orders a
                            // ghost by its root local so boundary pairs are kept once
                            const int jo = (half_ghost && j >= g.nparticles) ? c.root[j - g.nparticles] : j;
                            if (half != 0 && !(i > jo)) continue;
                            const double* pj = P(g.pos, j);
                            double dx = pi[0] - pj[0];
                            double dy = pi[1] - pj[1];
                            double dz = pi[2] - pj[2];
                            double rsq = dx * dx + dy * dy + dz * dz;
                            if (rsq <= cut2) {
                                if (cnt >= nbcap) {
                                    if (resize < cnt) resize = cnt;
                                } else {
                                    g.nb_lists[(size_t)i * nbcap + cnt] = j;
                                }
                                cnt++;
                            }
                        }
                    }
            g.nb_sizes[i] = cnt;
        }
        if (resize > 0) reallocate_neighborlist_capacity(resize * 2);
    }
}

// core/runtime.impala:188-201 -- the LJ closure.
inline void lj_pair(double rsq, double sigma6, double eps, double& f, double& sr6_out) {
    double sr2 = 1.0 / rsq;
    double sr6 = sr2 * sr2 * sr2 * sigma6;
    f = 48.0 * sr6 * (sr6 - 0.5) * sr2 * eps;
    sr6_out = sr6;
}

// core/compute.impala:1-48 with the LJ closure.  Also accumulates the
// (extension) potential energy 4*eps*sr6*(sr6-1) and virial f*rsq per list
// pair inside the cutoff.
void compute_lj(int half, double rc, double eps, double sigma) {
    const double sigma6 = ipow(sigma, 6);
    const double rsq_cut = rc * rc;
    const int N = g.nparticles;
    const int nbcap = g.nb_capacity;
    int64_t total = 0, inside = 0;
    double epot = 0.0, vir = 0.0;
    if (half) {
        for (int i = 0; i < N; ++i) P(g.force, i)[0] = P(g.force, i)[1] = P(g.force, i)[2] = 0.0;
        for (int i = 0; i < N; ++i) {
            const double* pi = P(g.pos, i);
            for (int n = 0; n < g.nb_sizes[i]; ++n) {
                int j = g.nb_lists[(size_t)i * nbcap + n];
                const double* pj = P(g.pos, j);
                double dx = pi[0] - pj[0], dy = pi[1] - pj[1], dz = pi[2] - pj[2];
                double rsq = dx * dx + dy * dy + dz * dz;
                if (rsq < rsq_cut) {
                    double f, sr6;
                    lj_pair(rsq, sigma6, eps, f, sr6);
                    double fx = dx * f, fy = dy * f, fz = dz * f;
                    double* Fi = P(g.force, i);
                    Fi[0] += fx; Fi[1] += fy; Fi[2] += fz;
                    const int jt = j < N ? j : (half_ghost ? c.root[j - N] : -1);
                    if (jt >= 0) {
                        double* Fj = P(g.force, jt);
                        Fj[0] += -fx; Fj[1] += -fy; Fj[2] += -fz;
                    }
                    epot += 4.0 * eps * sr6 * (sr6 - 1.0);
                    vir += f * rsq;
                    inside++;
                }
                total++;
            }
        }
    } else {
#pragma omp parallel for schedule(static) reduction(+ : total, inside, epot, vir)
        for (int i = 0; i < N; ++i) {
            const double* pi = P(g.pos, i);
            double fx = 0.0, fy = 0.0, fz = 0.0;
            double ei = 0.0, wi = 0.0;
            for (int n = 0; n < g.nb_sizes[i]; ++n) {
                int j = g.nb_lists[(size_t)i * nbcap + n];
                const double* pj = P(g.pos, j);
                double dx = pi[0] - pj[0], dy = pi[1] - pj[1], dz = pi[2] - pj[2];
                double rsq = dx * dx + dy * dy + dz * dz;
                if (rsq < rsq_cut) {
                    double f, sr6;
                    lj_pair(rsq, sigma6, eps, f, sr6);
                    fx = fx + dx * f;
                    fy = fy + dy * f;
                    fz = fz + dz * f;
                    ei += 4.0 * eps * sr6 * (sr6 - 1.0);
                    wi += f * rsq;
                    inside++;
                }
                total++;
            }
            double* Fi = P(g.force, i);
            Fi[0] = fx; Fi[1] = fy; Fi[2] = fz;
            epot += ei;
            vir += wi;
        }
    }
    force_iters = total;
    rsq_iters = inside;
    last_epot = epot;
    last_virial = vir;
}

// core/runtime.impala:203-247 -- the DEM closure.  With the reference
// condition (penetration_depth > 0 inside rsq < (2r)^2) the contact branch is
// unreachable, so the force is identically zero; that is reproduced.  The
// opt-in contact-fixed model (extension) uses radius = dem_radius, overlap
// delta = 2R - r > 0, a dissipative normal spring-dashpot and a Coulomb-capped
// tangential dashpot opposing the tangential relative velocity.
void dem_pair(int i, int j, const double* del, double rsq, double dn, double dt_, double k, double mu,
              double* out) {
    out[0] = out[1] = out[2] = 0.0;
    const double radius = dem_contact_fixed ? dem_radius : 1.0;
    if (!(rsq < (radius * 2.0) * (radius * 2.0))) return;
    double len = std::sqrt(rsq);
    double pen = len - radius * 2.0;
    if (!dem_contact_fixed) {
        if (!(pen > 0.0)) return;
        // reference formulas (unreachable, kept for completeness)
        double n[3] = {del[0] * (1.0 / len), del[1] * (1.0 / len), del[2] * (1.0 / len)};
        const double* v1 = P(g.vel, i);
        const double* v2 = P(g.vel, j);
        double rv[3] = {v1[0] - v2[0], v1[1] - v2[1], v1[2] - v2[2]};
        double vn = rv[0] * n[0] + rv[1] * n[1] + rv[2] * n[2];
        double vt[3] = {rv[0] - n[0] * vn, rv[1] - n[1] * vn, rv[2] - n[2] * vn};
        double vtl = std::sqrt(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
        double fn = dn * vn - k * pen;
        double t1 = dt_ * vtl, t2 = mu * fn;
        double ft = t1 < t2 ? t1 : t2;
        for (int d = 0; d < 3; ++d) out[d] = n[d] * fn + (vt[d] * (1.0 / vtl)) * ft;
        return;
    }
    if (!(len > 0.0)) return;
    double delta = radius * 2.0 - len;
    double inv = 1.0 / len;
    double n[3] = {del[0] * inv, del[1] * inv, del[2] * inv};
    const double* v1 = P(g.vel, i);
    const double* v2 = P(g.vel, j);
    double rv[3] = {v1[0] - v2[0], v1[1] - v2[1], v1[2] - v2[2]};
    double vn = rv[0] * n[0] + rv[1] * n[1] + rv[2] * n[2];
    double vt[3] = {rv[0] - n[0] * vn, rv[1] - n[1] * vn, rv[2] - n[2] * vn};
    double vtl = std::sqrt(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
    double fn = k * delta - dn * vn;
    if (fn < 0.0) fn = 0.0;
    double t1 = dt_ * vtl, t2 = mu * fn;
    double ft = t1 < t2 ? t1 : t2;
    double tinv = vtl > 0.0 ? 1.0 / vtl : 0.0;
    for (int d = 0; d < 3; ++d) out[d] = n[d] * fn - (vt[d] * tinv) * ft;
}

void compute_dem(int half, double rc, double dn, double dt_, double k, double mu) {
    const double rsq_cut = rc * rc;
    const int N = g.nparticles;
    const int nbcap = g.nb_capacity;
    int64_t total = 0, inside = 0;
    if (half) {
        for (int i = 0; i < N; ++i) P(g.force, i)[0] = P(g.force, i)[1] = P(g.force, i)[2] = 0.0;
        for (int i = 0; i < N; ++i) {
            const double* pi = P(g.pos, i);
            for (int n = 0; n < g.nb_sizes[i]; ++n) {
                int j = g.nb_lists[(size_t)i * nbcap + n];
                const double* pj = P(g.pos, j);
                double del[3] = {pi[0] - pj[0], pi[1] - pj[1], pi[2] - pj[2]};
                double rsq = del[0] * del[0] + del[1] * del[1] + del[2] * del[2];
                if (rsq < rsq_cut) {
                    double f[3];
                    dem_pair(i, j, del, rsq, dn, dt_, k, mu, f);
                    double* Fi = P(g.force, i);
                    Fi[0] += f[0]; Fi[1] += f[1]; Fi[2] += f[2];
                    const int jt = j < N ? j : (half_ghost ? c.root[j - N] : -1);
                    if (jt >= 0) {
                        double* Fj = P(g.force, jt);
                        Fj[0] += -f[0]; Fj[1] += -f[1]; Fj[2] += -f[2];
                    }
                    inside++;
                }
                total++;
            }
        }
    } else {
#pragma omp parallel for schedule(static) reduction(+ : total, inside)
        for (int i = 0; i < N; ++i) {
            const double* pi = P(g.pos, i);
            double F[3] = {0.0, 0.0, 0.0};
            for (int n = 0; n < g.nb_sizes[i]; ++n) {
                int j = g.nb_lists[(size_t)i * nbcap + n];
                const double* pj = P(g.pos, j);
                double del[3] = {pi[0] - pj[0], pi[1] - pj[1], pi[2] - pj[2]};
                double rsq = del[0] * del[0] + del[1] * del[1] + del[2] * del[2];
                if (rsq < rsq_cut) {
                    double f[3];
                    dem_pair(i, j, del, rsq, dn, dt_, k, mu, f);
                    F[0] = F[0] + f[0];
                    F[1] = F[1] + f[1];
                    F[2] = F[2] + f[2];
                    inside++;
                }
                total++;
            }
            double* Fi = P(g.force, i);
            Fi[0] = F[0]; Fi[1] = F[1]; Fi[2] = F[2];
        }
    }
    force_iters = total;
    rsq_iters = inside;
}

// core/thermo.impala:1-16
double temperature() {
    const double mass = 1.0;
    const double mvv2e = 1.0;
    int dof = g.nparticles * 3 - 3;
    double t_scale = mvv2e / (double)dof;
    double t = 0.0;
    for (int i = 0; i < g.nparticles; ++i) {
        const double* v = P(g.vel, i);
        t += (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * mass;
    }
    return t * t_scale;
}

}  // namespace

extern "C" {

// core/runtime.impala:7-37
int md_initialize_grid(const double* masses, const Vector3D* positions, const Vector3D* velocities, int n,
                       const double* aabb, const double* rank_aabb, double cell_spacing, int cell_capacity,
                       int neighborlist_capacity) {
    AABB world{aabb[0], aabb[1], aabb[2], aabb[3], aabb[4], aabb[5]};
    AABB ext{rank_aabb[0] - cell_spacing, rank_aabb[1] + cell_spacing, rank_aabb[2] - cell_spacing,
             rank_aabb[3] + cell_spacing, rank_aabb[4] - cell_spacing, rank_aabb[5] + cell_spacing};
    allocate_grid(world, ext, cell_spacing, cell_capacity, neighborlist_capacity);
    alloc_comm();
    // core/grid.impala:215-249 (insert_particle, sequential)
    for (int i = 0; i < n; ++i) {
        if (g.nparticles >= g.particle_capacity) {
            int cap = g.particle_capacity + g.particle_capacity / 10 + 10;
            reallocate_particle_capacity(cap);
        }
        int k = g.nparticles;
        g.mass[k] = masses[i];
        P(g.pos, k)[0] = positions[i].x; P(g.pos, k)[1] = positions[i].y; P(g.pos, k)[2] = positions[i].z;
        P(g.vel, k)[0] = velocities[i].x; P(g.vel, k)[1] = velocities[i].y; P(g.vel, k)[2] = velocities[i].z;
        P(g.force, k)[0] = P(g.force, k)[1] = P(g.force, k)[2] = 0.0;
        g.nb_sizes[k] = 0;
        g.nparticles++;
    }
    g_alive = true;
    return g.nparticles;
}

// core/runtime.impala:158-186
void md_create_velocity(double t_request) {
    int n = g.nparticles;
    double vt[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; ++i) {
        const double* v = P(g.vel, i);
        vt[0] = vt[0] + v[0]; vt[1] = vt[1] + v[1]; vt[2] = vt[2] + v[2];
    }
    vt[0] = vt[0] / (double)n; vt[1] = vt[1] / (double)n; vt[2] = vt[2] / (double)n;
    for (int i = 0; i < n; ++i) {
        double* v = P(g.vel, i);
        v[0] = v[0] - vt[0]; v[1] = v[1] - vt[1]; v[2] = v[2] - vt[2];
    }
    double t = temperature();
    double factor = std::sqrt(t_request / t);
    for (int i = 0; i < n; ++i) {
        double* v = P(g.vel, i);
        v[0] = v[0] * factor; v[1] = v[1] * factor; v[2] = v[2] * factor;
    }
}

void md_copy_data_to_accelerator(void) {}
void md_copy_data_from_accelerator(void) {}
void md_exchange_particles(void) {}  // comm/comm.impala:392-525: no remote ranks in one process
void md_borders(void) { borders(); }
void md_distribute_particles(void) { fill_cells(); }  // sort_particles() == false, core/grid.impala:54
void md_assemble_neighborlists(bool half, double cutoff) { assemble_neighborlists(half ? 1 : 0, cutoff); }
void md_synchronize_ghost_layer(void) { synchronize_ghost_layer(); }
void md_compute_lennard_jones(bool half, double rc, double eps, double sigma) {
    compute_lj(half ? 1 : 0, rc, eps, sigma);
}
void md_compute_dem(bool half, double rc, double damping_n, double damping_t, double stiffness, double friction) {
    compute_dem(half ? 1 : 0, rc, damping_n, damping_t, stiffness, friction);
}

// core/compute.impala:97-106
void md_initial_integration(double dt) {
    const int N = g.nparticles;
    const double h = 0.5 * dt;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        double* v = P(g.vel, i);
        const double* f = P(g.force, i);
        double* x = P(g.pos, i);
        v[0] = v[0] + f[0] * h; v[1] = v[1] + f[1] * h; v[2] = v[2] + f[2] * h;
        x[0] = x[0] + v[0] * dt; x[1] = x[1] + v[1] * dt; x[2] = x[2] + v[2] * dt;
    }
    integration_iters = N;
}

// core/compute.impala:108-116
void md_final_integration(double dt) {
    const int N = g.nparticles;
    const double h = 0.5 * dt;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        double* v = P(g.vel, i);
        const double* f = P(g.force, i);
        v[0] = v[0] + f[0] * h; v[1] = v[1] + f[1] * h; v[2] = v[2] + f[2] * h;
    }
    integration_iters = N;
}

// core/compute.impala:118-122
void md_enforce_pbc(void) {
    for (int i = 0; i < g.nparticles; ++i) pbc_correct(P(g.pos, i));
}

// core/grid.impala:483-499
int md_write_grid_data_to_arrays(double* m, Vector3D* x, Vector3D* v, Vector3D* f) {
    for (int i = 0; i < g.nparticles; ++i) {
        m[i] = g.mass[i];
        x[i] = {P(g.pos, i)[0], P(g.pos, i)[1], P(g.pos, i)[2]};
        v[i] = {P(g.vel, i)[0], P(g.vel, i)[1], P(g.vel, i)[2]};
        f[i] = {P(g.force, i)[0], P(g.force, i)[1], P(g.force, i)[2]};
    }
    return g.nparticles;
}

// core/grid.impala:501-518 (note: returns nparticles, as the reference does)
int md_write_grid_ghost_data_to_arrays(double* m, Vector3D* x, Vector3D* v, Vector3D* f) {
    for (int p = g.nparticles; p < g.nparticles + g.nghost; ++p) {
        int i = p - g.nparticles;
        m[i] = g.mass[p];
        x[i] = {P(g.pos, p)[0], P(g.pos, p)[1], P(g.pos, p)[2]};
        v[i] = {P(g.vel, p)[0], P(g.vel, p)[1], P(g.vel, p)[2]};
        f[i] = {P(g.force, p)[0], P(g.force, p)[1], P(g.force, p)[2]};
    }
    return g.nparticles;
}

// core/grid.impala:520-546
int md_write_grid_aabb_data_to_arrays(double* m, Vector3D* x, Vector3D* v, Vector3D* f) {
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int k = 0; k < 2; ++k) {
                int idx = k * 4 + j * 2 + i;
                m[idx] = 0.0;
                x[idx] = {i == 0 ? g.aabb.xmin : g.aabb.xmax, j == 0 ? g.aabb.ymin : g.aabb.ymax,
                          k == 0 ? g.aabb.zmin : g.aabb.zmax};
                v[idx] = {0.0, 0.0, 0.0};
                f[idx] = {0.0, 0.0, 0.0};
            }
    return g.nparticles;
}

int md_get_number_of_particles(void) { return g.nparticles; }
int md_get_number_of_ghost_particles(void) { return g.nghost; }
int md_get_world_size(void) { return 1; }
int md_get_world_rank(void) { return 0; }
void md_mpi_initialize(void) {}
void md_mpi_finalize(void) {}
void md_barrier(void) {}

// comm/comm.impala:254-331 with one rank
void md_get_node_bounding_box(const double* aabb, double (*rank)[6]) {
    double xl = (aabb[1] - aabb[0]) / 1.0, yl = (aabb[3] - aabb[2]) / 1.0, zl = (aabb[5] - aabb[4]) / 1.0;
    double xmin = aabb[0] + xl * 0.0, ymin = aabb[2] + yl * 0.0, zmin = aabb[4] + zl * 0.0;
    (*rank)[0] = xmin; (*rank)[1] = xmin + xl;
    (*rank)[2] = ymin; (*rank)[3] = ymin + yl;
    (*rank)[4] = zmin; (*rank)[5] = zmin + zl;
}

// core/runtime.impala:280-296
void md_report_iterations(void) {
    std::printf("ForceIters RsqIters IntegrationIters\n");
    std::printf("%lld %lld %lld \n", (long long)force_iters, (long long)rsq_iters, (long long)integration_iters);
    std::fflush(stdout);
}

// core/runtime.impala:298-316
void md_report_particles(void) {
    std::printf("# Local # Ghost Temp\n");
    std::printf("%d %d %g\n", g.nparticles, g.nghost, temperature());
    std::fflush(stdout);
}

void md_report_time(double total, double force, double neigh, double comm, double lb, double other) {
    std::printf("Total Force Neigh Comm Balance Other\n");
    std::printf("%g %g %g %g %g %g \n", total, force, neigh, comm, lb, other);
    std::fflush(stdout);
}

void md_deallocate_grid(void) {
    g = Grid();
    c = Comm();
    g_alive = false;
}

// ---- oracle_* introspection (tests only) ---------------------------------
void oracle_set_ghost_mode(int exact) { ghost_exact = exact; }
void oracle_set_half_mode(int ghost_pairs) { half_ghost = ghost_pairs ? 1 : 0; }
void oracle_set_dem_mode(int contact_fixed, double radius) {
    dem_contact_fixed = contact_fixed;
    dem_radius = radius;
}
void oracle_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}
int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
double oracle_temperature(void) { return temperature(); }
void oracle_grid_info(int* out) {  // nx ny nz ncells cell_capacity nb_capacity
    out[0] = g.nx; out[1] = g.ny; out[2] = g.nz; out[3] = g.ncells; out[4] = g.cell_capacity;
    out[5] = g.nb_capacity;
}
void oracle_aabb(double* out) {
    out[0] = g.aabb.xmin; out[1] = g.aabb.xmax; out[2] = g.aabb.ymin;
    out[3] = g.aabb.ymax; out[4] = g.aabb.zmin; out[5] = g.aabb.zmax;
}
// Positions of locals then ghosts, [n_all][3].
void oracle_positions(double* out) {
    int n = g.nparticles + g.nghost;
    std::memcpy(out, g.pos.data(), sizeof(double) * 3 * (size_t)n);
}
void oracle_velocities(double* out) { std::memcpy(out, g.vel.data(), sizeof(double) * 3 * (size_t)g.nparticles); }
void oracle_forces(double* out) { std::memcpy(out, g.force.data(), sizeof(double) * 3 * (size_t)g.nparticles); }
void oracle_set_positions(const double* in) {  // locals only
    std::memcpy(g.pos.data(), in, sizeof(double) * 3 * (size_t)g.nparticles);
}
void oracle_set_velocities(const double* in) {
    std::memcpy(g.vel.data(), in, sizeof(double) * 3 * (size_t)g.nparticles);
}
// Neighbour lists in reference index space: sizes[N], lists[N][cap] (row-major).
int oracle_neighbor_lists(int* sizes, int* lists, int cap) {
    for (int i = 0; i < g.nparticles; ++i) {
        sizes[i] = g.nb_sizes[i];
        for (int n = 0; n < g.nb_sizes[i] && n < cap; ++n) lists[(size_t)i * cap + n] = g.nb_lists[(size_t)i * g.nb_capacity + n];
    }
    return g.nb_capacity;
}
// Ghost bookkeeping: src[G], pbc[G][3], root[G], tshift[G][3].
void oracle_ghosts(int* src, int* pbc, int* root, int* tshift) {
    for (int s = 0; s < c.send_noffsets; ++s) {
        src[s] = c.send_offsets[s];
        root[s] = c.root[s];
        for (int d = 0; d < 3; ++d) {
            pbc[s * 3 + d] = c.send_pbc[(size_t)s * 3 + d];
            tshift[s * 3 + d] = c.tshift[(size_t)s * 3 + d];
        }
    }
}
// Cell lists: sizes[ncells], members[ncells][cell_capacity] (row-major).
void oracle_cells(int* sizes, int* members) {
    for (int ci = 0; ci < g.ncells; ++ci) {
        sizes[ci] = g.cell_sizes[ci];
        for (int k = 0; k < g.cell_sizes[ci] && k < g.cell_capacity; ++k)
            members[(size_t)ci * g.cell_capacity + k] = g.cell_particles[(size_t)ci * g.cell_capacity + k];
    }
}
// Last LJ force call: potential energy sum and virial sum over list pairs.
void oracle_last_thermo(double* out) { out[0] = last_epot; out[1] = last_virial; }
void oracle_iters(long long* out) { out[0] = force_iters; out[1] = rsq_iters; out[2] = integration_iters; }

}  // extern "C"
