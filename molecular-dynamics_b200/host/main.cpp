// main.cpp -- the md command-line driver (host side of the tinyMD path).
//
// Same flags, benchmark setups, run loop and report lines as the reference
// driver (main.cpp:33-803 of tinyMD; one process, no waLBerla), calling the
// md_* C ABI.  Additive options select the B200 forms (--precision,
// --ghost, --dem_model, --dem_radius) and print periodic thermo lines
// (--thermo) and throughput (--perf).
//
// Built twice: against libtinymd_b200.so (the product, molecular-dynamics_b200/
// build.py) and, with TINYMD_DRIVER_CPU_ORACLE, against the CPU oracle
// (oracle/Makefile), which is the timed CPU baseline.

#include <getopt.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#if defined(__x86_64__) || defined(__amd64__)
#include <xmmintrin.h>
#include <pmmintrin.h>
#endif

#include "driver_ext.h"
#include "setups.h"
#include "tinymd_b200.h"

namespace {

using Clock = std::chrono::high_resolution_clock;

enum Bucket { T_FORCE = 0, T_NEIGH, T_COMM, T_BALANCE, T_OTHER, T_COUNT };

// Per-run, per-bucket wall-clock accumulators in ms (the reference's
// MultiTimer, MultiTimer.h:7-54).  The reference's run total is summed with
// an int seed (MultiTimer.h:33) and so truncated; the total here is exact.
struct PhaseClock {
    std::vector<std::vector<double>> ms;
    Clock::time_point t0;
    size_t run = 0;
    explicit PhaseClock(size_t runs) : ms(runs, std::vector<double>(T_COUNT, 0.0)) {}
    void start() { t0 = Clock::now(); }
    void accum(int b) {
        auto t = Clock::now();
        ms[run][b] += std::chrono::duration<double, std::milli>(t - t0).count();
        t0 = Clock::now();
    }
    void finish() { ++run; }
    double avg(int b) const {
        double s = 0;
        for (auto& r : ms) s += r[b];
        return s / (double)ms.size();
    }
    double avg_total() const {
        double s = 0;
        for (int b = 0; b < T_COUNT; ++b) s += avg(b);
        return s;
    }
};

void usage(const char* name) {
    std::cout << "Usage: " << name << " [OPTION]...\n"
              << "Short-range molecular dynamics (tinyMD timestep) on " << drv::backend() << ".\n\n"
              << "\t-f, --force_field=STRING  force field: lj (default) or dem\n"
              << "\t-b, --benchmark=STRING    default, half, body_collision, granular_gas or granular_gas_fcc\n"
              << "\t-x, --nx=SIZE             unit cells in x (default 32)\n"
              << "\t-y, --ny=SIZE             unit cells in y (default 32)\n"
              << "\t-z, --nz=SIZE             unit cells in z (default 32)\n"
              << "\t-s, --timesteps=NUMBER    timesteps (default 100)\n"
              << "\t-r, --runs=NUMBER         runs (default 1)\n"
              << "\t-t, --threads=NUMBER      threads (reported; host threads of the CPU baseline build)\n"
              << "\t-a, --algorithm=STRING    load balancing algorithm (accepted; single process)\n"
              << "\t-v, --vtk=DIRECTORY       write VTK files of the first run into DIRECTORY\n"
              << "\t    --reneigh=NUMBER      steps between neighbour-list rebuilds (default 20)\n"
              << "\t    --rebalance=NUMBER    steps between load balancing (default 100)\n"
              << "\t    --dt=REAL             timestep (default 0.005)\n"
              << "\t    --temp=REAL           initial temperature (default 1.44)\n"
              << "\t    --cutoff=REAL         cutoff radius (default 2.5)\n"
              << "\t    --verlet=REAL         Verlet buffer (default 0.3)\n"
              << "\t    --epsilon=REAL        LJ epsilon (default 1.0)\n"
              << "\t    --sigma=REAL          LJ sigma (default 1.0)\n"
              << "\t    --damping_n=REAL      DEM normal damping (default 0.0)\n"
              << "\t    --damping_t=REAL      DEM tangential damping (default 0.0)\n"
              << "\t    --stiffness=REAL      DEM stiffness (default 0.0)\n"
              << "\t    --friction=REAL       DEM friction (default 0.0)\n"
              << "\t    --potmin=REAL         lattice constant / potential minimum (default 1.6796)\n"
              << "\t    --half_nb             half neighbour lists\n"
              << "\t    --prebalance          static load balancing before the run (accepted; single process)\n"
              << "\t    --precision=STRING    fp64 (default) or mixed (FP32 pair forces)\n"
              << "\t    --ghost=STRING        reference (default, two-phase ghost refresh) or exact\n"
              << "\t    --half_mode=STRING    reference (default: half lists drop periodic-boundary pairs) or ghost\n"
              << "\t    --dem_model=STRING    reference (default) or fixed (contact-fixed spring-dashpot)\n"
              << "\t    --dem_radius=REAL     contact radius of the fixed DEM model (default cutoff/2)\n"
              << "\t    --thermo=NUMBER       print a thermo line every NUMBER steps (0 = off)\n"
              << "\t    --perf                print throughput after the timing report\n"
              << "\t-h, --help                this help\n";
}

void write_vtk(const std::string& file, const std::vector<double>& m, const std::vector<Vector3D>& x,
               const std::vector<Vector3D>& v, const std::vector<Vector3D>& f) {
    std::ofstream o(file);
    const size_t n = x.size();
    o << "# vtk DataFile Version 2.0\nParticle data\nASCII\nDATASET UNSTRUCTURED_GRID\n";
    o << "POINTS " << n << " double\n" << std::fixed;
    for (auto& p : x) o << p.x << " " << p.y << " " << p.z << "\n";
    o << "\n\nCELLS " << n << " " << 2 * n << "\n";
    for (size_t i = 0; i < n; ++i) o << "1 " << i << "\n";
    o << "\n\nCELL_TYPES " << n << "\n";
    for (size_t i = 0; i < n; ++i) o << "1\n";
    o << "\n\nPOINT_DATA " << m.size() << "\n";
    o << "SCALARS mass double\nLOOKUP_TABLE default\n";
    for (double w : m) o << w << "\n";
    o << "\n";
    const char* names[6] = {"velocity_x", "velocity_y", "velocity_z", "force_x", "force_y", "force_z"};
    for (int q = 0; q < 6; ++q) {
        o << "SCALARS " << names[q] << " double\nLOOKUP_TABLE default\n";
        for (size_t i = 0; i < n; ++i) {
            const Vector3D& a = q < 3 ? v[i] : f[i];
            o << (q % 3 == 0 ? a.x : (q % 3 == 1 ? a.y : a.z)) << "\n";
        }
        o << "\n";
    }
}

void vtk_dump(const std::string& dir, int step) {
    for (int kind = 0; kind < 3; ++kind) {
        int n = kind == 0 ? md_get_number_of_particles() : (kind == 1 ? md_get_number_of_ghost_particles() : 8);
        std::vector<double> m(n);
        std::vector<Vector3D> x(n), v(n), f(n);
        if (kind == 0) md_write_grid_data_to_arrays(m.data(), x.data(), v.data(), f.data());
        if (kind == 1) md_write_grid_ghost_data_to_arrays(m.data(), x.data(), v.data(), f.data());
        if (kind == 2) md_write_grid_aabb_data_to_arrays(m.data(), x.data(), v.data(), f.data());
        const char* stem[3] = {"particles_", "ghost_", "aabb_"};
        write_vtk(dir + stem[kind] + std::to_string(step) + ".vtk", m, x, v, f);
    }
}

// thermo line: step, temperature (dof 3N-3), potential energy per atom,
// pressure, total energy per atom (extension; the reference prints none)
void print_thermo(int step, const double* t, bool half_nb, double volume) {
    const int n = md_get_number_of_particles();
    const double w = half_nb ? 1.0 : 0.5;
    const double epot = t[0] * w, vir = t[1] * w;
    const double dof = 3.0 * n - 3.0;
    const double temp = t[2] / dof;
    const double press = (temp * dof + vir) / (3.0 * volume);
    std::printf("thermo %d %.9e %.9e %.9e %.9e\n", step, temp, epot / n, press, (0.5 * t[2] + epot) / n);
    std::fflush(stdout);
}

// Thermo lines without stalling the timestep loop: a line's sums are requested when its step
// is enqueued (a copy into page-locked memory behind that step's work) and printed one thermo
// interval later, when the copy has long landed; the last line is printed after the loop.
struct ThermoLines {
    bool half_nb = false;
    double volume = 1.0;
    int pending_step = -1, pending_ticket = -1;
    void request(int step) {
        const int ticket = drv::thermo_request();
        flush();
        pending_step = step;
        pending_ticket = ticket;
    }
    void flush() {
        if (pending_step < 0) return;
        double t[3];
        drv::thermo_fetch(pending_ticket, t);
        print_thermo(pending_step, t, half_nb, volume);
        pending_step = -1;
    }
};

}  // namespace

int main(int argc, char** argv) {
#if defined(__x86_64__) || defined(__amd64__)
    // the reference flushes denormals to zero on the host (main.cpp:300-303)
    _mm_setcsr(_mm_getcsr() | (_MM_FLUSH_ZERO_ON | _MM_DENORMALS_ZERO_ON));
#endif
    std::string benchmark = "default", force_field = "lj", algorithm, vtk_dir;
    int gridsize[3] = {32, 32, 32};
    int steps = 100, runs = 1, nthreads = 1, reneigh_every = 20, rebalance_every = 100;
    double dt = 0.005, cutoff = 2.5, verlet = 0.3, epsilon = 1.0, sigma = 1.0, potmin = 1.6796, init_temp = 1.44;
    double damping_n = 0.0, damping_t = 0.0, stiffness = 0.0, friction = 0.0;
    bool half_nb = false, prebalance = false, perf = false;
    std::string precision = "fp64", ghost = "reference", dem_model = "reference", half_mode = "reference";
    double dem_radius = -1.0;
    int thermo_every = 0;

    enum {
        O_RENEIGH = 256, O_REBALANCE, O_DT, O_TEMP, O_CUTOFF, O_VERLET, O_EPS, O_SIGMA, O_DN, O_DT_, O_K, O_MU,
        O_POTMIN, O_HALF, O_PREBAL, O_PREC, O_GHOST, O_DEMMODEL, O_DEMR, O_THERMO, O_PERF, O_HALFMODE
    };
    static option opts[] = {{"force_field", required_argument, nullptr, 'f'},
                            {"benchmark", required_argument, nullptr, 'b'},
                            {"nx", required_argument, nullptr, 'x'},
                            {"ny", required_argument, nullptr, 'y'},
                            {"nz", required_argument, nullptr, 'z'},
                            {"timesteps", required_argument, nullptr, 's'},
                            {"runs", required_argument, nullptr, 'r'},
                            {"threads", required_argument, nullptr, 't'},
                            {"algorithm", required_argument, nullptr, 'a'},
                            {"vtk", required_argument, nullptr, 'v'},
                            {"help", no_argument, nullptr, 'h'},
                            {"reneigh", required_argument, nullptr, O_RENEIGH},
                            {"rebalance", required_argument, nullptr, O_REBALANCE},
                            {"dt", required_argument, nullptr, O_DT},
                            {"temp", required_argument, nullptr, O_TEMP},
                            {"cutoff", required_argument, nullptr, O_CUTOFF},
                            {"verlet", required_argument, nullptr, O_VERLET},
                            {"epsilon", required_argument, nullptr, O_EPS},
                            {"sigma", required_argument, nullptr, O_SIGMA},
                            {"damping_n", required_argument, nullptr, O_DN},
                            {"damping_t", required_argument, nullptr, O_DT_},
                            {"stiffness", required_argument, nullptr, O_K},
                            {"friction", required_argument, nullptr, O_MU},
                            {"potmin", required_argument, nullptr, O_POTMIN},
                            {"half_nb", no_argument, nullptr, O_HALF},
                            {"prebalance", no_argument, nullptr, O_PREBAL},
                            {"precision", required_argument, nullptr, O_PREC},
                            {"ghost", required_argument, nullptr, O_GHOST},
                            {"dem_model", required_argument, nullptr, O_DEMMODEL},
                            {"dem_radius", required_argument, nullptr, O_DEMR},
                            {"thermo", required_argument, nullptr, O_THERMO},
                            {"perf", no_argument, nullptr, O_PERF},
                            {"half_mode", required_argument, nullptr, O_HALFMODE},
                            {nullptr, 0, nullptr, 0}};
    int opt;
    while ((opt = getopt_long(argc, argv, "f:b:x:y:z:s:r:t:a:v:h", opts, nullptr)) != -1) {
        switch (opt) {
            case 'f': force_field = optarg; break;
            case 'b': benchmark = optarg; break;
            case 'x': gridsize[0] = std::atoi(optarg); break;
            case 'y': gridsize[1] = std::atoi(optarg); break;
            case 'z': gridsize[2] = std::atoi(optarg); break;
            case 's': steps = std::atoi(optarg); break;
            case 'r': runs = std::atoi(optarg); break;
            case 't': nthreads = std::atoi(optarg); break;
            case 'a': algorithm = optarg; break;
            case 'v': vtk_dir = optarg; break;
            case O_RENEIGH: reneigh_every = std::atoi(optarg); break;
            case O_REBALANCE: rebalance_every = std::atoi(optarg); break;
            case O_DT: dt = std::atof(optarg); break;
            case O_TEMP: init_temp = std::atof(optarg); break;
            case O_CUTOFF: cutoff = std::atof(optarg); break;
            case O_VERLET: verlet = std::atof(optarg); break;
            case O_EPS: epsilon = std::atof(optarg); break;
            case O_SIGMA: sigma = std::atof(optarg); break;
            case O_DN: damping_n = std::atof(optarg); break;
            case O_DT_: damping_t = std::atof(optarg); break;
            case O_K: stiffness = std::atof(optarg); break;
            case O_MU: friction = std::atof(optarg); break;
            case O_POTMIN: potmin = std::atof(optarg); break;
            case O_HALF: half_nb = true; break;
            case O_PREBAL: prebalance = true; break;
            case O_PREC: precision = optarg; break;
            case O_GHOST: ghost = optarg; break;
            case O_DEMMODEL: dem_model = optarg; break;
            case O_DEMR: dem_radius = std::atof(optarg); break;
            case O_THERMO: thermo_every = std::atoi(optarg); break;
            case O_PERF: perf = true; break;
            case O_HALFMODE: half_mode = optarg; break;
            default: usage(argv[0]); return EXIT_FAILURE;
        }
    }
    if (reneigh_every <= 0 || rebalance_every % reneigh_every != 0) {
        std::cerr << "Error: rebalancing timesteps must be multiple of reneighboring timesteps!" << std::endl;
        return EXIT_FAILURE;
    }
    int bench = -1;
    if (benchmark == "default") bench = tmd::BENCH_DEFAULT;
    else if (benchmark == "half") bench = tmd::BENCH_HALF;
    else if (benchmark == "granular_gas") bench = tmd::BENCH_GRANULAR_GAS;
    else if (benchmark == "body_collision") bench = tmd::BENCH_BODY_COLLISION;
    else if (benchmark == "granular_gas_fcc") bench = tmd::BENCH_GRANULAR_GAS_FCC;
    if (bench < 0) {
        std::cerr << "Invalid benchmark specified: \"" << benchmark << "\"" << std::endl;
        std::cerr << "Available options are default, half, body_collision, granular_gas and granular_gas_fcc"
                  << std::endl;
        return EXIT_FAILURE;
    }
    const bool dem = force_field == "dem";
    if (!dem && force_field != "lj") {
        std::cerr << "Invalid force field specified: \"" << force_field << "\"" << std::endl;
        return EXIT_FAILURE;
    }

    double world[6], rank[6], aabb1[6], aabb2[6];
    tmd::world_box(bench, gridsize, potmin, world, aabb1, aabb2);
    md_mpi_initialize();
    md_get_node_bounding_box(world, &rank);
    const double volume = (world[1] - world[0]) * (world[3] - world[2]) * (world[5] - world[4]);

    drv::enable_phase_timing();  // the time report's buckets come from the GPU timeline
    drv::set_precision(precision == "mixed" ? 1 : 0);
    drv::set_ghost_mode(ghost == "exact" ? 1 : 0);
    drv::set_half_mode(half_mode == "ghost" ? 1 : 0);
    drv::set_dem_model(dem_model == "fixed" ? 1 : 0, dem_radius > 0 ? dem_radius : 0.5 * cutoff);
    drv::set_threads(nthreads);
    drv::set_thermo(thermo_every > 0 ? 1 : 0);

    if (md_get_world_rank() == 0) {  // main.cpp:620-651
        std::cout << "Simulation settings:" << std::endl;
        std::cout << "- Force field: " << force_field << std::endl;
        if (dem) {
            std::cout << "- Normal damping: " << damping_n << std::endl;
            std::cout << "- Tangential damping: " << damping_t << std::endl;
            std::cout << "- Stiffness: " << stiffness << std::endl;
            std::cout << "- Friction: " << friction << std::endl;
        } else {
            std::cout << "- Epsilon: " << epsilon << std::endl;
            std::cout << "- Sigma: " << sigma << std::endl;
        }
        std::cout << "- Benchmark: " << benchmark << std::endl;
        std::cout << "- Unit cells (x, y, z): " << gridsize[0] << ", " << gridsize[1] << ", " << gridsize[2]
                  << std::endl;
        std::cout << "- Number of timesteps: " << steps << std::endl;
        std::cout << "- Number of runs: " << runs << std::endl;
        std::cout << "- Number of threads: " << nthreads << std::endl;
        std::cout << "- Reneighboring timesteps: " << reneigh_every << std::endl;
        std::cout << "- Rebalancing timesteps: " << rebalance_every << std::endl;
        std::cout << "- Timestep size: " << dt << std::endl;
        std::cout << "- Initial temperature: " << init_temp << std::endl;
        std::cout << "- Cutoff radius: " << cutoff << std::endl;
        std::cout << "- Verlet buffer: " << verlet << std::endl;
        std::cout << "- Potential minimum: " << potmin << std::endl;
        std::cout << "- Half neighbor lists: " << (half_nb ? "yes" : "no") << std::endl;
        std::cout << "- Walberla domain partitioning: no" << std::endl;
        std::cout << "- Prebalance: " << (prebalance ? "yes" : "no") << std::endl;
        std::cout << "- Dynamic load balancing algorithm: none" << std::endl;
        std::cout << "- VTK output directory: " << (vtk_dir.empty() ? "none" : vtk_dir) << std::endl;
        std::cout << "- Backend: " << drv::backend() << std::endl;
        std::cout << "- Precision: " << precision << std::endl;
        std::cout << "- Ghost refresh: " << ghost << std::endl << std::endl;
    }
    const bool vtk = !vtk_dir.empty();
    if (vtk && md_get_world_size() > 1) vtk_dir += std::to_string(md_get_world_rank());  // main.cpp:654-659
    if (vtk) vtk_dir += "/";

    PhaseClock timer((size_t)runs);
    std::vector<std::vector<double>> gpu_ms((size_t)runs, std::vector<double>(6, 0.0));
    double wall_ms_total = 0.0;
    long long atoms_total = 0;

    for (int run = 0; run < runs; ++run) {
        tmd::Particles parts;
        const double cell = cutoff + verlet;
        if (tmd::generate(bench, world, rank, aabb1, aabb2, potmin, parts) < 0) return EXIT_FAILURE;
        int n = md_initialize_grid(parts.mass.data(), parts.pos.data(), parts.vel.data(), (int)parts.mass.size(),
                                   world, rank, cell, 60, 100);
        if (n < 0) {
            std::cerr << "md_initialize_grid failed" << std::endl;
            return EXIT_FAILURE;
        }
        if (bench == tmd::BENCH_DEFAULT || bench == tmd::BENCH_HALF) md_create_velocity(init_temp);
        md_copy_data_to_accelerator();
        md_exchange_particles();
        md_borders();
        md_distribute_particles();
        md_assemble_neighborlists(half_nb, cell);
        auto force = [&]() {
            if (dem) md_compute_dem(half_nb, cutoff, damping_n, damping_t, stiffness, friction);
            else md_compute_lennard_jones(half_nb, cutoff, epsilon, sigma);
        };
        force();
        ThermoLines thermo;
        thermo.half_nb = half_nb;
        thermo.volume = volume;
        if (thermo_every > 0) {
            md_final_integration(0.0);  // a zero kick: drains the force and reduces v.v
            thermo.request(0);
        }
        if (vtk && run == 0) {
            md_copy_data_from_accelerator();
            vtk_dump(vtk_dir, 0);
        }
        md_barrier();
        double g0[6] = {0}, g1[6] = {0};
        drv::phase_times(g0);
        auto w0 = Clock::now();
        timer.start();
        for (int j = 0; j < steps; ++j) {
            md_initial_integration(dt);
            timer.accum(T_FORCE);
            if ((j + 1) % reneigh_every == 0) {
                md_exchange_particles();
                timer.accum(T_COMM);
                md_enforce_pbc();
                timer.accum(T_OTHER);
                md_borders();
                timer.accum(T_COMM);
                md_distribute_particles();
                timer.accum(T_OTHER);
                md_assemble_neighborlists(half_nb, cell);
                timer.accum(T_NEIGH);
            } else {
                md_synchronize_ghost_layer();
                timer.accum(T_COMM);
            }
            force();
            md_final_integration(dt);
            timer.accum(T_FORCE);
            if (thermo_every > 0 && ((j + 1) % thermo_every == 0 || j + 1 == steps)) thermo.request(j + 1);
            if (vtk && run == 0) {
                md_copy_data_from_accelerator();
                vtk_dump(vtk_dir, j + 1);
                timer.accum(T_OTHER);
            }
        }
        md_barrier();
        thermo.flush();
        timer.accum(T_OTHER);
        auto w1 = Clock::now();
        timer.finish();
        if (drv::phase_times(g1))
            for (int q = 0; q < 6; ++q) gpu_ms[run][q] = g1[q] - g0[q];
        wall_ms_total += std::chrono::duration<double, std::milli>(w1 - w0).count();
        atoms_total += (long long)n * steps;
        md_enforce_pbc();
        md_copy_data_from_accelerator();
        md_report_iterations();
        md_report_particles();
        md_deallocate_grid();
    }

    if (drv::kGpu) {  // phase times from the GPU timeline of the library stream
        double avg[6] = {0};
        for (auto& r : gpu_ms)
            for (int q = 0; q < 6; ++q) avg[q] += r[q] / runs;
        md_report_time(avg[0], avg[1], avg[2], avg[3], avg[4], avg[5]);
    } else {
        md_report_time(timer.avg_total(), timer.avg(T_FORCE), timer.avg(T_NEIGH), timer.avg(T_COMM),
                       timer.avg(T_BALANCE), timer.avg(T_OTHER));
    }
    if (perf) {
        double rate = wall_ms_total > 0 ? atoms_total / (wall_ms_total * 1e-3) : 0.0;
        std::printf("Performance: %.6e atom-steps/s (wall clock of the timestep loops)\n", rate);
    }
    md_mpi_finalize();
    return drv::failed() ? EXIT_FAILURE : EXIT_SUCCESS;
}
