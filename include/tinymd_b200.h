/*
 * tinymd_b200.h -- C ABI of the B200-native tinyMD short-range MD timestep.
 *
 * Drop-in replacement for the extern "C" interface tinyMD's host driver binds
 * (anydsl_includes.h:4-49, implemented in core/runtime.impala and
 * comm/lb.impala).  Every md_* entry point keeps the reference's name,
 * argument order and meaning; each comment names the reference line it
 * replaces.  One library instance owns one global grid (as
 * core/runtime.impala:1-2 does) on the current CUDA device.
 *
 * Execution model: calls enqueue CUDA work on one library-owned stream and
 * return.  Adjacent calls of one timestep are fused (md_initial_integration
 * followed by md_synchronize_ghost_layer becomes one kernel; the LJ force
 * followed by md_final_integration becomes one kernel).  Every call whose
 * result the host can observe (md_write_*, md_report_*, md_get_*,
 * md_copy_data_from_accelerator) first drains that pending work, so the
 * observable behaviour is the reference's synchronous one.
 *
 * Errors: the reference has none (capacities grow silently).  Here the void
 * entry points keep their signatures; failures are latched and readable with
 * md_last_error() / md_last_error_string().  Neighbour-list and ghost storage
 * grow on overflow and the step is redone, as the reference does.
 *
 * Everything below the "extensions" line is new API without a reference
 * counterpart: precision / ghost / DEM model selection, thermo reductions,
 * GPU phase timing and kernel profiling, parity introspection, benchmark
 * setups, and the differentiable (adjoint) form.
 */
#ifndef TINYMD_B200_H
#define TINYMD_B200_H

#ifdef __cplusplus
#include <cstdint>
extern "C" {
#else
#include <stdbool.h>
#include <stdint.h>
#endif

/* anydsl_includes.h:5-9 */
struct Vector3D {
    double x;
    double y;
    double z;
};
#ifndef __cplusplus
typedef struct Vector3D Vector3D;
#endif

/* ---- reference interface (anydsl_includes.h:10-48) ------------------------ */

/* anydsl_includes.h:10, core/runtime.impala:7-37.  Copies n particles (AoS
 * host arrays) into the library, builds the grid over rank_aabb extended by
 * one cell_spacing, returns the number of local particles. */
int md_initialize_grid(double const *masses, struct Vector3D const *positions, struct Vector3D const *velocities,
                       int nparticles, double const *world_aabb, double const *rank_aabb, double cell_spacing,
                       int cell_capacity, int neighborlist_capacity);
/* anydsl_includes.h:11, core/runtime.impala:39-50 (load balancing only: latches MD_ERR_UNSUPPORTED) */
void md_rescale_grid(double const *aabb);
/* anydsl_includes.h:12, core/grid.impala:369-374 (device -> host mirror) */
void md_copy_data_from_accelerator(void);
/* anydsl_includes.h:13, core/grid.impala:360-367 (host mirror -> device) */
void md_copy_data_to_accelerator(void);
/* anydsl_includes.h:14, core/compute.impala:97-106: v += dt/2 f; x += dt v */
void md_initial_integration(double dt);
/* anydsl_includes.h:15, core/compute.impala:108-116: v += dt/2 f */
void md_final_integration(double dt);
/* anydsl_includes.h:16, core/compute.impala:118-122 (single periodic wrap of locals) */
void md_enforce_pbc(void);
/* anydsl_includes.h:17, core/grid.impala:483-499: copies the host mirror of the
 * locals, in input order; returns the number of locals. */
int md_write_grid_data_to_arrays(double *masses, struct Vector3D *positions, struct Vector3D *velocities,
                                 struct Vector3D *forces);
/* anydsl_includes.h:18, core/grid.impala:501-518: ghosts in the reference's
 * ghost order; returns the number of LOCALS, as the reference does. */
int md_write_grid_ghost_data_to_arrays(double *masses, struct Vector3D *positions, struct Vector3D *velocities,
                                       struct Vector3D *forces);
/* anydsl_includes.h:19, core/grid.impala:520-546: the 8 grid box corners */
int md_write_grid_aabb_data_to_arrays(double *masses, struct Vector3D *positions, struct Vector3D *velocities,
                                      struct Vector3D *forces);
/* anydsl_includes.h:20, core/grid.impala:323-358: bins locals and ghosts into
 * cells (a counting sort that also reorders the device arrays by cell). */
void md_distribute_particles(void);
/* anydsl_includes.h:21, core/neighborlist.impala:18-78.  Returns before the build's status (list
 * overflow, locals outside the grid) is read: the next force starts on the new lists and the status
 * is read while it runs, the build and force redone on an overflow; a warning of the build is
 * latched by then, or by the next call that reads state or the error code. */
void md_assemble_neighborlists(bool half_neighborlist, double cutoff_distance);
/* anydsl_includes.h:22, core/runtime.impala:97-102 */
void md_deallocate_grid(void);
/* anydsl_includes.h:23-24, core/runtime.impala:146-156 */
void md_print_grid(void);
void md_print_ghost(void);
/* anydsl_includes.h:25, core/runtime.impala:158-186 (host mirror, before upload) */
void md_create_velocity(double temperature);
/* anydsl_includes.h:26, core/runtime.impala:188-201 */
void md_compute_lennard_jones(bool half_neighborlist, double cutoff_distance, double epsilon, double sigma);
/* anydsl_includes.h:27, core/runtime.impala:203-247 */
void md_compute_dem(bool half_neighborlist, double cutoff_distance, double damping_n, double damping_t,
                    double stiffness, double friction);
/* anydsl_includes.h:28-29, core/runtime.impala:250-251.  Several processes (one per GPU) form
 * one run when the environment names the world size and this process's rank
 * (TINYMD_WORLD_SIZE / TINYMD_RANK, else WORLD_SIZE / RANK as torchrun sets them, else
 * OMPI_COMM_WORLD_SIZE / OMPI_COMM_WORLD_RANK, else PMI_SIZE / PMI_RANK): md_mpi_initialize
 * connects them over TCP (rank 0 listens on TINYMD_ADDR or MASTER_ADDR, default 127.0.0.1,
 * port TINYMD_PORT, else MASTER_PORT + 17, else 29417), selects this rank's GPU
 * (TINYMD_DEVICE, else the launcher's local rank) and picks the transport of the halo data:
 * NCCL when every rank has its own GPU, else page-locked host buffers over the TCP mesh
 * (TINYMD_COMM=auto|socket|nccl).  Without those variables the run has one rank.
 * md_mpi_finalize releases the grid and the connections.  Several ranks run full neighbour
 * lists and exact ghosts; md_report_* print sums (times: maxima) over the ranks on rank 0. */
void md_mpi_initialize(void);
void md_mpi_finalize(void);
/* anydsl_includes.h:30, comm/comm.impala:334-388 */
void md_synchronize_ghost_layer(void);
/* anydsl_includes.h:31, comm/comm.impala:528-642 */
void md_borders(void);
/* anydsl_includes.h:32, comm/comm.impala:392-525 (one rank: nothing leaves; several: locals
 * beyond the rank box move to the rank that owns their new place) */
void md_exchange_particles(void);
/* anydsl_includes.h:33-35, core/runtime.impala:258-264 (MPI buffers: stubs) */
double md_get_send_buffer_value(int index);
void md_set_recv_buffer_value(int index, double value);
void md_resize_recv_buffer_capacity(int capacity);
/* anydsl_includes.h:36-37, core/runtime.impala:266-279 (load balancing: latch MD_ERR_UNSUPPORTED) */
int md_serialize_particles(double const *aabb);
void md_deserialize_particles(int nparticles);
/* anydsl_includes.h:38-39, core/runtime.impala:253-255 */
int md_get_world_size(void);
int md_get_world_rank(void);
/* anydsl_includes.h:40-41, core/runtime.impala:256-257 */
int md_get_number_of_particles(void);
int md_get_number_of_ghost_particles(void);
/* anydsl_includes.h:42, core/runtime.impala:52-70, comm/comm.impala:221-299 (the rank layout
 * that minimises the ranks' surface, a periodic row-major cart; one rank: the world box) */
void md_get_node_bounding_box(double const *world_aabb, double (*rank_aabb)[6]);
/* anydsl_includes.h:43-44, core/runtime.impala:72-95, comm/lb.impala:52-86 (load balancing: stubs) */
void md_compute_boundary_weights(double xmin, double xmax, double ymin, double ymax, double zmin, double zmax,
                                 unsigned long int *computational_weight, unsigned long int *communication_weight);
void md_update_neighborhood(int nranks, int total_aabbs, int const *ranks, int const *naabbs, double const *aabbs);
/* anydsl_includes.h:45-47, core/runtime.impala:280-337 (same output lines) */
void md_report_iterations(void);
void md_report_particles(void);
void md_report_time(double total, double force, double neigh, double comm, double balance, double other);
/* anydsl_includes.h:48, core/runtime.impala:253 */
void md_barrier(void);

/* ---- extensions (no reference counterpart) -------------------------------- */

enum md_error {
    MD_OK = 0,
    MD_ERR_CUDA = 1,          /* a CUDA call failed (message in md_last_error_string) */
    MD_ERR_STATE = 2,         /* call out of order (e.g. before md_initialize_grid) */
    MD_ERR_ARGUMENT = 3,      /* invalid argument */
    MD_ERR_UNSUPPORTED = 4,   /* multi-process / load-balancing entry point */
    MD_ERR_OUT_OF_GRID = 5,   /* locals outside the cell grid at binning (warning; they get no neighbours) */
    MD_ERR_NO_DEVICE = 6,     /* no CUDA device */
    MD_ERR_COMM = 7           /* the ranks could not connect, or an exchange between them failed */
};
int md_last_error(void);
const char *md_last_error_string(void);
void md_clear_error(void);

/* Precision of the pair forces: 0 = FP64 throughout (default, the drop-in),
 * 1 = mixed (FP64 state, integration, list cutoff and reductions; FP32 pair
 * arithmetic on cell-rebased FP32 positions and FP32 force accumulation). */
void md_set_precision(int mode);
/* Ghost refresh: 0 = reference two-phase update (chained edge/corner ghosts
 * lag by one step per chain link, comm/comm.impala:334-388; default),
 * 1 = exact periodic images (ghost = root local + total shift). */
void md_set_ghost_mode(int exact);
/* Half neighbour lists: 0 = the reference's (core/neighborlist.impala:34 keeps
 * j < i by particle index, which never admits a ghost, so every pair across
 * the periodic boundary is dropped; default), 1 = corrected: local-ghost
 * pairs are kept when the ghost's root local precedes i, and the reaction
 * force goes to that root. */
void md_set_half_mode(int ghost_pairs);
/* DEM contact model: 0 = the reference closure (its contact branch is
 * unreachable, so the force is zero; default), 1 = contact-fixed
 * spring-dashpot with contact radius `radius` (overlap 2R - r > 0). */
void md_set_dem_model(int contact_fixed, double radius);
/* When enabled, LJ force calls also reduce the potential energy and virial,
 * and final integrations reduce the kinetic energy (FP64, deterministic). */
void md_set_thermo(int enable);
/* out[0] = sum of pair energies 4 eps (s12 - s6) over list entries inside the
 * cutoff, out[1] = sum of f(r) r^2 over the same entries, out[2] = number of
 * list entries inside the cutoff, out[3] = sum of v.v of locals after the last
 * final integration.  Full lists count each pair twice.  With several ranks the sums are over
 * all ranks (every rank calls).  Returns 0 on success. */
int md_get_thermo(double *out);
/* The same sums without waiting: md_thermo_request enqueues a copy of them (as of the work
 * issued so far) into page-locked memory and returns a ticket; md_thermo_fetch(ticket, out)
 * waits for that copy alone and fills out[4] as md_get_thermo does.  Up to 8 requests stay
 * fetchable; returns 0, or -1 for an unknown ticket. */
int md_thermo_request(void);
int md_thermo_fetch(int ticket, double *out);
/* Blocks until all enqueued device work is done. */
void md_synchronize(void);
/* Use `stream` (a cudaStream_t) for all library work instead of the stream
 * the library creates; NULL selects the legacy default stream. */
void md_set_stream(void *stream);
/* GPU time per timer bucket since md_initialize_grid, in ms:
 * out = {total, force, neigh, comm, balance, other} (main.cpp:477-484 buckets).
 * Zero unless md_set_phase_timing(1): the phase boundaries are CUDA events on the stream. */
void md_get_phase_times(double *out);
void md_set_phase_timing(int enable); /* default 0 */
/* Kernel profiling with CUDA events on the library stream. */
void md_profile_enable(int enable);
/* Time one launch in `every` of each profiled kernel (default 1); md_profile_get then
 * counts and sums the timed launches only.  Each timed launch adds two events to the stream. */
void md_profile_sample(int every);
int md_profile_count(void);
const char *md_profile_name(int kernel_id);
int md_profile_get(int kernel_id, long long *launches, double *total_ms);
void md_profile_reset(void);
/* Number of kernel launches issued since md_initialize_grid. */
long long md_kernel_launches(void);
/* Device bytes held by the library. */
long long md_device_bytes(void);

/* Runs `steps` timesteps of the md driver loop (main.cpp:715-776) natively:
 * initial integration, ghost refresh -- or, when (step0 + k + 1) is a
 * multiple of reneigh_every, exchange / wrap / borders / binning / lists with
 * `list_cutoff` -- then the force of the last md_compute_* call and the final
 * integration.  When step_ms is not NULL each step is bracketed by CUDA
 * events and its device time stored; when flush_buf is not NULL, flush_bytes
 * of it are overwritten and then read back before each step, outside the
 * timed interval (an L2 flush for benchmarking: the read evicts the written
 * lines, so the step starts with a cold L2 that holds no dirty lines of the
 * flush).  Returns 0 on success. */
int md_run_timesteps(int steps, double dt, int reneigh_every, int step0, double list_cutoff, float *step_ms,
                     void *flush_buf, long long flush_bytes);

/* LJ forces and energy / virial sums over a caller-built full neighbour list,
 * allocating no device memory (no counterpart in the reference).  For callers
 * that cannot call cudaMalloc -- code inside another framework's memory pool,
 * code running while someone else captures a CUDA graph, hosts with a fixed
 * memory budget -- its per-block partial sums live in a fixed device array
 * compiled into the library (128 KiB, held by every GPU that loads the
 * library until exit), so the call only launches two kernels on `stream`.
 * Limit: n_local <= 1,048,576 (larger is rejected with MD_ERR_ARGUMENT).
 * All pointers are device memory: positions [n_all][4] (x, y, z, unused),
 * list_sizes [n_local], lists atom-fastest (entry k of atom i at
 * lists[k*stride + i], a plain index into positions), forces [n_local][4]
 * out, sums [4] out = {sum of 4 eps (s12 - s6), sum of f r^2, pairs inside the
 * cutoff, 0} over the list entries.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and should therefore come
 * before any stream capture; that address is kept for the life of the
 * process, so after a device reset the library must be loaded again.  Calls
 * share the array: calls that overlap on the GPU race.  Returns MD_OK or an
 * md_error code. */
int md_lj_forces_noalloc(const double *positions, int n_local, const int *list_sizes, const int *lists, int stride,
                         int max_neighbors, double cutoff, double epsilon, double sigma, double *forces, double *sums,
                         void *stream);

/* Parity introspection (reference index space: locals 0..N-1 in input order,
 * ghosts N..N+G-1 in the reference's ghost order).  Drain pending work. */
int md_get_neighbor_lists(int *sizes, int *lists, int capacity); /* row-major [N][capacity]; returns max size */
int md_get_ghost_info(int *src, int *pbc, int *root, int *tshift); /* per ghost; returns G */
int md_get_state(double *pos, double *vel, double *force);       /* pos [N+G][3], vel/force [N][3] */
int md_set_positions(double const *pos);                          /* locals [N][3] in input order */
int md_set_velocities(double const *vel);
/* Cell membership counts: out[c] = locals + ghosts in cell c (flattened). */
int md_get_cell_sizes(int *out, int ncells);
int md_get_grid_info(int *out); /* nx ny nz ncells N G nb_capacity nb_stride */

/* Benchmark setups of the md driver (main.cpp:491-521, initialize.h).
 * benchmark: 0 default, 1 half, 2 granular_gas, 3 body_collision,
 * 4 granular_gas_fcc (FCC kept where x/Lx + y/Ly < 1, zero velocities). */
int tmd_setup_world(int benchmark, int const *gridsize, double potmin, double *world, double *aabb1,
                    double *aabb2);
void tmd_setup_rank_box(double const *world, double *rank);
/* Generates into library-owned storage; returns the particle count (or -1). */
int tmd_setup_generate(int benchmark, double const *world, double const *rank, double const *aabb1,
                       double const *aabb2, double potmin);
/* Copies the last generated setup out (arrays of the returned count). */
int tmd_setup_fetch(double *masses, struct Vector3D *positions, struct Vector3D *velocities);
/* md_initialize_grid on the last generated setup. */
int tmd_setup_initialize(double const *world, double const *rank, double cell_spacing, int cell_capacity,
                         int neighborlist_capacity);

/* ---- rank layout and transport (several processes; md_mpi_initialize) ------ */
/* comm/comm.impala:221-257: the rank grid dims[3] for `world` ranks over a box of side
 * lengths len[3].  Returns 0, or -1 for world < 1. */
int tmd_node_config(int world, double const *len, int *dims);
/* The 26 regions around rank `rank` of the periodic row-major cart dims[3] (region
 * t = ez*9 + ey*3 + ex - 1, e per axis 0 inside, 1 above, 2 below): peer[26] their owners,
 * shift[26*3] the world lengths added to a position sent there, *selfmask the regions this
 * rank owns itself.  Returns 0, or -1 for a rank outside the cart. */
int tmd_topology(int rank, int const *dims, int *peer, int *shift, unsigned *selfmask);
/* This rank's halo at the last border pass: out[0] its own periodic ghosts, out[1] images sent
 * per step, out[2] ghosts received per step, out[3] neighbour ranks.  Returns -1 on one rank. */
int tmd_halo_info(int *out);
/* The NCCL binding on this GPU alone: a one-rank communicator sends `bytes` to itself through the
 * calls the halo exchange uses.  0 on a match, -2 when libnccl.so.2 is absent, -1 otherwise. */
int tmd_comm_nccl_selftest(long long bytes);
/* "none" (one rank), "socket" or "nccl": the transport of the halo data. */
const char *tmd_comm_transport(void);
/* Sum of v[n] over the ranks (rank order), on every rank.  Returns 0 or -1. */
int tmd_comm_allreduce_sum(double *v, int n);
/* One host message to rank `to` and one from rank `from` (bytes may be 0).  Returns 0 or -1. */
int tmd_comm_sendrecv(int to, void const *sbuf, long long sbytes, int from, void *rbuf, long long rbytes);

/* ---- differentiable form (adjoint) ---------------------------------------- */
/* Trajectory: VV with LJ over full lists, exact periodic ghosts, neighbour
 * lists rebuilt every `reneigh` steps and frozen inside a segment.  Loss:
 * L = (1/N) sum_i |x_T,i - x_0,i|^2 (unwrapped) + U(x_T)/N.  Checkpoints
 * (positions, velocities, image shifts) are kept per segment on the device. */
int md_adjoint_configure(int steps, int reneigh, double dt, double cutoff, double skin, int precision);
/* Runs the forward trajectory from the current grid state with initial
 * velocities v0 ([N][3], input order) and parameters eps, sigma; returns L. */
int md_adjoint_forward(double const *v0, double epsilon, double sigma, double *loss);
/* Reverse pass: dL/dv0 ([N][3], input order), dL/deps, dL/dsigma. */
int md_adjoint_backward(double *grad_v0, double *grad_eps, double *grad_sigma);
/* Loss energy: 0 = U as the reference defines pair energies (unshifted, hard
 * cutoff: L jumps when a pair crosses the cutoff; default), 1 = U shifted to
 * zero at the cutoff per pair (continuous in the parameters; same forces). */
int md_adjoint_set_loss(int shifted_energy);
/* GPU ms of the last forward and backward passes. */
int md_adjoint_times(double *forward_ms, double *backward_ms);

#ifdef __cplusplus
}
#endif

#endif /* TINYMD_B200_H */
