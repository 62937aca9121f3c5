// md_state.h -- host-side state of the tinyMD B200 library and the launch
// wrappers of its kernels.  One global State instance (the reference keeps
// one global grid too, core/runtime.impala:1-2).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdlib>
#include <new>
#include <string>
#include <utility>
#include <vector>

namespace tmd {

// Page-locked host memory for the host mirror, so host<->device copies go straight
// to and from it.  New elements are left uninitialised (every user overwrites them),
// and a failed page-locked allocation falls back to ordinary memory (the copies
// then stage through the driver); a 64-byte header records which kind a block is.
template <class T>
struct PinnedAlloc {
    using value_type = T;
    PinnedAlloc() = default;
    template <class U>
    PinnedAlloc(const PinnedAlloc<U>&) {}
    T* allocate(size_t n) {
        const size_t bytes = n * sizeof(T) + kHeader;
        void* p = nullptr;
        int kind = 1;
        if (cudaMallocHost(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            p = std::malloc(bytes);
            kind = 2;
            if (!p) throw std::bad_alloc();
        }
        *(int*)p = kind;
        return (T*)((char*)p + kHeader);
    }
    void deallocate(T* q, size_t) {
        void* p = (char*)q - kHeader;
        if (*(int*)p == 2) std::free(p);
        else if (cudaFreeHost(p) != cudaSuccess) cudaGetLastError();  // runtime already unloading: leave it
    }
    template <class U>
    void construct(U* p) noexcept { ::new ((void*)p) U; }
    template <class U, class... A>
    void construct(U* p, A&&... a) { ::new ((void*)p) U(std::forward<A>(a)...); }
    static constexpr size_t kHeader = 64;
};
template <class T, class U>
bool operator==(const PinnedAlloc<T>&, const PinnedAlloc<U>&) { return true; }
template <class T, class U>
bool operator!=(const PinnedAlloc<T>&, const PinnedAlloc<U>&) { return false; }
using HostVec = std::vector<double, PinnedAlloc<double>>;

enum Phase { PH_FORCE = 1, PH_NEIGH = 2, PH_COMM = 3, PH_BALANCE = 4, PH_OTHER = 5, PH_COUNT = 6 };

enum KernelId {
    K_FORCE_LJ = 0,   // LJ forces (any list / precision), possibly fused with the final kick
    K_FORCE_DEM,
    K_INTEGRATE,      // initial integration (+ ghost refresh when fused)
    K_GHOST_SYNC,     // stand-alone ghost refresh
    K_FINAL,          // stand-alone final integration
    K_PBC,
    K_BORDER,         // ghost generation (3 kernels)
    K_BIN,            // counting sort (5 kernels)
    K_NLIST,          // neighbour-list build
    K_SCAN,
    K_REDUCE,
    K_HVP,            // adjoint Hessian-vector product
    K_ADJ_STEP,       // adjoint elementwise updates
    K_MISC,
    K_COUNT
};
const char* kernel_name(int id);

template <class T>
struct DBuf {  // a double-buffered device array
    T* b[2] = {nullptr, nullptr};
};

struct Geometry {
    double world_lo[3], world_hi[3];
    double aabb_lo[3], aabb_hi[3];  // rank box extended by one cell spacing
    double len[3];                  // world lengths (periodic shifts)
    double spacing;
    int nx, ny, nz, ncells;
    // mixed form: dyadic rebasing grid (spacing rb_h > list cutoff)
    double rb_h;
};

// Device-side status words written by kernels and read back with one copy.
struct DevStatus {
    int nghost;         // ghosts produced by the last border pass
    // zeroed together before a binning (one memset): out_local .. img_over2
    int out_local;      // locals outside the cell grid at the last binning
    int out_ghost;      // ghosts outside the cell grid
    int nchain;         // ghosts whose two-phase source is a ghost (last distribution)
    int img_over1;      // locals with more than kImg1 direct images
    int img_over2;      // locals with more than kImg2 images in all
    int max_nb;         // longest neighbour list of the last build (zeroed before each build)
};

// periodic images a local can push (two-phase: its own first-pass images, one per face
// it is near; exact: all its images, up to seven where the box is wider than two
// ghost layers; a local with more leaves the map incomplete and the ghosts to a kernel)
constexpr int kImg1 = 6;
constexpr int kImg2 = 8;
constexpr int kImgW = kImg1 + kImg2;

constexpr int kThermoSlots = 8;  // asynchronous thermo reads in flight at most

// threads per block of the ghost count and emit kernels (and the migration's): the ghost offsets
// are scanned over 26 types x blocks, 13k values at 131k atoms, one look-back scan; 1,024-thread
// blocks kept that scan to 3.3k values for the one-block scan, but the emit runs a single
// half-occupied wave then (rebuild step 195 -> 192-193.5 us with 256)
#ifndef TMD_BORDER_THREADS
#define TMD_BORDER_THREADS 256
#endif
constexpr int kBorderThreads = TMD_BORDER_THREADS;
inline int border_blocks(int N) { return (N + kBorderThreads - 1) / kBorderThreads; }

// Multi-rank runs (comm.h): the images this rank sends into its neighbours' regions and the
// ghosts it receives from them.  Ghost order: the periodic images of this rank's own atoms
// (gself, the border pass's order), then the received ghosts peer by peer (ascending rank),
// each peer's in its send order.
struct Halo {
    bool on = false;          // more than one rank
    int gself = 0;            // ghosts that are images of this rank's own atoms
    int nsend = 0, nrecv = 0; // images sent / ghosts received by the last border pass
    int send_cap = 0;
    int* send_ref = nullptr;  // [send_cap] root reference index of each image sent, by region type
    int* send_type = nullptr; // its region type
    int* pk_ref = nullptr;    // the same in message order (peer by peer): the per-step packing
    int* pk_type = nullptr;
    int* tab = nullptr;       // [kHaloTab] device copy of the per-type offsets (see k_halo.cu)
    int* tab_host = nullptr;  // pinned: offsets read back, then the table to upload
    double* sbuf = nullptr;   // device message buffers
    double* rbuf = nullptr;
    size_t sbuf_cap = 0, rbuf_cap = 0;  // doubles
    HostVec hs, hr;           // page-locked staging when the transport is host sockets
    std::vector<int> send_cnt, recv_cnt;  // per peer rank (Topology::peers), at the last border pass
};
constexpr int kHaloTab = 128;

struct PendingForce {
    bool valid = false;
    bool dem = false;
    bool half = false;
    double rc = 0, eps = 0, sigma = 0;
    double dn = 0, dt_ = 0, k = 0, mu = 0;
};

struct State {
    bool alive = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool stream_set = false;   // a caller chose the stream (md_set_stream), NULL included
    Geometry geo{};

    // sizes
    int N = 0, G = 0;
    int capA = 0;       // slots for locals + ghosts
    int nb_cap = 0;     // neighbour-list capacity per atom (rows)
    int nb_stride = 0;  // column stride of the atom-fastest list
    int nblk_border = 0;
    int lists_valid = 0;
    bool lists_half = false;

    // modes
    int precision = 0;   // 0 FP64, 1 mixed
    int ghost_exact = 0;
    int half_ghost = 0;  // half lists keep local-ghost pairs (ordered by root) -- corrected half mode
    int dem_fixed = 0;
    double dem_radius = 1.0;
    int thermo = 0;

    // device arrays (slots: locals 0..N-1 sorted by cell, ghosts N..N+G-1)
    DBuf<double4> pos;   int pc = 0;   // positions
    DBuf<double4> vel;   int vc = 0;   // velocities
    DBuf<double4> frc;   DBuf<double> mass;  DBuf<int> ref;  DBuf<int> img;  int ac = 0;
    float4* frc32 = nullptr;   // mixed-form forces
    DBuf<float4> pos32;        // mixed-form rebased positions, double-buffered with pos (index pc)
    int* rbk = nullptr;        // packed rebasing cell of each slot
    int* slot_of_ref = nullptr;
    int* rref = nullptr;       // per slot: reference index of the root local (= ref for locals)
    int* gsrc = nullptr;       // ghost: source slot (reference two-phase refresh)
    int* groot = nullptr;      // ghost: root local slot
    int* gcode = nullptr;      // ghost: shifts (see md_common.cuh)
    // cells: starts of locals per cell [ncells+2] followed by ghosts per cell [ncells+2]
    int* cnt = nullptr;        // counts, same layout
    int* cstart = nullptr;     // exclusive scan of cnt (ghost starts include the N offset)
    int* bin_cell = nullptr;   // per slot: cell of the slot (or ncells when outside)
    int* bin_rank = nullptr;   // per slot: arrival rank within its cell
    int* tmp_key = nullptr;    // per sorted position: reference index
    int* tmp_src = nullptr;    // per sorted position: old slot
    int* slot_cell = nullptr;  // per (sorted) slot: its cell, ncells when outside the grid
    // ghost images by local (k_ghost_links at every distribution): the force kernel that does
    // the next initial integration writes them, so no separate ghost refresh is needed
    char* slab = nullptr;      // the one allocation the per-slot arrays are carved from (grow_atoms)
    double* dl_buf = nullptr;  // host-mirror transfers (mass, pos, vel, frc by reference): 10 doubles per slot
    int* img_cnt = nullptr;    // [2][capA]: direct two-phase images of a local, all its images
    int* img_slot = nullptr;   // [kImgW][capA]: their slots by plane (kImg1 two-phase planes, then
                               // kImg2 exact ones), -1 after a local's last image
    int* chain = nullptr;      // [capA]: ghost indices whose two-phase source is a ghost
    int nchain = 0;            // their number (status readback of the list build)
    int img_ok = 0;            // bit gm - 1: the map of ghost mode gm (1, 2) is complete
    int ghosts_pushed = 0;     // ghost mode whose images the last fused kernel wrote (0: none)
    // border pass
    unsigned* bmask = nullptr;   // per local (reference order): 26-bit ghost-type mask
    int* bcount = nullptr;       // [26][nblk] counts, scanned in place
    int* bsrc_ref = nullptr;     // per ghost (reference order): source reference index
    int* broot_ref = nullptr;    // per ghost: root local reference index
    int* bcode = nullptr;        // per ghost: shift code (reference order)
    // neighbour lists
    // list layout: quads of four consecutive entries of one atom, atom-fastest (nl_index);
    // nb_cap is a multiple of four
    int* nbn = nullptr;
    uint32_t* nbl = nullptr;
    double lists_cutoff = 0.0;
    // A list build's status (overflow, locals outside the grid, two-phase chain, image maps)
    // comes back while the next force kernel already runs: resolve_lists reads it.
    bool status_pending = false;
    bool status_half = false;  // the pending build's list mode (a redo after a capacity growth)
    cudaEvent_t ev_status = nullptr;
    // scan scratch, reductions, status
    int* scan_part = nullptr;  int scan_part_cap = 0;
    double* red_part = nullptr; int red_part_cap = 0;
    double* thermo_dev = nullptr;   // [8]
    DevStatus* status_dev = nullptr;
    DevStatus* status_host = nullptr;  // pinned
    cudaEvent_t ev_counted = nullptr;  // the ghost count's readback (run_borders)
    cudaEvent_t ev_scanned = nullptr;  // the ghost offsets scanned (the readback waits on it)
    cudaStream_t copy_stream = nullptr;  // the ghost count's readback, beside the emit kernel
    int scan_attr_device = -1;         // device whose k_scan_single shared-memory attribute is set
    unsigned long long* lb_tiles = nullptr;  // look-back scan: one word per tile (k_neigh.cu)
    int lb_tile_cap = 0;
    unsigned lb_epoch = 0;             // look-back scan launches so far (tags the tile words)
    double* thermo_host = nullptr;     // pinned [kThermoSlots][4]: asynchronous thermo reads
    cudaEvent_t thermo_ev[8] = {};     // one per slot: its copy has landed
    long long thermo_slot_ticket[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
    long long thermo_tickets = 0;      // tickets issued by md_thermo_request

    // host mirror in reference order (core/grid.impala ArrayData host buffers)
    // md_copy_data_from_accelerator gathers the device state into dl_buf and leaves the copy
    // to the host pending: bit 0 the locals, bit 1 the ghosts of that snapshot (mirror_n locals,
    // mirror_na slots).  Readers copy what they need; anything that would overwrite dl_buf
    // first completes the mirror (materialize_mirror).
    int mirror_pending = 0;
    int mirror_n = 0, mirror_na = 0;
    bool mirror_frc_zero = false;  // the mirror's forces are all zero (not yet written)
    bool x0_in_pos = false;        // h_x0 is still h_pos (the positions md_initialize_grid got)
    HostVec h_mass;                 // [N+G]
    HostVec h_pos, h_vel, h_frc;    // [(N+G)*3]
    HostVec h_x0;                   // initial positions (adjoint), once the mirror's are overwritten

    PendingForce pend_force;
    PendingForce force_cfg;   // parameters of the last md_compute_* call
    bool pend_init = false;
    double pend_dt = 0.0;
    // a full-list LJ force whose final integration was requested: launched when the next
    // call is known, fused with the next step's initial integration when that is the call
    bool pend_final = false;
    double pend_final_dt = 0.0;
    // the final kick of a half-list or DEM force, held back to join the next initial integration
    bool pend_kick = false;
    double pend_kick_dt = 0.0;
    PendingForce final_cfg;
    // locals were integrated by that fused kernel; ghosts still to be refreshed or carried
    bool pend_ghost = false;
    // md_enforce_pbc held back: md_borders does the wrap in its first kernel, any other call
    // launches it alone
    bool pend_pbc = false;
    // the cell counters and binning status were zeroed by the last border pass (cleared by
    // the binning that uses them)
    bool bin_zeroed = false;
    bool build_zeroed = false;  // likewise the list-build status, by the binning's reorder kernel
    bool pend_links = false;    // ghost links of the last binning not yet launched (see flush_links)

    Halo halo;  // multi-rank only

    // reported iteration counters (core/runtime.impala:3-5)
    long long force_iters = 0, rsq_iters = 0, integration_iters = 0;
    int last_force_half = 0;
    double last_rc = 0, last_eps = 0, last_sigma = 0;

    // bookkeeping
    long long launches = 0;
    long long dev_bytes = 0;
    int last_error = 0;
    std::string last_error_msg;
};

extern State g_state;

// ---- error helpers ---------------------------------------------------------
void set_error(int code, const std::string& msg);
bool cuda_ok(cudaError_t e, const char* what);
#define TMD_CUDA(call) ::tmd::cuda_ok((call), #call)
void launched(int kernel_id);  // counts a launch, checks the launch error

// ---- timing ------------------------------------------------------------------
void phase_mark(int phase);
void phase_times(double* out6);
void phase_reset();
void prof_begin(int kernel_id);
void prof_end(int kernel_id);
void prof_reset();

// ---- kernels (launch wrappers, all on g_state.stream) ---------------------
struct KLaunch;  // fwd
void run_enforce_pbc(State& s);
void flush_links(State& s);                      // the deferred ghost links of a binning, if pending
void run_borders(State& s, bool wrap = false);   // ghost generation, reference order (wrap: the periodic wrap first)
void run_distribute(State& s);                    // binning + reorder
// defer: the status readback is left in flight (resolve_lists completes it)
int run_build_lists(State& s, bool half, double cutoff, bool defer = false);  // returns 0 or error
// completes a deferred list build: 0 when the lists stand, 1 when they were rebuilt (a force
// kernel launched on them speculatively returned without writing), -1 on an error
int resolve_lists(State& s);
void run_force_lj(State& s, const PendingForce& p, bool fuse_final, double dt);
void run_force_dem(State& s, const PendingForce& p);
// kick_dt >= 0: the previous step's final kick of kick_dt is applied first (held back by
// md_final_integration for forces whose kernel cannot take it)
void run_integrate(State& s, double dt, bool fuse_ghosts, double kick_dt = -1.0);
void run_ghost_sync(State& s);
void run_final(State& s, double dt);
void run_refresh_pos32(State& s);
// completes the pending host-mirror copies of the last md_copy_data_from_accelerator (parts:
// bit 0 locals, bit 1 ghosts)
void materialize_mirror(State& s, int parts = 3);
void release_adjoint();  // frees the differentiable form's device buffers (adjoint.cu)
// list pairs inside the cutoff rc (FP64), the reference's rsq_iters of a force call on the
// current lists and positions
long long count_pairs_inside(State& s, double rc);
// the LJ force (full list) with the final kick of dt_final and the next step's initial
// integration of dt_init fused into its epilogue (plain-list kernels); writes the locals of
// the other position buffer, which becomes current (ghosts: run_ghost_refresh)
void run_force_lj_init(State& s, const PendingForce& p, double dt_final, double dt_init);
bool force_init_fusable(const State& s, const PendingForce& p);
// ghosts of the current buffer from their sources after run_force_lj_init: gm 0 carries
// them over, 1 is the reference two-phase refresh, 2 exact images
void run_ghost_refresh(State& s, int gm);
void run_reduce_thermo(State& s, int nblocks, int nq);
// multi-rank (k_halo.cu): atoms that left the rank box go to their new owners (the caller
// flushed pending work); the remote part of a border pass (after its emit); the ghosts
// received from other ranks refreshed from the current positions of their roots
bool run_migrate(State& s);
bool halo_plan_borders(State& s, const int* boff, int nblk);
bool halo_finish_borders(State& s);
bool run_halo_sync(State& s);
void halo_free(State& s);
// the per-local arrays sized by the local count (border masks and counts, list stride) hold n
bool ensure_locals(State& s, int n);
// sums the [q][nblocks] per-block partials of quantities q0..q1-1 into thermo_dev[q]
void run_reduce_partials(State& s, int nblocks, int q0, int q1);
void exclusive_scan(State& s, const int* in, int* out, int n);
void ensure_scan_scratch(State& s, int n);
void ensure_red_scratch(State& s, int n);

// device memory helpers
void dev_alloc(void** p, size_t bytes);
void dev_free(void** p);
template <class T>
inline void dalloc(T** p, size_t n) { dev_alloc(reinterpret_cast<void**>(p), n * sizeof(T)); }
template <class T>
inline void dfree(T** p) { dev_free(reinterpret_cast<void**>(p)); }

}  // namespace tmd
