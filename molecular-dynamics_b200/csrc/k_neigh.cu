// k_neigh.cu -- reneighbour kernels of the tinyMD B200 timestep:
//   * periodic wrap of locals        (core/compute.impala:118-122, comm/comm.impala:152-162)
//   * ghost generation (borders)     (comm/comm.impala:105-127, 528-642, 723-734; comm/lb.impala:88-100)
//   * cell binning as a counting sort that reorders the device arrays by cell
//                                    (core/grid.impala:280-321, 406-426)
//   * neighbour-list build, one warp per cell with a home atom per lane, the
//     stencil's candidates filtered by the homes' bounding box and staged in
//     shared memory               (core/neighborlist.impala:1-78)
//
// Ghost order.  The reference runs six passes (x+, x-, y+, y-, z+, z-); a
// pass scans locals then all earlier ghosts in order and appends the ones
// within one cell of the face, shifted by one box length.  A ghost is
// therefore identified by its root local r and its pass combination
// (ex, ey, ez) with e in {0 none, 1 plus pass, 2 minus pass}, and the
// reference appends them grouped by base-3 type index ez*9 + ey*3 + ex - 1,
// in increasing r inside a type.  The kernels below compute that order
// directly: one mask per local, per-type counts, one exclusive scan, emit.
//
// In-cell order.  The reference fills cells sequentially by particle index,
// so a cell lists its locals in input order, then its ghosts in ghost order.
// The counting sort here ranks each cell's members by that reference index,
// which makes list order -- and hence FP64 force summation order -- equal to
// the reference's.

#include <cstdio>

#include "comm.h"
#include "md_common.cuh"
#include "md_state.h"

namespace tmd {

namespace {

struct GeoArgs {
    double wlo[3], whi[3], alo[3], ahi[3], len[3];
    double spacing;
    int nx, ny, nz, ncells;
    double rb_h, inv_rb_h;
};

GeoArgs geo_args(const Geometry& g) {
    GeoArgs a;
    for (int d = 0; d < 3; ++d) {
        a.wlo[d] = g.world_lo[d];
        a.whi[d] = g.world_hi[d];
        a.alo[d] = g.aabb_lo[d];
        a.ahi[d] = g.aabb_hi[d];
        a.len[d] = g.len[d];
    }
    a.spacing = g.spacing;
    a.nx = g.nx;
    a.ny = g.ny;
    a.nz = g.nz;
    a.ncells = g.ncells;
    a.rb_h = g.rb_h;
    a.inv_rb_h = 1.0 / g.rb_h;
    return a;
}

__device__ __forceinline__ double comp(const double4& p, int d) { return d == 0 ? p.x : (d == 1 ? p.y : p.z); }

// core/grid.impala:406-411 and 419-426: floor per axis, flattened, with only
// the global range check.  Returns ncells when outside.
__device__ __forceinline__ int flat_cell(const double4& p, const GeoArgs& a) {
    int i = (int)floor(ddiv(dsub(p.x, a.alo[0]), a.spacing));
    int j = (int)floor(ddiv(dsub(p.y, a.alo[1]), a.spacing));
    int k = (int)floor(ddiv(dsub(p.z, a.alo[2]), a.spacing));
    int c = (k * a.ny + j) * a.nx + i;
    return (c >= 0 && c < a.ncells) ? c : a.ncells;
}

// The rebasing cell is computed here only (the binning's move) and stored, so every kernel sees
// the same cell; a product with 1 / h instead of a correctly rounded division is enough (a pair
// within the list cutoff stays within one cell step whatever the rounding at a cell boundary).
__device__ __forceinline__ int rebase_cell(const double4& p, const GeoArgs& a) {
    int i = (int)floor((p.x - a.alo[0]) * a.inv_rb_h);
    int j = (int)floor((p.y - a.alo[1]) * a.inv_rb_h);
    int k = (int)floor((p.z - a.alo[2]) * a.inv_rb_h);
    return pack3(i, j, k);
}

}  // namespace

// ---- periodic wrap ---------------------------------------------------------
// comm/comm.impala:152-162: one wrap per axis with strict comparisons against
// the world box.  img counts wraps so the adjoint can unwrap displacements.
__device__ __forceinline__ double4 wrap_local(double4* __restrict__ pos, int* __restrict__ img, int i,
                                              const GeoArgs& a) {
    double4 p = pos[i];
    double c[3] = {p.x, p.y, p.z};
    int im = img[i];
    int w[3] = {unpack_axis(im, 0), unpack_axis(im, 1), unpack_axis(im, 2)};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double v = comp(p, d);
        if (v < a.wlo[d]) { c[d] = dadd(c[d], a.len[d]); w[d] -= 1; }
        if (v > a.whi[d]) { c[d] = dsub(c[d], a.len[d]); w[d] += 1; }
    }
    p = make_double4(c[0], c[1], c[2], p.w);
    pos[i] = p;
    img[i] = pack3(w[0], w[1], w[2]);
    return p;
}

__global__ void k_enforce_pbc(double4* __restrict__ pos, int* __restrict__ img, int N, GeoArgs a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    wrap_local(pos, img, i, a);
}

// ---- borders ---------------------------------------------------------------
// Mask of the 26 ghost types of one local (bit t = ez*9 + ey*3 + ex - 1) in
// bits 0-25 and the six periodic flags of its passes in bits 26-31
// (x+, x-, y+, y-, z+, z-): flag set means the pass shifts that axis.
__device__ __forceinline__ unsigned border_mask(const double4& p, const GeoArgs& a) {
    const double dsp = dmul(a.spacing, 2.0);
    unsigned has[3] = {0, 0, 0};  // bit0 plus pass, bit1 minus pass
    unsigned flags = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double v = comp(p, d);
        // comm/comm.impala:116-127 (grid.aabb is the extended rank box)
        if (v > dsub(a.ahi[d], dsp)) has[d] |= 1u;
        if (v < dadd(a.alo[d], dsp)) has[d] |= 2u;
        // comm/lb.impala:88-100 with the pass direction
        if (v > dsub(a.whi[d], a.spacing)) flags |= 1u << (2 * d);
        if (v < dadd(a.wlo[d], a.spacing)) flags |= 1u << (2 * d + 1);
    }
    unsigned mask = 0;
    for (int ez = 0; ez < 3; ++ez) {
        if (ez && !(has[2] & (1u << (ez - 1)))) continue;
        for (int ey = 0; ey < 3; ++ey) {
            if (ey && !(has[1] & (1u << (ey - 1)))) continue;
            for (int ex = 0; ex < 3; ++ex) {
                if (ex && !(has[0] & (1u << (ex - 1)))) continue;
                int t = ez * 9 + ey * 3 + ex;
                if (t) mask |= 1u << (t - 1);
            }
        }
    }
    return mask | (flags << 26);
}

// Pass 1: masks in reference order and per-block per-type counts [26][nblk].  WRAP: the
// periodic wrap of each local (k_enforce_pbc's) is done here first, one launch fewer.
template <bool WRAP>
__global__ void __launch_bounds__(kBorderThreads) k_border_count(double4* __restrict__ pos, int* __restrict__ img, const int* __restrict__ slot_of_ref,
                               unsigned* __restrict__ bmask, int* __restrict__ bcount, int N, int nblk, GeoArgs a,
                               int* __restrict__ cnt, int nseg, DevStatus* st) {
    __shared__ int wc[kBorderThreads / 32][26];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // the binning that follows starts from zeroed cell counters and status (no memsets there)
    for (int g = r; g < nseg; g += gridDim.x * blockDim.x) cnt[g] = 0;
    if (r == 0) st->out_local = st->out_ghost = st->nchain = st->img_over1 = st->img_over2 = 0;
    unsigned m = 0;
    if (r < N) {
        const int sl = slot_of_ref[r];
        m = border_mask(WRAP ? wrap_local(pos, img, sl, a) : pos[sl], a);
        bmask[r] = m;
    }
    for (int t = 0; t < 26; ++t) {
        unsigned b = __ballot_sync(0xffffffffu, (m >> t) & 1u);
        if (lane == 0) wc[wid][t] = __popc(b);
    }
    __syncthreads();
    if (threadIdx.x < 26) {
        int s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += wc[w][threadIdx.x];
        bcount[threadIdx.x * nblk + blockIdx.x] = s;
    }
}

// Pass 2 (after an exclusive scan of bcount into boff): writes every ghost at
// slot N + g, g its reference ghost index, with its source / root links.
// MR (several ranks): only the types in selfmask are periodic ghosts of this rank; the others
// are images for the neighbour ranks, listed (root, type) in type order for the halo pack.
// tab[t] / tab[26 + t]: images of the other kind before type t (k_halo.cu's table).
struct RemoteOut {
    const int* tab;
    int* send_ref;
    int* send_type;
    unsigned selfmask;
};

template <bool MR>
__global__ void __launch_bounds__(kBorderThreads) k_border_emit(double4* __restrict__ pos, double4* __restrict__ vel, double4* __restrict__ frc,
                              double* __restrict__ mass, int* __restrict__ ref, int* __restrict__ slot_of_ref,
                              const unsigned* __restrict__ bmask, const int* __restrict__ boff,
                              int* __restrict__ gsrc, int* __restrict__ groot, int* __restrict__ gcode,
                              int* __restrict__ bsrc_ref, int* __restrict__ broot_ref, int* __restrict__ bcode,
                              int N, int nblk, int capA, GeoArgs a, int sync_vel, RemoteOut ro) {
    __shared__ int wpre[kBorderThreads / 32][26];
    __shared__ unsigned char s_rank[26][kBorderThreads];  // a thread's rank among its warp's ghosts of each type
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned m = r < N ? bmask[r] : 0u;
    const unsigned lt = lanemask_lt();
    for (int t = 0; t < 26; ++t) {
        unsigned b = __ballot_sync(0xffffffffu, (m >> t) & 1u);
        s_rank[t][threadIdx.x] = (unsigned char)__popc(b & lt);
        if (lane == 0) wpre[wid][t] = __popc(b);
    }
    __syncthreads();
    if (threadIdx.x < 26) {  // exclusive prefix over warps, per type
        int s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            int c = wpre[w][threadIdx.x];
            wpre[w][threadIdx.x] = s;
            s += c;
        }
    }
    __syncthreads();
    if (r >= N || (m & 0x03ffffffu) == 0) return;
    const int s_root = slot_of_ref[r];
    const double4 p = pos[s_root];
    const double mroot = mass[s_root];
    const double4 vroot = vel[s_root];
    const unsigned flags = m >> 26;
    // index of this root's ghost of type t (a type whose bit is set)
    auto gidx = [&](int t) { return boff[t * nblk + blockIdx.x] + wpre[wid][t] + s_rank[t][threadIdx.x]; };
    for (int t = 0; t < 26; ++t) {
        if (!((m >> t) & 1u)) continue;
        if (MR && !((ro.selfmask >> t) & 1u)) {
            const int k = gidx(t) - ro.tab[26 + t];
            ro.send_ref[k] = r;
            ro.send_type[k] = t;
            continue;
        }
        const int g = gidx(t) - (MR ? ro.tab[t] : 0);
        const int slot = N + g;
        if (slot >= capA) continue;  // the host grows the arrays and redoes the pass
        const int tt = t + 1;
        const int e[3] = {tt % 3, (tt / 3) % 3, tt / 9};
        int last = e[2] ? 2 : (e[1] ? 1 : 0);
        double c[3] = {p.x, p.y, p.z};
        int tot[3] = {0, 0, 0};
        int lastsh = 0;
        for (int d = 0; d < 3; ++d) {
            if (!e[d]) continue;
            // plus pass shifts by -1 when the flag holds, minus pass by +1
            int sh = 0;
            if (e[d] == 1 && (flags & (1u << (2 * d)))) sh = -1;
            if (e[d] == 2 && (flags & (1u << (2 * d + 1)))) sh = 1;
            c[d] = dadd(c[d], dmul(a.len[d], (double)sh));
            tot[d] = sh;
            if (d == last) lastsh = sh;
        }
        // source of the last pass: the ghost of the same root without the last axis, or the root
        const int tsrc = tt - e[last] * (last == 0 ? 1 : (last == 1 ? 3 : 9));
        const int src_ref = tsrc == 0 ? r : N + gidx(tsrc - 1) - (MR ? ro.tab[tsrc - 1] : 0);
        const int src_slot = tsrc == 0 ? s_root : src_ref;  // a ghost's slot is its reference index
        int code = 0;
        for (int d = 0; d < 3; ++d) {
            int ls = (d == last) ? lastsh : 0;
            code |= (ls + 1) << (2 * d);
            code |= (tot[d] + 1) << (8 + 2 * d);
        }
        pos[slot] = make_double4(c[0], c[1], c[2], 0.0);
        mass[slot] = mroot;
        frc[slot] = make_double4(0.0, 0.0, 0.0, 0.0);
        vel[slot] = sync_vel ? vroot : make_double4(0.0, 0.0, 0.0, 0.0);
        ref[slot] = slot;
        slot_of_ref[slot] = slot;
        gsrc[g] = src_slot;
        groot[g] = s_root;
        gcode[g] = code;
        bsrc_ref[g] = src_ref;
        broot_ref[g] = r;
        bcode[g] = code;
    }
}

// ---- binning (counting sort) -----------------------------------------------
// cnt / cstart layout: [0, ncells] locals per cell (index ncells = outside
// the grid), [ncells+1, 2*ncells+1] ghosts per cell.
__global__ void k_bin_count(const double4* __restrict__ pos, int* __restrict__ cnt, int* __restrict__ bin_cell,
                            int* __restrict__ bin_rank, DevStatus* st, int N, int NA, GeoArgs a) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= NA) return;
    int c = flat_cell(pos[s], a);
    if (c == a.ncells) atomicAdd(s < N ? &st->out_local : &st->out_ghost, 1);
    int seg = s < N ? c : (a.ncells + 1) + c;
    bin_cell[s] = c;
    bin_rank[s] = atomicAdd(&cnt[seg], 1);
}

__global__ void k_bin_scatter(const int* __restrict__ ref, const int* __restrict__ bin_cell,
                              const int* __restrict__ bin_rank, const int* __restrict__ cstart,
                              int* __restrict__ tmp_key, int* __restrict__ tmp_src, int N, int NA, int ncells) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= NA) return;
    int c = bin_cell[s];
    int seg = s < N ? c : (ncells + 1) + c;
    int p = cstart[seg] + bin_rank[s];
    tmp_key[p] = ref[s];
    tmp_src[p] = s;
}

// The members of a segment (a cell's locals or its ghosts) ranked by reference index (keys are
// unique), each moved from its old slot to its new one (cstart[segment] + rank).  The two
// outside-the-grid buckets keep arrival order: their members have no neighbours and are
// nobody's neighbour, so their order is not observable.
struct MoveArgs {
    const double4* pos_o; double4* pos_n;
    const double4* vel_o; double4* vel_n;
    const double4* frc_o; double4* frc_n;
    const double* mass_o; double* mass_n;
    const int* ref_o; int* ref_n;
    const int* img_o; int* img_n;
    int* slot_of_ref; int* rref; int* rbk;
    const int* bin_cell; int* slot_cell;
    float4* pos32; int* img_cnt; int* img_slot;
    int capA, N, mixed;
};

__device__ __forceinline__ void move_slot(int n, int o, const MoveArgs& m, const GeoArgs& a) {
    m.slot_cell[n] = m.bin_cell[o];
    const double4 p = m.pos_o[o];
    m.pos_n[n] = p;
    m.vel_n[n] = m.vel_o[o];
    m.frc_n[n] = m.frc_o[o];
    m.mass_n[n] = m.mass_o[o];
    const int r = m.ref_o[o];
    m.ref_n[n] = r;
    if (n < m.N) {
        m.img_n[n] = m.img_o[o];
        m.rref[n] = r;
        // empty image records for k_ghost_links to fill
        m.img_cnt[n] = 0;
        m.img_cnt[m.capA + n] = 0;
#pragma unroll
        for (int k = 0; k < kImgW; ++k) m.img_slot[(size_t)k * m.capA + n] = -1;
    }
    m.slot_of_ref[r] = n;
    const int k = rebase_cell(p, a);
    m.rbk[n] = k;
    if (m.mixed) m.pos32[n] = rebased32(p, k, a.alo, a.rb_h);
}

// One thread per new slot: the slot's segment (cell, locals or ghosts) from its old slot's cell,
// its rank among the segment's members by reference index, then the move.  (A warp per segment
// left ~45 % of the lanes idle and half the warps on the empty ghost segments of inner cells.)
__global__ void k_rank_move(const int* __restrict__ cstart, const int* __restrict__ tmp_key,
                            const int* __restrict__ tmp_src, int NA, int ncells, MoveArgs m, GeoArgs ga,
                            DevStatus* st) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    // the list build that follows starts from a zeroed status (no memset there)
    if (e == 0) st->max_nb = 0;
    if (e >= NA) return;
    const int o = tmp_src[e];
    const int key = tmp_key[e];
    const int c = m.bin_cell[o];
    int n = e;  // atoms outside the grid keep their bucket order
    if (c != ncells) {
        const int seg = o < m.N ? c : ncells + 1 + c;
        const int a = cstart[seg], b = cstart[seg + 1];
        int rank = 0;
        for (int f = a; f < b; ++f) rank += tmp_key[f] < key;
        n = a + rank;
    }
    move_slot(n, o, m, ga);
}

// Per ghost: its source, root and shift code in slot terms, and its place in the image
// records of the locals (k_rank_move emptied them): a local's direct two-phase images (ghosts
// whose source it is) and all its images (ghosts whose root it is), one plane per image
// number (filled in order, -1 beyond the last); ghosts whose two-phase source is another
// ghost go to `chain`.  The order within a record follows the atomics, but every ghost is
// written exactly once, so the result is deterministic.
struct LinkArgs {
    const int* ref; const int* slot_of_ref; const int* bsrc_ref; const int* broot_ref; const int* bcode;
    int* gsrc; int* groot; int* gcode; int* rref; int* img_cnt; int* img_slot; int* chain;
    DevStatus* st;
    int N, G, capA;
};

__device__ __forceinline__ void ghost_link(int h, const LinkArgs& l) {
    const int N = l.N, capA = l.capA;
    int g = l.ref[N + h] - N;
    if (l.broot_ref[g] < 0) {  // received from another rank: refreshed by the halo exchange
        l.gsrc[h] = l.groot[h] = -1;
        l.gcode[h] = 0;
        l.rref[N + h] = -1;
        return;
    }
    const int s1 = l.slot_of_ref[l.bsrc_ref[g]];
    const int r = l.slot_of_ref[l.broot_ref[g]];
    l.gsrc[h] = s1;
    l.groot[h] = r;
    l.gcode[h] = l.bcode[g];
    l.rref[N + h] = l.broot_ref[g];
    const int t = N + h;
    if (s1 < N) {
        const int k = atomicAdd(&l.img_cnt[s1], 1);
        if (k < kImg1) l.img_slot[(size_t)k * capA + s1] = t;
        else atomicAdd(&l.st->img_over1, 1);
    } else {
        l.chain[atomicAdd(&l.st->nchain, 1)] = h;
    }
    const int k2 = atomicAdd(&l.img_cnt[capA + r], 1);
    if (k2 < kImg2) l.img_slot[(size_t)(kImg1 + k2) * capA + r] = t;
    else atomicAdd(&l.st->img_over2, 1);
}

__global__ void k_ghost_links(LinkArgs l) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h < l.G) ghost_link(h, l);
}

// ---- neighbour lists ---------------------------------------------------------
// rebasing cell k relative to b as dx + 4 dy + 16 dz (signed offsets per axis): for two atoms
// whose offsets differ by at most 1 on every axis, (c - i) + 21 is exactly the list code
// (dx+1) | (dy+1) << 2 | (dz+1) << 4 of the pair, each term being 0, 1 or 2 with no carry
__device__ __forceinline__ int rel_code(int k, int b) {
    return wrap_diff(unpack_axis(k, 0), unpack_axis(b, 0)) + 4 * wrap_diff(unpack_axis(k, 1), unpack_axis(b, 1)) +
           16 * wrap_diff(unpack_axis(k, 2), unpack_axis(b, 2));
}
constexpr int kCodeBias = 1 + 4 + 16;  // dk + 1 on every axis

// The reference's exact FP64 membership test for a pair near the list cutoff (core/neighborlist.impala:
// 18-78), which the FP32 prefilter cannot decide (~1 candidate in 150)
__device__ __forceinline__ bool exact_within(const double4* __restrict__ pos, int i, int j, double cut2) {
    const double4 pi = pos[i], pj = pos[j];
    return len2_strict(dsub(pi.x, pj.x), dsub(pi.y, pj.y), dsub(pi.z, pj.z)) <= cut2;
}

// Warp per cell (core/neighborlist.impala:18-78), one home atom per lane (32 at a time).  The
// 27 stencil cells' candidates (locals then ghosts per cell, stencil order) are staged in shared
// memory, keeping only those within the list cutoff (with the FP32 margin) of the bounding box
// of the homes, in order; then every lane walks the kept candidates (one broadcast read each)
// and appends its own pairs, so each list comes out in stencil order -- the reference's, which
// fixes the FP64 summation order -- with no cross-lane compaction.  Lanes without a home sit
// far away and never match.  Pairs near the cutoff take the reference's FP64 test
// (rsq <= cutoff^2), so membership is exactly the reference's.
//
// List layout: quads of four consecutive entries of one atom, atom-fastest (nl_index): a force
// kernel reads four entries with one 16-byte load, and the quads of a warp's 32 atoms form one
// 512-byte line.  An entry is slot << 6 | code, code = dk + 1 per axis, dk the neighbour's
// rebasing cell minus the home's (mixed form).  A list's last quad is padded with the home
// itself one rebasing cell away on every axis (code 42), which every force kernel skips by
// count or finds beyond its cutoff.
#ifndef TMD_NL_WARPS
#define TMD_NL_WARPS 4
#endif
#ifndef TMD_NL_TILE
#define TMD_NL_TILE 128
#endif
#ifndef TMD_NL_MINB
#define TMD_NL_MINB 8  // 64 registers: eight blocks of four warps per SM
#endif
#ifndef TMD_NL_UNROLL
#define TMD_NL_UNROLL 4
#endif
constexpr int kNlWarps = TMD_NL_WARPS;    // warps (cells) per block
constexpr int kNlTile = TMD_NL_TILE;      // kept candidates staged per warp before the homes walk them
constexpr int kNlUnroll = TMD_NL_UNROLL;  // candidates per step of a home's walk
constexpr uint32_t kPadCode = 42u;        // dk = +1 on every axis

struct NlArgs {
    double cut2;     // cutoff^2 (FP64, the reference's membership test)
    float lo2, hi2;  // FP32 prefilter: certainly inside below lo2, certainly outside above hi2
    int nbcap, stride, N, ncells, nx, nxy;
    double alo[3], spacing;
};

template <int HM, typename IDX>
__global__ void __launch_bounds__(kNlWarps * 32, TMD_NL_MINB)
k_build_list(const double4* __restrict__ pos, const int* __restrict__ ref, const int* __restrict__ rbk,
             const int* __restrict__ cstart, int* __restrict__ nbn, uint32_t* __restrict__ nbl, DevStatus* st,
             NlArgs a, int cell_blocks, LinkArgs la) {
    // kept candidate position (cell-centre relative); w = slot << 6 + its rebasing cell relative to
    // the first home's (rel_code) + kCodeBias, from which a home's entry is one subtraction
    __shared__ float4 s_cpos[kNlWarps][kNlTile];
    __shared__ int s_cref[kNlWarps][HM ? kNlTile : 1];
    __shared__ int s_rstart[kNlWarps][54];
    __shared__ int s_rpre[kNlWarps][55];

    if (blockIdx.x >= cell_blocks) {  // blocks past the cells link the ghosts (k_ghost_links' work)
        const int h = (blockIdx.x - cell_blocks) * blockDim.x + threadIdx.x;
        if (h < la.G) ghost_link(h, la);
        return;
    }
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * kNlWarps + wid;
    if (c >= a.ncells) return;
    const int h0 = cstart[c], h1 = cstart[c + 1];
    if (h0 == h1) return;
    const unsigned lt = lanemask_lt();

    // 27 stencil cells in the reference order (z, y, x offsets -1..1), each contributing
    // its locals then its ghosts (54 ranges); lane l owns ranges 2l and 2l + 1
    {
        int start = 0, len = 0, gs = 0, gl = 0;
        if (lane < 27) {
            const int oz = lane / 9 - 1, oy = (lane / 3) % 3 - 1, ox = lane % 3 - 1;
            const int nb = c + oz * a.nxy + oy * a.nx + ox;
            if (nb >= 0 && nb < a.ncells) {
                start = cstart[nb];
                len = cstart[nb + 1] - start;
                gs = cstart[a.ncells + 1 + nb];
                gl = cstart[a.ncells + 2 + nb] - gs;
            }
        }
        int incl = len + gl;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane < 27) {
            const int ex = incl - len - gl;
            s_rstart[wid][2 * lane] = start;
            s_rstart[wid][2 * lane + 1] = gs;
            s_rpre[wid][2 * lane] = ex;
            s_rpre[wid][2 * lane + 1] = ex + len;
        }
        if (lane == 26) s_rpre[wid][54] = incl;
    }
    __syncwarp();
    const int M = s_rpre[wid][54];

    const int cz = c / a.nxy, cy = (c / a.nx) % (a.nxy / a.nx), cx = c % a.nx;
    const double ctr[3] = {a.alo[0] + ((double)cx + 0.5) * a.spacing, a.alo[1] + ((double)cy + 0.5) * a.spacing,
                           a.alo[2] + ((double)cz + 0.5) * a.spacing};
    const int rb0 = __ldg(rbk + h0);  // rebasing cells are staged relative to the first home's
    int maxcnt = 0;

    for (int hb = h0; hb < h1; hb += 32) {
        const int hn = min(32, h1 - hb);
        const bool home = lane < hn;
        const int i = hb + (home ? lane : 0);
        float hx = 1e18f, hy = 1e18f, hz = 1e18f;  // no home: never within the cutoff
        int irel = 0, iref = 0;
        if (home) {
            const double4 p = pos[i];
            hx = (float)(p.x - ctr[0]);
            hy = (float)(p.y - ctr[1]);
            hz = (float)(p.z - ctr[2]);
            irel = rel_code(rbk[i], rb0);
            if (HM) iref = ref[i];
        }
        // a candidate's staged w minus irel is the entry slot << 6 | code; it equals i6 only for
        // the home itself (within the cutoff the two rebasing parts differ by less than 64)
        const uint32_t i6 = ((uint32_t)i << kCodeBits) + (uint32_t)(irel + kCodeBias);
        // nl_index in the list's index type: 32-bit unless the list holds 2^32 entries or more
        // (the 64-bit index arithmetic made the build 15 % slower)
        const IDX i4 = HM ? 0 : (IDX)i * 4u, stride4 = HM ? 0 : (IDX)a.stride * 4u;  // (the half lists: nl_index)
        // bounding box of the homes, widened by the list cutoff (with the FP32 margin)
        float lo[3] = {home ? hx : INFINITY, home ? hy : INFINITY, home ? hz : INFINITY};
        float hi[3] = {home ? hx : -INFINITY, home ? hy : -INFINITY, home ? hz : -INFINITY};
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], off));
                hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], off));
            }
        int cnt = 0;
        int t0 = 0;  // next candidate to stage (M > 0: the home cell is in the stencil)
        do {
            int nk = 0;  // kept candidates staged (warp-uniform)
            // stage: keep candidates in order until the next chunk might not fit
            while (t0 < M && nk + 32 <= kNlTile) {
                const int m = t0 + lane;
                bool keep = false;
                float4 cp;
                int cref = 0;
                if (m < M) {
                    int lo_r = 0, hi_r = 53;  // the range of candidate m: the last one starting at or before m
                    while (lo_r < hi_r) {
                        const int mid = (lo_r + hi_r + 1) >> 1;
                        if (s_rpre[wid][mid] <= m) lo_r = mid;
                        else hi_r = mid - 1;
                    }
                    const int slot = s_rstart[wid][lo_r] + (m - s_rpre[wid][lo_r]);
                    // the candidate's position, rebasing cell and key load together (one latency)
                    const double4 p = pos[slot];
                    const int kb = __ldg(rbk + slot);
                    if (HM) cref = __ldg(ref + slot);  // root reference index (ref for locals)
                    cp = make_float4((float)(p.x - ctr[0]), (float)(p.y - ctr[1]), (float)(p.z - ctr[2]),
                                     __uint_as_float(((uint32_t)slot << kCodeBits) +
                                                     (uint32_t)(rel_code(kb, rb0) + kCodeBias)));
                    const float ex = fmaxf(fmaxf(lo[0] - cp.x, cp.x - hi[0]), 0.f);
                    const float ey = fmaxf(fmaxf(lo[1] - cp.y, cp.y - hi[1]), 0.f);
                    const float ez = fmaxf(fmaxf(lo[2] - cp.z, cp.z - hi[2]), 0.f);
                    keep = fmaf(ex, ex, fmaf(ey, ey, ez * ez)) <= a.hi2;
                }
                const unsigned bal = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int at = nk + __popc(bal & lt);
                    s_cpos[wid][at] = cp;
                    if (HM) s_cref[wid][at] = cref;
                }
                nk += __popc(bal);
                t0 += 32;
            }
            __syncwarp();
            // every home walks the kept candidates in order
#pragma unroll kNlUnroll
            for (int k = 0; k < nk; ++k) {
                const float4 cp = s_cpos[wid][k];
                const float dx = hx - cp.x, dy = hy - cp.y, dz = hz - cp.z;
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const uint32_t s6 = __float_as_uint(cp.w);
                bool in = r2 < a.lo2;
                // near the cutoff (|dk| <= 1 still holds there): s6 - irel is the entry, its slot the candidate's
                if (!in && r2 <= a.hi2) in = exact_within(pos, i, (s6 - (uint32_t)irel) >> kCodeBits, a.cut2);
                // core/neighborlist.impala:34: half lists keep i > j (reference index); HM == 2
                // compares ghosts by their root so pairs across the periodic boundary are kept once
                const bool take = in && s6 != i6 && (!HM || s_cref[wid][HM ? k : 0] < iref);
                // the entry slot << 6 | code: the list cutoff below the rebasing spacing keeps
                // every |dk| <= 1 within it (checked on the host)
                if (HM) {
                    // half lists: the append without a branch (measured faster there, while
                    // the full-list walk is faster with the branch)
                    if (take && cnt < a.nbcap) nbl[nl_index(cnt, i, a.stride)] = s6 - (uint32_t)irel;
                    cnt += take ? 1 : 0;
                } else if (take) {
                    // (a store at every step, without the branch: 147 -> 182 us at 131k atoms)
                    if (cnt < a.nbcap) nbl[(IDX)(cnt >> 2) * stride4 + i4 + (IDX)(cnt & 3)] = s6 - (uint32_t)irel;
                    ++cnt;
                }
            }
            __syncwarp();
        } while (t0 < M);
        if (home) {
            nbn[i] = cnt;
            // the last quad's padding
            const uint32_t pad = ((uint32_t)i << kCodeBits) | kPadCode;
            for (int q = cnt; (q & 3) != 0 && q < a.nbcap; ++q) nbl[nl_index(q, i, a.stride)] = pad;
            maxcnt = max(maxcnt, cnt);
        }
    }
    maxcnt = warp_max(maxcnt);
    if (lane == 0) atomicMax(&st->max_nb, maxcnt);
}

// Locals outside the grid (bucket ncells) get empty lists.
__global__ void k_clear_lists(int* __restrict__ nbn, int a, int b) {
    int i = a + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < b) nbn[i] = 0;
}

// ---- exclusive scan ------------------------------------------------------------
__device__ __forceinline__ int block_exscan(int v, int* total, int* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int nw = blockDim.x >> 5;
        int w = lane < nw ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        sh[lane] = w;  // inclusive prefix of warp sums
    }
    __syncthreads();
    int r = x - v + (wid ? sh[wid - 1] : 0);
    *total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return r;
}

constexpr int kScanThreads = 1024, kScanItems = 4, kScanBlock = kScanThreads * kScanItems;

// per-block totals of the input
__global__ void k_scan_sums(const int* __restrict__ in, int* __restrict__ part, int n) {
    __shared__ int sh[32];
    int base = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
    int s = 0;
    for (int k = 0; k < kScanItems; ++k) s += (base + k < n) ? in[base + k] : 0;
    int tot;
    block_exscan(s, &tot, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// exclusive scan of the block totals in place (one block); part[nb] = grand total
__global__ void k_scan_part(int* __restrict__ part, int nb) {
    __shared__ int sh[32];
    int carry = 0;
    for (int b0 = 0; b0 < nb; b0 += kScanThreads) {
        int i = b0 + threadIdx.x;
        int v = i < nb ? part[i] : 0;
        int tot;
        int ex = block_exscan(v, &tot, sh);
        if (i < nb) part[i] = carry + ex;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) part[nb] = carry;
}

__global__ void k_scan_apply(const int* __restrict__ in, int* __restrict__ out, const int* __restrict__ part,
                             int n, int nb) {
    __shared__ int sh[32];
    int base = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    int tot;
    int ex = block_exscan(s, &tot, sh) + part[blockIdx.x];
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = ex;
        ex += v[k];
    }
    if (blockIdx.x == nb - 1 && threadIdx.x == 0) out[n] = part[nb];
}

// Exclusive scan of up to kScanSingleMax values in one block: the values are staged in
// shared memory by coalesced loads, each thread scans a run of consecutive values there,
// the block scans the run totals, and the results leave by coalesced stores.  One launch
// instead of three for the counts of a rebuild (tens of thousands of values).
constexpr int kScanSingleMax = 32768;  // 128 KiB of shared memory
__global__ void __launch_bounds__(kScanThreads) k_scan_single(const int* __restrict__ in, int* __restrict__ out,
                                                               int n) {
    extern __shared__ int sv[];
    __shared__ int sh[32];
#pragma unroll 8
    for (int k = threadIdx.x; k < n; k += kScanThreads) sv[k] = in[k];
    __syncthreads();
    const int run = (n + kScanThreads - 1) / kScanThreads;
    const int base = threadIdx.x * run;
    const int end = min(base + run, n);
    int s = 0;
    for (int k = base; k < end; ++k) s += sv[k];
    int tot;
    int ex = block_exscan(s, &tot, sh);
    for (int k = base; k < end; ++k) {
        const int v = sv[k];
        sv[k] = ex;
        ex += v;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = threadIdx.x; k < n; k += kScanThreads) out[k] = sv[k];
    if (threadIdx.x == 0) out[n] = tot;
}

// ---- host wrappers ---------------------------------------------------------------
// Single-pass exclusive scan of a long array (decoupled look-back): block b scans tile b,
// publishes its total, then adds the totals of the tiles before it -- a tile that already
// knows its inclusive prefix ends the walk -- and publishes that prefix.  A tile word holds
// (launch epoch << 2 | state) << 32 | value, so nothing is reset between launches.  The wait
// for a predecessor is bounded: past the limit the block sums that predecessor's inputs (and
// all before it) directly, so the result never depends on the wait ending (the grids here
// are a few dozen blocks, all resident at once).  One launch with ~11 blocks for the 21k cell
// counts of a 131k-atom rebuild, where one block walked all of them.
constexpr int kLbThreads = 256, kLbItems = 8, kLbTile = kLbThreads * kLbItems;
constexpr int kLbSpinLimit = 1 << 14;  // polls of a predecessor's word (64 ns apart) before summing it directly

__device__ __forceinline__ unsigned long long lb_word(unsigned epoch, unsigned state, int v) {
    return ((unsigned long long)((epoch << 2) | state) << 32) | (unsigned)v;
}

__global__ void __launch_bounds__(kLbThreads)
k_scan_lookback(const int* __restrict__ in, int* __restrict__ out, int n, int ntiles,
                unsigned long long* __restrict__ tiles, unsigned epoch) {
    __shared__ int sh[32];
    __shared__ int s_prefix, s_missing;
    const int tile = blockIdx.x;
    const int base = tile * kLbTile + threadIdx.x * kLbItems;
    int v[kLbItems];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kLbItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        sum += v[k];
    }
    int total;
    const int ex = block_exscan(sum, &total, sh);
    if (threadIdx.x == 0) {
        int excl = 0, missing = -1;
        volatile unsigned long long* tw = tiles;
        if (tile == 0) {
            tw[0] = lb_word(epoch, 2u, total);
        } else {
            tw[tile] = lb_word(epoch, 1u, total);
            const unsigned want = epoch & 0x3fffffffu;
            for (int j = tile - 1; j >= 0; --j) {
                unsigned long long w = tw[j];
                int spins = 0;
                while (((unsigned)(w >> 34) != want || ((w >> 32) & 3u) == 0u) && spins < kLbSpinLimit) {
                    __nanosleep(64);
                    w = tw[j];
                    ++spins;
                }
                if ((unsigned)(w >> 34) != want || ((w >> 32) & 3u) == 0u) {
                    missing = j;
                    break;
                }
                excl += (int)(unsigned)w;
                if (((w >> 32) & 3u) == 2u) break;
            }
            if (missing < 0) tw[tile] = lb_word(epoch, 2u, excl + total);
        }
        s_prefix = excl;
        s_missing = missing;
    }
    __syncthreads();
    int prefix = s_prefix;
    if (s_missing >= 0) {  // the inputs of tiles 0..missing summed directly
        const int end = min(n, (s_missing + 1) * kLbTile);
        int part = 0;
        for (int i = threadIdx.x; i < end; i += kLbThreads) part += in[i];
        int all;
        block_exscan(part, &all, sh);
        prefix += all;
        if (threadIdx.x == 0) ((volatile unsigned long long*)tiles)[tile] = lb_word(epoch, 2u, prefix + total);
    }
    int e = prefix + ex;
#pragma unroll
    for (int k = 0; k < kLbItems; ++k) {
        if (base + k < n) out[base + k] = e;
        e += v[k];
    }
    if (tile == ntiles - 1 && threadIdx.x == 0) out[n] = prefix + total;
}

static inline int nblocks(long long n, int t) { return (int)((n + t - 1) / t); }

void ensure_scan_scratch(State& s, int n) {
    int nb = nblocks(n, kScanBlock) + 1;
    if (nb > s.scan_part_cap) {
        dfree(&s.scan_part);
        s.scan_part_cap = nb + 64;
        dalloc(&s.scan_part, s.scan_part_cap);
    }
}

// look-back scans from this many values on (below, one block is as fast)
#ifndef TMD_LB_MIN
#define TMD_LB_MIN 8192
#endif
constexpr int kLookbackMin = TMD_LB_MIN;

static bool ensure_lookback(State& s, int ntiles) {
    if (ntiles <= s.lb_tile_cap) return true;
    dfree(&s.lb_tiles);
    s.lb_tile_cap = ntiles + 64;
    dalloc(&s.lb_tiles, s.lb_tile_cap);
    if (!s.lb_tiles) {
        s.lb_tile_cap = 0;
        return false;
    }
    TMD_CUDA(cudaMemsetAsync(s.lb_tiles, 0, sizeof(unsigned long long) * s.lb_tile_cap, s.stream));
    return true;
}

// out[0..n-1] = exclusive prefix sums of in, out[n] = total (in != out allowed only)
void exclusive_scan(State& s, const int* in, int* out, int n) {
    if (n >= kLookbackMin) {
        const int ntiles = nblocks(n, kLbTile);
        if (ensure_lookback(s, ntiles)) {
            k_scan_lookback<<<ntiles, kLbThreads, 0, s.stream>>>(in, out, n, ntiles, s.lb_tiles, ++s.lb_epoch);
            launched(K_SCAN);
            return;
        }
    }
    if (n <= kScanSingleMax) {
        if (s.scan_attr_device != s.device) {  // a function attribute is set per device
            TMD_CUDA(cudaFuncSetAttribute(k_scan_single, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kScanSingleMax * (int)sizeof(int)));
            s.scan_attr_device = s.device;
        }
        k_scan_single<<<1, kScanThreads, (size_t)n * sizeof(int), s.stream>>>(in, out, n);
        launched(K_SCAN);
        return;
    }
    int nb = nblocks(n, kScanBlock);
    if (nb < 1) nb = 1;
    ensure_scan_scratch(s, n);
    k_scan_sums<<<nb, kScanThreads, 0, s.stream>>>(in, s.scan_part, n);
    launched(K_SCAN);
    k_scan_part<<<1, kScanThreads, 0, s.stream>>>(s.scan_part, nb);
    launched(K_SCAN);
    k_scan_apply<<<nb, kScanThreads, 0, s.stream>>>(in, out, s.scan_part, n, nb);
    launched(K_SCAN);
}

void run_enforce_pbc(State& s) {
    if (s.N == 0) return;
    GeoArgs a = geo_args(s.geo);
    prof_begin(K_PBC);
    k_enforce_pbc<<<nblocks(s.N, 256), 256, 0, s.stream>>>(s.pos.b[s.pc], s.img.b[s.ac], s.N, a);
    launched(K_PBC);
    prof_end(K_PBC);
}

bool grow_atoms(State& s, int need);  // api.cu

void run_borders(State& s, bool wrap) {
    GeoArgs a = geo_args(s.geo);
    const int N = s.N;
    const int nblk = border_blocks(N);
    if (N == 0 && !s.halo.on) {
        s.G = 0;
        return;
    }
    prof_begin(K_BORDER);
    const int nseg = 2 * (a.ncells + 1);
    const int n = 26 * nblk;
    // boff = exclusive scan of bcount, stored after the counts
    int* boff = s.bcount + n;
    if (s.halo.on) {
        // several ranks: the per-type totals first (they split the images into this rank's
        // periodic ghosts and the ones for other ranks), then the emit, then the exchange;
        // a rank without locals still takes part in the exchange
        if (N > 0) {
            if (wrap)
                k_border_count<true><<<nblk, kBorderThreads, 0, s.stream>>>(s.pos.b[s.pc], s.img.b[s.ac], s.slot_of_ref,
                                                                  s.bmask, s.bcount, N, nblk, a, s.cnt, nseg,
                                                                  s.status_dev);
            else
                k_border_count<false><<<nblk, kBorderThreads, 0, s.stream>>>(s.pos.b[s.pc], s.img.b[s.ac], s.slot_of_ref,
                                                                   s.bmask, s.bcount, N, nblk, a, s.cnt, nseg,
                                                                   s.status_dev);
            s.bin_zeroed = true;
            launched(K_BORDER);
            exclusive_scan(s, s.bcount, boff, n);
        }
        bool ok = halo_plan_borders(s, N > 0 ? boff : nullptr, nblk);
        if (ok && N + s.halo.gself > s.capA) ok = grow_atoms(s, N + s.halo.gself);
        if (ok && N > 0) {
            RemoteOut ro{s.halo.tab, s.halo.send_ref, s.halo.send_type, comm().topo.selfmask};
            k_border_emit<true><<<nblk, kBorderThreads, 0, s.stream>>>(s.pos.b[s.pc], s.vel.b[s.vc], s.frc.b[s.ac],
                                                             s.mass.b[s.ac], s.ref.b[s.ac], s.slot_of_ref, s.bmask, boff,
                                                             s.gsrc, s.groot, s.gcode, s.bsrc_ref, s.broot_ref,
                                                             s.bcode, N, nblk, s.capA, a, s.dem_fixed, ro);
            launched(K_BORDER);
        }
        if (ok) ok = halo_finish_borders(s);
        if (!ok) s.G = 0;
        prof_end(K_BORDER);
        s.lists_valid = 0;
        return;
    }
    if (wrap)
        k_border_count<true><<<nblk, kBorderThreads, 0, s.stream>>>(s.pos.b[s.pc], s.img.b[s.ac], s.slot_of_ref, s.bmask,
                                                          s.bcount, N, nblk, a, s.cnt, nseg, s.status_dev);
    else
        k_border_count<false><<<nblk, kBorderThreads, 0, s.stream>>>(s.pos.b[s.pc], s.img.b[s.ac], s.slot_of_ref, s.bmask,
                                                           s.bcount, N, nblk, a, s.cnt, nseg, s.status_dev);
    s.bin_zeroed = true;
    launched(K_BORDER);
    exclusive_scan(s, s.bcount, boff, n);
    // The ghost count comes back while the emit kernel already runs: emit writes only the
    // slots below the capacity, so when the count shows the capacity was short the host
    // grows the arrays (which waits for that emit) and emits again.  The host thus enqueues
    // the next kernels before emit finishes instead of leaving the GPU idle for a round trip.
    // The readback runs on a second stream, so the emit kernel does not queue behind the copy
    // (a rebuild's ghost phase 40 -> 33 us at 131k atoms).
    TMD_CUDA(cudaEventRecord(s.ev_scanned, s.stream));
    TMD_CUDA(cudaStreamWaitEvent(s.copy_stream, s.ev_scanned, 0));
    TMD_CUDA(cudaMemcpyAsync(&s.status_host->nghost, boff + n, sizeof(int), cudaMemcpyDeviceToHost, s.copy_stream));
    TMD_CUDA(cudaEventRecord(s.ev_counted, s.copy_stream));
    auto emit = [&]() {
        k_border_emit<false><<<nblk, kBorderThreads, 0, s.stream>>>(s.pos.b[s.pc], s.vel.b[s.vc], s.frc.b[s.ac], s.mass.b[s.ac],
                                                  s.ref.b[s.ac], s.slot_of_ref, s.bmask, boff, s.gsrc, s.groot,
                                                  s.gcode, s.bsrc_ref, s.broot_ref, s.bcode, N, nblk, s.capA,
                                                  a, s.dem_fixed, RemoteOut{nullptr, nullptr, nullptr, 0u});
        launched(K_BORDER);
    };
    emit();
    TMD_CUDA(cudaEventSynchronize(s.ev_counted));
    const int G = s.status_host->nghost;
    if (N + G > s.capA) {
        if (!grow_atoms(s, N + G)) {  // no room: no ghosts rather than writes past the arrays
            s.G = 0;
            s.lists_valid = 0;
            prof_end(K_BORDER);
            return;
        }
        emit();
    }
    prof_end(K_BORDER);
    s.G = G;
    s.lists_valid = 0;
}

void run_distribute(State& s) {
    GeoArgs a = geo_args(s.geo);
    const int N = s.N, NA = s.N + s.G;
    const int nseg = 2 * (a.ncells + 1);
    if (NA == 0) return;
    prof_begin(K_BIN);
    if (!s.bin_zeroed) {  // else zeroed by the border pass's first kernel
        TMD_CUDA(cudaMemsetAsync(s.cnt, 0, sizeof(int) * nseg, s.stream));
        TMD_CUDA(cudaMemsetAsync(&s.status_dev->out_local, 0, 5 * sizeof(int), s.stream));  // .. img_over2
    }
    s.bin_zeroed = false;
    k_bin_count<<<nblocks(NA, 256), 256, 0, s.stream>>>(s.pos.b[s.pc], s.cnt, s.bin_cell, s.bin_rank, s.status_dev,
                                                        N, NA, a);
    launched(K_BIN);
    exclusive_scan(s, s.cnt, s.cstart, nseg);
    k_bin_scatter<<<nblocks(NA, 256), 256, 0, s.stream>>>(s.ref.b[s.ac], s.bin_cell, s.bin_rank, s.cstart,
                                                          s.tmp_key, s.tmp_src, N, NA, a.ncells);
    launched(K_BIN);
    const int np = 1 - s.pc, nv = 1 - s.vc, na = 1 - s.ac;
    MoveArgs m;
    m.pos_o = s.pos.b[s.pc]; m.pos_n = s.pos.b[np];
    m.vel_o = s.vel.b[s.vc]; m.vel_n = s.vel.b[nv];
    m.frc_o = s.frc.b[s.ac]; m.frc_n = s.frc.b[na];
    m.mass_o = s.mass.b[s.ac]; m.mass_n = s.mass.b[na];
    m.ref_o = s.ref.b[s.ac]; m.ref_n = s.ref.b[na];
    m.img_o = s.img.b[s.ac]; m.img_n = s.img.b[na];
    m.slot_of_ref = s.slot_of_ref; m.rref = s.rref; m.rbk = s.rbk;
    m.bin_cell = s.bin_cell; m.slot_cell = s.slot_cell;
    m.pos32 = s.pos32.b[np]; m.img_cnt = s.img_cnt; m.img_slot = s.img_slot;
    m.capA = s.capA; m.N = N; m.mixed = s.precision;
    k_rank_move<<<nblocks(NA, 256), 256, 0, s.stream>>>(s.cstart, s.tmp_key, s.tmp_src, NA, a.ncells, m, a,
                                                         s.status_dev);
    launched(K_BIN);
    s.build_zeroed = true;
    s.pc = np;
    s.vc = nv;
    s.ac = na;
    // the ghost links run as extra blocks of the list build that follows, or alone
    // (flush_links) before anything else that reads them
    s.pend_links = s.G > 0;
    s.img_ok = 0;  // known after the status readback of the list build
    s.nchain = 0;
    prof_end(K_BIN);
    s.lists_valid = 0;
}

void grow_lists(State& s, int rows);  // api.cu

LinkArgs link_args(State& s) {
    LinkArgs l;
    l.ref = s.ref.b[s.ac];
    l.slot_of_ref = s.slot_of_ref;
    l.bsrc_ref = s.bsrc_ref;
    l.broot_ref = s.broot_ref;
    l.bcode = s.bcode;
    l.gsrc = s.gsrc;
    l.groot = s.groot;
    l.gcode = s.gcode;
    l.rref = s.rref;
    l.img_cnt = s.img_cnt;
    l.img_slot = s.img_slot;
    l.chain = s.chain;
    l.st = s.status_dev;
    l.N = s.N;
    l.G = s.G;
    l.capA = s.capA;
    return l;
}

void flush_links(State& s) {
    if (!s.pend_links) return;
    s.pend_links = false;
    k_ghost_links<<<nblocks(s.G, 256), 256, 0, s.stream>>>(link_args(s));
    launched(K_BIN);
}

template <int HM>
void launch_build_list(State& s, bool wide, int blocks, const int* ref, const NlArgs& a, int nb, const LinkArgs& la) {
    if (wide)
        k_build_list<HM, size_t><<<blocks, kNlWarps * 32, 0, s.stream>>>(s.pos.b[s.pc], ref, s.rbk, s.cstart, s.nbn,
                                                                         s.nbl, s.status_dev, a, nb, la);
    else
        k_build_list<HM, uint32_t><<<blocks, kNlWarps * 32, 0, s.stream>>>(s.pos.b[s.pc], ref, s.rbk, s.cstart,
                                                                           s.nbn, s.nbl, s.status_dev, a, nb, la);
}

// A list build's status, read back: the locals outside the grid get empty lists, the two-phase
// chain and image-map state of the links; 0 when the lists stand, 1 when the capacity was short
// (grown: the build is to be redone).
static int finish_build(State& s, bool half) {
    const Geometry& g = s.geo;
    if (s.status_host->out_local > 0) {
        int first_out = 0;
        // locals outside the grid sit at [cstart[ncells], N): empty lists
        TMD_CUDA(cudaMemcpyAsync(&first_out, s.cstart + g.ncells, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
        TMD_CUDA(cudaStreamSynchronize(s.stream));
        k_clear_lists<<<nblocks(s.N - first_out, 256), 256, 0, s.stream>>>(s.nbn, first_out, s.N);
        launched(K_NLIST);
        set_error(5, "locals outside the cell grid at binning (they have no neighbours)");
    }
    s.nchain = s.status_host->nchain;
    s.img_ok = (s.status_host->img_over1 == 0 ? 1 : 0) | (s.status_host->img_over2 == 0 ? 2 : 0);
    const int mx = s.status_host->max_nb;
    if (mx <= s.nb_cap) {
        s.lists_valid = 1;
        s.lists_half = half;
        return 0;
    }
    // core/neighborlist.impala:74-76: grow to twice the overflow and redo
    std::printf("0> reallocate_neighborlist_capacity(): %d\n", mx * 2);
    grow_lists(s, mx * 2);
    return 1;
}

int run_build_lists(State& s, bool half, double cutoff, bool defer) {
    const Geometry& g = s.geo;
    s.lists_cutoff = cutoff;
    s.status_pending = false;
    if (s.N == 0) {
        s.lists_valid = 1;
        s.lists_half = half;
        return 0;
    }
    // the half lists that keep boundary pairs read the ghosts' root references, which the
    // links write: they run first, alone
    if (half && s.half_ghost) flush_links(s);
    NlArgs a;
    a.cut2 = cutoff * cutoff;
    const double margin = 1e-3 * a.cut2 + 1e-6;
    a.lo2 = (float)(a.cut2 - margin);
    a.hi2 = (float)(a.cut2 + margin);
    a.N = s.N;
    a.ncells = g.ncells;
    a.nx = g.nx;
    a.nxy = g.nx * g.ny;
    a.stride = s.nb_stride;
    for (int d = 0; d < 3; ++d) a.alo[d] = g.aabb_lo[d];
    a.spacing = g.spacing;
    const int nb = nblocks(g.ncells, kNlWarps);
    for (int attempt = 0; attempt < 8; ++attempt) {
        a.nbcap = s.nb_cap;
        if (attempt > 0 || !s.build_zeroed)  // else zeroed by the binning's reorder kernel
            TMD_CUDA(cudaMemsetAsync(&s.status_dev->max_nb, 0, sizeof(int), s.stream));
        s.build_zeroed = false;
        prof_begin(K_NLIST);
        // the pending ghost links ride along as extra blocks (once: they count with atomics)
        const LinkArgs la = link_args(s);
        const int lb = s.pend_links ? nblocks(s.G, kNlWarps * 32) : 0;
        s.pend_links = false;
        const bool wide = (size_t)s.nb_cap * s.nb_stride > 0xffffffffull;  // list index beyond 32 bits
        if (half && s.half_ghost)
            launch_build_list<2>(s, wide, nb + lb, s.rref, a, nb, la);
        else if (half)
            launch_build_list<1>(s, wide, nb + lb, s.ref.b[s.ac], a, nb, la);
        else
            launch_build_list<0>(s, wide, nb + lb, s.ref.b[s.ac], a, nb, la);
        launched(K_NLIST);
        prof_end(K_NLIST);
        TMD_CUDA(cudaMemcpyAsync(s.status_host, s.status_dev, sizeof(DevStatus), cudaMemcpyDeviceToHost, s.stream));
        if (defer && attempt == 0) {
            // the host goes on; the next force kernel is launched on these lists at once and
            // resolve_lists reads the status while it runs
            TMD_CUDA(cudaEventRecord(s.ev_status, s.stream));
            s.status_pending = true;
            s.status_half = half;
            s.lists_valid = 0;
            return 0;
        }
        TMD_CUDA(cudaStreamSynchronize(s.stream));
        if (finish_build(s, half) == 0) return 0;
    }
    set_error(2, "neighbour list capacity did not converge");
    return -1;
}

int resolve_lists(State& s) {
    if (!s.status_pending) return 0;
    s.status_pending = false;
    TMD_CUDA(cudaEventSynchronize(s.ev_status));
    const bool outside = s.status_host->out_local > 0;
    if (finish_build(s, s.status_half) == 0) return outside ? 1 : 0;
    // the capacity was short: the build again, on the grown lists
    return run_build_lists(s, s.status_half, s.lists_cutoff) == 0 ? 1 : -1;
}

}  // namespace tmd
