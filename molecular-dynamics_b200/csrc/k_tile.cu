// k_tile.cu -- tiled full neighbour lists and the staged mixed LJ force kernel.
//
// Row blocks.  Locals are sorted by flat cell index (x fastest), so the locals
// of one (y, z) row of the cell grid are contiguous slots.  Each row's locals
// are split into blocks of at most 128 consecutive slots ("homes").  The
// candidates of a block's homes -- the 3 x 3 rows around its row, over the
// home cells widened by one cell on each side -- are 18 contiguous slot
// ranges: locals and ghosts of 9 row runs (ghosts are sorted by cell too, in
// their own slot range).  Their concatenation is the block's halo; keeping a
// block inside one row bounds the halo by 9 runs of (home cells + 2) cells.
//
// k_row_blocks / k_block_desc: per-row block counts, then one descriptor per
// block (its homes, runs and ranges), once per list build.
//
// k_build_tiles: one thread per home.  The halo's positions are staged in
// shared memory relative to the block's first home cell; each thread walks
// its own 27 stencil cells in the reference order (core/neighborlist.impala:
// 1-78: z, y, x offsets, the cell's locals then its ghosts), prefilters in
// FP32 and takes the exact FP64 membership test near the cutoff, recording the
// halo index of each hit in shared memory.  A second pass writes the plain
// list (slot << 6 | code, read by the FP64, half, DEM and adjoint kernels) and
// the tiled list (16-bit halo indices, four per 8 bytes), row by row of the
// atom-fastest layout so a warp's stores are coalesced.  Entry order is the
// reference's, so both lists equal the ones k_build_list writes.
//
// k_lj_tile_mixed: stages the halo's rebased FP32 positions in shared memory
// (16 bytes per atom, a plain copy: pos32.w carries the rebasing cell) and
// runs the pair loop against it, reading two bytes of list per neighbour.
// The pair arithmetic and the FP64 fallback are those of the plain-list mixed
// kernel (k_lj_mixed_bf); the summation order differs, so the forces agree with
// it to FP32 rounding.

#include <algorithm>
#include <cmath>
#include <cstdio>

#include "lj_args.cuh"
#include "md_common.cuh"
#include "md_state.h"

namespace tmd {

namespace {

constexpr int kBlockHomes = 128;   // homes (= threads) per block at most
constexpr int kBlockCells = 8;     // home cells per block the split aims at (bounds sparse rows' halos)
constexpr int kRunCellsMax = 64;   // cells per row run (home cells + 2) at most
constexpr int kRanges = 18;        // 9 runs x (locals, ghosts)
constexpr int kThermoQ = 4;
constexpr int kDescThreads = 32;

struct TileGeo {
    int nx, ny, nz, ncells, nrows;
};

struct BlockDesc {
    int h0, h1;            // home slots [h0, h1); h0 == h1 for an unused block
    int xa, ncell, u0;     // x of the runs' first cell, cells per run, run cell of the first home cell
    int y, z;              // the row
    int cfirst[9];         // flat index of run r's first cell, -1 when the run lies outside the grid
    int start[kRanges];    // first slot of range q = 2 r + {0 locals, 1 ghosts}
    int base[kRanges + 1]; // halo index of range q's first member; base[kRanges] = halo size
};
constexpr int kDescInts = (int)((sizeof(BlockDesc) + sizeof(int) - 1) / sizeof(int));

// ---- block table ------------------------------------------------------------------
// One thread per row: in-grid locals of the row and the number of blocks they
// take: ceil(homes / 128), more when the homes span more than kBlockCells cells
// (a sparse row -- e.g. in the partly filled last plane -- would otherwise give
// one block a halo of many dense neighbour cells).
__global__ void k_row_blocks(const int* __restrict__ cstart, int* __restrict__ rowblocks, TileGeo g) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= g.nrows) return;
    const int rc = row * g.nx;
    const int h = cstart[rc + g.nx] - cstart[rc];
    int nb = 0;
    if (h > 0) {
        int xlo = 0, xhi = g.nx - 1;
        while (cstart[rc + xlo + 1] == cstart[rc]) ++xlo;      // first cell holding a local
        while (cstart[rc + xhi] == cstart[rc + g.nx]) --xhi;   // last one
        const int span = xhi - xlo + 1;
        nb = max((h + kBlockHomes - 1) / kBlockHomes, (span + kBlockCells - 1) / kBlockCells);
        nb = min(nb, h);
    }
    rowblocks[row] = nb;
}

// Descriptor of block blockIdx.x (one warp per block).  rowoff = exclusive scan of the
// per-row block counts (rowoff[nrows] = total); block k of a row with h homes takes
// homes [k h / nb, (k + 1) h / nb) of the row.
__global__ void __launch_bounds__(kDescThreads)
k_block_desc(const int* __restrict__ cstart, const int* __restrict__ rowoff, const int* __restrict__ slot_cell,
             int* __restrict__ desc, DevStatus* st, TileGeo g) {
    __shared__ BlockDesc d;
    const int b = blockIdx.x;
    // more blocks than descriptors launched (cannot happen within the bound): no tiled lists
    if (b == 0 && threadIdx.x == 0 && rowoff[g.nrows] > (int)gridDim.x) atomicAdd(&st->tile_overflow, 1);
    if (threadIdx.x == 0) {
        d.h0 = d.h1 = 0;
        d.xa = d.ncell = d.u0 = d.y = d.z = 0;
        for (int q = 0; q <= kRanges; ++q) d.base[q] = 0;
        if (b < rowoff[g.nrows]) {
            int lo = 0, hi = g.nrows - 1;  // row with rowoff[row] <= b < rowoff[row + 1]
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (rowoff[mid] <= b) lo = mid;
                else hi = mid - 1;
            }
            const int row = lo, k = b - rowoff[row], nb = rowoff[row + 1] - rowoff[row];
            const int rc = row * g.nx;
            const int r0 = cstart[rc], h = cstart[rc + g.nx] - r0;
            d.h0 = r0 + (int)((long long)k * h / nb);
            d.h1 = r0 + (int)((long long)(k + 1) * h / nb);
            const int xlo = slot_cell[d.h0] - rc, xhi = slot_cell[d.h1 - 1] - rc;
            d.xa = max(xlo - 1, 0);
            d.ncell = min(xhi + 2, g.nx) - d.xa;
            d.u0 = xlo - d.xa;
            d.y = row % g.ny;
            d.z = row / g.ny;
            if (d.ncell > kRunCellsMax) {  // homes spread over too many cells: no tiled lists
                atomicAdd(&st->tile_overflow, 1);
                d.h1 = d.h0;
            }
        }
    }
    __syncwarp();
    const int G0 = g.ncells + 1;  // ghost segments of cstart
    if (threadIdx.x < 9 && d.h1 > d.h0) {
        const int r = threadIdx.x;
        const int yy = d.y + (r % 3) - 1, zz = d.z + (r / 3) - 1;
        int ls = 0, ll = 0, gs = 0, gl = 0, cf = -1;
        if (yy >= 0 && yy < g.ny && zz >= 0 && zz < g.nz) {
            cf = (zz * g.ny + yy) * g.nx + d.xa;
            ls = cstart[cf];
            ll = cstart[cf + d.ncell] - ls;
            gs = cstart[G0 + cf];
            gl = cstart[G0 + cf + d.ncell] - gs;
        }
        d.cfirst[r] = cf;
        d.start[2 * r] = ls;
        d.start[2 * r + 1] = gs;
        d.base[2 * r] = ll;  // lengths, scanned below
        d.base[2 * r + 1] = gl;
    }
    __syncwarp();
    if (threadIdx.x == 0 && d.h1 > d.h0) {
        int acc = 0;
        for (int q = 0; q < kRanges; ++q) {
            const int l = d.base[q];
            d.base[q] = acc;
            acc += l;
        }
        d.base[kRanges] = acc;
    }
    __syncwarp();
    const int* src = reinterpret_cast<const int*>(&d);
    for (int q = threadIdx.x; q < kDescInts; q += blockDim.x) desc[(size_t)b * kDescInts + q] = src[q];
}

// the calling block's descriptor into shared memory; ends with a barrier
__device__ __forceinline__ void load_desc(BlockDesc& d, const int* __restrict__ desc) {
    int* dst = reinterpret_cast<int*>(&d);
    for (int k = threadIdx.x; k < kDescInts; k += blockDim.x) dst[k] = __ldg(desc + (size_t)blockIdx.x * kDescInts + k);
    __syncthreads();
}

// halo index of home slot i: homes lie in the locals range of the centre run (r = 4)
__device__ __forceinline__ int home_hid(const BlockDesc& d, int i) { return d.base[8] + (i - d.start[8]); }

// slot of halo index m
__device__ __forceinline__ int halo_slot(const BlockDesc& d, int m) {
    int lo = 0, hi = kRanges - 1;
    while (lo < hi) {  // last range whose base is <= m (empty ranges share the next one's base)
        const int mid = (lo + hi + 1) >> 1;
        if (d.base[mid] <= m) lo = mid;
        else hi = mid - 1;
    }
    return d.start[lo] + (m - d.base[lo]);
}

__device__ __forceinline__ void put_partial(double* part, int q, double v, double* scratch) {
    const double r = block_sum(v, scratch);
    if (threadIdx.x == 0) part[q * gridDim.x + blockIdx.x] = r;
}

struct TileListArgs {
    double cut2;     // list cutoff^2 (FP64, the reference's membership test)
    float lo2, hi2;  // FP32 prefilter: certainly inside below lo2, certainly outside above hi2
    int nbcap, stride;
    double alo[3], spacing;
};

constexpr int kWarps = kBlockHomes / 32;

// exclusive prefix sum over the warp; *total = warp sum
__device__ __forceinline__ int warp_exscan(int v, int* total) {
    const int lane = threadIdx.x & 31;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    *total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

// ---- tiled list build ---------------------------------------------------------
// Warp w of a block owns homes [h0 + 32 w, h0 + 32 w + 32).  The warp walks the union of its
// homes' stencil cells -- for each of the 9 runs in order, the cells from its lowest home cell
// - 1 to its highest + 1 in increasing x, each cell's locals then ghosts -- broadcasting every
// candidate to all lanes; a lane takes the candidates of the three cells around its own (the
// same run cells in the same order as its reference stencil), so its hits come out in the
// reference order.  Hits are recorded as halo indices in shared memory; a second pass writes
// the plain list and the warp's stream: its homes' halo-index lists concatenated home-major
// (uint16, region [gw][32 nbcap] for global warp gw), stored so a warp writes and later reads
// 32 consecutive entries at a time.
//
// Dynamic shared memory: float4 s_rel[cap] (position relative to the block's first home cell
// centre, w = packed rebasing cell), int s_slot[cap], uint16 s_hit[nbcap][kBlockHomes].  A
// block whose halo exceeds `cap` only reports its size (halo_max); the host rebuilds with a
// larger cap.
__global__ void __launch_bounds__(kBlockHomes)
k_build_tiles(const double4* __restrict__ pos, const int* __restrict__ rbk, const int* __restrict__ cstart,
              const int* __restrict__ desc, int* __restrict__ nbn, uint32_t* __restrict__ nbl,
              uint16_t* __restrict__ stream, DevStatus* st, TileGeo g, TileListArgs a, int cap) {
    __shared__ BlockDesc d;
    __shared__ int s_lc[9][kRunCellsMax + 1];  // halo index of the first local of run r's cell u
    __shared__ int s_gc[9][kRunCellsMax + 1];  // ... of the first ghost
    __shared__ int s_off[kWarps][33];          // per warp: exclusive offsets of its homes' lists
    extern __shared__ float4 s_dyn[];
    float4* s_rel = s_dyn;
    int* s_slot = reinterpret_cast<int*>(s_dyn + cap);
    uint16_t* s_hit = reinterpret_cast<uint16_t*>(s_slot + cap);

    load_desc(d, desc);
    const int M = d.base[kRanges];
    if (d.h1 <= d.h0) return;
    if (threadIdx.x == 0) atomicMax(&st->halo_max, M);
    if (M > cap) return;
    const double ctr[3] = {a.alo[0] + ((double)(d.xa + d.u0) + 0.5) * a.spacing,
                           a.alo[1] + ((double)d.y + 0.5) * a.spacing, a.alo[2] + ((double)d.z + 0.5) * a.spacing};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = warp; q < kRanges; q += kWarps) {
        const int len = d.base[q + 1] - d.base[q], s0 = d.start[q], b = d.base[q];
        for (int x = lane; x < len; x += 32) {
            const double4 p = pos[s0 + x];
            s_rel[b + x] = make_float4((float)(p.x - ctr[0]), (float)(p.y - ctr[1]), (float)(p.z - ctr[2]),
                                       __int_as_float(rbk[s0 + x]));
            s_slot[b + x] = s0 + x;
        }
    }
    const int G0 = g.ncells + 1;
    for (int v = threadIdx.x; v < 9 * (kRunCellsMax + 1); v += blockDim.x) {
        const int r = v / (kRunCellsMax + 1), u = v % (kRunCellsMax + 1);
        int lc = 0, gc = 0;
        if (d.cfirst[r] >= 0 && u <= d.ncell) {
            lc = d.base[2 * r] + __ldg(cstart + d.cfirst[r] + u) - d.start[2 * r];
            gc = d.base[2 * r + 1] + __ldg(cstart + G0 + d.cfirst[r] + u) - d.start[2 * r + 1];
        }
        s_lc[r][u] = lc;
        s_gc[r][u] = gc;
    }
    __syncthreads();

    const int i = d.h0 + threadIdx.x;
    const bool home = i < d.h1;
    int hid = -1, u = 0;
    float4 own = make_float4(0.f, 0.f, 0.f, 0.f);
    double4 pi = make_double4(0.0, 0.0, 0.0, 0.0);
    if (home) {
        hid = home_hid(d, i);
        u = d.u0;  // the home's cell within the runs
        while (s_lc[4][u + 1] <= hid) ++u;
        own = s_rel[hid];
        pi = pos[i];
    }
    int ulo = home ? u : (1 << 30), uhi = home ? u : -1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ulo = min(ulo, __shfl_xor_sync(0xffffffffu, ulo, o));
        uhi = max(uhi, __shfl_xor_sync(0xffffffffu, uhi, o));
    }
    int cnt = 0;
    // pass 1 (warp-uniform loops): halo indices of the members, in the reference order
    if (uhi >= 0) {
        for (int r = 0; r < 9; ++r) {  // r = 3 (oz + 1) + (oy + 1)
            if (d.cfirst[r] < 0) continue;
            const int ua = max(ulo - 1, 0), ub = min(uhi + 1, d.ncell - 1);
            for (int uu = ua; uu <= ub; ++uu) {
                const bool win = home && uu >= u - 1 && uu <= u + 1;
#pragma unroll
                for (int part = 0; part < 2; ++part) {  // the cell's locals, then its ghosts
                    const int m0 = part ? s_gc[r][uu] : s_lc[r][uu];
                    const int m1 = part ? s_gc[r][uu + 1] : s_lc[r][uu + 1];
                    for (int m = m0; m < m1; ++m) {
                        const float4 cp = s_rel[m];
                        const float dx = own.x - cp.x, dy = own.y - cp.y, dz = own.z - cp.z;
                        const float r2 = dx * dx + dy * dy + dz * dz;
                        bool in = win && r2 < a.lo2;
                        if (win && !in && r2 <= a.hi2) {
                            // near the cutoff: the reference's exact FP64 test
                            const double4 pj = pos[s_slot[m]];
                            in = len2_strict(dsub(pi.x, pj.x), dsub(pi.y, pj.y), dsub(pi.z, pj.z)) <= a.cut2;
                        }
                        if (in && m != hid) {
                            if (cnt < a.nbcap) s_hit[cnt * kBlockHomes + threadIdx.x] = (uint16_t)m;
                            ++cnt;
                        }
                    }
                }
            }
        }
    }
    // pass 2: the plain list, one row of the atom-fastest layout per iteration
    const int n = min(cnt, a.nbcap);
    bool wrapped = false;
    if (home) {
        const int irbk = __float_as_int(own.w);
        for (int k = 0; k < n; ++k) {
            const int m = s_hit[k * kBlockHomes + threadIdx.x];
            const int cr = __float_as_int(s_rel[m].w);
            int dk[3];
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                const int raw = unpack_axis(cr, ax) - unpack_axis(irbk, ax);
                dk[ax] = wrap_diff(unpack_axis(cr, ax), unpack_axis(irbk, ax));
                wrapped |= raw < -1 || raw > 1;  // the staged kernel decodes unwrapped fields
            }
            if (dk[0] < -1 || dk[0] > 1 || dk[1] < -1 || dk[1] > 1 || dk[2] < -1 || dk[2] > 1) {
                atomicAdd(&st->bad_code, 1);
                dk[0] = dk[1] = dk[2] = 0;
            }
            const uint32_t code = (uint32_t)((dk[0] + 1) | ((dk[1] + 1) << 2) | ((dk[2] + 1) << 4));
            nbl[(size_t)k * a.stride + i] = ((uint32_t)s_slot[m] << kCodeBits) | code;
        }
        nbn[i] = cnt;
    }
    // the warp's stream: position p of the home-major concatenation, 32 positions per step
    int P;
    const int off = warp_exscan(n, &P);
    s_off[warp][lane] = off;
    if (lane == 31) s_off[warp][32] = P;
    __syncwarp();
    uint16_t* ws = stream + (size_t)(blockIdx.x * kWarps + warp) * (32 * (size_t)a.nbcap);
    int t = 0;
    for (int p0 = 0; p0 < P; p0 += 32) {
        const int p = p0 + lane;
        if (p < P) {
            while (s_off[warp][t + 1] <= p) ++t;
            ws[p] = s_hit[(p - s_off[warp][t]) * kBlockHomes + warp * 32 + t];
        }
    }
    if (__any_sync(0xffffffffu, wrapped) && lane == 0) atomicAdd(&st->tile_overflow, 1);
    const int maxcnt = warp_max(cnt);
    if (lane == 0 && maxcnt > 0) atomicMax(&st->max_nb, maxcnt);
}

// ---- staged mixed LJ ----------------------------------------------------------
// Shared memory holds pos32 of the halo: the FP32 offset from the centre of
// the atom's rebasing cell, and in w that cell packed 10 bits per axis.  For a
// list pair the fields differ by dk in {-1, 0, 1} (the builder checks that no
// field wraps), so w_j - w_i + 0x00100401 holds dk + 1 in bits 0-1 (x), 10-11
// (y) and 20-21 (z) without borrows, and dk * (-rb_h) is built exactly as in
// k_lj_mixed_bf: an integer OR into the float 2^23, one subtraction, and a scale
// (-rb_h, -rb_h / 2^10, -rb_h / 2^20: exact for rb_h a multiple of 1/8).  The
// pair arithmetic and the FP64 fallback are k_lj_mixed_bf's.
//
// Work distribution: a warp walks its stream 32 consecutive positions at a
// time (lane l takes position p0 + l), so every lane has a pair in every step
// whatever the list lengths.  A lane keeps running sums for the home T that
// the warp's running sums belong to; in a step where the homes change, the
// warp sums the finished home's lane sums with a fixed butterfly and lane 0
// stores them, so the result is deterministic.  FP64 contributions (close
// pairs, pairs at the cutoff) are rare: they live in separate running sums
// that are only reduced when some lane has one.
__device__ __forceinline__ float warp_fsum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_dsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

constexpr int kGroup = 4;  // stream steps whose entries are in flight together

// One step of a warp's stream walk: lane `lane` takes position p0 + lane (halo index m).
template <bool THERMO>
__device__ __forceinline__ void stream_step(int p0, int m, int lane, int warp, int hw, int P, const BlockDesc& d,
                                            const LjArgs& a, const float4* s_p, const int (*s_off)[33],
                                            float (*s_f32)[32][3], double (*s_f64)[32][3],
                                            const double4* __restrict__ pos, int& t, int& T, int& tj, float4& ri,
                                            int& wi, float& ax, float& ay, float& az, double& bx, double& by,
                                            double& bz, bool& any64, float& ef, float& wf, double& e, double& w,
                                            int& ncnt) {
    const int p = p0 + lane;
    const bool act = p < P;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    bool d64 = false;
    double cx = 0.0, cy = 0.0, cz = 0.0;
    if (act) {
        while (s_off[warp][t + 1] <= p) ++t;
        if (t != tj) {
            tj = t;
            ri = s_p[home_hid(d, hw + t)];
            wi = __float_as_int(ri.w);
        }
        const float4 rj = s_p[m];
        const uint32_t dd = (uint32_t)(__float_as_int(rj.w) - wi + 0x00100401);
        const float sx = __int_as_float((int)((dd & 0x3u) | 0x4B000000u)) - 8388609.0f;
        const float sy = __int_as_float((int)((dd & 0xC00u) | 0x4B000000u)) - 8389632.0f;
        const float sz = __int_as_float((int)((dd & 0x300000u) | 0x4B000000u)) - 9437184.0f;
        const float dx = fmaf(a.hx, sx, ri.x - rj.x);
        const float dy = fmaf(a.hy, sy, ri.y - rj.y);
        const float dz = fmaf(a.hz, sz, ri.z - rj.z);
        const float rsq = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        if (rsq < a.rc2_hi) {
            if (rsq < a.rc2_lo && rsq >= a.close2) {
                float sr2;  // hardware reciprocal, as in k_lj_mixed_bf
                asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(sr2) : "f"(rsq));
                const float sr6 = sr2 * sr2 * sr2 * a.sig6f;
                const float f = a.eps48f * sr6 * (sr6 - 0.5f) * sr2;
                fx = dx * f;
                fy = dy * f;
                fz = dz * f;
                if (THERMO) {
                    ef += a.eps4f * sr6 * (sr6 - 1.0f);
                    wf += f * rsq;
                    ncnt++;
                }
            } else {
                // FP64 path: exact cutoff decision and close-contact accuracy
                const double4 pi = pos[hw + t];
                const double4 pj = pos[halo_slot(d, m)];
                const double ex = dsub(pi.x, pj.x), ey = dsub(pi.y, pj.y), ez = dsub(pi.z, pj.z);
                const double r2 = len2_strict(ex, ey, ez);
                if (r2 < a.rc2) {
                    const double sr2 = 1.0 / r2;
                    const double sr6 = sr2 * sr2 * sr2 * a.sigma6;
                    const double f = 48.0 * sr6 * (sr6 - 0.5) * sr2 * a.eps;
                    cx = ex * f;
                    cy = ey * f;
                    cz = ez * f;
                    d64 = true;
                    if (THERMO) {
                        e += 4.0 * a.eps * sr6 * (sr6 - 1.0);
                        w += f * r2;
                        ncnt++;
                    }
                }
            }
        }
    }
    // positions rise with the lane, so the last active lane holds the step's highest home
    const int tmax = __shfl_sync(0xffffffffu, t, min(31, P - p0 - 1));
    if (tmax == T) {  // every active lane is still on home T
        ax += fx;
        ay += fy;
        az += fz;
        if (d64) {
            bx += cx;
            by += cy;
            bz += cz;
            any64 = true;
        }
        return;
    }
    // home T ends in this step
    {
        const bool on = act && t == T;
        const float vx = warp_fsum(ax + (on ? fx : 0.f));
        const float vy = warp_fsum(ay + (on ? fy : 0.f));
        const float vz = warp_fsum(az + (on ? fz : 0.f));
        if (lane == 0) {
            s_f32[warp][T][0] = vx;
            s_f32[warp][T][1] = vy;
            s_f32[warp][T][2] = vz;
        }
        const bool h64 = any64 || (on && d64);
        if (__any_sync(0xffffffffu, h64)) {
            const double ux = warp_dsum(bx + (on && d64 ? cx : 0.0));
            const double uy = warp_dsum(by + (on && d64 ? cy : 0.0));
            const double uz = warp_dsum(bz + (on && d64 ? cz : 0.0));
            if (lane == 0) {
                s_f64[warp][T][0] = ux;
                s_f64[warp][T][1] = uy;
                s_f64[warp][T][2] = uz;
            }
        }
    }
    // homes that begin and end inside this step (lists shorter than a step)
    for (int h = T + 1; h < tmax; ++h) {
        const bool on = act && t == h;
        const float vx = warp_fsum(on ? fx : 0.f);
        const float vy = warp_fsum(on ? fy : 0.f);
        const float vz = warp_fsum(on ? fz : 0.f);
        if (lane == 0) {
            s_f32[warp][h][0] = vx;
            s_f32[warp][h][1] = vy;
            s_f32[warp][h][2] = vz;
        }
        if (__any_sync(0xffffffffu, on && d64)) {
            const double ux = warp_dsum(on && d64 ? cx : 0.0);
            const double uy = warp_dsum(on && d64 ? cy : 0.0);
            const double uz = warp_dsum(on && d64 ? cz : 0.0);
            if (lane == 0) {
                s_f64[warp][h][0] = ux;
                s_f64[warp][h][1] = uy;
                s_f64[warp][h][2] = uz;
            }
        }
    }
    // home tmax continues into the next step
    const bool on = act && t == tmax;
    ax = on ? fx : 0.f;
    ay = on ? fy : 0.f;
    az = on ? fz : 0.f;
    any64 = on && d64;
    bx = any64 ? cx : 0.0;
    by = any64 ? cy : 0.0;
    bz = any64 ? cz : 0.0;
    T = tmax;
}

template <bool FUSE, bool THERMO>
__global__ void __launch_bounds__(kBlockHomes)
k_lj_tile_mixed(const float4* __restrict__ pos32, const double4* __restrict__ pos, float4* __restrict__ frc32,
                double4* __restrict__ vel, const int* __restrict__ nbn, const uint16_t* __restrict__ stream,
                const int* __restrict__ desc, double* __restrict__ part, LjArgs a) {
    __shared__ BlockDesc d;
    __shared__ double scratch[kWarps];
    __shared__ int s_off[kWarps][33];
    __shared__ float s_f32[kWarps][32][3];   // per home: FP32 force sum
    __shared__ double s_f64[kWarps][32][3];  // per home: FP64 force sum
    extern __shared__ float4 s_p[];
    load_desc(d, desc);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int hw = d.h0 + warp * 32;  // the warp's first home slot
    const int i = hw + lane;
    const bool home = i < d.h1;
    const int n = home ? min(nbn[i], a.nbcap) : 0;
    int P;
    const int off = warp_exscan(n, &P);
    s_off[warp][lane] = off;
    if (lane == 31) s_off[warp][32] = P;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        s_f32[warp][lane][c] = 0.f;
        s_f64[warp][lane][c] = 0.0;
    }
    const uint16_t* ws = stream + (size_t)(blockIdx.x * kWarps + warp) * (32 * (size_t)a.nbcap);
    if (lane == 0 && P > 0) {  // the warp's stream into L2 (16-byte aligned, whole 16-byte units)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(ws), "r"(((P * 2 + 15) / 16) * 16)
                     : "memory");
    }
    for (int q = warp; q < kRanges; q += kWarps) {
        const int len = d.base[q + 1] - d.base[q], s0 = d.start[q], b = d.base[q];
        for (int x = lane; x < len; x += 32) s_p[b + x] = pos32[s0 + x];
    }
    __syncthreads();

    double e = 0.0, w = 0.0, cnt = 0.0, ke = 0.0;
    float ef = 0.f, wf = 0.f;
    int ncnt = 0;
    int t = 0;  // home of this lane's current position
    while (t < 31 && s_off[warp][t + 1] <= lane) ++t;
    int T = __shfl_sync(0xffffffffu, t, 0);  // home of the warp's running sums
    float ax = 0.f, ay = 0.f, az = 0.f;       // this lane's share of home T, FP32
    double bx = 0.0, by = 0.0, bz = 0.0;      // ... FP64
    bool any64 = false;
    int tj = -1;  // home whose position the lane holds
    float4 ri = make_float4(0.f, 0.f, 0.f, 0.f);
    int wi = 0;
    // entries of kGroup steps are loaded while the previous group is processed
    int mb[kGroup], mn[kGroup];
#pragma unroll
    for (int u = 0; u < kGroup; ++u) {
        const int pp = u * 32 + lane;
        mb[u] = pp < P ? (int)ws[pp] : 0;
    }
    for (int g0 = 0; g0 < P; g0 += 32 * kGroup) {
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
            const int pp = g0 + (kGroup + u) * 32 + lane;
            mn[u] = pp < P ? (int)ws[pp] : 0;
        }
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
            const int p0 = g0 + u * 32;
            if (p0 < P)
                stream_step<THERMO>(p0, mb[u], lane, warp, hw, P, d, a, s_p, s_off, s_f32, s_f64, pos, t, T, tj, ri,
                                    wi, ax, ay, az, bx, by, bz, any64, ef, wf, e, w, ncnt);
        }
#pragma unroll
        for (int u = 0; u < kGroup; ++u) mb[u] = mn[u];
    }
    // the last home of the stream
    if (P > 0) {
        const float vx = warp_fsum(ax), vy = warp_fsum(ay), vz = warp_fsum(az);
        if (lane == 0) {
            s_f32[warp][T][0] = vx;
            s_f32[warp][T][1] = vy;
            s_f32[warp][T][2] = vz;
        }
        if (__any_sync(0xffffffffu, any64)) {
            const double ux = warp_dsum(bx), uy = warp_dsum(by), uz = warp_dsum(bz);
            if (lane == 0) {
                s_f64[warp][T][0] = ux;
                s_f64[warp][T][1] = uy;
                s_f64[warp][T][2] = uz;
            }
        }
    }
    __syncwarp();
    if (home) {
        const double Fx = (double)s_f32[warp][lane][0] + s_f64[warp][lane][0];
        const double Fy = (double)s_f32[warp][lane][1] + s_f64[warp][lane][1];
        const double Fz = (double)s_f32[warp][lane][2] + s_f64[warp][lane][2];
        const float4 F = make_float4((float)Fx, (float)Fy, (float)Fz, 0.f);
        frc32[i] = F;
        if (FUSE) {
            double4 v = vel[i];
            v.x += (double)F.x * a.h;
            v.y += (double)F.y * a.h;
            v.z += (double)F.z * a.h;
            vel[i] = v;
            if (THERMO) ke = v.x * v.x + v.y * v.y + v.z * v.z;
        }
    }
    if (THERMO) {
        e += (double)ef;
        w += (double)wf;
        cnt = (double)ncnt;
        put_partial(part, 0, e, scratch);
        put_partial(part, 1, w, scratch);
        put_partial(part, 2, cnt, scratch);
        if (FUSE) put_partial(part, 3, ke, scratch);
    }
}

TileGeo tile_geo(const State& s) {
    TileGeo t;
    t.nx = s.geo.nx;
    t.ny = s.geo.ny;
    t.nz = s.geo.nz;
    t.ncells = s.geo.ncells;
    t.nrows = s.geo.ny * s.geo.nz;
    return t;
}

size_t build_smem(const State& s, int cap) {
    return (sizeof(float4) + sizeof(int)) * (size_t)cap + sizeof(uint16_t) * (size_t)s.nb_cap * kBlockHomes;
}

constexpr size_t kSmemLimit = 200 * 1024;  // dynamic shared memory a tiled launch may request

}  // namespace

bool tiles_usable(const State& s) {
    // the flat 27-cell stencil only reaches cells of other rows across the grid
    // edge, and those are at least one cell spacing away, when every axis has
    // three cells or more
    return s.tile_mode != 0 && s.geo.nx >= 3 && s.geo.ny >= 3 && s.geo.nz >= 3 &&
           build_smem(s, s.tile_cap) <= kSmemLimit;
}

bool tile_cap_fits(const State& s, int cap) { return build_smem(s, cap) <= kSmemLimit; }

// Upper bound on the number of row blocks: each row takes at most
// ceil(h / 128) + ceil(span / kBlockCells) blocks.
int tile_block_bound(const State& s) {
    const int nrows = s.geo.ny * s.geo.nz;
    return s.N / kBlockHomes + 2 * nrows + (int)(((long long)nrows * s.geo.nx) / kBlockCells) + 2;
}

int run_build_tiles(State& s, double cutoff) {
    if (!tiles_usable(s)) return 0;
    const TileGeo g = tile_geo(s);
    const int bound = tile_block_bound(s);
    if (bound > s.tile_desc_blocks) {
        dfree(&s.tile_desc);
        dalloc(&s.tile_desc, (size_t)bound * kDescInts);
        dfree(&s.tile_rows);
        dalloc(&s.tile_rows, (size_t)2 * (g.nrows + 1));
        s.tile_desc_blocks = bound;
    }
    // streams: per warp of every block, 32 lists of up to nb_cap halo indices
    const size_t stream_len = (size_t)bound * kBlockHomes * s.nb_cap;
    if (stream_len > s.tile_stream_len) {
        dfree(&s.tile_stream);
        dalloc(&s.tile_stream, stream_len);
        s.tile_stream_len = stream_len;
    }
    int* rowblocks = s.tile_rows;
    int* rowoff = s.tile_rows + (g.nrows + 1);
    k_row_blocks<<<(g.nrows + 127) / 128, 128, 0, s.stream>>>(s.cstart, rowblocks, g);
    launched(K_NLIST);
    exclusive_scan(s, rowblocks, rowoff, g.nrows);
    TMD_CUDA(cudaMemcpyAsync(&s.status_dev->tile_blocks, rowoff + g.nrows, sizeof(int), cudaMemcpyDeviceToDevice,
                             s.stream));
    k_block_desc<<<bound, kDescThreads, 0, s.stream>>>(s.cstart, rowoff, s.slot_cell, s.tile_desc, s.status_dev, g);
    launched(K_NLIST);
    TileListArgs a;
    a.cut2 = cutoff * cutoff;
    const double margin = 1e-3 * a.cut2 + 1e-6;
    a.lo2 = (float)(a.cut2 - margin);
    a.hi2 = (float)(a.cut2 + margin);
    a.nbcap = s.nb_cap;
    a.stride = s.nb_stride;
    for (int d = 0; d < 3; ++d) a.alo[d] = s.geo.aabb_lo[d];
    a.spacing = s.geo.spacing;
    const size_t smem = build_smem(s, s.tile_cap);
    TMD_CUDA(cudaFuncSetAttribute(k_build_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_build_tiles<<<bound, kBlockHomes, smem, s.stream>>>(s.pos.b[s.pc], s.rbk, s.cstart, s.tile_desc, s.nbn, s.nbl,
                                                         s.tile_stream, s.status_dev, g, a, s.tile_cap);
    return 1;  // the caller counts this launch and reads the status (block count included)
}

void run_force_lj_tiles(State& s, const PendingForce& p, bool fuse_final, double dt) {
    LjArgs a = lj_args(s, p, dt);
    a.hx = (float)(-s.geo.rb_h);
    a.hy = (float)(-s.geo.rb_h / 1024.0);
    a.hz = (float)(-s.geo.rb_h / 1048576.0);
    const int nb = std::max(s.tile_blocks, 1);
    const bool thermo = s.thermo != 0;
    if (thermo) ensure_red_scratch(s, kThermoQ * nb);
    const size_t smem = sizeof(float4) * (size_t)std::max(s.tile_halo_max, 1);
    double4* vel = s.vel.b[s.vc];
    prof_begin(K_FORCE_LJ);
#define TMD_TILE_LAUNCH(F, T)                                                                                      \
    do {                                                                                                           \
        static size_t smem_set = 0;                                                                                \
        if (smem > smem_set) {                                                                                     \
            TMD_CUDA(cudaFuncSetAttribute(k_lj_tile_mixed<F, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                          (int)smem));                                                             \
            smem_set = smem;                                                                                       \
        }                                                                                                          \
        k_lj_tile_mixed<F, T><<<nb, kBlockHomes, smem, s.stream>>>(s.pos32.b[s.pc], s.pos.b[s.pc], s.frc32, vel, s.nbn,   \
                                                                   s.tile_stream, s.tile_desc, s.red_part, a);    \
    } while (0)
    if (fuse_final) {
        if (thermo) TMD_TILE_LAUNCH(true, true);
        else TMD_TILE_LAUNCH(true, false);
    } else {
        if (thermo) TMD_TILE_LAUNCH(false, true);
        else TMD_TILE_LAUNCH(false, false);
    }
#undef TMD_TILE_LAUNCH
    launched(K_FORCE_LJ);
    prof_end(K_FORCE_LJ);
    if (fuse_final) s.integration_iters = s.N;
    if (thermo) run_reduce_partials(s, nb, 0, fuse_final ? kThermoQ : 3);
}

}  // namespace tmd
