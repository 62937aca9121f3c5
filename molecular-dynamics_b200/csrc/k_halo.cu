// k_halo.cu -- the multi-rank part of the timestep (one process per GPU, comm.h):
//   * migration: locals that left the rank box go to the rank owning their new place
//     (comm/comm.impala:392-525, exchange_particles)
//   * the remote half of the border pass: this rank's images inside its neighbours' halos,
//     and the ghosts received from them (comm/comm.impala:528-642, borders)
//   * the per-step halo refresh (comm/comm.impala:334-388, synchronize_ghost_layer)
//
// The reference sweeps six directions in three rounds (x, then y over the locals and the
// x ghosts, then z), each round a host-staged MPI exchange.  Here every local is tested
// once against the 26 regions around the rank box (the border pass's ghost types): a
// region owned by this rank makes a periodic ghost as on one rank, a region owned by
// another rank an image sent there directly with the periodic shift its crossing needs.
// The ghost set is the reference's (an image through two faces reaches the diagonal rank
// in one message instead of two hops), every exchange is one round, and the per-step
// refresh is one pack kernel, one send/receive per neighbour rank and one unpack kernel.
// With NCCL (a GPU per rank) the messages go device to device on the library stream and a
// step needs no host synchronisation; over host sockets they are staged through
// page-locked buffers.
//
// Multi-rank ghosts are exact (each image is its root's current position plus the shift).

#include <algorithm>
#include <cstdio>
#include <string>

#include "comm.h"
#include "md_common.cuh"
#include "md_state.h"
#include "tinymd_b200.h"

namespace tmd {

bool grow_atoms(State& s, int need);  // api.cu

namespace {

constexpr int kClasses = 27;  // migration: 0 stays, 1 + t leaves into region t

// device table (Halo::tab): migration  [c] = message offset of class c's first atom;
// borders [t] = remote images of types before t, [26 + t] = periodic ghosts of types before
// t, [52 + t] = index of type t's first image among the remote ones, [78 + t] = message
// offset of that image
constexpr int kTabRemBefore = 0, kTabSelfBefore = 26, kTabRemStart = 52, kTabMsgOff = 78;
constexpr int kTabUpload = 64;  // pinned host side: readbacks in [0, 64), the upload in [64, 64 + kHaloTab)

struct Regions {
    int sh[26][3];
    double len[3];
};

Regions regions(const State& s) {
    Regions r;
    const Topology& t = comm().topo;
    for (int k = 0; k < 26; ++k)
        for (int d = 0; d < 3; ++d) r.sh[k][d] = t.shift[k][d];
    for (int d = 0; d < 3; ++d) r.len[d] = s.geo.len[d];
    return r;
}

// the image of p in region t's frame (as a periodic ghost of the border pass: one shift per axis)
__device__ __forceinline__ double4 image(const double4& p, int t, const Regions& a) {
    return make_double4(dadd(p.x, dmul(a.len[0], (double)a.sh[t][0])), dadd(p.y, dmul(a.len[1], (double)a.sh[t][1])),
                        dadd(p.z, dmul(a.len[2], (double)a.sh[t][2])), 0.0);
}

struct Box {
    double lo[3], hi[3];
    int split[3];  // axes divided among ranks (the others are periodic within this rank)
};

__device__ __forceinline__ double axis(const double4& p, int d) { return d == 0 ? p.x : (d == 1 ? p.y : p.z); }

// comm/comm.impala:116-127 (exchange_positions: strictly beyond a face of the rank box)
__device__ __forceinline__ int leave_class(const double4& p, const Box& b) {
    int c = 0, w = 1;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double v = axis(p, d);
        int e = 0;
        if (b.split[d]) e = v > b.hi[d] ? 1 : (v < b.lo[d] ? 2 : 0);
        c += e * w;
        w *= 3;
    }
    return c;
}

// per-warp counts of each class into w[warp][class] (zeroed by the caller); returns this
// thread's rank among its warp's members of its class
__device__ __forceinline__ int warp_class_rank(int c, int (*w)[kClasses]) {
    const unsigned same = __match_any_sync(0xffffffffu, c);
    const int lane = threadIdx.x & 31;
    if (c >= 0 && lane == __ffs(same) - 1) w[threadIdx.x >> 5][c] = __popc(same);
    return __popc(same & lanemask_lt());
}

__global__ void __launch_bounds__(kBorderThreads)
k_mig_count(const double4* __restrict__ pos, const int* __restrict__ slot_of_ref, unsigned* __restrict__ cls,
            int* __restrict__ mcount, int N, int nblk, Box b) {
    __shared__ int wc[kBorderThreads / 32][kClasses];
    for (int i = threadIdx.x; i < (kBorderThreads / 32) * kClasses; i += blockDim.x) (&wc[0][0])[i] = 0;
    __syncthreads();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    int c = -1;
    if (r < N) {
        c = leave_class(pos[slot_of_ref[r]], b);
        cls[r] = (unsigned)c;
    }
    warp_class_rank(c, wc);
    __syncthreads();
    if (threadIdx.x < kClasses) {
        int s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += wc[w][threadIdx.x];
        mcount[threadIdx.x * nblk + blockIdx.x] = s;
    }
}

struct Slots {  // one generation of the double-buffered per-slot arrays
    double4* pos;
    double4* vel;
    double4* frc;
    double* mass;
    int* ref;
    int* img;
};

// staying locals compacted into the other buffers in reference order (new reference index =
// rank among the stayers), leaving ones packed into the message buffer (mass, position,
// velocity: core/grid.impala's seven values) peer by peer
__global__ void __launch_bounds__(kBorderThreads)
k_mig_emit(const unsigned* __restrict__ cls, const int* __restrict__ moff, const int* __restrict__ tab,
           const int* __restrict__ slot_of_ref, Slots o, Slots n, double* __restrict__ sbuf, int N, int nblk) {
    __shared__ int wpre[kBorderThreads / 32][kClasses];
    for (int i = threadIdx.x; i < (kBorderThreads / 32) * kClasses; i += blockDim.x) (&wpre[0][0])[i] = 0;
    __syncthreads();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = r < N ? (int)cls[r] : -1;
    const int wr = warp_class_rank(c, wpre);
    __syncthreads();
    if (threadIdx.x < kClasses) {  // exclusive prefix over warps, per class
        int s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            const int k = wpre[w][threadIdx.x];
            wpre[w][threadIdx.x] = s;
            s += k;
        }
    }
    __syncthreads();
    if (r >= N) return;
    const int k = moff[c * nblk + blockIdx.x] - moff[c * nblk] + wpre[threadIdx.x >> 5][c] + wr;
    const int s = slot_of_ref[r];
    const double4 p = o.pos[s];
    const double4 v = o.vel[s];
    if (c == 0) {
        n.pos[k] = p;
        n.vel[k] = v;
        n.frc[k] = make_double4(0.0, 0.0, 0.0, 0.0);
        n.mass[k] = o.mass[s];
        n.ref[k] = k;
        n.img[k] = o.img[s];
        return;
    }
    double* q = sbuf + 7 * (size_t)(tab[c] + k);
    q[0] = o.mass[s];
    q[1] = p.x;
    q[2] = p.y;
    q[3] = p.z;
    q[4] = v.x;
    q[5] = v.y;
    q[6] = v.z;
}

// arrivals appended after the stayers; every local's slot is its reference index
__global__ void k_mig_unpack(const double* __restrict__ rbuf, Slots n, int* __restrict__ slot_of_ref, int nstay,
                             int N) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    slot_of_ref[r] = r;
    if (r < nstay) return;
    const double* q = rbuf + 7 * (size_t)(r - nstay);
    n.mass[r] = q[0];
    n.pos[r] = make_double4(q[1], q[2], q[3], 0.0);
    n.vel[r] = make_double4(q[4], q[5], q[6], 0.0);
    n.frc[r] = make_double4(0.0, 0.0, 0.0, 0.0);
    n.ref[r] = r;
    n.img[r] = 0;
}

// the border pass's remote images in message order: mass and image position (and velocity
// for the contact-fixed DEM model, whose ghosts carry their root's), with the packing
// recorded for the per-step refresh
__global__ void k_halo_pack_borders(const int* __restrict__ send_ref, const int* __restrict__ send_type,
                                    const int* __restrict__ tab, int* __restrict__ pk_ref, int* __restrict__ pk_type,
                                    const int* __restrict__ slot_of_ref, const double4* __restrict__ pos,
                                    const double4* __restrict__ vel, const double* __restrict__ mass,
                                    double* __restrict__ sbuf, int nsend, int stride, Regions a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsend) return;
    const int t = send_type[k];
    const int r = send_ref[k];
    const int o = tab[kTabMsgOff + t] + (k - tab[kTabRemStart + t]);
    pk_ref[o] = r;
    pk_type[o] = t;
    const int s = slot_of_ref[r];
    const double4 p = image(pos[s], t, a);
    double* q = sbuf + (size_t)stride * o;
    q[0] = mass[s];
    q[1] = p.x;
    q[2] = p.y;
    q[3] = p.z;
    if (stride == 7) {
        const double4 v = vel[s];
        q[4] = v.x;
        q[5] = v.y;
        q[6] = v.z;
    }
}

// received ghosts after this rank's own periodic ones (slot = reference index before the
// binning); they have no source on this rank (links -1)
__global__ void k_halo_unpack_borders(const double* __restrict__ rbuf, int stride, Slots n, int* __restrict__ slot_of_ref,
                                      int* __restrict__ gsrc, int* __restrict__ groot, int* __restrict__ gcode,
                                      int* __restrict__ bsrc_ref, int* __restrict__ broot_ref, int* __restrict__ bcode,
                                      int N, int gself, int nrecv) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrecv) return;
    const int g = gself + k;
    const int slot = N + g;
    const double* q = rbuf + (size_t)stride * k;
    n.mass[slot] = q[0];
    n.pos[slot] = make_double4(q[1], q[2], q[3], 0.0);
    n.vel[slot] = stride == 7 ? make_double4(q[4], q[5], q[6], 0.0) : make_double4(0.0, 0.0, 0.0, 0.0);
    n.frc[slot] = make_double4(0.0, 0.0, 0.0, 0.0);
    n.ref[slot] = slot;
    slot_of_ref[slot] = slot;
    gsrc[g] = groot[g] = -1;
    gcode[g] = 0;
    bsrc_ref[g] = broot_ref[g] = -1;
    bcode[g] = 0;
}

struct Frame {
    double alo[3], rb_h;
};

// per step: the images' current positions (comm/comm.impala:334-356) ...
__global__ void k_halo_pack(const int* __restrict__ pk_ref, const int* __restrict__ pk_type,
                            const int* __restrict__ slot_of_ref, const double4* __restrict__ pos,
                            const double4* __restrict__ vel, double* __restrict__ sbuf, int nsend, int stride,
                            Regions a) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nsend) return;
    const int s = slot_of_ref[pk_ref[o]];
    const double4 p = image(pos[s], pk_type[o], a);
    double* q = sbuf + (size_t)stride * o;
    q[0] = p.x;
    q[1] = p.y;
    q[2] = p.z;
    if (stride == 6) {
        const double4 v = vel[s];
        q[3] = v.x;
        q[4] = v.y;
        q[5] = v.z;
    }
}

// ... written into the received ghosts' current slots (comm/comm.impala:377-381), with their
// FP32 rebased copies for the mixed form
__global__ void k_halo_unpack(const double* __restrict__ rbuf, int stride, const int* __restrict__ slot_of_ref,
                              double4* __restrict__ pos, double4* __restrict__ vel, float4* __restrict__ pos32,
                              const int* __restrict__ rbk, int N, int gself, int nrecv, int mixed, Frame f) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrecv) return;
    const int slot = slot_of_ref[N + gself + k];
    const double* q = rbuf + (size_t)stride * k;
    const double4 x = make_double4(q[0], q[1], q[2], 0.0);
    pos[slot] = x;
    if (stride == 6) vel[slot] = make_double4(q[3], q[4], q[5], 0.0);
    if (mixed) pos32[slot] = rebased32(x, rbk[slot], f.alo, f.rb_h);
}

int blocks(long long n, int t) { return (int)std::max<long long>(1, (n + t - 1) / t); }

bool comm_fail(const char* what) {
    set_error(MD_ERR_COMM, std::string(what) + ": " + comm().error());
    return false;
}

bool ensure_dev(double** p, size_t* cap, size_t need) {
    if (need <= *cap) return true;
    dfree(p);
    *cap = need + need / 4 + 1024;
    dalloc(p, *cap);
    if (!*p) {
        *cap = 0;
        return false;
    }
    return true;
}

// one message per peer in each direction, of the given element counts (doubles per element
// `per`), from sbuf / into rbuf in peer order; device to device with NCCL, else staged
bool exchange_payload(State& s, const std::vector<int>& to, const std::vector<int>& from, int per) {
    Comm& c = comm();
    const std::vector<int>& peers = c.topo.peers;
    size_t ns = 0, nr = 0;
    for (size_t i = 0; i < peers.size(); ++i) {
        ns += (size_t)to[i];
        nr += (size_t)from[i];
    }
    if (ns == 0 && nr == 0) return true;
    Halo& h = s.halo;
    std::vector<HostMsg> tx, rx;
    const bool dev = c.device_direct();
    if (!dev) {
        if (h.hs.size() < ns * per) h.hs.resize(ns * per + 1024);
        if (h.hr.size() < nr * per) h.hr.resize(nr * per + 1024);
        if (ns) TMD_CUDA(cudaMemcpyAsync(h.hs.data(), h.sbuf, sizeof(double) * ns * per, cudaMemcpyDeviceToHost, s.stream));
        TMD_CUDA(cudaStreamSynchronize(s.stream));
    }
    double* sb = dev ? h.sbuf : h.hs.data();
    double* rb = dev ? h.rbuf : h.hr.data();
    size_t os = 0, orr = 0;
    for (size_t i = 0; i < peers.size(); ++i) {
        if (to[i]) tx.push_back({peers[i], sb + os * per, sizeof(double) * (size_t)to[i] * per});
        if (from[i]) rx.push_back({peers[i], rb + orr * per, sizeof(double) * (size_t)from[i] * per});
        os += (size_t)to[i];
        orr += (size_t)from[i];
    }
    if (dev) return c.exchange_device(tx, rx, s.stream) || comm_fail("halo exchange");
    if (!c.exchange(tx, rx)) return comm_fail("halo exchange");
    if (nr) TMD_CUDA(cudaMemcpyAsync(h.rbuf, h.hr.data(), sizeof(double) * nr * per, cudaMemcpyHostToDevice, s.stream));
    return true;
}

// element counts per peer: mine to them, theirs to me
bool exchange_counts(const std::vector<int>& to, std::vector<int>& from) {
    Comm& c = comm();
    const std::vector<int>& peers = c.topo.peers;
    from.assign(peers.size(), 0);
    std::vector<HostMsg> tx, rx;
    for (size_t i = 0; i < peers.size(); ++i) {
        tx.push_back({peers[i], const_cast<int*>(&to[i]), sizeof(int)});
        rx.push_back({peers[i], &from[i], sizeof(int)});
    }
    return c.exchange(tx, rx) || comm_fail("count exchange");
}

Slots slots(State& s, int pc, int vc, int ac) {
    return Slots{s.pos.b[pc], s.vel.b[vc], s.frc.b[ac], s.mass.b[ac], s.ref.b[ac], s.img.b[ac]};
}

}  // namespace

void halo_free(State& s) {
    Halo& h = s.halo;
    dfree(&h.send_ref);
    dfree(&h.send_type);
    dfree(&h.pk_ref);
    dfree(&h.pk_type);
    dfree(&h.tab);
    dfree(&h.sbuf);
    dfree(&h.rbuf);
    if (h.tab_host) cudaFreeHost(h.tab_host);
    h.tab_host = nullptr;
    h.sbuf_cap = h.rbuf_cap = 0;
    h.send_cap = 0;
    h.gself = h.nsend = h.nrecv = 0;
    h.send_cnt.clear();
    h.recv_cnt.clear();
}

static bool ensure_tables(State& s) {
    Halo& h = s.halo;
    if (!h.tab) dalloc(&h.tab, kHaloTab);
    if (!h.tab_host) TMD_CUDA(cudaMallocHost((void**)&h.tab_host, sizeof(int) * (kTabUpload + kHaloTab)));
    return h.tab && h.tab_host;
}

// ---- migration -------------------------------------------------------------------------------
bool run_migrate(State& s) {
    Comm& c = comm();
    Halo& h = s.halo;
    if (!h.on || !ensure_tables(s)) return h.on ? false : true;
    const Topology& t = c.topo;
    const int N = s.N;
    const int nblk = border_blocks(std::max(N, 1));
    Box b;
    for (int d = 0; d < 3; ++d) {
        b.lo[d] = s.geo.aabb_lo[d] + s.geo.spacing;  // the rank box (the grid adds one cell per side)
        b.hi[d] = s.geo.aabb_hi[d] - s.geo.spacing;
        b.split[d] = t.dims[d] > 1;
    }
    // class counts per block [27][nblk] in bcount (room for 2 * 26 * nblk + 1), their scan after them
    int* mcount = s.bcount;
    int* moff = s.bcount + kClasses * nblk;
    int* tot = h.tab_host;
    if (N > 0) {
        k_mig_count<<<nblk, kBorderThreads, 0, s.stream>>>(s.pos.b[s.pc], s.slot_of_ref, s.bmask, mcount, N, nblk, b);
        launched(K_BORDER);
        exclusive_scan(s, mcount, moff, kClasses * nblk);
        TMD_CUDA(cudaMemcpy2DAsync(tot, sizeof(int), moff, sizeof(int) * nblk, sizeof(int), kClasses, cudaMemcpyDeviceToHost,
                                   s.stream));
        TMD_CUDA(cudaMemcpyAsync(tot + kClasses, moff + kClasses * nblk, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
        TMD_CUDA(cudaStreamSynchronize(s.stream));
    } else {
        for (int k = 0; k <= kClasses; ++k) tot[k] = 0;
    }
    // per peer: atoms to send; message offsets per class, peer by peer then class order
    std::vector<int> to(t.peers.size(), 0), from;
    int* off = h.tab_host + kTabUpload;
    for (int k = 0; k < kClasses; ++k) off[k] = 0;
    const int nstay = tot[1] - tot[0];
    size_t run = 0;
    for (size_t i = 0; i < t.peers.size(); ++i) {
        for (int k = 1; k < kClasses; ++k) {
            if (t.peer[k - 1] != t.peers[i]) continue;
            off[k] = (int)run;
            const int n = tot[k + 1] - tot[k];
            run += (size_t)n;
            to[i] += n;
        }
    }
    if (!exchange_counts(to, from)) return false;
    long long nrecv = 0;
    for (int v : from) nrecv += v;
    const long long Nn = (long long)nstay + nrecv;
    if (Nn >= kMaxSlots / 2) {
        set_error(MD_ERR_ARGUMENT, "md_exchange_particles: too many locals on this rank");
        return false;
    }
    if (!ensure_dev(&h.sbuf, &h.sbuf_cap, 7 * run + 7) || !ensure_dev(&h.rbuf, &h.rbuf_cap, 7 * (size_t)nrecv + 7))
        return false;
    if (Nn > s.capA && !grow_atoms(s, (int)Nn)) return false;
    const int np = 1 - s.pc, nv = 1 - s.vc, na = 1 - s.ac;
    const Slots o = slots(s, s.pc, s.vc, s.ac), n = slots(s, np, nv, na);
    if (N > 0) {
        TMD_CUDA(cudaMemcpyAsync(h.tab, off, sizeof(int) * kClasses, cudaMemcpyHostToDevice, s.stream));
        k_mig_emit<<<nblk, kBorderThreads, 0, s.stream>>>(s.bmask, moff, h.tab, s.slot_of_ref, o, n, h.sbuf, N, nblk);
        launched(K_BORDER);
    }
    if (!exchange_payload(s, to, from, 7)) return false;
    if (Nn > 0) {
        k_mig_unpack<<<blocks(Nn, 256), 256, 0, s.stream>>>(h.rbuf, n, s.slot_of_ref, nstay, (int)Nn);
        launched(K_BORDER);
    }
    s.pc = np;
    s.vc = nv;
    s.ac = na;
    s.N = (int)Nn;
    s.G = 0;
    h.gself = h.nsend = h.nrecv = 0;
    s.lists_valid = 0;
    s.img_ok = 0;
    // the per-local arrays follow the new count (the classes in bmask are no longer needed)
    return ensure_locals(s, (int)Nn);
}

// ---- borders -------------------------------------------------------------------------------------
// boff: the border pass's scanned ghost offsets ([26][nblk] and the total after them; null
// when this rank has no locals).  Reads back the offset of each type's first block, splits the
// images into this rank's periodic ghosts and the ones for other ranks, and uploads the offset
// table the emit and pack kernels use.
bool halo_plan_borders(State& s, const int* boff, int nblk) {
    Halo& h = s.halo;
    const Topology& t = comm().topo;
    if (!ensure_tables(s)) return false;
    int* type_off = h.tab_host;
    if (boff) {
        TMD_CUDA(cudaMemcpy2DAsync(type_off, sizeof(int), boff, sizeof(int) * nblk, sizeof(int), 26,
                                   cudaMemcpyDeviceToHost, s.stream));
        TMD_CUDA(cudaMemcpyAsync(type_off + 26, boff + 26 * nblk, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
        TMD_CUDA(cudaStreamSynchronize(s.stream));
    } else {
        for (int k = 0; k <= 26; ++k) type_off[k] = 0;
    }
    int* up = h.tab_host + kTabUpload;
    int nself = 0, nrem = 0;
    for (int k = 0; k < 26; ++k) {
        const int n = type_off[k + 1] - type_off[k];
        up[kTabRemBefore + k] = nrem;
        up[kTabSelfBefore + k] = nself;
        up[kTabRemStart + k] = type_off[k] - nself;
        if ((t.selfmask >> k) & 1u) nself += n;
        else nrem += n;
    }
    h.send_cnt.assign(t.peers.size(), 0);
    int run = 0;
    for (size_t i = 0; i < t.peers.size(); ++i)
        for (int k = 0; k < 26; ++k) {
            if (((t.selfmask >> k) & 1u) || t.peer[k] != t.peers[i]) continue;
            up[kTabMsgOff + k] = run;
            const int n = type_off[k + 1] - type_off[k];
            run += n;
            h.send_cnt[i] += n;
        }
    for (int k = 0; k < 26; ++k)
        if ((t.selfmask >> k) & 1u) up[kTabMsgOff + k] = 0;
    h.gself = nself;
    h.nsend = nrem;
    if (nrem > h.send_cap) {
        const int cap = nrem + nrem / 4 + 1024;
        int** arr[] = {&h.send_ref, &h.send_type, &h.pk_ref, &h.pk_type};
        for (int** a : arr) {
            dfree(a);
            dalloc(a, cap);
            if (!*a) return false;
        }
        h.send_cap = cap;
    }
    TMD_CUDA(cudaMemcpyAsync(h.tab, up, sizeof(int) * (kTabMsgOff + 26), cudaMemcpyHostToDevice, s.stream));
    return true;
}

// after the border emit (periodic ghosts written, remote images listed by type): pack and send
// the images, receive the neighbours' and append them as ghosts
bool halo_finish_borders(State& s) {
    Halo& h = s.halo;
    const int stride = s.dem_fixed ? 7 : 4;
    if (!ensure_dev(&h.sbuf, &h.sbuf_cap, (size_t)stride * h.nsend + 8)) return false;
    const Regions a = regions(s);
    if (h.nsend > 0) {
        k_halo_pack_borders<<<blocks(h.nsend, 256), 256, 0, s.stream>>>(h.send_ref, h.send_type, h.tab, h.pk_ref, h.pk_type,
                                                                      s.slot_of_ref, s.pos.b[s.pc], s.vel.b[s.vc],
                                                                      s.mass.b[s.ac], h.sbuf, h.nsend, stride, a);
        launched(K_BORDER);
    }
    if (!exchange_counts(h.send_cnt, h.recv_cnt)) return false;
    long long nrecv = 0;
    for (int v : h.recv_cnt) nrecv += v;
    const long long NA = (long long)s.N + h.gself + nrecv;
    if (NA >= kMaxSlots) {
        set_error(MD_ERR_ARGUMENT, "md_borders: too many ghosts on this rank");
        return false;
    }
    if (!ensure_dev(&h.rbuf, &h.rbuf_cap, (size_t)stride * nrecv + 8)) return false;
    if (NA > s.capA && !grow_atoms(s, (int)NA)) return false;
    if (!exchange_payload(s, h.send_cnt, h.recv_cnt, stride)) return false;
    if (nrecv > 0) {
        k_halo_unpack_borders<<<blocks(nrecv, 256), 256, 0, s.stream>>>(h.rbuf, stride, slots(s, s.pc, s.vc, s.ac),
                                                                        s.slot_of_ref, s.gsrc, s.groot, s.gcode,
                                                                        s.bsrc_ref, s.broot_ref, s.bcode, s.N, h.gself,
                                                                        (int)nrecv);
        launched(K_BORDER);
    }
    h.nrecv = (int)nrecv;
    s.G = h.gself + h.nrecv;
    return true;
}

// ---- per-step refresh --------------------------------------------------------------------------
bool run_halo_sync(State& s) {
    Halo& h = s.halo;
    if (!h.on) return true;
    const int stride = s.dem_fixed ? 6 : 3;
    if (!ensure_dev(&h.sbuf, &h.sbuf_cap, (size_t)stride * h.nsend + 8) ||
        !ensure_dev(&h.rbuf, &h.rbuf_cap, (size_t)stride * h.nrecv + 8))
        return false;
    prof_begin(K_GHOST_SYNC);
    if (h.nsend > 0) {
        k_halo_pack<<<blocks(h.nsend, 256), 256, 0, s.stream>>>(h.pk_ref, h.pk_type, s.slot_of_ref, s.pos.b[s.pc],
                                                               s.vel.b[s.vc], h.sbuf, h.nsend, stride, regions(s));
        launched(K_GHOST_SYNC);
    }
    if (!exchange_payload(s, h.send_cnt, h.recv_cnt, stride)) return false;
    if (h.nrecv > 0) {
        Frame f;
        for (int d = 0; d < 3; ++d) f.alo[d] = s.geo.aabb_lo[d];
        f.rb_h = s.geo.rb_h;
        k_halo_unpack<<<blocks(h.nrecv, 256), 256, 0, s.stream>>>(h.rbuf, stride, s.slot_of_ref, s.pos.b[s.pc],
                                                                 s.vel.b[s.vc], s.pos32.b[s.pc], s.rbk, s.N, h.gself,
                                                                 h.nrecv, s.precision == 1, f);
        launched(K_GHOST_SYNC);
    }
    prof_end(K_GHOST_SYNC);
    return true;
}

}  // namespace tmd
