// k_step.cu -- per-timestep kernels of the tinyMD B200 path:
//   * LJ forces over full or half lists, FP64 (bit-identical to the CPU
//     restatement for full lists) or mixed (FP32 pair arithmetic on rebased
//     FP32 positions), optionally fused with the final velocity half-kick
//     (core/compute.impala:1-95 and 108-116, core/runtime.impala:188-201)
//   * DEM spring-dashpot forces (core/runtime.impala:203-247)
//   * initial integration fused with the periodic ghost refresh
//     (core/compute.impala:97-106, comm/comm.impala:334-388)
//   * stand-alone ghost refresh and final integration
//   * deterministic FP64 reductions of energy, virial and kinetic energy
//
// Thread per local atom; the atom-fastest list makes the index loads of a
// warp one coalesced 128-byte line per neighbour slot, and neighbour
// positions come through the read-only path.

#include "lj_args.cuh"
#include "md_common.cuh"
#include "md_state.h"

namespace tmd {

namespace {

// 128-thread blocks: 1,024 blocks for 131k atoms spread evenly over 148 SMs (6-7 each);
// 256-thread blocks left 68 SMs with four and 80 with three, and ran 5 % (mixed) to 11 %
// (FP64) slower in the force kernels
#ifndef TMD_THREADS
#define TMD_THREADS 128
#endif
constexpr int kThreads = TMD_THREADS;
constexpr int kThermoQ = 4;  // partials: energy, virial, pairs inside the cutoff, v.v

inline int nblocks(long long n, int t) { return (int)((n + t - 1) / t); }

struct StepArgs {
    int N, G, stride;
    double dt, h;  // h = 0.5 * dt as the reference computes it
    double len[3], alo[3], rb_h;
    int pre;       // k_integrate first applies the previous step's final kick v += hp f
    double hp;
};

struct DemArgs {
    int N, stride, nbcap, fixed;
    double rc2, dn, dt_, k, mu, radius;
};

__device__ __forceinline__ double4 ldg_d4(const double4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// writes the per-block partial of quantity q (kThermoQ-major layout)
__device__ __forceinline__ void put_partial(double* part, int q, double v, double* scratch) {
    double r = block_sum(v, scratch);
    if (threadIdx.x == 0) part[q * gridDim.x + blockIdx.x] = r;
}

// ---- prefetch ------------------------------------------------------------------------
// The force kernels do not prefetch their list rows: a bulk L2 prefetch of every block's rows at
// the start queued ~40 MB ahead of the first demand loads and cost 2.4 us (cold L2) and 1.4 us
// (warm) per launch of the mixed kernel at 131k atoms, and one of only the first 2-8 rows still
// 0.5-0.9 us (cold); the quad loads one batch ahead suffice.

// quad b of atom i's list (entries 4b .. 4b + 3)
__device__ __forceinline__ uint4 list_quad(const uint32_t* nbl, int b, int i, int stride) {
    return __ldg(reinterpret_cast<const uint4*>(nbl) + (size_t)b * stride + i);
}
// this block's share of a per-slot array (bytes a multiple of 16), prefetched into L2 by
// warp 0 in pieces of at most 4 KiB: the gathered neighbour positions and the block's own
// rows arrive at DRAM bandwidth instead of on first touch (cold L2 after other work)
__device__ __forceinline__ void prefetch_share(const void* base, size_t bytes) {
    if (threadIdx.x >= 32 || bytes == 0) return;
    const size_t share = ((bytes + gridDim.x - 1) / gridDim.x + 15) & ~(size_t)15;
    const size_t lo = share * blockIdx.x;
    if (lo >= bytes) return;
    const size_t hi = min(bytes, lo + share);
    for (size_t o = lo + (size_t)threadIdx.x * 4096; o < hi; o += (size_t)32 * 4096) {
        const unsigned len = (unsigned)min((size_t)4096, hi - o);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"((const char*)base + o), "r"(len) : "memory");
    }
}

// one vector atomic (sm_90+: red.global.add.v4.f32) instead of three scalar ones for a
// half-list reaction on an FP32 force; w stays zero
__device__ __forceinline__ void add_force32(float4* f, float x, float y, float z) {
    atomicAdd(f, make_float4(x, y, z, 0.f));
}

// target of the reaction force of a half-list pair: the local itself or a ghost's root
__device__ __forceinline__ int reaction_slot(int j, int N, const int* groot) { return j < N ? j : groot[j - N]; }

// ---- FP64 LJ ------------------------------------------------------------------
#ifndef TMD_MINB
// seven 128-thread blocks per SM cap registers at 72 per thread, and 7 x 148 blocks still hold the
// 1,024 blocks of 131k atoms in one wave (the mixed kernel: 37.4 -> 36.9 us against 64 registers)
#define TMD_MINB 7
#endif
// v += dt/2 f; x += dt v (core/compute.impala:97-106) in the reference's operand order
__device__ __forceinline__ double4 integrate_one(const double4& x, double4& v, double fx, double fy, double fz,
                                                 double dt, double h) {
    v.x = dadd(v.x, dmul(fx, h));
    v.y = dadd(v.y, dmul(fy, h));
    v.z = dadd(v.z, dmul(fz, h));
    return make_double4(dadd(x.x, dmul(v.x, dt)), dadd(x.y, dmul(v.y, dt)), dadd(x.z, dmul(v.z, dt)), x.w);
}

constexpr int kB64 = 4;  // neighbours per batch (FP64): one list quad
constexpr int kB32 = 4;  // neighbours per batch (mixed): one list quad
// list quads with FP64-path pairs a mixed thread queues (more: the atom is redone in place, rare)
constexpr int kQQ = 8;

// Ghost images written by the force kernel that integrates (maps from k_ghost_links): each
// local writes the ghosts that are its images, from its new position, and extra threads
// write the two-phase ghosts whose source is another ghost, from that source's previous
// value.  The arithmetic is k_ghost_refresh's, so the ghosts are bit-identical to it.
struct PushArgs {
    const int* slot = nullptr;   // first image plane of the ghost mode (planes `plane` apart)
    const int* chain = nullptr;  // two-phase ghosts whose source is a ghost
    const int* gsrc = nullptr;
    const int* gcode = nullptr;
    const int* rbk = nullptr;
    int nchain = 0;              // two-phase mode only
    const int* nchain_dev = nullptr;  // the count on the device (nchain is then a bound)
    int base = 0;                // shift field of the code: 0 last pass, 8 total
    int planes = 0;              // image planes of the mode
    int plane = 0;               // plane stride (slot capacity)
    int G = 0;
    double len[3] = {0.0, 0.0, 0.0};
};

template <bool MIXED>
__device__ __forceinline__ void write_ghost(int t, const double4& xs, int code, const PushArgs& pa,
                                            double4* __restrict__ pos_n, float4* __restrict__ pos32_n,
                                            const double* alo, double rb_h) {
    double4 x;
    x.x = dadd(xs.x, dmul(pa.len[0], (double)shift_axis(code, pa.base, 0)));
    x.y = dadd(xs.y, dmul(pa.len[1], (double)shift_axis(code, pa.base, 1)));
    x.z = dadd(xs.z, dmul(pa.len[2], (double)shift_axis(code, pa.base, 2)));
    x.w = 0.0;
    pos_n[t] = x;
    if (MIXED) pos32_n[t] = rebased32(x, pa.rbk[t], alo, rb_h);
}

// the first three planes are read together (a local near one face, edge or corner of the box
// has one, two or three two-phase images); further ones, for thin boxes, one by one
template <bool MIXED>
__device__ __forceinline__ void push_images(int i, const double4& x, int N, const PushArgs& pa,
                                            double4* __restrict__ pos_n, float4* __restrict__ pos32_n,
                                            const double* alo, double rb_h) {
    int t[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) t[k] = pa.slot[(size_t)k * pa.plane + i];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (t[k] < 0) return;
        write_ghost<MIXED>(t[k], x, pa.gcode[t[k] - N], pa, pos_n, pos32_n, alo, rb_h);
    }
    for (int k = 3; k < pa.planes; ++k) {
        const int tk = pa.slot[(size_t)k * pa.plane + i];
        if (tk < 0) return;
        write_ghost<MIXED>(tk, x, pa.gcode[tk - N], pa, pos_n, pos32_n, alo, rb_h);
    }
}

// L2 prefetch of what the pushes read: the first image planes, ghost codes, rebasing cells
__device__ __forceinline__ void prefetch_push(const PushArgs& pa, int N) {
#pragma unroll
    for (int k = 0; k < 3; ++k) prefetch_share(pa.slot + (size_t)k * pa.plane, (size_t)((N + 3) & ~3) * sizeof(int));
    prefetch_share(pa.gcode, (size_t)((pa.G + 3) & ~3) * sizeof(int));
    prefetch_share(pa.rbk, (size_t)((N + pa.G + 3) & ~3) * sizeof(int));
}

template <bool MIXED>
__device__ __forceinline__ void push_chain(int q, const double4* __restrict__ pos_o, int N, const PushArgs& pa,
                                           double4* __restrict__ pos_n, float4* __restrict__ pos32_n,
                                           const double* alo, double rb_h) {
    const int h = pa.chain[q];
    write_ghost<MIXED>(N + h, pos_o[pa.gsrc[h]], pa.gcode[h], pa, pos_n, pos32_n, alo, rb_h);
}

// INIT (with FUSE, full lists): the epilogue also does the next step's initial integration
// and writes the atom's new position to pos_n, the other buffer (neighbours read pos)
// PUSH (with INIT): the kernel also writes the ghosts (PushArgs)
template <bool HALF, bool FUSE, bool THERMO, bool INIT = false, bool PUSH = false>
__global__ void __launch_bounds__(kThreads)
k_lj_fp64(const double4* __restrict__ pos, double4* __restrict__ frc, double4* __restrict__ vel,
          const int* __restrict__ nbn, const uint32_t* __restrict__ nbl, const int* __restrict__ groot,
          double* __restrict__ part, LjArgs a, double4* __restrict__ pos_n = nullptr, PushArgs pa = PushArgs()) {
    __shared__ double scratch[kThreads / 32];
    if (INIT && lists_failed(a)) return;  // the whole grid returns: nothing written
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = i < a.N ? min(nbn[i], a.nbcap) : 0;
    prefetch_share(pos, (size_t)a.NA * sizeof(double4));
    if (FUSE) prefetch_share(vel, (size_t)a.N * sizeof(double4));
    if (PUSH) prefetch_push(pa, a.N);
    double e = 0.0, w = 0.0, cnt = 0.0, ke = 0.0;
    if (i < a.N) {
        const double4 pi = pos[i];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        // quads of four entries; the next quad loads while this one's gathers are in flight
        // (entries past n are padding, skipped below)
        const int nq = (n + 3) >> 2;
        uint4 eq = n > 0 ? list_quad(nbl, 0, i, a.stride) : make_uint4(0u, 0u, 0u, 0u);
        for (int b = 0; b < nq; ++b) {
            const int k0 = 4 * b;
            const uint32_t ent[kB64] = {eq.x, eq.y, eq.z, eq.w};
            int j[kB64];
            double4 pj[kB64];
#pragma unroll
            for (int u = 0; u < kB64; ++u) j[u] = (int)(ent[u] >> kCodeBits);
#pragma unroll
            for (int u = 0; u < kB64; ++u) pj[u] = ldg_d4(pos + j[u]);
            eq = list_quad(nbl, min(b + 1, nq - 1), i, a.stride);
#pragma unroll
            for (int u = 0; u < kB64; ++u) {
                const double dx = dsub(pi.x, pj[u].x), dy = dsub(pi.y, pj[u].y), dz = dsub(pi.z, pj[u].z);
                const double rsq = len2_strict(dx, dy, dz);
                if (k0 + u >= n) continue;
                if (rsq < a.rc2) {
                    const double sr2 = ddiv(1.0, rsq);
                    const double sr6 = dmul(dmul(dmul(sr2, sr2), sr2), a.sigma6);
                    const double f = dmul(dmul(dmul(dmul(48.0, sr6), dsub(sr6, 0.5)), sr2), a.eps);
                    const double px = dmul(dx, f), py = dmul(dy, f), pz = dmul(dz, f);
                    fx = dadd(fx, px);
                    fy = dadd(fy, py);
                    fz = dadd(fz, pz);
                    if (HALF) {
                        const int t = reaction_slot(j[u], a.N, groot);
                        atomicAdd(&frc[t].x, -px);
                        atomicAdd(&frc[t].y, -py);
                        atomicAdd(&frc[t].z, -pz);
                    }
                    if (THERMO) {
                        e += 4.0 * a.eps * sr6 * (sr6 - 1.0);
                        w += f * rsq;
                        cnt += 1.0;
                    }
                }
            }
        }
        if (HALF) {
            atomicAdd(&frc[i].x, fx);
            atomicAdd(&frc[i].y, fy);
            atomicAdd(&frc[i].z, fz);
        } else {
            frc[i] = make_double4(fx, fy, fz, 0.0);
            if (FUSE) {  // core/compute.impala:108-116
                double4 v = vel[i];
                v.x = dadd(v.x, dmul(fx, a.h));
                v.y = dadd(v.y, dmul(fy, a.h));
                v.z = dadd(v.z, dmul(fz, a.h));
                if (THERMO) ke = v.x * v.x + v.y * v.y + v.z * v.z;
                if (INIT) {  // positions carry w = 0
                    double4 x = integrate_one(pi, v, fx, fy, fz, a.dt_i, a.h_i);
                    x.w = 0.0;
                    pos_n[i] = x;
                    if (PUSH) push_images<false>(i, x, a.N, pa, pos_n, nullptr, a.alo, a.rb_h);
                }
                vel[i] = v;
            }
        }
    } else if (PUSH && i < a.N + (pa.nchain_dev ? *pa.nchain_dev : pa.nchain)) {
        push_chain<false>(i - a.N, pos, a.N, pa, pos_n, nullptr, a.alo, a.rb_h);
    }
    if (THERMO) {
        put_partial(part, 0, e, scratch);
        put_partial(part, 1, w, scratch);
        put_partial(part, 2, cnt, scratch);
        if (FUSE) put_partial(part, 3, ke, scratch);
    }
}

// ---- mixed LJ -----------------------------------------------------------------
// 1/x for the mixed form's FP64 pairs: the hardware's approximate FP64 reciprocal refined by
// two Newton-Raphson steps (y <- y + y (1 - x y), quadratic convergence), relative error far
// below the 1e-7 the mixed form's FP64 pairs need, without a full IEEE division
__device__ __forceinline__ double recip64(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    y = fma(y, fma(-x, y, 1.0), y);
    return fma(y, fma(-x, y, 1.0), y);
}

// FP64 evaluation of one list pair (the mixed form's fallback for close pairs
// and pairs at the cutoff): accumulates the force on i into c and the thermo sums
template <bool THERMO>
__device__ __forceinline__ void fp64_lj(const double4& pi, int j, const double4* __restrict__ pos, const LjArgs& a,
                                        double& cx, double& cy, double& cz, double& e, double& w, int& ncnt) {
    const double4 pj = ldg_d4(pos + j);
    const double ex = dsub(pi.x, pj.x), ey = dsub(pi.y, pj.y), ez = dsub(pi.z, pj.z);
    const double r2 = len2_strict(ex, ey, ez);
    if (r2 < a.rc2) {
        const double sr2 = recip64(r2);
        const double sr6 = sr2 * sr2 * sr2 * a.sigma6;
        const double f = 48.0 * sr6 * (sr6 - 0.5) * sr2 * a.eps;
        cx += ex * f;
        cy += ey * f;
        cz += ez * f;
        if (THERMO) {
            e += 4.0 * a.eps * sr6 * (sr6 - 1.0);
            w += f * r2;
            ncnt++;
        }
    }
}

// FP32 pair arithmetic on positions rebased to a dyadic grid of spacing rb_h:
// del = (r_i - r_j) - dk*rb_h, with dk in {-1,0,1}^3 decoded from the list
// entry's low bits (exact float construction, 3 operations per axis) and the
// product exact, so del carries one rounding more than r_i - r_j.  Pairs
// closer than 1.04 sigma (large forces, ~1 per atom in a dense LJ liquid) and
// pairs within 2e-5 (relative) of the squared cutoff take the FP64 path, so list
// membership and the cutoff test stay exactly the FP64 decisions (lj_args).
//
// Half lists: each pair once, the reaction added atomically to j (or to the root of
// a ghost j); forces must be zeroed before the launch.

// del and r^2 of one mixed-form pair from its list entry (the rebasing shift decoded from the
// entry's code) and the fast-window test, shared by the kernels so that they decide alike
__device__ __forceinline__ float mixed_del(uint32_t en, const float4& ri, const float4& rj, const LjArgs& a,
                                           float& dx, float& dy, float& dz) {
    const float sx = __int_as_float((int)((en & 0x03u) | 0x4B000000u)) - 8388609.0f;
    const float sy = __int_as_float((int)((en & 0x0Cu) | 0x4B000000u)) - 8388612.0f;
    const float sz = __int_as_float((int)((en & 0x30u) | 0x4B000000u)) - 8388624.0f;
    dx = fmaf(a.hx, sx, ri.x - rj.x);
    dy = fmaf(a.hy, sy, ri.y - rj.y);
    dz = fmaf(a.hz, sz, ri.z - rj.z);
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}
__device__ __forceinline__ bool mixed_fast(float rsq, const LjArgs& a) {
    return fabsf(rsq - a.fast_mid) < a.fast_half;
}
// f/r of a pair from sr2 = 1/r^2 (five FP32 operations), and t = 1/r^6 for the energy
__device__ __forceinline__ float mixed_force(float sr2, const LjArgs& a, float& t) {
    t = sr2 * sr2 * sr2;
    return (t * sr2) * fmaf(a.lj_a, t, a.lj_b);
}

// FP64 evaluation of one half-list pair of the mixed form, its reaction added to j's root
template <bool THERMO>
__device__ __forceinline__ void fp64_lj_half(const double4& pi, int j, const double4* __restrict__ pos,
                                             float4* __restrict__ frc32, const int* __restrict__ groot,
                                             const LjArgs& a, double& cx, double& cy, double& cz, double& e,
                                             double& w, int& ncnt) {
    const double4 pj = ldg_d4(pos + j);
    const double ex = dsub(pi.x, pj.x), ey = dsub(pi.y, pj.y), ez = dsub(pi.z, pj.z);
    const double r2 = len2_strict(ex, ey, ez);
    if (r2 < a.rc2) {
        const double sr2 = recip64(r2);
        const double sr6 = sr2 * sr2 * sr2 * a.sigma6;
        const double f = 48.0 * sr6 * (sr6 - 0.5) * sr2 * a.eps;
        cx += ex * f;
        cy += ey * f;
        cz += ez * f;
        add_force32(frc32 + reaction_slot(j, a.N, groot), (float)(-ex * f), (float)(-ey * f), (float)(-ez * f));
        if (THERMO) {
            e += 4.0 * a.eps * sr6 * (sr6 - 1.0);
            w += f * r2;
            ncnt++;
        }
    }
}

// The full-list kernel's arrangement over half lists: the FP32 pair force of a quad without
// branches, the reaction added (one vector atomic) for the pairs in the fast window, and the quads
// holding FP64-path pairs queued and worked off after the loop (49.1 -> 42.5 us at 131k atoms
// against one branch per pair with the FP64 path inline).
template <bool THERMO>
__global__ void __launch_bounds__(kThreads, TMD_MINB)
k_lj_mixed_half(const float4* __restrict__ pos32, const double4* __restrict__ pos, float4* __restrict__ frc32,
                const int* __restrict__ nbn, const uint32_t* __restrict__ nbl, const int* __restrict__ groot,
                double* __restrict__ part, LjArgs a) {
    __shared__ double scratch[kThreads / 32];
    __shared__ int s_q[kQQ + 1][kThreads];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = i < a.N ? min(nbn[i], a.nbcap) : 0;
    prefetch_share(pos32, (size_t)a.NA * sizeof(float4));
    prefetch_share(pos, (size_t)a.N * sizeof(double4));
    double e = 0.0, w = 0.0, cnt = 0.0;
    if (i < a.N) {
        const float4 ri = pos32[i];
        float fx = 0.f, fy = 0.f, fz = 0.f, ef = 0.f, wf = 0.f;
        double cx = 0.0, cy = 0.0, cz = 0.0;
        int ncnt = 0;
        int nq = 0;
        // the last quad's padding (the atom itself one rebasing cell away) is in no window
        const int nquad = (n + 3) >> 2;
        uint4 eq = n > 0 ? list_quad(nbl, 0, i, a.stride) : make_uint4(0u, 0u, 0u, 0u);
        for (int b = 0; b < nquad; ++b) {
            const uint32_t cur[kB32] = {eq.x, eq.y, eq.z, eq.w};
            float4 rj[kB32];
#pragma unroll
            for (int u = 0; u < kB32; ++u) rj[u] = __ldg(pos32 + (cur[u] >> kCodeBits));
            eq = list_quad(nbl, b + 1, i, a.stride);  // the last read lands in the spare row
            unsigned slow = 0;
#pragma unroll
            for (int u = 0; u < kB32; ++u) {
                float dx, dy, dz;
                const float rsq = mixed_del(cur[u], ri, rj[u], a, dx, dy, dz);
                const bool fast = mixed_fast(rsq, a);
                float sr2, t;
                asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(sr2) : "f"(rsq));
                float f = mixed_force(sr2, a, t);
                f = fast ? f : 0.f;
                const float px = dx * f, py = dy * f, pz = dz * f;
                fx += px;
                fy += py;
                fz += pz;
                if (fast) add_force32(frc32 + reaction_slot((int)(cur[u] >> kCodeBits), a.N, groot), -px, -py, -pz);
                if (THERMO) {
                    ef += fast ? t * fmaf(a.lj_c, t, a.lj_d) : 0.f;
                    wf = fmaf(f, rsq, wf);
                    ncnt += fast ? 1 : 0;
                }
                slow |= (!fast && rsq < a.rc2_hi) ? (1u << u) : 0u;
            }
            s_q[min(nq, kQQ)][threadIdx.x] = (b << kB32) | (int)slow;
            nq += slow != 0u ? 1 : 0;
        }
        if (nq > 0) {
            const double4 pi = ldg_d4(pos + i);
            if (nq > kQQ) {
                // more queued quads than the queue holds: every quad is tested again (the same
                // arithmetic, so the same pairs) and its FP64 pairs evaluated in place
                for (int b = 0; b < nquad; ++b) {
                    const uint4 e4 = list_quad(nbl, b, i, a.stride);
                    const uint32_t c4[kB32] = {e4.x, e4.y, e4.z, e4.w};
                    for (int u = 0; u < kB32; ++u) {
                        float dx, dy, dz;
                        const float rsq = mixed_del(c4[u], ri, __ldg(pos32 + (c4[u] >> kCodeBits)), a, dx, dy, dz);
                        if (!mixed_fast(rsq, a) && rsq < a.rc2_hi)
                            fp64_lj_half<THERMO>(pi, (int)(c4[u] >> kCodeBits), pos, frc32, groot, a, cx, cy, cz, e, w,
                                                 ncnt);
                    }
                }
            } else {
                uint4 nx4 = list_quad(nbl, s_q[0][threadIdx.x] >> kB32, i, a.stride);
                for (int q = 0; q < nq; ++q) {
                    const int wq = s_q[q][threadIdx.x];
                    const uint4 e4 = nx4;
                    if (q + 1 < nq) nx4 = list_quad(nbl, s_q[q + 1][threadIdx.x] >> kB32, i, a.stride);
                    unsigned bits = (unsigned)wq & ((1u << kB32) - 1u);
                    while (bits) {
                        const int u = __ffs(bits) - 1;
                        bits &= bits - 1u;
                        const uint32_t en = u == 0 ? e4.x : (u == 1 ? e4.y : (u == 2 ? e4.z : e4.w));
                        fp64_lj_half<THERMO>(pi, (int)(en >> kCodeBits), pos, frc32, groot, a, cx, cy, cz, e, w, ncnt);
                    }
                }
            }
        }
        add_force32(frc32 + i, (float)((double)fx + cx), (float)((double)fy + cy), (float)((double)fz + cz));
        if (THERMO) {
            e += (double)ef;
            w += (double)wf;
            cnt = (double)ncnt;
        }
    }
    if (THERMO) {
        put_partial(part, 0, e, scratch);
        put_partial(part, 1, w, scratch);
        put_partial(part, 2, cnt, scratch);
    }
}

// ---- mixed LJ, branch-free batches (full lists) --------------------------------
// The pair arithmetic of k_lj_mixed_half, each pair seen from both atoms (no atomics),
// arranged for instruction-level parallelism: the FP32 fast path of a batch's kB32 pairs (one
// list quad) runs without branches (the force of a pair outside [close2, rc2_lo) is masked to
// zero), so the compiler interleaves the pairs' dependent chains; a quad holding FP64-path pairs
// is queued in shared memory (one store per quad, no branch) and its FP64 pairs are evaluated
// after the loop, in list order (1 -> 0.99 of the time of a queue of pairs with a per-quad
// room check, which also spilled in the thermo variants).  The next batch's list entries are loaded before
// the current batch's gathers, so a batch waits for one memory latency, not two.
// The atom's FP64 position is re-read where it is needed (FP64 pairs, the epilogue)
// instead of occupying registers through the loop.
template <bool THERMO>
__device__ __forceinline__ void fp64_lj_i(const double4* __restrict__ pos, int i, int j, const LjArgs& a, double& cx,
                                          double& cy, double& cz, double& e, double& w, int& ncnt) {
    fp64_lj<THERMO>(ldg_d4(pos + i), j, pos, a, cx, cy, cz, e, w, ncnt);
}

// One FP32 pair of k_lj_mixed_bf: the rebasing shift from the entry's code, del, r^2 and, for a
// fast pair (close2 <= r^2 < rc2_lo), its force added without a branch; returns whether the pair
// takes the FP64 path (closer than close2, or within the window around the cutoff).
template <bool THERMO>
__device__ __forceinline__ bool mixed_pair(uint32_t en, const float4& ri, const float4& rj, const LjArgs& a,
                                           float& fx, float& fy, float& fz, float& ef, float& wf, int& ncnt) {
    float dx, dy, dz;
    const float rsq = mixed_del(en, ri, rj, a, dx, dy, dz);
    const bool fast = mixed_fast(rsq, a);
    float sr2, t;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(sr2) : "f"(rsq));
    float f = mixed_force(sr2, a, t);
    f = fast ? f : 0.f;
    fx = fmaf(dx, f, fx);
    fy = fmaf(dy, f, fy);
    fz = fmaf(dz, f, fz);
    if (THERMO) {
        ef += fast ? t * fmaf(a.lj_c, t, a.lj_d) : 0.f;
        wf = fmaf(f, rsq, wf);
        ncnt += fast ? 1 : 0;
    }
    return !fast && rsq < a.rc2_hi;
}

template <bool FUSE, bool THERMO, bool INIT = false, bool PUSH = false>
__global__ void __launch_bounds__(kThreads, TMD_MINB)
k_lj_mixed_bf(const float4* __restrict__ pos32, const double4* __restrict__ pos, float4* __restrict__ frc32,
              double4* __restrict__ vel, const int* __restrict__ nbn, const uint32_t* __restrict__ nbl,
              double* __restrict__ part, LjArgs a, double4* __restrict__ pos_n = nullptr,
              float4* __restrict__ pos32_n = nullptr, const int* __restrict__ rbk = nullptr,
              PushArgs pa = PushArgs()) {
    __shared__ double scratch[kThreads / 32];
    // each thread's queue of list quads holding FP64-path pairs: quad index << kB32 | pair bits;
    // row kQQ takes the writes past a full queue
    __shared__ int s_q[kQQ + 1][kThreads];
    if (INIT && lists_failed(a)) return;  // the whole grid returns: nothing written
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = i < a.N ? min(nbn[i], a.nbcap) : 0;
    prefetch_share(pos32, (size_t)a.NA * sizeof(float4));
    prefetch_share(pos, (size_t)a.N * sizeof(double4));
    if (FUSE) prefetch_share(vel, (size_t)a.N * sizeof(double4));
    if (INIT) prefetch_share(rbk, (size_t)((a.N + 3) & ~3) * sizeof(int));
    if (PUSH) prefetch_push(pa, a.N);
    double e = 0.0, w = 0.0, cnt = 0.0, ke = 0.0;
    if (i < a.N) {
        const float4 ri = pos32[i];
        float fx = 0.f, fy = 0.f, fz = 0.f, ef = 0.f, wf = 0.f;
        double cx = 0.0, cy = 0.0, cz = 0.0;
        int ncnt = 0;
        int nq = 0;  // list quads with FP64-path pairs, queued in s_q[0..nq)[threadIdx.x]
        // the last quad is padded with the atom itself one rebasing cell away on every axis
        // (rsq = 3h^2 with h above the list cutoff, beyond every window), so a padding entry
        // is neither a fast nor a queued pair and the loop needs no count test
        const int nquad = (n + 3) >> 2;
        uint4 eq = n > 0 ? list_quad(nbl, 0, i, a.stride) : make_uint4(0u, 0u, 0u, 0u);
        for (int b = 0; b < nquad; ++b) {
            const uint32_t cur[kB32] = {eq.x, eq.y, eq.z, eq.w};
            float4 rj[kB32];
#pragma unroll
            for (int u = 0; u < kB32; ++u) rj[u] = __ldg(pos32 + (cur[u] >> kCodeBits));
            // the next quad loads while this one's gathers are in flight
            eq = list_quad(nbl, b + 1, i, a.stride);  // the last read lands in the spare row
            unsigned slow = 0;
#pragma unroll
            for (int u = 0; u < kB32; ++u)
                slow |= mixed_pair<THERMO>(cur[u], ri, rj[u], a, fx, fy, fz, ef, wf, ncnt) ? (1u << u) : 0u;
            // a quad with FP64-path pairs is queued: the slot is written always, counted only then
            s_q[min(nq, kQQ)][threadIdx.x] = (b << kB32) | (int)slow;
            nq += slow != 0u ? 1 : 0;
        }
        if (nq > kQQ) {
            // more quads with FP64-path pairs than the queue holds (dense states): the atom is
            // redone with its FP64 pairs evaluated in place
            fx = fy = fz = ef = wf = 0.f;
            ncnt = 0;
            const double4 pi = ldg_d4(pos + i);
            for (int b = 0; b < nquad; ++b) {
                const uint4 e4 = list_quad(nbl, b, i, a.stride);
                const uint32_t c4[kB32] = {e4.x, e4.y, e4.z, e4.w};
                for (int u = 0; u < kB32; ++u) {
                    const int j = (int)(c4[u] >> kCodeBits);
                    if (mixed_pair<THERMO>(c4[u], ri, __ldg(pos32 + j), a, fx, fy, fz, ef, wf, ncnt))
                        fp64_lj<THERMO>(pi, j, pos, a, cx, cy, cz, e, w, ncnt);
                }
            }
        } else if (nq > 0) {
            // the FP64 pairs of the whole list, worked off together in list order: the warp's
            // lanes run them side by side instead of one lane at a time inside the loop
            const double4 pi = ldg_d4(pos + i);
            uint4 nx4 = list_quad(nbl, s_q[0][threadIdx.x] >> kB32, i, a.stride);
            for (int q = 0; q < nq; ++q) {
                const int wq = s_q[q][threadIdx.x];
                // the next queued quad loads while this one's pairs run (cold L2: 36.6 -> 35.8 us at 131k)
                const uint4 e4 = nx4;
                if (q + 1 < nq) nx4 = list_quad(nbl, s_q[q + 1][threadIdx.x] >> kB32, i, a.stride);
                unsigned bits = (unsigned)wq & ((1u << kB32) - 1u);
                while (bits) {
                    const int u = __ffs(bits) - 1;
                    bits &= bits - 1u;
                    const uint32_t en = u == 0 ? e4.x : (u == 1 ? e4.y : (u == 2 ? e4.z : e4.w));
                    fp64_lj<THERMO>(pi, (int)(en >> kCodeBits), pos, a, cx, cy, cz, e, w, ncnt);
                }
            }
        }
        const double Fx = (double)fx + cx, Fy = (double)fy + cy, Fz = (double)fz + cz;
        const float4 F = make_float4((float)Fx, (float)Fy, (float)Fz, 0.f);
        frc32[i] = F;
        if (FUSE) {
            double4 v = vel[i];
            v.x += (double)F.x * a.h;
            v.y += (double)F.y * a.h;
            v.z += (double)F.z * a.h;
            if (THERMO) ke = v.x * v.x + v.y * v.y + v.z * v.z;
            if (INIT) {
                double4 x = integrate_one(ldg_d4(pos + i), v, (double)F.x, (double)F.y, (double)F.z, a.dt_i, a.h_i);
                x.w = 0.0;  // positions carry w = 0
                pos_n[i] = x;
                pos32_n[i] = rebased32(x, rbk[i], a.alo, a.rb_h);
                if (PUSH) push_images<true>(i, x, a.N, pa, pos_n, pos32_n, a.alo, a.rb_h);
            }
            vel[i] = v;
        }
        if (THERMO) {
            e += (double)ef;
            w += (double)wf;
            cnt = (double)ncnt;
        }
    } else if (PUSH && i < a.N + (pa.nchain_dev ? *pa.nchain_dev : pa.nchain)) {
        push_chain<true>(i - a.N, pos, a.N, pa, pos_n, pos32_n, a.alo, a.rb_h);
    }
    if (THERMO) {
        put_partial(part, 0, e, scratch);
        put_partial(part, 1, w, scratch);
        put_partial(part, 2, cnt, scratch);
        if (FUSE) put_partial(part, 3, ke, scratch);
    }
}

// ---- DEM ----------------------------------------------------------------------
// core/runtime.impala:203-247.  With the reference condition the contact
// branch can never run (penetration r - 2R > 0 inside r < 2R); `fixed`
// selects the contact-fixed model (overlap 2R - r > 0, dissipative normal
// spring-dashpot, Coulomb-capped tangential dashpot), which needs ghost
// velocities (refreshed with the ghosts).
__device__ __forceinline__ void dem_pair(const double4& del, double rsq, const double4& v1, const double4& v2,
                                         const DemArgs& a, double* out) {
    out[0] = out[1] = out[2] = 0.0;
    const double radius = a.fixed ? a.radius : 1.0;
    const double d2 = dmul(radius, 2.0);
    if (!(rsq < dmul(d2, d2))) return;
    const double len = __dsqrt_rn(rsq);
    const double pen = dsub(len, d2);
    if (!a.fixed) {
        if (!(pen > 0.0)) return;
        const double il = ddiv(1.0, len);
        const double n[3] = {dmul(del.x, il), dmul(del.y, il), dmul(del.z, il)};
        const double rv[3] = {dsub(v1.x, v2.x), dsub(v1.y, v2.y), dsub(v1.z, v2.z)};
        const double vn = dadd(dadd(dmul(rv[0], n[0]), dmul(rv[1], n[1])), dmul(rv[2], n[2]));
        const double vt[3] = {dsub(rv[0], dmul(n[0], vn)), dsub(rv[1], dmul(n[1], vn)), dsub(rv[2], dmul(n[2], vn))};
        const double vtl = __dsqrt_rn(len2_strict(vt[0], vt[1], vt[2]));
        const double fn = dsub(dmul(a.dn, vn), dmul(a.k, pen));
        const double t1 = dmul(a.dt_, vtl), t2 = dmul(a.mu, fn);
        const double ft = t1 < t2 ? t1 : t2;
        const double iv = ddiv(1.0, vtl);
        for (int d = 0; d < 3; ++d) out[d] = dadd(dmul(n[d], fn), dmul(dmul(vt[d], iv), ft));
        return;
    }
    if (!(len > 0.0)) return;
    const double delta = dsub(d2, len);
    const double inv = ddiv(1.0, len);
    const double n[3] = {dmul(del.x, inv), dmul(del.y, inv), dmul(del.z, inv)};
    const double rv[3] = {dsub(v1.x, v2.x), dsub(v1.y, v2.y), dsub(v1.z, v2.z)};
    const double vn = dadd(dadd(dmul(rv[0], n[0]), dmul(rv[1], n[1])), dmul(rv[2], n[2]));
    const double vt[3] = {dsub(rv[0], dmul(n[0], vn)), dsub(rv[1], dmul(n[1], vn)), dsub(rv[2], dmul(n[2], vn))};
    const double vtl = __dsqrt_rn(len2_strict(vt[0], vt[1], vt[2]));
    double fn = dsub(dmul(a.k, delta), dmul(a.dn, vn));
    if (fn < 0.0) fn = 0.0;
    const double t1 = dmul(a.dt_, vtl), t2 = dmul(a.mu, fn);
    const double ft = t1 < t2 ? t1 : t2;
    const double tinv = vtl > 0.0 ? ddiv(1.0, vtl) : 0.0;
    for (int d = 0; d < 3; ++d) out[d] = dsub(dmul(n[d], fn), dmul(dmul(vt[d], tinv), ft));
}

template <bool HALF>
__global__ void __launch_bounds__(kThreads)
k_dem_fp64(const double4* __restrict__ pos, const double4* __restrict__ vel, double4* __restrict__ frc,
           const int* __restrict__ nbn, const uint32_t* __restrict__ nbl, const int* __restrict__ groot, DemArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.N) return;
    const double4 pi = pos[i];
    const double4 vi = vel[i];
    // the reference closure's pair force is exactly zero (r < 2R gives sqrt(r^2) <= 2R, so its
    // penetration test never passes): the loop would only add +0.0
    const int n = a.fixed ? min(nbn[i], a.nbcap) : 0;
    double F[3] = {0.0, 0.0, 0.0};
    uint4 eq = make_uint4(0u, 0u, 0u, 0u);
    for (int k = 0; k < n; ++k) {
        if ((k & 3) == 0) eq = list_quad(nbl, k >> 2, i, a.stride);
        const int j = (int)((k & 2 ? (k & 1 ? eq.w : eq.z) : (k & 1 ? eq.y : eq.x)) >> kCodeBits);
        const double4 pj = ldg_d4(pos + j);
        const double4 del = make_double4(dsub(pi.x, pj.x), dsub(pi.y, pj.y), dsub(pi.z, pj.z), 0.0);
        const double rsq = len2_strict(del.x, del.y, del.z);
        if (rsq < a.rc2) {
            double f[3];
            dem_pair(del, rsq, vi, ldg_d4(vel + j), a, f);
            F[0] = dadd(F[0], f[0]);
            F[1] = dadd(F[1], f[1]);
            F[2] = dadd(F[2], f[2]);
            if (HALF) {
                const int t = reaction_slot(j, a.N, groot);
                atomicAdd(&frc[t].x, -f[0]);
                atomicAdd(&frc[t].y, -f[1]);
                atomicAdd(&frc[t].z, -f[2]);
            }
        }
    }
    if (HALF) {
        atomicAdd(&frc[i].x, F[0]);
        atomicAdd(&frc[i].y, F[1]);
        atomicAdd(&frc[i].z, F[2]);
    } else {
        frc[i] = make_double4(F[0], F[1], F[2], 0.0);
    }
}

// Mixed DEM: the contact-fixed model's pair force in FP32 (same expression order
// as dem_pair) on rebased positions and FP32 relative velocities.  Pairs within a
// relative 1e-4 of the force cutoff or of the contact distance 2R take dem_pair
// in FP64, so both decisions are the FP64 ones.  The reference closure's force
// is zero (its contact branch is unreachable), as in k_dem_fp64.
struct DemMixedArgs {
    float rc2_lo, rc2_hi, c2_lo, c2_hi;  // margins around rc^2 and (2R)^2
    float d2, dn, dt_, k, mu;            // 2R and the model parameters
    float hx, hy, hz;                    // rebasing shift decode scales (as k_lj_mixed_bf)
};

template <bool HALF>
__global__ void __launch_bounds__(kThreads)
k_dem_mixed(const float4* __restrict__ pos32, const double4* __restrict__ pos, const double4* __restrict__ vel,
            float4* __restrict__ frc32, const int* __restrict__ nbn, const uint32_t* __restrict__ nbl,
            const int* __restrict__ groot, DemArgs a, DemMixedArgs b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.N) return;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    double cx = 0.0, cy = 0.0, cz = 0.0;
    if (a.fixed) {
        const float4 ri = pos32[i];
        const double4 vi = vel[i];
        const float vix = (float)vi.x, viy = (float)vi.y, viz = (float)vi.z;
        const int n = min(nbn[i], a.nbcap);
        uint4 eq = make_uint4(0u, 0u, 0u, 0u);
        for (int k = 0; k < n; ++k) {
            if ((k & 3) == 0) eq = list_quad(nbl, k >> 2, i, a.stride);
            const uint32_t en = k & 2 ? (k & 1 ? eq.w : eq.z) : (k & 1 ? eq.y : eq.x);
            const int j = (int)(en >> kCodeBits);
            const float4 rj = __ldg(pos32 + j);
            const float sx = __int_as_float((int)((en & 0x03u) | 0x4B000000u)) - 8388609.0f;
            const float sy = __int_as_float((int)((en & 0x0Cu) | 0x4B000000u)) - 8388612.0f;
            const float sz = __int_as_float((int)((en & 0x30u) | 0x4B000000u)) - 8388624.0f;
            const float dx = fmaf(b.hx, sx, ri.x - rj.x);
            const float dy = fmaf(b.hy, sy, ri.y - rj.y);
            const float dz = fmaf(b.hz, sz, ri.z - rj.z);
            const float rsq = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (!(rsq < b.rc2_hi) || !(rsq < b.c2_hi)) continue;  // beyond the cutoff or no contact
            if (rsq >= b.rc2_lo || rsq >= b.c2_lo) {
                // near a decision: the FP64 pair
                const double4 pi = pos[i], pj = pos[j];
                const double4 del = make_double4(dsub(pi.x, pj.x), dsub(pi.y, pj.y), dsub(pi.z, pj.z), 0.0);
                const double r2 = len2_strict(del.x, del.y, del.z);
                if (r2 < a.rc2) {
                    double o[3];
                    dem_pair(del, r2, vi, ldg_d4(vel + j), a, o);
                    cx += o[0];
                    cy += o[1];
                    cz += o[2];
                    if (HALF) {
                        const int t = reaction_slot(j, a.N, groot);
                        add_force32(frc32 + t, (float)(-o[0]), (float)(-o[1]), (float)(-o[2]));
                    }
                }
                continue;
            }
            const double4 vj = ldg_d4(vel + j);
            // |del| and 1/|del| from one reciprocal square root (against a rounded square root and
            // a division: the force 33.0 -> 28.9 us on the 48^3 FCC split)
            if (!(rsq > 0.f)) continue;
            const float inv = rsqrtf(rsq);
            const float len = rsq * inv;
            const float delta = b.d2 - len;
            const float nx = dx * inv, ny = dy * inv, nz = dz * inv;
            const float rvx = vix - (float)vj.x, rvy = viy - (float)vj.y, rvz = viz - (float)vj.z;
            const float vn = rvx * nx + rvy * ny + rvz * nz;
            const float vtx = rvx - nx * vn, vty = rvy - ny * vn, vtz = rvz - nz * vn;
            const float vt2 = vtx * vtx + vty * vty + vtz * vtz;
            const float tinv = vt2 > 0.f ? rsqrtf(vt2) : 0.f;
            const float vtl = vt2 * tinv;
            float fn = b.k * delta - b.dn * vn;
            if (fn < 0.f) fn = 0.f;
            const float t1 = b.dt_ * vtl, t2 = b.mu * fn;
            const float ft = t1 < t2 ? t1 : t2;
            const float px = nx * fn - vtx * tinv * ft;
            const float py = ny * fn - vty * tinv * ft;
            const float pz = nz * fn - vtz * tinv * ft;
            fx += px;
            fy += py;
            fz += pz;
            if (HALF) {
                const int t = reaction_slot(j, a.N, groot);
                add_force32(frc32 + t, -px, -py, -pz);
            }
        }
    }
    const float Fx = (float)((double)fx + cx), Fy = (float)((double)fy + cy), Fz = (float)((double)fz + cz);
    if (HALF) {
        add_force32(frc32 + i, Fx, Fy, Fz);
    } else {
        frc32[i] = make_float4(Fx, Fy, Fz, 0.f);
    }
}

// ---- integration + ghost refresh ------------------------------------------------
// GM: 0 = locals only, ghost positions carried over unchanged;
//     1 = reference two-phase refresh: ghost = (its source's value in this
//         step) + one shift, where a local source is integrated here and a
//         ghost source still holds the previous step's value (so chained
//         edge / corner ghosts lag, exactly like comm/comm.impala:334-388);
//     2 = exact periodic images: ghost = integrated root + total shift.

// v += h f in the reference's operand order (core/compute.impala:108-116), as k_final does it
__device__ __forceinline__ void kick(double4& v, double fx, double fy, double fz, double h) {
    v.x = dadd(v.x, dmul(fx, h));
    v.y = dadd(v.y, dmul(fy, h));
    v.z = dadd(v.z, dmul(fz, h));
}

template <bool MIXED>
__device__ __forceinline__ void load_force(const double4* frc, const float4* frc32, int i, double& fx, double& fy,
                                           double& fz) {
    if (MIXED) {
        const float4 f = frc32[i];
        fx = f.x; fy = f.y; fz = f.z;
    } else {
        const double4 f = frc[i];
        fx = f.x; fy = f.y; fz = f.z;
    }
}

template <int GM, bool MIXED, bool DEMV>
__global__ void __launch_bounds__(kThreads)
k_integrate(const double4* __restrict__ pos_o, double4* __restrict__ pos_n, const double4* __restrict__ vel_o,
            double4* __restrict__ vel_n, const double4* __restrict__ frc, const float4* __restrict__ frc32,
            const float4* __restrict__ pos32_o, float4* __restrict__ pos32_n, const int* __restrict__ rbk,
            const int* __restrict__ gsrc, const int* __restrict__ groot, const int* __restrict__ gcode, StepArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < a.N) {
        double4 v = vel_o[t];
        double fx, fy, fz;
        load_force<MIXED>(frc, frc32, t, fx, fy, fz);
        if (a.pre) kick(v, fx, fy, fz, a.hp);
        const double4 x = integrate_one(pos_o[t], v, fx, fy, fz, a.dt, a.h);
        pos_n[t] = x;
        vel_n[t] = v;
        if (MIXED) pos32_n[t] = rebased32(x, rbk[t], a.alo, a.rb_h);
        return;
    }
    if (t >= a.N + a.G) return;
    const int g = t - a.N;
    if (GM == 0) {
        pos_n[t] = pos_o[t];
        if (MIXED) pos32_n[t] = pos32_o[t];
        if (DEMV) vel_n[t] = vel_o[t];
        return;
    }
    const int s = GM == 1 ? gsrc[g] : groot[g];
    if (s < 0) return;  // a ghost received from another rank: the halo exchange refreshes it
    const int code = gcode[g];
    double4 xs;
    if (s < a.N) {
        double4 vs = vel_o[s];
        double fx, fy, fz;
        load_force<MIXED>(frc, frc32, s, fx, fy, fz);
        if (a.pre) kick(vs, fx, fy, fz, a.hp);
        xs = integrate_one(pos_o[s], vs, fx, fy, fz, a.dt, a.h);
    } else {
        xs = pos_o[s];
    }
    const int base = GM == 1 ? 0 : 8;
    double4 x;
    x.x = dadd(xs.x, dmul(a.len[0], (double)shift_axis(code, base, 0)));
    x.y = dadd(xs.y, dmul(a.len[1], (double)shift_axis(code, base, 1)));
    x.z = dadd(xs.z, dmul(a.len[2], (double)shift_axis(code, base, 2)));
    x.w = 0.0;
    pos_n[t] = x;
    if (MIXED) pos32_n[t] = rebased32(x, rbk[t], a.alo, a.rb_h);
    if (DEMV) {  // contact-fixed DEM: ghost velocity = its root's, after this half-kick
        const int r = groot[g];
        double4 vr = vel_o[r];
        double fx, fy, fz;
        load_force<MIXED>(frc, frc32, r, fx, fy, fz);
        if (a.pre) kick(vr, fx, fy, fz, a.hp);
        kick(vr, fx, fy, fz, a.h);
        vel_n[t] = vr;
    }
}

// stand-alone ghost refresh (no pending integration): locals carried over
template <int GM, bool MIXED>
__global__ void __launch_bounds__(kThreads)
k_ghost_sync(const double4* __restrict__ pos_o, double4* __restrict__ pos_n, const float4* __restrict__ pos32_o,
             float4* __restrict__ pos32_n, double4* __restrict__ vel, int demv, const int* __restrict__ rbk,
             const int* __restrict__ gsrc, const int* __restrict__ groot, const int* __restrict__ gcode,
             StepArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < a.N) {
        pos_n[t] = pos_o[t];
        if (MIXED) pos32_n[t] = pos32_o[t];
        return;
    }
    if (t >= a.N + a.G) return;
    const int g = t - a.N;
    const int s = GM == 1 ? gsrc[g] : groot[g];
    if (s < 0) return;  // received from another rank (halo exchange)
    const int code = gcode[g];
    const double4 xs = pos_o[s];
    const int base = GM == 1 ? 0 : 8;
    double4 x;
    x.x = dadd(xs.x, dmul(a.len[0], (double)shift_axis(code, base, 0)));
    x.y = dadd(xs.y, dmul(a.len[1], (double)shift_axis(code, base, 1)));
    x.z = dadd(xs.z, dmul(a.len[2], (double)shift_axis(code, base, 2)));
    x.w = 0.0;
    pos_n[t] = x;
    if (MIXED) pos32_n[t] = rebased32(x, rbk[t], a.alo, a.rb_h);
    if (demv) vel[t] = vel[groot[g]];  // ghost slots only; roots are locals
}

// ghosts after a force kernel that also did the next initial integration of the locals
// (k_lj_*<.., INIT>): pos_n/pos32_n hold the new locals, pos_o the previous buffer.
// GM 0 carries the ghosts over; 1 and 2 give exactly what k_integrate<1|2> computes, since
// the new local equals its on-the-fly integration there.
template <int GM, bool MIXED>
__global__ void __launch_bounds__(kThreads)
k_ghost_refresh(const double4* __restrict__ pos_o, double4* __restrict__ pos_n, const float4* __restrict__ pos32_o,
                float4* __restrict__ pos32_n, const int* __restrict__ rbk, const int* __restrict__ gsrc,
                const int* __restrict__ groot, const int* __restrict__ gcode, StepArgs a) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.G) return;
    const int t = a.N + g;
    if (GM == 0) {
        pos_n[t] = pos_o[t];
        if (MIXED) pos32_n[t] = pos32_o[t];
        return;
    }
    const int s = GM == 1 ? gsrc[g] : groot[g];
    if (s < 0) return;  // received from another rank (halo exchange)
    const int code = gcode[g];
    const double4 xs = s < a.N ? pos_n[s] : pos_o[s];
    const int base = GM == 1 ? 0 : 8;
    double4 x;
    x.x = dadd(xs.x, dmul(a.len[0], (double)shift_axis(code, base, 0)));
    x.y = dadd(xs.y, dmul(a.len[1], (double)shift_axis(code, base, 1)));
    x.z = dadd(xs.z, dmul(a.len[2], (double)shift_axis(code, base, 2)));
    x.w = 0.0;
    pos_n[t] = x;
    if (MIXED) pos32_n[t] = rebased32(x, rbk[t], a.alo, a.rb_h);
}

template <bool MIXED, bool THERMO>
__global__ void __launch_bounds__(kThreads)
k_final(double4* __restrict__ vel, const double4* __restrict__ frc, const float4* __restrict__ frc32,
        double* __restrict__ part, int N, double h) {
    __shared__ double scratch[kThreads / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ke = 0.0;
    if (i < N) {
        double fx, fy, fz;
        load_force<MIXED>(frc, frc32, i, fx, fy, fz);
        double4 v = vel[i];
        v.x = dadd(v.x, dmul(fx, h));
        v.y = dadd(v.y, dmul(fy, h));
        v.z = dadd(v.z, dmul(fz, h));
        vel[i] = v;
        if (THERMO) ke = v.x * v.x + v.y * v.y + v.z * v.z;
    }
    if (THERMO) put_partial(part, 3, ke, scratch);
}

// List pairs inside the force cutoff (rsq < rc^2 in the reference's FP64 evaluation order):
// the reference's rsq_iters of the last force call (core/runtime.impala:188-201, 203-247),
// counted on demand at report time from the lists and positions that call used.
__global__ void k_count_inside(const double4* __restrict__ pos, const int* __restrict__ nbn,
                               const uint32_t* __restrict__ nbl, int N, int stride, int nbcap, double rc2,
                               unsigned long long* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned c = 0;
    if (i < N) {
        const double4 pi = pos[i];
        const int n = min(nbn[i], nbcap);
        for (int k = 0; k < n; ++k) {
            const double4 pj = ldg_d4(pos + (int)(nbl[nl_index(k, i, stride)] >> kCodeBits));
            c += len2_strict(dsub(pi.x, pj.x), dsub(pi.y, pj.y), dsub(pi.z, pj.z)) < rc2 ? 1u : 0u;
        }
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, (unsigned long long)c);
}

__global__ void k_refresh_pos32(const double4* __restrict__ pos, float4* __restrict__ pos32,
                                const int* __restrict__ rbk, int NA, StepArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < NA) pos32[t] = rebased32(pos[t], rbk[t], a.alo, a.rb_h);
}

__global__ void k_zero4(double4* __restrict__ d, float4* __restrict__ f, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    if (d) d[t] = make_double4(0.0, 0.0, 0.0, 0.0);
    if (f) f[t] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// sums part[q][0..nb) in a fixed order for q in [q0, q1) into out[q]
__global__ void k_reduce_partials(const double* __restrict__ part, double* __restrict__ out, int nb, int q0,
                                  int q1) {
    __shared__ double scratch[32];
    for (int q = q0; q < q1; ++q) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) v += part[q * nb + b];
        double r = block_sum(v, scratch);
        if (threadIdx.x == 0) out[q] = r;
    }
}

StepArgs step_args(const State& s, double dt) {
    StepArgs a;
    a.N = s.N;
    a.G = s.G;
    a.stride = s.nb_stride;
    a.dt = dt;
    a.h = 0.5 * dt;
    for (int d = 0; d < 3; ++d) {
        a.len[d] = s.geo.len[d];
        a.alo[d] = s.geo.aabb_lo[d];
    }
    a.rb_h = s.geo.rb_h;
    a.pre = 0;
    a.hp = 0.0;
    return a;
}

// INIT: the kernels write the integrated locals into the other position buffer
template <bool HALF, bool FUSE, bool THERMO, bool INIT = false, bool PUSH = false>
void launch_lj(State& s, const LjArgs& a, int nb, const PushArgs& pa = PushArgs()) {
    double4* vel = s.vel.b[s.vc];
    double4* pn = INIT ? s.pos.b[1 - s.pc] : nullptr;
    if (s.precision == 1) {
        if constexpr (HALF)
            k_lj_mixed_half<THERMO><<<nb, kThreads, 0, s.stream>>>(s.pos32.b[s.pc], s.pos.b[s.pc], s.frc32, s.nbn,
                                                                   s.nbl, s.groot, s.red_part, a);
        else
            k_lj_mixed_bf<FUSE, THERMO, INIT, PUSH><<<nb, kThreads, 0, s.stream>>>(
                s.pos32.b[s.pc], s.pos.b[s.pc], s.frc32, vel, s.nbn, s.nbl, s.red_part, a, pn,
                INIT ? s.pos32.b[1 - s.pc] : nullptr, s.rbk, pa);
    } else
        k_lj_fp64<HALF, FUSE, THERMO, INIT, PUSH><<<nb, kThreads, 0, s.stream>>>(
            s.pos.b[s.pc], s.frc.b[s.ac], vel, s.nbn, s.nbl, s.groot, s.red_part, a, pn, pa);
}

}  // namespace

void ensure_red_scratch(State& s, int n) {
    if (n > s.red_part_cap) {
        dfree(&s.red_part);
        s.red_part_cap = n + 1024;
        dalloc(&s.red_part, s.red_part_cap);
    }
}

void run_reduce_thermo(State& s, int nb, int nq) {
    (void)nq;
    k_reduce_partials<<<1, 256, 0, s.stream>>>(s.red_part, s.thermo_dev, nb, 0, kThermoQ);
    launched(K_REDUCE);
}

void run_reduce_partials(State& s, int nb, int q0, int q1) {
    k_reduce_partials<<<1, 256, 0, s.stream>>>(s.red_part, s.thermo_dev, nb, q0, q1);
    launched(K_REDUCE);
}

// The mixed kernel pads a batch with the atom itself one rebasing cell away on every
// axis (rsq = 3h^2), which must lie beyond the cutoff window; h exceeds the cell
// spacing, so only a cutoff beyond sqrt(3) cell spacings (where the 27-cell stencil
// misses pairs anyway) breaks this.  Latches MD_ERR_ARGUMENT (3).
void check_mixed_cutoff(const State& s, const LjArgs& a) {
    if (3.0 * s.geo.rb_h * s.geo.rb_h <= (double)a.rc2_hi)
        set_error(3, "mixed form: LJ cutoff beyond sqrt(3) cell spacings");
}

// A list entry's code holds one rebasing-cell step per axis, which needs every listed pair
// closer than the rebasing spacing (above the cell spacing): a list cutoff beyond it, or a
// grid too wide for the packed cells, leaves the mixed form's codes invalid.  Latches 3.
bool mixed_lists_ok(const State& s) {
    const Geometry& g = s.geo;
    bool ok = s.lists_cutoff < g.rb_h;
    for (int d = 0; d < 3; ++d) ok = ok && (g.aabb_hi[d] - g.aabb_lo[d]) / g.rb_h < 1000.0;
    if (!ok) set_error(3, "mixed form: list cutoff beyond the rebasing spacing or grid too wide");
    return ok;
}

void run_force_lj(State& s, const PendingForce& p, bool fuse_final, double dt) {
    const int N = s.N;
    if (N == 0) return;
    LjArgs a = lj_args(s, p, dt);
    if (s.precision == 1 && !p.half) check_mixed_cutoff(s, a);
    if (s.precision == 1) mixed_lists_ok(s);
    // the list entry's code holds dk + 1 in bits 0-1 (x), 2-3 (y), 4-5 (z)
    a.hx = (float)(-s.geo.rb_h);
    a.hy = (float)(-s.geo.rb_h / 4.0);
    a.hz = (float)(-s.geo.rb_h / 16.0);
    const int nb = nblocks(N, kThreads);
    const bool half = p.half;
    const bool thermo = s.thermo != 0;
    if (thermo) ensure_red_scratch(s, kThermoQ * nb);
    if (half) {
        if (s.precision == 1)
            k_zero4<<<nblocks(N, kThreads), kThreads, 0, s.stream>>>(nullptr, s.frc32, N);
        else
            k_zero4<<<nblocks(N, kThreads), kThreads, 0, s.stream>>>(s.frc.b[s.ac], nullptr, N);
        launched(K_MISC);
        fuse_final = false;
    }
    prof_begin(K_FORCE_LJ);
    if (half) {
        if (thermo) launch_lj<true, false, true>(s, a, nb);
        else launch_lj<true, false, false>(s, a, nb);
    } else if (fuse_final) {
        if (thermo) launch_lj<false, true, true>(s, a, nb);
        else launch_lj<false, true, false>(s, a, nb);
    } else {
        if (thermo) launch_lj<false, false, true>(s, a, nb);
        else launch_lj<false, false, false>(s, a, nb);
    }
    launched(K_FORCE_LJ);
    prof_end(K_FORCE_LJ);
    if (fuse_final) s.integration_iters = N;
    if (thermo) {
        if (!fuse_final) {
            // energy/virial only; the kinetic partial comes from the next final kick
            k_reduce_partials<<<1, 256, 0, s.stream>>>(s.red_part, s.thermo_dev, nb, 0, 3);
        } else {
            k_reduce_partials<<<1, 256, 0, s.stream>>>(s.red_part, s.thermo_dev, nb, 0, kThermoQ);
        }
        launched(K_REDUCE);
    }
}

bool force_init_fusable(const State& s, const PendingForce& p) {
    // ghost velocities of the contact-fixed DEM model come from k_integrate
    return !p.dem && !p.half && !s.lists_half && s.dem_fixed == 0;
}

void run_force_lj_init(State& s, const PendingForce& p, double dt_final, double dt_init) {
    const int N = s.N;
    if (N == 0) {
        resolve_lists(s);
        return;  // no ghosts either
    }
    LjArgs a = lj_args(s, p, dt_final);
    if (s.precision == 1) {
        check_mixed_cutoff(s, a);
        mixed_lists_ok(s);
    }
    a.hx = (float)(-s.geo.rb_h);
    a.hy = (float)(-s.geo.rb_h / 4.0);
    a.hz = (float)(-s.geo.rb_h / 16.0);
    a.dt_i = dt_init;
    a.h_i = 0.5 * dt_init;
    // Right after a list build whose status is still in flight the kernel runs on the lists at
    // once: it returns without writing if that build failed, the two-phase chain count comes
    // from the device, and the image maps are taken as complete (checked below).
    const bool spec = s.status_pending;
    if (spec) a.spec = s.status_dev;
    // the ghosts of the current mode are written too when the image maps are complete
    const int gm = s.ghost_exact ? 2 : 1;
    const bool push = s.G > 0 && (spec || ((s.img_ok >> (gm - 1)) & 1));
    PushArgs pa;
    if (push) {
        pa.slot = s.img_slot + (gm == 2 ? (size_t)kImg1 * s.capA : 0);
        pa.planes = gm == 2 ? kImg2 : kImg1;
        pa.plane = s.capA;
        pa.G = s.G;
        pa.chain = s.chain;
        pa.gsrc = s.gsrc;
        pa.gcode = s.gcode;
        pa.rbk = s.rbk;
        pa.nchain = gm == 1 ? (spec ? s.G : s.nchain) : 0;
        if (spec && gm == 1) pa.nchain_dev = &s.status_dev->nchain;
        pa.base = gm == 1 ? 0 : 8;
        for (int d = 0; d < 3; ++d) pa.len[d] = s.geo.len[d];
    }
    const int nb = nblocks(N + pa.nchain, kThreads);
    const bool thermo = s.thermo != 0;
    if (thermo) ensure_red_scratch(s, kThermoQ * nb);
    prof_begin(K_FORCE_LJ);
    if (push) {
        if (thermo) launch_lj<false, true, true, true, true>(s, a, nb, pa);
        else launch_lj<false, true, false, true, true>(s, a, nb, pa);
    } else {
        if (thermo) launch_lj<false, true, true, true>(s, a, nb);
        else launch_lj<false, true, false, true>(s, a, nb);
    }
    launched(K_FORCE_LJ);
    prof_end(K_FORCE_LJ);
    bool pushed = push;
    if (spec) {
        const int r = resolve_lists(s);
        if (r != 0) {
            // the kernel returned without writing: the lists are rebuilt (or the error latched)
            if (r > 0) run_force_lj_init(s, p, dt_final, dt_init);
            return;
        }
        pushed = push && ((s.img_ok >> (gm - 1)) & 1);  // incomplete maps: the ghosts are refreshed
    }
    s.pc = 1 - s.pc;  // the locals of the other buffer are current; its ghosts follow
    s.ghosts_pushed = (pushed || s.G == 0) ? gm : 0;
    s.integration_iters = N;
    if (thermo) {
        k_reduce_partials<<<1, 256, 0, s.stream>>>(s.red_part, s.thermo_dev, nb, 0, kThermoQ);
        launched(K_REDUCE);
    }
}

void run_ghost_refresh(State& s, int gm) {
    if (s.G == 0) return;
    StepArgs a = step_args(s, 0.0);
    const double4* po = s.pos.b[1 - s.pc];
    double4* pn = s.pos.b[s.pc];
    const float4* p32o = s.pos32.b[1 - s.pc];
    float4* p32n = s.pos32.b[s.pc];
    const int nb = nblocks(s.G, kThreads);
    const bool mixed = s.precision == 1;
#define TMD_GR(GM_, MX_) \
    k_ghost_refresh<GM_, MX_><<<nb, kThreads, 0, s.stream>>>(po, pn, p32o, p32n, s.rbk, s.gsrc, s.groot, s.gcode, a)
    prof_begin(K_GHOST_SYNC);
    if (gm == 0) { if (mixed) TMD_GR(0, true); else TMD_GR(0, false); }
    else if (gm == 1) { if (mixed) TMD_GR(1, true); else TMD_GR(1, false); }
    else { if (mixed) TMD_GR(2, true); else TMD_GR(2, false); }
#undef TMD_GR
    launched(K_GHOST_SYNC);
    prof_end(K_GHOST_SYNC);
}

void run_force_dem(State& s, const PendingForce& p) {
    const int N = s.N;
    if (N == 0) return;
    DemArgs a;
    a.N = N;
    a.stride = s.nb_stride;
    a.nbcap = s.nb_cap;
    a.fixed = s.dem_fixed;
    a.rc2 = p.rc * p.rc;
    a.dn = p.dn;
    a.dt_ = p.dt_;
    a.k = p.k;
    a.mu = p.mu;
    a.radius = s.dem_radius;
    if (s.precision == 1) {  // the mixed form's integrators read frc32
        mixed_lists_ok(s);
        DemMixedArgs b;
        const double d2 = 2.0 * (s.dem_fixed ? s.dem_radius : 1.0);
        b.rc2_lo = (float)(a.rc2 * (1.0 - 1e-4));
        b.rc2_hi = (float)(a.rc2 * (1.0 + 1e-4));
        b.c2_lo = (float)(d2 * d2 * (1.0 - 1e-4));
        b.c2_hi = (float)(d2 * d2 * (1.0 + 1e-4));
        b.d2 = (float)d2;
        b.dn = (float)p.dn;
        b.dt_ = (float)p.dt_;
        b.k = (float)p.k;
        b.mu = (float)p.mu;
        b.hx = (float)(-s.geo.rb_h);
        b.hy = (float)(-s.geo.rb_h / 4.0);
        b.hz = (float)(-s.geo.rb_h / 16.0);
        if (p.half) {
            k_zero4<<<nblocks(N, kThreads), kThreads, 0, s.stream>>>(nullptr, s.frc32, N);
            launched(K_MISC);
        }
        prof_begin(K_FORCE_DEM);
        if (p.half)
            k_dem_mixed<true><<<nblocks(N, kThreads), kThreads, 0, s.stream>>>(
                s.pos32.b[s.pc], s.pos.b[s.pc], s.vel.b[s.vc], s.frc32, s.nbn, s.nbl, s.groot, a, b);
        else
            k_dem_mixed<false><<<nblocks(N, kThreads), kThreads, 0, s.stream>>>(
                s.pos32.b[s.pc], s.pos.b[s.pc], s.vel.b[s.vc], s.frc32, s.nbn, s.nbl, s.groot, a, b);
        launched(K_FORCE_DEM);
        prof_end(K_FORCE_DEM);
        return;
    }
    if (p.half) {
        k_zero4<<<nblocks(N, kThreads), kThreads, 0, s.stream>>>(s.frc.b[s.ac], nullptr, N);
        launched(K_MISC);
    }
    prof_begin(K_FORCE_DEM);
    if (p.half)
        k_dem_fp64<true><<<nblocks(N, kThreads), kThreads, 0, s.stream>>>(s.pos.b[s.pc], s.vel.b[s.vc],
                                                                          s.frc.b[s.ac], s.nbn, s.nbl, s.groot, a);
    else
        k_dem_fp64<false><<<nblocks(N, kThreads), kThreads, 0, s.stream>>>(s.pos.b[s.pc], s.vel.b[s.vc],
                                                                           s.frc.b[s.ac], s.nbn, s.nbl, s.groot, a);
    launched(K_FORCE_DEM);
    prof_end(K_FORCE_DEM);
}

void run_integrate(State& s, double dt, bool fuse_ghosts, double kick_dt) {
    const int NA = s.N + s.G;
    if (NA == 0) return;
    StepArgs a = step_args(s, dt);
    if (kick_dt >= 0.0) {  // the previous step's final kick first (k_final's arithmetic)
        a.pre = 1;
        a.hp = 0.5 * kick_dt;
    }
    const int gm = fuse_ghosts ? (s.ghost_exact ? 2 : 1) : 0;
    const bool mixed = s.precision == 1;
    const bool demv = s.dem_fixed != 0;
    const double4* po = s.pos.b[s.pc];
    double4* pn = s.pos.b[1 - s.pc];
    const double4* vo = s.vel.b[s.vc];
    double4* vn = s.vel.b[1 - s.vc];
    const float4* p32o = s.pos32.b[s.pc];
    float4* p32n = s.pos32.b[1 - s.pc];
    const int nb = nblocks(NA, kThreads);
#define TMD_INT(GM_, MX_, DV_)                                                                                 \
    k_integrate<GM_, MX_, DV_><<<nb, kThreads, 0, s.stream>>>(po, pn, vo, vn, s.frc.b[s.ac], s.frc32, p32o, p32n,  \
                                                              s.rbk, s.gsrc, s.groot, s.gcode, a)
    prof_begin(K_INTEGRATE);
    if (gm == 0) {
        if (mixed) { if (demv) TMD_INT(0, true, true); else TMD_INT(0, true, false); }
        else { if (demv) TMD_INT(0, false, true); else TMD_INT(0, false, false); }
    } else if (gm == 1) {
        if (mixed) { if (demv) TMD_INT(1, true, true); else TMD_INT(1, true, false); }
        else { if (demv) TMD_INT(1, false, true); else TMD_INT(1, false, false); }
    } else {
        if (mixed) { if (demv) TMD_INT(2, true, true); else TMD_INT(2, true, false); }
        else { if (demv) TMD_INT(2, false, true); else TMD_INT(2, false, false); }
    }
#undef TMD_INT
    launched(K_INTEGRATE);
    prof_end(K_INTEGRATE);
    s.pc = 1 - s.pc;
    s.vc = 1 - s.vc;
    s.integration_iters = s.N;
}

void run_ghost_sync(State& s) {
    const int NA = s.N + s.G;
    if (NA == 0) return;
    StepArgs a = step_args(s, 0.0);
    const double4* po = s.pos.b[s.pc];
    double4* pn = s.pos.b[1 - s.pc];
    const float4* p32o = s.pos32.b[s.pc];
    float4* p32n = s.pos32.b[1 - s.pc];
    const int nb = nblocks(NA, kThreads);
    prof_begin(K_GHOST_SYNC);
    if (s.ghost_exact) {
        if (s.precision == 1) k_ghost_sync<2, true><<<nb, kThreads, 0, s.stream>>>(po, pn, p32o, p32n, s.vel.b[s.vc], s.dem_fixed, s.rbk, s.gsrc, s.groot, s.gcode, a);
        else k_ghost_sync<2, false><<<nb, kThreads, 0, s.stream>>>(po, pn, p32o, p32n, s.vel.b[s.vc], s.dem_fixed, s.rbk, s.gsrc, s.groot, s.gcode, a);
    } else {
        if (s.precision == 1) k_ghost_sync<1, true><<<nb, kThreads, 0, s.stream>>>(po, pn, p32o, p32n, s.vel.b[s.vc], s.dem_fixed, s.rbk, s.gsrc, s.groot, s.gcode, a);
        else k_ghost_sync<1, false><<<nb, kThreads, 0, s.stream>>>(po, pn, p32o, p32n, s.vel.b[s.vc], s.dem_fixed, s.rbk, s.gsrc, s.groot, s.gcode, a);
    }
    launched(K_GHOST_SYNC);
    prof_end(K_GHOST_SYNC);
    s.pc = 1 - s.pc;
}

void run_final(State& s, double dt) {
    const int N = s.N;
    if (N == 0) return;
    const int nb = nblocks(N, kThreads);
    const bool thermo = s.thermo != 0;
    if (thermo) ensure_red_scratch(s, kThermoQ * nb);
    prof_begin(K_FINAL);
    const double h = 0.5 * dt;
    if (s.precision == 1) {
        if (thermo) k_final<true, true><<<nb, kThreads, 0, s.stream>>>(s.vel.b[s.vc], s.frc.b[s.ac], s.frc32, s.red_part, N, h);
        else k_final<true, false><<<nb, kThreads, 0, s.stream>>>(s.vel.b[s.vc], s.frc.b[s.ac], s.frc32, s.red_part, N, h);
    } else {
        if (thermo) k_final<false, true><<<nb, kThreads, 0, s.stream>>>(s.vel.b[s.vc], s.frc.b[s.ac], s.frc32, s.red_part, N, h);
        else k_final<false, false><<<nb, kThreads, 0, s.stream>>>(s.vel.b[s.vc], s.frc.b[s.ac], s.frc32, s.red_part, N, h);
    }
    launched(K_FINAL);
    prof_end(K_FINAL);
    if (thermo) {
        k_reduce_partials<<<1, 256, 0, s.stream>>>(s.red_part, s.thermo_dev, nb, 3, 4);
        launched(K_REDUCE);
    }
    s.integration_iters = N;
}

void run_refresh_pos32(State& s) {
    const int NA = s.N + s.G;
    if (NA == 0) return;
    StepArgs a = step_args(s, 0.0);
    k_refresh_pos32<<<nblocks(NA, kThreads), kThreads, 0, s.stream>>>(s.pos.b[s.pc], s.pos32.b[s.pc], s.rbk, NA, a);
    launched(K_MISC);
}

long long count_pairs_inside(State& s, double rc) {
    if (s.N == 0 || !s.lists_valid) return 0;
    unsigned long long* d = reinterpret_cast<unsigned long long*>(s.thermo_dev + 6);  // spare words
    TMD_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), s.stream));
    k_count_inside<<<nblocks(s.N, kThreads), kThreads, 0, s.stream>>>(s.pos.b[s.pc], s.nbn, s.nbl, s.N, s.nb_stride,
                                                                      s.nb_cap, rc * rc, d);
    launched(K_MISC);
    unsigned long long h = 0;
    TMD_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s.stream));
    TMD_CUDA(cudaStreamSynchronize(s.stream));
    return (long long)h;
}

}  // namespace tmd
