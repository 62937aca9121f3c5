// noalloc.cu -- LJ forces with energy / virial sums that allocate no device memory.
//
// Some callers cannot call cudaMalloc: code running inside another
// framework's memory pool (which forbids allocations outside it), code
// executing while a CUDA graph is being captured by someone else, or
// embedded hosts with a fixed memory budget.  The regular path keeps its
// per-block partial sums in memory the library allocates; this variant keeps
// them in a file-scope device array of fixed size instead, so a call only
// launches kernels on the caller's stream and touches the caller's buffers.
//
// The array is sized for kNoAllocMaxBlocks blocks of kNoAllocThreads atoms
// (1,048,576 local atoms); larger systems are rejected.  It lives in every
// GPU that loads the library until the process exits.  Every call shares it
// and it keeps the last call's contents; each call overwrites exactly the
// entries it then reads, so nothing needs clearing -- but two calls whose
// kernels overlap on the GPU (different streams, no ordering) race on it.

#include <cstdio>

#include "md_common.cuh"
#include "md_state.h"
#include "tinymd_b200.h"

namespace tmd {
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxBlocks = 4096;
constexpr int kNoAllocQ = 3;  // energy, virial, pairs inside the cutoff

// per-block partial sums, quantity-major: [kNoAllocQ][kNoAllocMaxBlocks]
static __device__ __align__(256) double g_noalloc_partials[kNoAllocQ * kNoAllocMaxBlocks];

// device address of g_noalloc_partials, looked up once per device; a device reset (or a
// primary context destroyed and made again) invalidates it, so such a reset needs the library
// to be loaded again before this entry point is called
constexpr int kMaxDevices = 64;
void* g_partials_addr[kMaxDevices] = {nullptr};

struct NoAllocArgs {
    int n, stride, max_nb;
    double rc2, sigma6, eps;
};

// The FP64 LJ force of k_lj_fp64 (full list, no fused kick, with thermo): same
// operand order, so the forces equal the regular path bit for bit on the same
// list.  List entries are plain neighbour indices here.
__global__ void __launch_bounds__(kNoAllocThreads)
k_lj_fp64_noalloc(const double4* __restrict__ pos, const int* __restrict__ nbn, const int* __restrict__ nbl,
                  double4* __restrict__ frc, double* __restrict__ part, NoAllocArgs a) {
    __shared__ double scratch[kNoAllocThreads / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0, w = 0.0, cnt = 0.0;
    if (i < a.n) {
        const double4 pi = pos[i];
        const int n = min(nbn[i], a.max_nb);
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int k = 0; k < n; ++k) {
            const int j = __ldg(nbl + (size_t)k * a.stride + i);
            const double4 pj = pos[j];
            const double dx = dsub(pi.x, pj.x), dy = dsub(pi.y, pj.y), dz = dsub(pi.z, pj.z);
            const double rsq = len2_strict(dx, dy, dz);
            if (rsq < a.rc2) {
                const double sr2 = ddiv(1.0, rsq);
                const double sr6 = dmul(dmul(dmul(sr2, sr2), sr2), a.sigma6);
                const double f = dmul(dmul(dmul(dmul(48.0, sr6), dsub(sr6, 0.5)), sr2), a.eps);
                fx = dadd(fx, dmul(dx, f));
                fy = dadd(fy, dmul(dy, f));
                fz = dadd(fz, dmul(dz, f));
                e += 4.0 * a.eps * sr6 * (sr6 - 1.0);
                w += f * rsq;
                cnt += 1.0;
            }
        }
        frc[i] = make_double4(fx, fy, fz, 0.0);
    }
    const double qs[kNoAllocQ] = {e, w, cnt};
    for (int q = 0; q < kNoAllocQ; ++q) {
        const double r = block_sum(qs[q], scratch);
        if (threadIdx.x == 0) part[q * kNoAllocMaxBlocks + blockIdx.x] = r;
    }
}

// sums the nb partials of each quantity in a fixed order into out[0..2]; out[3] = 0
__global__ void k_noalloc_reduce(const double* __restrict__ part, double* __restrict__ out, int nb) {
    __shared__ double scratch[32];
    for (int q = 0; q < kNoAllocQ; ++q) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) v += part[q * kNoAllocMaxBlocks + b];
        const double r = block_sum(v, scratch);
        if (threadIdx.x == 0) out[q] = r;
    }
    if (threadIdx.x == 0) out[3] = 0.0;
}

double pow6(double x) {  // utils/utilities.impala:27-36 for n = 6
    const double x3 = x * (x * x);
    return x3 * x3;
}

}  // namespace
}  // namespace tmd

using namespace tmd;

extern "C" int md_lj_forces_noalloc(const double* positions, int n_local, const int* list_sizes,
                                    const int* lists, int stride, int max_neighbors, double cutoff,
                                    double epsilon, double sigma, double* forces, double* sums, void* stream) {
    if (n_local < 0) {
        set_error(MD_ERR_ARGUMENT, "md_lj_forces_noalloc: invalid arguments (negative local atom count)");
        return MD_ERR_ARGUMENT;
    }
    if (n_local > kNoAllocMaxBlocks * kNoAllocThreads) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "md_lj_forces_noalloc: %d local atoms exceed the fixed scratch (at most %d)",
                      n_local, kNoAllocMaxBlocks * kNoAllocThreads);
        set_error(MD_ERR_ARGUMENT, msg);
        return MD_ERR_ARGUMENT;
    }
    if (stride < n_local || max_neighbors < 0 || !positions || !list_sizes || !lists || !forces || !sums) {
        set_error(MD_ERR_ARGUMENT, "md_lj_forces_noalloc: invalid arguments");
        return MD_ERR_ARGUMENT;
    }
    // once per device, with that device current: the device address of the scratch array
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice")) return MD_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) {
        set_error(MD_ERR_ARGUMENT, "md_lj_forces_noalloc: device index out of range");
        return MD_ERR_ARGUMENT;
    }
    if (!g_partials_addr[dev]) {
        void* p = nullptr;
        if (!cuda_ok(cudaGetSymbolAddress(&p, g_noalloc_partials), "cudaGetSymbolAddress")) return MD_ERR_CUDA;
        g_partials_addr[dev] = p;
    }
    double* part = static_cast<double*>(g_partials_addr[dev]);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    NoAllocArgs a;
    a.n = n_local;
    a.stride = stride;
    a.max_nb = max_neighbors;
    a.rc2 = cutoff * cutoff;
    a.sigma6 = pow6(sigma);
    a.eps = epsilon;
    const int nb = n_local > 0 ? (n_local + kNoAllocThreads - 1) / kNoAllocThreads : 1;
    k_lj_fp64_noalloc<<<nb, kNoAllocThreads, 0, st>>>(reinterpret_cast<const double4*>(positions), list_sizes,
                                                      lists, reinterpret_cast<double4*>(forces), part, a);
    if (!cuda_ok(cudaGetLastError(), "md_lj_forces_noalloc launch")) return MD_ERR_CUDA;
    k_noalloc_reduce<<<1, 256, 0, st>>>(part, sums, nb);
    if (!cuda_ok(cudaGetLastError(), "md_lj_forces_noalloc reduce launch")) return MD_ERR_CUDA;
    return MD_OK;
}
