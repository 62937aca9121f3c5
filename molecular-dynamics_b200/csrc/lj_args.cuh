// lj_args.cuh -- parameters of the LJ force kernels (core/runtime.impala:188-201)
// of k_step.cu: every form evaluates a pair with the same constants.
#pragma once

#include "md_state.h"

namespace tmd {

struct LjArgs {
    int N, NA, stride, nbcap;  // NA = locals + ghosts
    double rc2, sigma6, eps, h;
    double dt_i, h_i;          // the next step's initial integration (fused kernels only)
    double alo[3], rb_h;       // rebasing grid (mixed form's positions)
    // mixed form
    float rc2_lo, rc2_hi, close2;
    float fast_mid, fast_half;  // the FP32 window [close2, rc2_lo) as |rsq - mid| < half
    float lj_a, lj_b;           // force: f/r = t/r^2 (lj_a t + lj_b), t = 1/r^6
    float lj_c, lj_d;           // energy: t (lj_c t + lj_d)
    float hx, hy, hz;  // shift decode scales (see the kernels)
    // a launch on lists whose build status is still in flight: the kernel returns without
    // writing when that build overflowed the capacity or left locals outside the grid
    const DevStatus* spec = nullptr;
};

__device__ __forceinline__ bool lists_failed(const LjArgs& a) {
    return a.spec != nullptr && (a.spec->max_nb > a.nbcap || a.spec->out_local > 0);
}

// utils/utilities.impala:27-36 (recursive squaring) for integer powers
inline double ipow(double x, int n) {
    if (n == 1) return x;
    if (n % 2 == 0) {
        double y = ipow(x, n / 2);
        return y * y;
    }
    return x * ipow(x, n - 1);
}

// hx, hy, hz are left to the caller (they depend on how the kernel packs dk)
inline LjArgs lj_args(const State& s, const PendingForce& p, double dt) {
    LjArgs a;
    a.N = s.N;
    a.NA = s.N + s.G;
    a.stride = s.nb_stride;
    a.nbcap = s.nb_cap;
    a.rc2 = p.rc * p.rc;
    a.sigma6 = ipow(p.sigma, 6);
    a.eps = p.eps;
    a.h = 0.5 * dt;
    a.dt_i = a.h_i = 0.0;
    for (int d = 0; d < 3; ++d) a.alo[d] = s.geo.aabb_lo[d];
    a.rb_h = s.geo.rb_h;
    // FP32 rsq of a list pair is within ~4e-6 of the FP64 value (del components
    // carry at most ~3.6e-7 error); pairs inside this window take the FP64 test
    const double margin = 2e-5 * a.rc2 + 1e-7;
    a.rc2_lo = (float)(a.rc2 - margin);
    a.rc2_hi = (float)(a.rc2 + margin);
    // pairs closer than 1.04 sigma take the FP64 path: the force's steep r^-13 branch magnifies
    // the FP32 rounding of del there.  On the 131k-atom LJ liquid (emulated FP32 arithmetic
    // against FP64), max |dF| / rms(F) after 25 / 220 / 1000 steps is 1.30e-5 / 7.2e-6 / 8.0e-6
    // with a threshold of sigma (~0.1-0.3 FP64 pairs per atom), 9.6e-6 after 25 steps with
    // 1.02 sigma, 4.5e-6 / 4.7e-6 after 220 / 1000 steps with 1.04 sigma (~1.0 FP64 pair per
    // atom) and 5.7e-6 / 3.9e-6 / 3.8e-6 with 1.05 sigma (~1.2-1.4 FP64 pairs per atom)
    a.close2 = (float)((1.04 * p.sigma) * (1.04 * p.sigma));
    // one comparison of |rsq - mid| instead of two: its edges move by an ulp at most, and a pair
    // on either side of an edge is exact enough in both forms (both edges are margins)
    a.fast_mid = (float)(0.5 * ((double)a.rc2_lo + (double)a.close2));
    a.fast_half = (float)(0.5 * ((double)a.rc2_lo - (double)a.close2));
    // with t = 1/r^6: sr6 = sigma^6 t, f/r = 48 eps sr6 (sr6 - 1/2) / r^2 = t/r^2 (A t + B) and
    // 4 eps sr6 (sr6 - 1) = t (C t + D)
    a.lj_a = (float)(48.0 * p.eps * a.sigma6 * a.sigma6);
    a.lj_b = (float)(-24.0 * p.eps * a.sigma6);
    a.lj_c = (float)(4.0 * p.eps * a.sigma6 * a.sigma6);
    a.lj_d = (float)(-4.0 * p.eps * a.sigma6);
    a.hx = a.hy = a.hz = 0.0f;
    return a;
}

}  // namespace tmd
