// driver_ext.h -- the md driver's hooks into extensions of the library it is
// linked against.  Linked against libtinymd_b200.so (the product) the hooks
// call the extension entry points of include/tinymd_b200.h; built with
// TINYMD_DRIVER_CPU_ORACLE (the CPU baseline, oracle/Makefile) they call the
// test oracle's equivalents, and GPU-only options are ignored.
#pragma once

#include "tinymd_b200.h"

#ifdef TINYMD_DRIVER_CPU_ORACLE
extern "C" {
void oracle_set_ghost_mode(int exact);
void oracle_set_half_mode(int ghost_pairs);
void oracle_set_dem_mode(int contact_fixed, double radius);
void oracle_set_threads(int n);
int oracle_max_threads(void);
double oracle_temperature(void);
void oracle_last_thermo(double* out);
}
namespace drv {
constexpr bool kGpu = false;
inline void set_precision(int) {}
inline void set_ghost_mode(int exact) { oracle_set_ghost_mode(exact); }
inline void set_half_mode(int g) { oracle_set_half_mode(g); }
inline void set_dem_model(int fixed, double radius) { oracle_set_dem_mode(fixed, radius); }
inline void set_threads(int n) { oracle_set_threads(n); }
inline void set_thermo(int) {}
// {pair energy sum, virial sum, v.v sum}
inline void thermo(double* out) {
    double t[2];
    oracle_last_thermo(t);
    out[0] = t[0];
    out[1] = t[1];
    int n = md_get_number_of_particles();
    out[2] = oracle_temperature() * (3.0 * n - 3.0);
}
// the oracle runs synchronously: a request takes the sums at once and a fetch returns them
inline double* thermo_ring() {
    static double ring[8][3];
    return &ring[0][0];
}
inline int thermo_request() {
    static int t = 0;
    thermo(thermo_ring() + 3 * (t % 8));
    return t++;
}
inline void thermo_fetch(int ticket, double* out) {
    for (int q = 0; q < 3; ++q) out[q] = thermo_ring()[3 * (ticket % 8) + q];
}
inline bool phase_times(double*) { return false; }
inline void enable_phase_timing() {}
inline const char* backend() { return "cpu oracle (restatement of the reference cpu backend)"; }
inline bool failed() { return false; }
}  // namespace drv
#else
namespace drv {
constexpr bool kGpu = true;
inline void set_precision(int m) { md_set_precision(m); }
inline void set_ghost_mode(int exact) { md_set_ghost_mode(exact); }
inline void set_half_mode(int g) { md_set_half_mode(g); }
inline void set_dem_model(int fixed, double radius) { md_set_dem_model(fixed, radius); }
inline void set_threads(int) {}
inline void set_thermo(int on) { md_set_thermo(on); }
inline void thermo(double* out) {
    double t[4];
    md_get_thermo(t);
    out[0] = t[0];
    out[1] = t[1];
    out[2] = t[3];
}
// the sums go to page-locked memory behind the enqueued work; fetching waits for that copy only
inline int thermo_request() { return md_thermo_request(); }
inline void thermo_fetch(int ticket, double* out) {
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    md_thermo_fetch(ticket, t);
    out[0] = t[0];
    out[1] = t[1];
    out[2] = t[3];
}
inline bool phase_times(double* out6) {
    md_get_phase_times(out6);
    return true;
}
inline void enable_phase_timing() { md_set_phase_timing(1); }
inline const char* backend() { return "B200 (sm_100a CUDA kernels)"; }
inline bool failed() { return md_last_error() == MD_ERR_CUDA || md_last_error() == MD_ERR_NO_DEVICE; }
}  // namespace drv
#endif
