/*
 * rhmc_legacy.h -- the extern "C" GPU entry points of coppolachan/RHMC-on-GPU, implemented by
 * librhmc_b200 with the same names, signatures and semantics, so that the reference's host
 * code (lib/Main/Gpu/gpu.cc, lib/Action/Inverter/cu_inverter.cc, the lib/Update sources,
 * lib/Action/fermionforce.cc, lib/Tools/RationalApprox/rationalapprox.cc, findminmax.cc,
 * chiralmeas.cc) links against this library in place of its lib/Cuda directory.
 *
 * The reference keeps its GPU state in file-scope device globals and reads its compile-time
 * constants (include/parameters.h) and packed host buffers (include/global_var.h:90-98)
 * directly.  A library cannot see either, so the host program makes one extra call,
 * rhmc_legacy_bind, before the first cuda_init0 (for example at the end of initialize(),
 * lib/Main/init.cc:14-116, once the packed buffers exist).  After that the functions below
 * behave as their lib/Cuda counterparts: void, print and exit on error (cudaSafe,
 * lib/Cuda/cuda_err.cu:5-13), host buffers in the packer formats of lib/Tools/Packer/packer.cc.
 *
 * Differences, all in the direction of accuracy: every kernel computes in FP64 (the reference
 * GPU uses FP32 for the force, the exponential and the power iteration); the link exponential
 * is the 6th-order Taylor of the CPU code (su3.cc:187-219) instead of the GPU's 5th order
 * (cuda_exponentiate.cu:54-311); the single-precision inverter keeps FP64 scalars.
 */
#ifndef RHMC_LEGACY_H
#define RHMC_LEGACY_H

#include "rhmc_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny, nz, nt;     /* include/parameters.h:7-10 */
    int ferm_temp_bc;       /* parameters.h:29 */
    double mass, beta;      /* parameters.h:15-16 */
    int no_ps;              /* parameters.h:58 */
    int max_approx_order;   /* include/global_const.h:11 */
    int max_cg;             /* parameters.h:57 */
    int device;             /* parameters.h:76 */
    /* the host program's packed buffers (include/global_var.h:90-98, allocated in init.cc:79-97) */
    float *gauge_field_packed;    /* float[2*12*no_links], smartpack_gauge (packer.cc:8-71) */
    float *chi_packed;            /* float[6*sizeh*no_ps*2], smartpack_multifermion (packer.cc:278-319) */
    float *simple_fermion_packed; /* float[6*sizeh*2], smartpack_fermion_d (packer.cc:192-230) */
    float *ipdot_packed;          /* float[8*no_links], smartpack_tamatrix (packer.cc:443-469) */
    float *momenta_packed;        /* float[8*no_links], smartpack_thmatrix (packer.cc:508-534) */
    const int *shift_table;       /* int[8*size], make_shift_table (packer.cc:415-439); checked */
    const int *eta;               /* int[4*size] (geometry.cc:107-153); checked */
} rhmc_legacy_config;

/* No counterpart in the reference: hands the compile-time constants and the packed buffers to
 * the library.  Call once, before cuda_init0; calling it again releases the device state of the
 * previous binding.  Returns RHMC_OK or an error code. */
int rhmc_legacy_bind(const rhmc_legacy_config *cfg);
/* The context the legacy entry points operate on (for mixing with the handle API), or NULL. */
rhmc_ctx *rhmc_legacy_context(void);

/* lib/Cuda/cuda_init.h:4-11 */
void cuda_init0(void);
void cuda_init1(void);
void cuda_meas_init(void);
void cuda_meas_end(void);
void cuda_end(void);
void cuda_get_conf(void);
void cuda_get_momenta(void);
void cuda_put_momenta(void);
/* lib/Cuda/cuda_inverter.h:4-14 */
void cuda_shifted_inverter(const double residual, const double *shifts, const int num_shifts, const int psferm, int *ncount);
void cuda_shifted_inverter_d(const double residual, const double *shifts, const int num_shifts, const int psferm, int *ncount);
/* lib/Cuda/cuda_sol_sum.h:4 */
void cuda_sol_sum(const int num_shifts, const double mult_const, const double *numerators);
/* lib/Cuda/cuda_fermion_force.h:4 */
void cuda_fermion_force(int num_shifts, float *numerators);
/* lib/Cuda/cuda_deriv.h:4 */
void cuda_gauge_deriv(int ipdot_init);
/* lib/Cuda/cuda_exponentiate.h:4 */
void cuda_exp_su3(float step);
/* lib/Cuda/cuda_mom_sum_mul.h:4 */
void cuda_momenta_sum_multiply(float step);
/* lib/Cuda/cuda_find_min_max.h:6-7 (REAL = double, include/global_macro.h:5) */
void cuda_find_max(double *max);
void cuda_find_min(double *min, const double max);
/* lib/Cuda/DeviceInfo/device_info.h:4-6 (called by lib/Main/rhmc.cc:318): selects the device and
 * prints its properties. */
void GPUDeviceInfo(const int gpu_device);

/* The power iterations behind cuda_find_max/min through the handle API (FP64): start is a
 * host spinor in the reference layout; stops when the relative change is below 5e-4
 * (cuda_find_min_max.cu:133,210). */
int rhmc_find_max(rhmc_ctx *ctx, const double *start, double *max);
int rhmc_find_min(rhmc_ctx *ctx, const double *start, double max, double *min);

#ifdef __cplusplus
}
#endif
#endif /* RHMC_LEGACY_H */
