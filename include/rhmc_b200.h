/*
 * rhmc_b200.h -- C ABI of librhmc_b200, the B200 (sm_100a) implementation of the RHMC hot
 * path of coppolachan/RHMC-on-GPU: even/odd staggered Dslash, multi-shift CG on
 * M^dag M + sigma_i, fermion force, gauge-force staples and the SU(3) momentum/link update.
 *
 * Plain C types only.  Every function returns an int status (RHMC_OK or a negative
 * RHMC_ERR_*); rhmc_last_error() describes the last failure of the calling thread.
 * Device work is issued on the context's stream (rhmc_set_stream); functions that return
 * host values synchronise that stream first.
 *
 * Field layouts at this boundary are the reference's CPU layouts (complex = two doubles):
 *   links, momenta, ipdot : complex[4V][3][3], index mu*V + site   (Conf::u_work,
 *                           include/configuration.h:9-10; Momenta, Ipdot)
 *   spinor (one parity)   : complex[Vh][3]                        (Fermion, lib/Action/fermions.h:12)
 * with sites numbered even-first (lib/Main/Geometry/geometry.cc:5-11,86) and the staggered
 * phases folded into the links (lib/Main/Conf/conf.cc:36,49).
 * "Internal" spinors are the device layout the kernels use: colour planes [3][Vh] of
 * complex (double2 for FP64 formats, float2 for FP32 formats); n right-hand sides are
 * consecutive spinors.
 *
 * The reference's own extern "C" GPU entry points (the lib/Cuda headers) are provided, with their
 * signatures and semantics, by rhmc_legacy.h.
 */
#ifndef RHMC_B200_H
#define RHMC_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rhmc_ctx rhmc_ctx;

enum {
    RHMC_OK = 0,
    RHMC_ERR_ARG = -1,       /* invalid argument (null pointer, bad size, bad enum) */
    RHMC_ERR_CUDA = -2,      /* a CUDA runtime call failed */
    RHMC_ERR_MAXITER = -3,   /* a solver hit its iteration cap (reference: exit(1), cu_inverter.cc:62-69) */
    RHMC_ERR_NONFINITE = -4, /* NaN/Inf detected in a solver reduction */
    RHMC_ERR_STATE = -5      /* call out of order (e.g. no gauge field set) */
};

/* Link storage formats used by the Dslash kernels (derived from the FP64 master copy). */
enum {
    RHMC_LINKS_F64_18 = 0, /* FP64, all 18 reals */
    RHMC_LINKS_F64_12 = 1, /* FP64, rows 0-1; row 2 = eta*conj(row0 x row1) (lib/Cuda/cuda_rhmc.cuh:32-45) */
    RHMC_LINKS_F32_18 = 2, /* FP32, all 18 reals */
    RHMC_LINKS_F32_12 = 3, /* FP32, rows 0-1, reconstructed */
    RHMC_LINKS_F16_12 = 4  /* half precision rows 0-1, reconstructed in FP32; spinors of this format are
                              half precision scaled per site, one 16-byte vector per site: three __half2
                              (the colour components divided by the site's largest |re|,|im|) and that
                              scale as a float (internal stride Vh vectors) */
};

enum { RHMC_HOST = 0, RHMC_DEVICE = 1 };

/* Run parameters; the reference fixes them at compile time (include/parameters.h:7-76). */
typedef struct {
    int nx, ny, nz, nt; /* lattice extents, all even (parameters.h:7-10) */
    int ferm_temp_bc;   /* 0: antiperiodic fermion time b.c. (parameters.h:29) */
    double mass;        /* bare staggered mass (parameters.h:16) */
    double beta;        /* Wilson gauge coupling (parameters.h:15) */
    int device;         /* CUDA device ordinal (parameters.h:76) */
} rhmc_params;

/* ------------------------------------------------------------------ lifecycle */
const char *rhmc_last_error(void);
/* Allocates the device-resident fields; replaces the per-trajectory cudaMalloc of
 * cuda_init0/cuda_init1 (lib/Cuda/cuda_init.cu:5-109). */
int rhmc_create(const rhmc_params *p, rhmc_ctx **out);
int rhmc_destroy(rhmc_ctx *ctx);
/* Issue subsequent work on a caller stream (cudaStream_t); NULL restores the context's own. */
int rhmc_set_stream(rhmc_ctx *ctx, void *stream);
int rhmc_sync(rhmc_ctx *ctx);
/* Number of kernels this context has launched so far. */
int rhmc_launch_count(const rhmc_ctx *ctx, long *count);

/* ------------------------------------------------------------------ geometry */
/* Neighbour table int[8V] (nnm mu=0..3 then nnp mu=0..3; make_shift_table,
 * lib/Tools/Packer/packer.cc:415-439) and staggered phases int[4V] (init_geo,
 * lib/Main/Geometry/geometry.cc:26-161), computed on the device into host buffers.
 * Either pointer may be NULL. */
int rhmc_geometry(rhmc_ctx *ctx, int *table, int *eta);

/* ------------------------------------------------------------------ fields */
/* Gauge field in the reference layout; replaces the gauge half of cuda_init0 / cuda_end
 * (lib/Cuda/cuda_init.cu:5-58, 187-211) without the float hi/lo split. */
int rhmc_set_gauge(rhmc_ctx *ctx, const double *u, int location);
int rhmc_get_gauge(rhmc_ctx *ctx, double *u, int location);
/* Momenta (traceless hermitian) and ipdot (traceless anti-hermitian) as full 3x3 matrices
 * in the reference layout; stored internally as 8 reals per link.  Replaces the P/ipdot
 * parts of cuda_init1 / cuda_end / cuda_get_momenta / cuda_put_momenta. */
int rhmc_set_momenta(rhmc_ctx *ctx, const double *p, int location);
int rhmc_get_momenta(rhmc_ctx *ctx, double *p, int location);
int rhmc_set_ipdot(rhmc_ctx *ctx, const double *ip, int location);
int rhmc_get_ipdot(rhmc_ctx *ctx, double *ip, int location);

/* Spinor conversion between the reference layout (n consecutive complex[Vh][3]) and the
 * internal device layout of format `fmt` precision.  `internal` is a device pointer. */
int rhmc_spinor_to_internal(rhmc_ctx *ctx, int fmt, void *internal, const double *ref, int n, int location);
int rhmc_spinor_from_internal(rhmc_ctx *ctx, int fmt, double *ref, const void *internal, int n, int location);

/* ------------------------------------------------------------------ Dslash */
/* out = D in onto parity `parity_out` (0: Deo, 1: Doe; lib/Action/fermionmatrix.cc:8-97,
 * including the factor 1/2), for n right-hand sides sharing each link load.  in/out are
 * internal-layout device spinors of the precision of `fmt`. */
int rhmc_dslash(rhmc_ctx *ctx, int fmt, int parity_out, void *out, const void *in, int n);
/* `repeats` times: odd = D_oe even, then even = D_eo odd (n RHS), issued back to back from C
 * so that timing loops measure the kernels and not the caller's launch overhead. */
int rhmc_dslash_repeat(rhmc_ctx *ctx, int fmt, void *even, void *odd, int n, int repeats);
/* Reference-facing form of Deo/Doe (lib/Action/fermionmatrix.cc:8-97): host spinors in the
 * reference layout (Vec3[Vh]), FP64 links; blocking.  The input is uploaded in chunks of
 * t-slabs that the Dslash consumes as they arrive; a page-locked `out` is written by the kernel
 * directly, any other `out` through a copy per chunk. */
int rhmc_dslash_host(rhmc_ctx *ctx, int parity_out, double *out, const double *in);
/* No counterpart in the reference.  The half-Dslash onto the output sites [k_lo, k_lo + k_count) of
 * parity parity_out only, FP64 18-real links, device spinors in the reference's site-major layout
 * (complex[Vh][3]); the other output sites are not written.  For domain decomposition: a rank's
 * context holds its t-slab extended by one ghost slice each side, and this computes its interior. */
int rhmc_dslash_sites(rhmc_ctx *ctx, int parity_out, double *out, const double *in, long k_lo, long k_count);
/* out = (M^dag M + shift) in on even sites = (mass^2 + shift) in - Deo Doe in
 * (lib/Action/Inverter/inverter.cc:3, 206-216); internal-layout device spinors. */
int rhmc_mdagm(rhmc_ctx *ctx, int fmt, void *out, const void *in, double shift, int n);

/* ------------------------------------------------------------------ multi-shift CG */
enum {
    RHMC_MSOLVE_FP64 = 0,  /* the reference algorithm in FP64 (multips_shifted_invert,
                              lib/Action/Inverter/inverter.cc:142-339): base operator M^dag M,
                              shift frozen when sqrt(|r|^2 zeta^2) < residual */
    RHMC_MSOLVE_MIXED = 1, /* multi-shift on the smallest pole with all RHS batched.  FP32 or half
                              fmt: precision schedule -- FP64 vectors and 12-real FP64 links until
                              |r| <= tol_phase_a |b|, then the same recurrences resumed with FP32
                              links and base vectors (FP64 shifted vectors, FP64 reliable update of
                              the base residual every 32 iterations) to `residual`.  FP64 fmt: FP64
                              vectors throughout (12-real links when fmt says so).  Then FP32 CG
                              per system inside FP64 defect correction for every system whose FP64
                              true residual |b - (M^dag M + sigma_i) x_i| is still above `residual` */
    RHMC_MSOLVE_FP32 = 2   /* the reference algorithm with FP32 links and vectors (its
                              single-precision path, lib/Cuda/cuda_inverter.cu:647-857, used
                              when residual >= 1e-4, cu_inverter.cc:45-60); FP64 scalars */
};

typedef struct {
    int nshift;            /* number of poles, 1..32 (max_approx_order, include/global_const.h:11) */
    const double *shifts; /* sigma_i >= 0: the rescaled RA_b (rationalapprox.cc:162-170) */
    int nrhs;              /* right-hand sides (pseudofermions) solved together */
    double residual;       /* absolute stopping residual (residue_metro / residue_md, parameters.h:68,73) */
    int max_iter;          /* iteration cap (max_cg, parameters.h:57) */
    int mode;              /* RHMC_MSOLVE_* */
    int fmt;               /* link format of the multi-shift phase (FP64 ones for RHMC_MSOLVE_FP64,
                              FP32 ones for RHMC_MSOLVE_FP32, any for RHMC_MSOLVE_MIXED; in mixed mode
                              RHMC_LINKS_F16_12 means an FP32 12-real multi-shift phase followed by a
                              refinement whose sloppy CG runs on half links and half spinors) */
    double tol_phase_a;    /* mixed mode, FP32/half fmt: relative residual |r|/|b| at which the FP64
                              part of the precision schedule hands over to FP32; 0: automatic,
                              1e-3 |b| but no more than 1e7 x `residual` above the target (the FP32
                              part leaves the shifted systems near 1e-7 of the hand-over residual)
                              and no less than 1e-4 |b| */
    double ru_delta;       /* mixed mode: FP32 residual reduction between FP64 updates (0: 0.05) */
    int certify;           /* FP64 mode: afterwards refine, by FP64 CG one system at a time, every system
                              whose FP64 true residual is still above `residual` (the reference's
                              iterated-residual test alone can stop above it) */
    const double *rhs_shifts; /* optional [nrhs][nshift]: a pole set per right-hand side (overrides
                              shifts), e.g. the pseudofermions of several fermion species solved in
                              one batch; NULL: `shifts` for every right-hand side */
} rhmc_msolve_params;

typedef struct {
    int status;            /* RHMC_OK or the error returned */
    int iters[8];          /* multi-shift iterations of right-hand sides 0..7 only (see iters_total
                              and iters_max for any nrhs) */
    long refine_iters;     /* mixed mode: batched refinement iterations (sum over batches) */
    int reliable_updates;  /* mixed mode: FP64 residual recomputations */
    double seconds;        /* wall time of the call */
    double seconds_phase_a;/* mixed mode / certified FP64: wall time of the multi-shift phase */
    int systems_refined;   /* mixed mode / certified FP64: (rhs, shift) systems that needed refinement */
    long iters_total;      /* multi-shift iterations summed over every right-hand side */
    int iters_max;         /* largest multi-shift iteration count of any right-hand side */
    long iters_fp64;       /* mixed mode: multi-shift iterations run in FP64 (summed over RHS 0..7) */
    int ms_reliable_updates; /* mixed mode, FP32/half fmt: FP64 reliable updates of the multi-shift */
} rhmc_msolve_info;

/* (M^dag M + sigma_i) x_{r,i} = b_r for every shift i and RHS r (cuda_shifted_inverter /
 * cuda_shifted_inverter_d, lib/Cuda/cuda_inverter.cu:647-857, cuda_inverter_d.cu:752-968,
 * called per pseudofermion by cu_multips_shifted_invert, lib/Action/Inverter/cu_inverter.cc:21-72).
 * b: nrhs FP64 internal spinors (device); x: nrhs*nshift FP64 internal spinors, RHS-major
 * (the ShiftMultiFermion order [no_ps][order][sizeh], lib/Action/fermions.h:114).
 * Returns RHMC_ERR_MAXITER instead of the reference's exit(1) at max_cg. */
int rhmc_msolve(rhmc_ctx *ctx, const rhmc_msolve_params *p, double *x, const double *b, rhmc_msolve_info *info);
/* Same with host arrays in the reference layout: b complex[nrhs][Vh][3], x complex[nrhs][nshift][Vh][3]. */
int rhmc_msolve_host(rhmc_ctx *ctx, const rhmc_msolve_params *p, double *x, const double *b, rhmc_msolve_info *info);
/* |b_r - (M^dag M + sigma_i) x_{r,i}| in FP64 for every (r, i); out: host double[nrhs][nshift].
 * The check of inverter.cc:306-338 / cu_inverter.cc:79-120 without the debug build. */
int rhmc_true_residuals(rhmc_ctx *ctx, int nshift, const double *shifts, int nrhs, const double *x, const double *b, double *out);

/* ------------------------------------------------------------------ forces and updates */
/* ipdot (=|+ when add) TA((U beta/3) staples): calc_ipdot_gauge (lib/Update/ipdot.cc:25-49) with
 * calc_staples (lib/Action/staples.cc:16-74); cuda_gauge_deriv (lib/Cuda/cuda_deriv.cu:697-744). */
int rhmc_gauge_force(rhmc_ctx *ctx, int add);
/* ipdot (=|+ when add) TA(U F), F = sum over rhs r and shift i of numerators[i] times the outer
 * products of fermionforce (lib/Action/fermionforce.cc:46-104) built from x_{r,i} and Doe x_{r,i};
 * cuda_fermion_force (lib/Cuda/cuda_fermion_force.cu:346-418).  x: FP64 internal device spinors
 * [nrhs][nshift]; numerators: host double[nshift] (rescaled RA_a). */
int rhmc_fermion_force(rhmc_ctx *ctx, int nrhs, int nshift, const double *numerators, const double *x, int add);
/* P += i step ipdot: momenta_sum_multiply(i step) (lib/Update/momenta.cc:82-115); cuda_momenta_sum_multiply. */
int rhmc_mom_update(rhmc_ctx *ctx, double step);
/* U <- exp(i step P) U, unitarised with the phases: conf_left_exp_multiply(i step)
 * (lib/Update/momenta.cc:42-78, Su3::exp su3.cc:187-219, unitarize_with_eta conf.cc:235-251);
 * cuda_exp_su3 (lib/Cuda/cuda_exponentiate.cu:783-828), here 6th order and FP64 throughout. */
int rhmc_link_update(rhmc_ctx *ctx, double step);
/* sum_x sum_{mu<nu} beta/3 ReTr(plaquette) (Conf::loc_action, lib/Action/action.cc:6-61). */
int rhmc_gauge_action(rhmc_ctx *ctx, double *out);
/* sum over links of 1/2 Tr P^2 (calc_action, lib/Action/action.cc:122-134). */
int rhmc_momentum_action(rhmc_ctx *ctx, double *out);
/* spatial and temporal plaquette as Conf::calc_plaq (lib/Measurements/gaugemeas.cc:7-65). */
int rhmc_plaquette(rhmc_ctx *ctx, double *spatial, double *temporal);
/* Polyakov loop as Conf::calc_poly (lib/Measurements/gaugemeas.cc:66-106): the average over spatial
 * points of -Tr/3 of the ordered product of the temporal links (the minus sign undoes the
 * antiperiodic phase folded into them). */
int rhmc_polyakov(rhmc_ctx *ctx, double *re, double *im);
/* chiral_meas (lib/Measurements/chiralmeas.cc:18-194, without imaginary chemical potential) for
 * nrand pairs of noise vectors (even, odd; n consecutive spinors of the reference layout, host or
 * device per `location`; the reference draws Z2 noise, the caller supplies it here):
 * phi_e = m rnd_e - Deo rnd_o, (M^dag M) chi_e = phi_e solved in FP64 to the absolute `residual`,
 * chi_o = (rnd_o - Doe chi_e) / m, then out[8] = chiral condensate, energy, baryon and pressure
 * densities as (re, im) pairs, averaged over the noise pairs. */
int rhmc_chiral_meas(rhmc_ctx *ctx, int nrand, int no_flavours, const double *noise_e, const double *noise_o, double residual,
                     int max_iter, int location, double *out);

/* ------------------------------------------------------------------ configuration files */
/* The reference's text configuration (Conf::write_last, lib/Main/Conf/conf.cc:175-200): a header
 * "nx ny nz nt beta mass no_flavours update_iteration" (beta and mass of the context), then every
 * link of the current gauge field (eta folded in) as 3 rows of "(re,im)" numbers, 16 digits. */
int rhmc_write_conf(rhmc_ctx *ctx, const char *path, int no_flavours, long update_iteration);
/* Reads such a file into the gauge field (the stored-conf start of Conf::Conf, conf.cc:55-94);
 * fails on a lattice-size mismatch.  reunitarize = 1 applies the reunitarisation with eta that
 * the reference's reader means to apply but does not (its calls act on u_work before u_work is
 * overwritten); 0 keeps the stored numbers as the reference does.  Header values are returned
 * through the non-null pointers. */
int rhmc_read_conf(rhmc_ctx *ctx, const char *path, int reunitarize, double *beta, double *mass, int *no_flavours,
                   long *update_iteration);
/* sum over n internal FP64 spinors of Re<a, b> (fermion_action, lib/Action/action.cc:65-107). */
int rhmc_rdot(rhmc_ctx *ctx, const double *a, const double *b, int n, double *out);
/* out_r = a0 b_r + sum_i a_i x_{r,i} (rationalapprox.cc:300-311; cuda_sol_sum, lib/Cuda/cuda_sol_sum.cu:168-221);
 * FP64 internal device spinors, a: host double[nshift]. */
int rhmc_rational_sum(rhmc_ctx *ctx, int nrhs, int nshift, double a0, const double *a, const double *x, const double *b,
                      double *out);

/* ------------------------------------------------------------------ molecular-dynamics driver */
/* Integrators: the reference's use_multistep values (parameters.h:48, update.cc:29-43) plus the
 * leapfrog of leapfrog.cc with the kick sign of the wired integrators. */
enum { RHMC_INT_2MN = 0, RHMC_INT_MULTISTEP_2MN = 1, RHMC_INT_MULTISTEP_4MN = 2, RHMC_INT_LEAPFROG = 3 };

typedef struct {
    int no_flavours;      /* parameters.h:14 */
    int no_ps;            /* pseudofermions, parameters.h:58 */
    int no_md;            /* MD steps per unit trajectory, parameters.h:47 */
    int gauge_scale;      /* gauge steps per fermion step in the multistep integrators, parameters.h:49 */
    int integrator;       /* RHMC_INT_* */
    int max_cg;           /* parameters.h:57 */
    double residue_metro; /* heatbath and action solves, parameters.h:68 */
    double residue_md;    /* force solves, parameters.h:73 */
    int metro_mode, metro_fmt; /* RHMC_MSOLVE_* and link format of the heatbath/action solves */
    int md_mode, md_fmt;       /* ... of the force solves */
    int auto_bounds;      /* spectral bounds of M^dag M: 0 from rhmc_set_eig_bounds; 1 by FP64 power
                             iterations for lambda_max and lambda_min (findminmax, findminmax.cc:12-183)
                             at the start of every trajectory, instead of at every rescaling as the
                             reference does; 2 lambda_max by power iteration, lambda_min = mass^2 (the
                             exact lower bound of M^dag M, no slow lambda_min iteration) */
    int single_rhs;       /* 1: every pseudofermion of every species in its own multi-shift solve (the
                             reference's loop over pseudofermions, inverter.cc:164); 0: all of them
                             batched into one solve (one link read serves every right-hand side) */
    int pole_group;       /* 0: all poles of an approximation in one multi-shift solve, every shifted
                             solution held on the device at once (the reference keeps them all,
                             smf_device, lib/Cuda/cuda_fermion_force.cu:346-418); G > 0: the poles
                             in groups of at most G, each group solved, used (its share of the
                             rational sum, force or action accumulated) and dropped before the
                             next: the shifted vectors of a solve shrink by order/G at the cost of
                             repeating the Krylov iterations once per group (no counterpart in
                             the reference; for volumes or batches whose shifted solutions do not
                             fit in HBM) */
} rhmc_driver_params;

/* Configures the driver of lib/Update (update.cc, ipdot.cc, momenta.cc, MD_integrators).
 * no_flavours and no_ps describe species 0, the fermions at the context mass. */
int rhmc_driver_setup(rhmc_ctx *ctx, const rhmc_driver_params *p);
/* No counterpart in the reference (one species only): adds a fermion species of its own mass
 * (>= the context mass), no_flavours and no_ps, e.g. the strange quark of N_f = 2+1, and returns
 * its index (1, 2, ...).  It gets its own pseudofermions, rational approximations and eigenvalue
 * bounds; heatbath, actions and forces then sum over all species.  Its solves run on the
 * context's M^dag M with every pole shifted by mass^2 - context mass^2. */
int rhmc_driver_add_species(rhmc_ctx *ctx, double mass, int no_flavours, int no_ps, int *index);
/* Selects the species that rhmc_set_approx, rhmc_set_eig_bounds and rhmc_set/get_phi/chi act on
 * (0 after setup). */
int rhmc_driver_select_species(rhmc_ctx *ctx, int index);
/* Normalised rational approximation on [min_eps, 1] (RationalApprox, rationalapprox.h:13-47):
 * which = 0 first (heatbath, x^(N_f/(8 N_ps))), 1 md (force), 2 last (action) (x^(-N_f/(4 N_ps))).
 * The coefficients rationalapprox_calc (rationalapprox_calc.cc:8-177) would compute at start-up. */
int rhmc_set_approx(rhmc_ctx *ctx, int which, int order, double a0, const double *a, const double *b, double min_eps);
/* Spectral bounds of M^dag M (at the selected species' mass) that findminmax would return (findminmax.cc:140-183); the rescaling
 * widens them by 0.95 / 1.05 like RationalApprox::*_inv_approx_coeff (rationalapprox.cc:134-266). */
int rhmc_set_eig_bounds(rhmc_ctx *ctx, double min, double max);
/* The bounds the driver currently holds for the selected species (set, or computed when
 * auto_bounds is on). */
int rhmc_get_eig_bounds(rhmc_ctx *ctx, double *min, double *max);
/* Pseudofermions phi and chi, reference layout complex[no_ps][Vh][3] (MultiFermion). */
int rhmc_set_phi(rhmc_ctx *ctx, const double *phi, int location);
int rhmc_get_phi(rhmc_ctx *ctx, double *phi, int location);
int rhmc_set_chi(rhmc_ctx *ctx, const double *chi, int location);
int rhmc_get_chi(rhmc_ctx *ctx, double *chi, int location);
/* chi = r_first(M^dag M) phi / phi = r_last(M^dag M) chi (rationalapprox.cc:269-369). */
int rhmc_first_inv_approx_calc(rhmc_ctx *ctx, double res);
int rhmc_last_inv_approx_calc(rhmc_ctx *ctx, double res);
/* calc_ipdot, calc_ipdot_gauge, calc_ipdot_fermion (lib/Update/ipdot.cc:25-196). */
int rhmc_calc_ipdot(rhmc_ctx *ctx);
int rhmc_calc_ipdot_gauge(rhmc_ctx *ctx);
int rhmc_calc_ipdot_fermion(rhmc_ctx *ctx);
/* The action whose link derivative rhmc_calc_ipdot_fermion is: S_f = sum over pseudofermions of
 * chi^dag r_md(M^dag M) chi = a0 |chi|^2 + sum_i a_i Re<chi, (M^dag M + b_i)^-1 chi> with the
 * rescaled md approximation and the md solver settings (the pole set fermionforce solves for,
 * lib/Action/fermionforce.cc:27-38).  With U -> exp(i t Q) U on one link (Q hermitian),
 * dS_f/dt = Re(i Tr(Q ipdot)) for the ipdot of rhmc_calc_ipdot_fermion: the action/force pair
 * checked by finite differences. */
int rhmc_fermion_action(rhmc_ctx *ctx, double *out);
/* One MD trajectory with the configured integrator (update_nometro, update.cc:17-53). */
int rhmc_update_nometro(rhmc_ctx *ctx);
/* One RHMC trajectory (update, update.cc:58-152) from the momenta and phi set by the caller:
 * heatbath, initial action, integration, action solve, final action, Metropolis against
 * `uniform`; *acc = 1 accepted / 0 rejected (configuration restored), *delta_s = S_new - S_old. */
int rhmc_update(rhmc_ctx *ctx, double uniform, int *acc, double *delta_s);
/* Conf::save / Conf::copy_saved (lib/Main/Conf/conf.cc:104-140). */
int rhmc_save_conf(rhmc_ctx *ctx);
int rhmc_copy_saved(rhmc_ctx *ctx);
int rhmc_driver_stats(rhmc_ctx *ctx, long *force_evals, long *solves);
/* Sums of the rhmc_msolve_info of every solve the driver ran since rhmc_driver_setup (or the last
 * reset): which = 0 the force (md) solves, 1 the heatbath and action (metro) solves.  Counts,
 * iterations and seconds are added up, iters_max is the largest, iters[] holds the last solve's
 * and status the last error.  No counterpart in the reference (its inverter prints an iteration
 * count per solve).  reset != 0 zeroes both sums after reading. */
int rhmc_driver_solver_stats(rhmc_ctx *ctx, int which, rhmc_msolve_info *out, int reset);
/* Device memory held by the context's workspaces (solver vectors, shifted solutions, driver
 * fields, reduction buffers), in bytes; no counterpart in the reference.  Workspaces grow to
 * the largest request and are kept until rhmc_workspace_release or rhmc_destroy. */
int rhmc_workspace_bytes(rhmc_ctx *ctx, long *bytes);
/* Synchronises the context's stream, then frees every workspace and instantiated solver graph
 * of the context except the state the driver carries between calls (phi, chi and the saved
 * configuration; links, momenta and ipdot are not workspaces); later calls allocate again what
 * they need.  No counterpart in the reference. */
int rhmc_workspace_release(rhmc_ctx *ctx);

/* CUDA-core FMA throughput of this GPU in TFLOP/s (fp64 = 1: FP64, 0: FP32), measured by a
 * microbenchmark (8 independent FMA chains per thread, 8 blocks of 256 threads per SM, CUDA
 * events): the compute roofline of the FP64 gauge force and link exponentiation. */
int rhmc_fma_peak(rhmc_ctx *ctx, int fp64, double *tflops);

/* ------------------------------------------------------------------ launch-configuration autotuner
 * No counterpart in the reference (it fixes 128 threads per block, include/global_macro.h:8).
 * Every Dslash instantiation is built in three launch shapes (threads per block, minimum resident
 * blocks per SM; shape 0 is the compiled-in default).  The first launch of an instantiation on a
 * device at a volume, outside a stream capture, times the three on scratch spinors with CUDA
 * events and keeps the fastest; the solvers look their shapes up before capturing their graphs.
 * Dslash calls with n >= 5 right-hand sides likewise time their RHS packings (launches of at most
 * 8, 4 or 3 right-hand sides).  Choices are keyed by device name, volume and kernel.  The shapes
 * change no arithmetic: results are bit-identical whichever shape runs. */
/* Turns tuning on (default; RHMC_AUTOTUNE=0 in the environment starts with it off) or off (every
 * launch uses shape 0 and the default packing).  Returns the previous setting. */
int rhmc_autotune(int enable);
/* candidate >= 0: every tuned launch uses that candidate (0..2) instead of the tuned choice;
 * -1: tuned choices again.  Returns the previous value.  For tests and diagnostics. */
int rhmc_autotune_override(int candidate);
/* JSON cache of the choices: load merges the entries of `path` (a missing file is an empty cache)
 * and makes it the file every new choice is saved to; save writes the table to `path` (NULL: the
 * cache file).  The environment variable RHMC_TUNE_CACHE names a cache file loaded at first use. */
int rhmc_tune_cache_load(const char *path);
int rhmc_tune_cache_save(const char *path);
/* The table as JSON into buf (at most len bytes, NUL-terminated); returns the length needed. */
long rhmc_tune_report(char *buf, long len);
/* Forgets every choice (the next launches tune again). */
int rhmc_tune_clear(void);

/* No counterpart in the reference.  The same values as rhmc_true_residuals, for callers that
 * must not allocate device memory where they check their solutions: programs whose own pool
 * owns all device memory after start-up, chains sharing a GPU under a fixed memory budget, and
 * code that cannot accept the device-wide synchronisation an allocation may imply.  This entry
 * point takes its scratch from one fixed device array compiled into the library
 * (RHMC_NOALLOC_SCRATCH_BYTES, held on every GPU that loads the library until the process
 * exits) and calls no allocator.  Limits: Vh <= RHMC_NOALLOC_MAX_VH sites per parity and
 * nrhs*nshift <= RHMC_NOALLOC_MAX_SYSTEMS; larger requests return RHMC_ERR_ARG.  The array is
 * shared by all calls on a device and keeps the last call's contents: calls whose GPU work
 * overlaps race.  The call is host-synchronous (it waits for the context's stream and writes
 * `out` before returning).  The first call on a device looks up the array's device address
 * with that device current; make it before any stream capture.  x, b: FP64 internal device
 * spinors; out: host double[nrhs][nshift]. */
#define RHMC_NOALLOC_MAX_VH 65536
#define RHMC_NOALLOC_MAX_SYSTEMS 256
#define RHMC_NOALLOC_SCRATCH_BYTES (2u * 3u * 65536u * 16u + 256u * 8u + 256u * 8u)
int rhmc_true_residuals_noalloc(rhmc_ctx *ctx, int nshift, const double *shifts, int nrhs, const double *x, const double *b,
                                double *out);

#ifdef __cplusplus
}
#endif
#endif /* RHMC_B200_H */
