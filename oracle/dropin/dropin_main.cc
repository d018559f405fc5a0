// dropin_main.cc -- TEST INFRASTRUCTURE ONLY.
//
// A host program made of the reference's own, unmodified sources: the lib/ tree of
// coppolachan/RHMC-on-GPU compiled as it lies, with this file in place of its main program
// (lib/Main/rhmc.cc:26-200).  Built twice by oracle/dropin/build_dropin.py:
//   * without USE_GPU: the reference's CPU trajectory;
//   * with USE_GPU, linked against librhmc_b200.so in place of the reference's lib/Cuda: the
//     reference's GPU code path (update.cc:58-152 -> gpu.cc, cu_inverter.cc, fermionforce.cc,
//     ipdot.cc, momenta.cc, rationalapprox.cc) running on this library's entry points.
// Both run the same trajectories from the same seed (the reference's own RNG draws the momenta,
// pseudofermions and Metropolis uniforms), so their outputs can be compared.
//
// Beyond what rhmc.cc does, this program
//   * supplies rationalapprox_calc (rationalapprox_calc.cc:8-177 needs MPFR/GMP, absent here):
//     the normalised approximations are read from the file named by RHMC_DROPIN_COEFFS;
//   * supplies findminmax (findminmax.cc:140-183) as fixed bounds from the same file, so that the
//     CPU and GPU builds rescale identically;
//   * in the GPU build calls rhmc_legacy_bind once after initialize() and before the first
//     gpu_init0 (the library cannot see the program's compile-time constants and buffers);
//   * prints the plaquette after every trajectory and sets cout to 17 digits, so that the
//     "Delta S" update() prints is exact.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#define DEFINE_GLOBALS
#include "include/rhmc_include.h"
#include "include/global_var.h"
#include "include/init.h"
#include "include/parameters.h"
#include "include/tools.h"
#include "include/update.h"
#include "lib/Action/Findminmax/findminmax.h"
#ifdef USE_GPU
#include "include/gpu.h"
#include "rhmc_legacy.h"
#endif

static REAL g_min_bound, g_max_bound;

// File format (whitespace separated):
//   bounds <lambda_min> <lambda_max>
//   approx <which: 0 first, 1 md, 2 last> <order> <min_eps> <a0> <a_1..a_order> <b_1..b_order>
void rationalapprox_calc(void)
{
    const char *path = getenv("RHMC_DROPIN_COEFFS");
    std::ifstream in(path ? path : "");
    if (!in) {
        std::cerr << "dropin: set RHMC_DROPIN_COEFFS to the coefficient file\n";
        exit(3);
    }
    std::string tag;
    RationalApprox *which_ptr[3] = {nullptr, nullptr, nullptr};
    while (in >> tag) {
        if (tag == "bounds") {
            in >> g_min_bound >> g_max_bound;
        } else if (tag == "approx") {
            int which, n;
            REAL eps, a0;
            in >> which >> n >> eps >> a0;
            std::vector<REAL> a(n), b(n);
            for (int i = 0; i < n; i++) in >> a[i];
            for (int i = 0; i < n; i++) in >> b[i];
            if (which < 0 || which > 2 || n < 1 || n > max_approx_order) {
                std::cerr << "dropin: bad approximation record\n";
                exit(3);
            }
            which_ptr[which] = new RationalApprox(eps, n, a0, a.data(), b.data());
        }
    }
    if (!which_ptr[0] || !which_ptr[1] || !which_ptr[2]) {
        std::cerr << "dropin: the coefficient file needs approximations 0, 1 and 2\n";
        exit(3);
    }
    first_inv_approx_norm_coeff = which_ptr[0];
    md_inv_approx_norm_coeff = which_ptr[1];
    last_inv_approx_norm_coeff = which_ptr[2];
    meas_inv_coeff = new RationalApprox(*which_ptr[2]);  // used by the measurements only
}

void findminmax(REAL &min, REAL &max)
{
    min = g_min_bound;
    max = g_max_bound;
}

int main(int argc, char **argv)
{
    const int ntraj = argc > 1 ? atoi(argv[1]) : 5;
    if (initialize() != 0) return 1;
    std::cout.precision(17);
#ifdef USE_GPU
    rhmc_legacy_config cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.nx = nx;
    cfg.ny = ny;
    cfg.nz = nz;
    cfg.nt = nt;
    cfg.ferm_temp_bc = ferm_temp_bc;
    cfg.mass = mass;
    cfg.beta = beta;
    cfg.no_ps = no_ps;
    cfg.max_approx_order = max_approx_order;
    cfg.max_cg = max_cg;
    cfg.device = gpu_device_to_use;
    cfg.gauge_field_packed = gauge_field_packed;
    cfg.chi_packed = chi_packed;
    cfg.simple_fermion_packed = simple_fermion_packed;
    cfg.ipdot_packed = ipdot_packed;
    cfg.momenta_packed = momenta_packed;
    cfg.shift_table = shift_table;
    cfg.eta = eta;
    if (rhmc_legacy_bind(&cfg) != RHMC_OK) {
        std::cerr << "dropin: rhmc_legacy_bind failed: " << rhmc_last_error() << "\n";
        return 2;
    }
#endif
    for (int t = 0; t < ntraj; t++) {
#ifdef USE_GPU
        gpu_init0();
#endif
        int acc = 0;
        update(acc);
        REAL pls, plt;
        gauge_conf->calc_plaq(pls, plt);
        printf("TRAJ %d acc %d plaq %.17g %.17g\n", t, acc, (double)pls, (double)plt);
        fflush(stdout);
        update_iteration++;
    }
    return 0;
}
