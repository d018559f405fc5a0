// ref_harness.cc -- TEST INFRASTRUCTURE ONLY (the reference side of the oracle).
//
// Compiled together with the UNMODIFIED CPU sources of coppolachan/RHMC-on-GPU by
// oracle/build_ref.py into oracle/_ref/libref_<tag>.so.  The reference keeps its fields in
// private arrays of Conf / Fermion / MultiFermion / ShiftMultiFermion / Momenta / Ipdot and
// reaches them only through friend functions declared in its headers (packer, CUDA glue).
// This file supplies its own bodies for those friend functions, which copy the private
// arrays exactly (FP64) from/to caller buffers, so that tests can inject identical inputs
// into the reference and into the CUDA path and compare outputs.  The reference's own code
// does all of the physics; nothing here re-implements it except the harness leapfrog, which
// composes the reference primitives with the sign of the wired integrators.
//
// The friend bodies below are declared by the reference with float array parameters
// (e.g. lib/Tools/Packer/packer.h:6-24); the harness passes double buffers cast to float*.

#define DEFINE_GLOBALS
#include "include/global_var.h"
#include "include/tools.h"
#include "include/geometry.h"
#include "lib/Action/fermions.h"
#include "lib/Action/fermionforce.h"
#include "lib/Action/action.h"
#include "lib/Action/staples.h"
#include "lib/Update/momenta.h"
#include "lib/Update/ipdot.h"
#include "lib/Update/MD_integrators/md_integrators.h"
#include "lib/Tools/RationalApprox/rationalapprox.h"
#include "lib/Action/Findminmax/findminmax.h"

void chiral_meas(complex<REAL> &chiral, complex<REAL> &e_dens, complex<REAL> &b_dens, complex<REAL> &p_dens);

#include <cstring>

static double h_min = 1.0e-3, h_max = 64.0;

// findminmax (lib/Action/Findminmax/findminmax.cc:140-183) is replaced by fixed bounds so that
// rescaling (lib/Tools/RationalApprox/rationalapprox.cc:134-266) is deterministic.  The power
// iterations of that file (findmaxeig, findmineig) are linked in unmodified (the recipe renames
// only its findminmax) and exposed below.
void findminmax(REAL &min, REAL &max) { min = h_min; max = h_max; }
void findmaxeig(REAL &max);
void findmineig(REAL &min, const REAL &max);

// ------------------------------------------------------------------ friend I/O hooks
void smartpack_gauge(float out[2 * 12 * no_links], const Conf *in)
{
    double *o = reinterpret_cast<double *>(out);
    for (long r = 0; r < no_links; r++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                o[r * 18 + i * 6 + j * 2] = real(in->u_work[r].comp[i][j]);
                o[r * 18 + i * 6 + j * 2 + 1] = imag(in->u_work[r].comp[i][j]);
            }
}

void smartunpack_gauge(Conf *out, const float in[2 * 12 * no_links])
{
    const double *s = reinterpret_cast<const double *>(in);
    complex<REAL> a[3][3];
    for (long r = 0; r < no_links; r++) {
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) a[i][j] = complex<REAL>(s[r * 18 + i * 6 + j * 2], s[r * 18 + i * 6 + j * 2 + 1]);
        out->u_work[r] = Su3(a);
    }
}

void smartpack_multifermion(float out[6 * sizeh * no_ps * 2], const MultiFermion *in)
{
    double *o = reinterpret_cast<double *>(out);
    for (int ps = 0; ps < no_ps; ps++)
        for (long i = 0; i < sizeh; i++)
            for (int c = 0; c < 3; c++) {
                o[(ps * sizeh + i) * 6 + c * 2] = real(in->fermion[ps][i].comp[c]);
                o[(ps * sizeh + i) * 6 + c * 2 + 1] = imag(in->fermion[ps][i].comp[c]);
            }
}

void smartunpack_multifermion(MultiFermion *out, const float in[6 * sizeh * no_ps * 2])
{
    const double *s = reinterpret_cast<const double *>(in);
    complex<REAL> a[3];
    for (int ps = 0; ps < no_ps; ps++)
        for (long i = 0; i < sizeh; i++) {
            for (int c = 0; c < 3; c++) a[c] = complex<REAL>(s[(ps * sizeh + i) * 6 + c * 2], s[(ps * sizeh + i) * 6 + c * 2 + 1]);
            out->fermion[ps][i] = Vec3(a);
        }
}

// Used in the READ direction: copies fermion_shiftmulti out into the (cast) buffer.
void smartunpack_multishiftfermion(ShiftMultiFermion *out, const float in[6 * sizeh * max_approx_order * no_ps * 2], int order)
{
    double *o = const_cast<double *>(reinterpret_cast<const double *>(in));
    for (int ps = 0; ps < no_ps; ps++)
        for (int k = 0; k < order; k++)
            for (long i = 0; i < sizeh; i++)
                for (int c = 0; c < 3; c++) {
                    long b = ((long)(ps * order + k) * sizeh + i) * 6 + c * 2;
                    o[b] = real(out->fermion[ps][k][i].comp[c]);
                    o[b + 1] = imag(out->fermion[ps][k][i].comp[c]);
                }
}

void smartpack_fermion_d(float out[6 * sizeh * 2], const Fermion *in)
{
    double *o = reinterpret_cast<double *>(out);
    for (long i = 0; i < sizeh; i++)
        for (int c = 0; c < 3; c++) {
            o[i * 6 + c * 2] = real(in->fermion[i].comp[c]);
            o[i * 6 + c * 2 + 1] = imag(in->fermion[i].comp[c]);
        }
}

void smartunpack_fermion_d(Fermion *out, const float in[6 * sizeh * 2])
{
    const double *s = reinterpret_cast<const double *>(in);
    complex<REAL> a[3];
    for (long i = 0; i < sizeh; i++) {
        for (int c = 0; c < 3; c++) a[c] = complex<REAL>(s[i * 6 + c * 2], s[i * 6 + c * 2 + 1]);
        out->fermion[i] = Vec3(a);
    }
}

void smartpack_tamatrix(float out[8 * no_links], Ipdot *in)
{
    double *o = reinterpret_cast<double *>(out);
    for (long r = 0; r < no_links; r++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                o[r * 18 + i * 6 + j * 2] = real(in->ipdot[r].comp[i][j]);
                o[r * 18 + i * 6 + j * 2 + 1] = imag(in->ipdot[r].comp[i][j]);
            }
}

void smartunpack_tamatrix(Ipdot *out, float in[8 * no_links])
{
    const double *s = reinterpret_cast<const double *>(in);
    complex<REAL> a[3][3];
    for (long r = 0; r < no_links; r++) {
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) a[i][j] = complex<REAL>(s[r * 18 + i * 6 + j * 2], s[r * 18 + i * 6 + j * 2 + 1]);
        out->ipdot[r] = Su3(a);
    }
}

void smartpack_thmatrix(float out[8 * no_links], Momenta *in)
{
    double *o = reinterpret_cast<double *>(out);
    for (long r = 0; r < no_links; r++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                o[r * 18 + i * 6 + j * 2] = real(in->momenta[r].comp[i][j]);
                o[r * 18 + i * 6 + j * 2 + 1] = imag(in->momenta[r].comp[i][j]);
            }
}

void smartunpack_thmatrix(Momenta *out, float in[8 * no_links])
{
    const double *s = reinterpret_cast<const double *>(in);
    complex<REAL> a[3][3];
    for (long r = 0; r < no_links; r++) {
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) a[i][j] = complex<REAL>(s[r * 18 + i * 6 + j * 2], s[r * 18 + i * 6 + j * 2 + 1]);
        out->momenta[r] = Su3(a);
    }
}

// The reference packer itself (lib/Tools/Packer/packer.cc), compiled unmodified with its
// functions renamed refpk_* (oracle/build_ref.py), for pinning the packed host formats.
void refpk_smartpack_gauge(float out[2 * 12 * no_links], const Conf *in);
void refpk_smartunpack_gauge(Conf *out, const float in[2 * 12 * no_links]);
void refpk_smartpack_fermion(float out[6 * sizeh], const Fermion *in);
void refpk_smartpack_fermion_d(float out[6 * sizeh * 2], const Fermion *in);
void refpk_smartunpack_fermion_d(Fermion *out, const float in[6 * sizeh * 2]);
void refpk_smartpack_multifermion(float out[6 * sizeh * no_ps * 2], const MultiFermion *in);
void refpk_smartunpack_multifermion(MultiFermion *out, const float in[6 * sizeh * no_ps * 2]);
void refpk_smartunpack_multishiftfermion(ShiftMultiFermion *out, const float in[6 * sizeh * max_approx_order * no_ps * 2],
                                         int order);
void refpk_make_shift_table(int table[8 * size]);
void refpk_smartpack_tamatrix(float out[8 * no_links], Ipdot *in);
void refpk_smartunpack_tamatrix(Ipdot *out, float in[8 * no_links]);
void refpk_smartpack_thmatrix(float out[8 * no_links], Momenta *in);
void refpk_smartunpack_thmatrix(Momenta *out, float in[8 * no_links]);

// ------------------------------------------------------------------ extern "C" surface
static Fermion *h_in = 0, *h_out = 0;

extern "C" {

int ref_dims(int *d)
{
    d[0] = nx; d[1] = ny; d[2] = nz; d[3] = nt;
    d[4] = no_ps; d[5] = max_approx_order; d[6] = no_md; d[7] = gauge_scale;
    return 0;
}

double ref_param(int which)
{
    switch (which) {
    case 0: return mass;
    case 1: return beta;
    case 2: return no_flavours;
    case 3: return residue_metro;
    case 4: return residue_md;
    case 5: return max_cg;
    default: return 0.0;
    }
}

// Allocation as in initialize() (lib/Main/init.cc:14-116), without Remez and without the
// run-time start configuration (fields are injected by the caller instead).
void ref_setup(unsigned long seed)
{
    initrand(seed);
    eta = new int[no_links];
    init_geo();
    gauge_conf = new Conf(0);
    gauge_staples = new Staples();
    gauge_momenta = new Momenta();
    gauge_ipdot = new Ipdot();
    d_vector1 = new double[size];
    d_vector2 = new double[size];
    c_vector1 = new complex<double>[size];
    c_vector2 = new complex<double>[size];
    plaq_test = new double[size];
    fermion_phi = new MultiFermion;
    fermion_chi = new MultiFermion;
    loc_r = new Fermion;
    loc_h = new Fermion;
    loc_s = new Fermion;
    loc_p = new Fermion;
    p_shiftferm = new ShiftFermion;
    fermion_shiftmulti = new ShiftMultiFermion;
    h_in = new Fermion;
    h_out = new Fermion;
    chi_e = new Fermion;  // the measurement fields (lib/Main/init.cc:71-76)
    chi_o = new Fermion;
    phi_e = new Fermion;
    phi_o = new Fermion;
    rnd_e = new Fermion;
    rnd_o = new Fermion;
    first_inv_approx_norm_coeff = new RationalApprox;
    md_inv_approx_norm_coeff = new RationalApprox;
    last_inv_approx_norm_coeff = new RationalApprox;
    update_iteration = 0;
}

// make_shift_table (lib/Tools/Packer/packer.cc:415-439) reads the same globals
// the reference's CPU power iterations for the bounds of M^dag M on the current links
// (findminmax.cc:12-137): each starts from a Gaussian vector of the reference's own generator and
// stops when the norm changes by less than 1e-5 relative
double ref_findmaxeig()
{
    REAL mx = 0;
    findmaxeig(mx);
    return mx;
}

double ref_findmineig(double max)
{
    REAL mn = 0;
    findmineig(mn, max);
    return mn;
}

void ref_tables(int *table, int *eta_out)
{
    for (long i = 0; i < size; i++)
        for (int mu = 0; mu < 4; mu++) {
            table[i + mu * size] = (int)nnm[i][mu];
            table[i + (4 + mu) * size] = (int)nnp[i][mu];
        }
    for (long i = 0; i < no_links; i++) eta_out[i] = eta[i];
}

// packer I/O: the reference packer between the harness's exact fields and packed floats
void ref_pk_gauge(float *out) { refpk_smartpack_gauge(out, gauge_conf); }
void ref_unpk_gauge(const float *in) { refpk_smartunpack_gauge(gauge_conf, in); }
void ref_pk_chi(float *out) { refpk_smartpack_multifermion(out, fermion_chi); }
void ref_unpk_chi(const float *in) { refpk_smartunpack_multifermion(fermion_chi, in); }
void ref_pk_fermion(float *out, const double *in)
{
    smartunpack_fermion_d(h_in, reinterpret_cast<const float *>(in));
    refpk_smartpack_fermion(out, h_in);
}
void ref_pk_fermion_d(float *out, const double *in)
{
    smartunpack_fermion_d(h_in, reinterpret_cast<const float *>(in));
    refpk_smartpack_fermion_d(out, h_in);
}
void ref_unpk_fermion_d(double *out, const float *in)
{
    refpk_smartunpack_fermion_d(h_in, in);
    smartpack_fermion_d(reinterpret_cast<float *>(out), h_in);
}
void ref_unpk_shifted(const float *in, int order) { refpk_smartunpack_multishiftfermion(fermion_shiftmulti, in, order); }
void ref_pk_ipdot(float *out) { refpk_smartpack_tamatrix(out, gauge_ipdot); }
void ref_unpk_ipdot(const float *in) { refpk_smartunpack_tamatrix(gauge_ipdot, const_cast<float *>(in)); }
void ref_pk_momenta(float *out) { refpk_smartpack_thmatrix(out, gauge_momenta); }
void ref_unpk_momenta(const float *in) { refpk_smartunpack_thmatrix(gauge_momenta, const_cast<float *>(in)); }
void ref_shift_table(int *table) { refpk_make_shift_table(table); }

void ref_set_links(const double *u) { smartunpack_gauge(gauge_conf, reinterpret_cast<const float *>(u)); gauge_conf->save(); }
void ref_get_links(double *u) { smartpack_gauge(reinterpret_cast<float *>(u), gauge_conf); }
void ref_unitarize_with_eta(void) { gauge_conf->unitarize_with_eta(); }
void ref_set_momenta(const double *p) { smartunpack_thmatrix(gauge_momenta, const_cast<float *>(reinterpret_cast<const float *>(p))); }
void ref_get_momenta(double *p) { smartpack_thmatrix(reinterpret_cast<float *>(p), gauge_momenta); }
void ref_set_ipdot(const double *p) { smartunpack_tamatrix(gauge_ipdot, const_cast<float *>(reinterpret_cast<const float *>(p))); }
void ref_get_ipdot(double *p) { smartpack_tamatrix(reinterpret_cast<float *>(p), gauge_ipdot); }
void ref_set_phi(const double *f) { smartunpack_multifermion(fermion_phi, reinterpret_cast<const float *>(f)); }
void ref_get_phi(double *f) { smartpack_multifermion(reinterpret_cast<float *>(f), fermion_phi); }
void ref_set_chi(const double *f) { smartunpack_multifermion(fermion_chi, reinterpret_cast<const float *>(f)); }
void ref_get_chi(double *f) { smartpack_multifermion(reinterpret_cast<float *>(f), fermion_chi); }
void ref_get_shifted(double *f, int order) { smartunpack_multishiftfermion(fermion_shiftmulti, reinterpret_cast<const float *>(f), order); }

// Deo / Doe: lib/Action/fermionmatrix.cc:8-97
void ref_deo(double *out, const double *in)
{
    smartunpack_fermion_d(h_in, reinterpret_cast<const float *>(in));
    Deo(h_out, h_in);
    smartpack_fermion_d(reinterpret_cast<float *>(out), h_out);
}

void ref_doe(double *out, const double *in)
{
    smartunpack_fermion_d(h_in, reinterpret_cast<const float *>(in));
    Doe(h_out, h_in);
    smartpack_fermion_d(reinterpret_cast<float *>(out), h_out);
}

// Repeated application for the CPU baseline timing (no copies inside the loop).
void ref_dslash_loop(int n, const double *in)
{
    smartunpack_fermion_d(h_in, reinterpret_cast<const float *>(in));
    for (int k = 0; k < n; k++) {
        Doe(h_out, h_in);
        Deo(h_in, h_out);
    }
}

// Rational approximations (normalised, on [min_eps, 1]); which = 0 first (heatbath),
// 1 md (force), 2 last (action).  They are rescaled by the reference with findminmax bounds.
void ref_set_approx(int which, int order, double min_eps, double a0, const double *a, const double *b)
{
    RationalApprox ra(min_eps, order, a0, a, b);
    if (which == 0) *first_inv_approx_norm_coeff = ra;
    else if (which == 1) *md_inv_approx_norm_coeff = ra;
    else *last_inv_approx_norm_coeff = ra;
}

void ref_set_minmax(double mn, double mx) { h_min = mn; h_max = mx; }

// multips_shifted_invert (lib/Action/Inverter/inverter.cc:142-339) on fermion_chi with
// the given (already rescaled) shifts; results stay in fermion_shiftmulti.
void ref_msolve(double res, int order, const double *shifts)
{
    double a[max_approx_order];
    double b[max_approx_order];
    for (int i = 0; i < max_approx_order; i++) { a[i] = 1.0; b[i] = (i < order) ? shifts[i] : 0.0; }
    RationalApprox ra(1.0, order, 0.0, a, b);
    multips_shifted_invert(fermion_shiftmulti, fermion_chi, res, ra);
}

void ref_first_inv_approx_calc(double res) { first_inv_approx_calc(res); }
void ref_last_inv_approx_calc(double res) { last_inv_approx_calc(res); }

void ref_calc_ipdot(void) { calc_ipdot(); }
void ref_calc_ipdot_gauge(void) { calc_ipdot_gauge(); }
void ref_calc_ipdot_fermion(void) { calc_ipdot_fermion(); }
void ref_calc_staples(double *st)
{
    calc_staples();
    // staples are private to Staples; ipdot is used as the carrier through its friend hook
    (void)st;
}

void ref_mom_update(double step) { momenta_sum_multiply(complex<REAL>(0.0, step)); }
void ref_link_update(double step) { conf_left_exp_multiply(complex<REAL>(0.0, step)); }

// calc_action (lib/Action/action.cc:111-156) begin/end; ref_action_end returns
// de = action_new - action_old exactly as update() forms it (lib/Update/update.cc:112-114).
void ref_action_begin(void) { calc_action(plaq_test, 0); }
double ref_action_end(void)
{
    calc_action(plaq_test, -1);
    global_sum(plaq_test, size);
    return -plaq_test[0];
}

// Conf::calc_poly (lib/Measurements/gaugemeas.cc:66-106) measures u_save; saved first.
void ref_polyakov(double *re, double *im)
{
    gauge_conf->save();
    REAL r, i;
    gauge_conf->calc_poly(r, i);
    *re = r;
    *im = i;
}

// chiral_meas (lib/Measurements/chiralmeas.cc:18-194) draws its own Z2 noise (rand_vect = 1) and
// solves with the CPU CG; the noise it used is copied out afterwards so that the CUDA path can be
// given the same vectors.  out: chiral, energy, baryon and pressure densities as (re, im).
void ref_chiral_meas(double *out, double *noise_e, double *noise_o)
{
    complex<REAL> ch, ed, bd, pd;
    chiral_meas(ch, ed, bd, pd);
    out[0] = real(ch); out[1] = imag(ch);
    out[2] = real(ed); out[3] = imag(ed);
    out[4] = real(bd); out[5] = imag(bd);
    out[6] = real(pd); out[7] = imag(pd);
    smartpack_fermion_d(reinterpret_cast<float *>(noise_e), rnd_e);
    smartpack_fermion_d(reinterpret_cast<float *>(noise_o), rnd_o);
}

// Conf::write_last (lib/Main/Conf/conf.cc:175-200) into ./config, and the stored-conf start of
// Conf::Conf (conf.cc:55-94) from ./config, whose links are copied out exactly.
void ref_write_conf(void)
{
    gauge_conf->save();
    gauge_conf->write_last();
}

void ref_read_conf(double *u)
{
    Conf *t = new Conf(2);
    smartpack_gauge(reinterpret_cast<float *>(u), t);
    delete t;
}

// Conf::calc_plaq measures u_save; the harness saves u_work first.
void ref_plaquette(double *pls, double *plt)
{
    gauge_conf->save();
    REAL s, t;
    gauge_conf->calc_plaq(s, t);
    *pls = s;
    *plt = t;
}

void ref_minimum_norm2_A(void) { minimum_norm2_A(); }
void ref_multistep_2MN(void) { multistep_2MN(); }
void ref_multistep_4MN(void) { multistep_4MN(); }

// Leapfrog composed of the reference primitives with the momentum kick sign of the wired
// integrators (minimum_norm2.cc:52 uses -iepsh); lib/Update/MD_integrators/leapfrog.cc:39,53
// kicks with +ieps, a sign that no wired integrator uses.
void ref_leapfrog_wired(void)
{
    conf_left_exp_multiply(iepsh);
    for (int md = 1; md < no_md; md++) {
        calc_ipdot();
        momenta_sum_multiply(-ieps);
        conf_left_exp_multiply(ieps);
    }
    calc_ipdot();
    momenta_sum_multiply(-ieps);
    conf_left_exp_multiply(iepsh);
}

// One trajectory with injected momenta/phi (update(), lib/Update/update.cc:58-152, without
// its RNG draws): heatbath, initial action, integrator, action solve, final action,
// Metropolis against the injected uniform.  integrator: 0 2MN, 1 multistep 2MN,
// 2 multistep 4MN, 3 wired-sign leapfrog.  Returns Delta S; *acc = 1 accepted, 0 rejected.
double ref_trajectory(int integrator, double uniform, int *acc)
{
    first_inv_approx_calc(residue_metro);
    calc_action(plaq_test, 0);
    if (integrator == 0) minimum_norm2_A();
    else if (integrator == 1) multistep_2MN();
    else if (integrator == 2) multistep_4MN();
    else ref_leapfrog_wired();
    last_inv_approx_calc(residue_metro);
    calc_action(plaq_test, -1);
    global_sum(plaq_test, size);
    double de = -plaq_test[0];
    if (de < 0 || uniform < exp(-de)) { *acc = 1; gauge_conf->save(); }
    else { *acc = 0; gauge_conf->copy_saved(); }
    return de;
}

}  // extern "C"
