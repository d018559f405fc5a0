// driver.cu -- the molecular-dynamics driver of lib/Update on device-resident fields.
//
// Mirrors, with the same steps and coefficients:
//   first/last_inv_approx_calc   lib/Tools/RationalApprox/rationalapprox.cc:134-369 (rescale by the
//                                eigenvalue bounds, shifted solve, chi = a0 phi + sum a_i x_i)
//   fermionforce / calc_ipdot*   lib/Action/fermionforce.cc:10-110, lib/Update/ipdot.cc:25-196
//   minimum_norm2_A              lib/Update/MD_integrators/minimum_norm2.cc:28-105
//   multistep_2MN(_gauge)        multistep_2MN.cc:31-168
//   multistep_4MN(_gauge)        multistep_4MN.cc:30-300
//   leapfrog                     leapfrog.cc:18-62, with the momentum kick sign of the wired
//                                integrators (-i eps); the reference kicks with +i eps, a sign no
//                                reachable code path uses (update.cc:29-43)
//   update / update_nometro      lib/Update/update.cc:17-152 with the momenta, the pseudofermions and
//                                the Metropolis uniform supplied by the caller instead of drawn
//                                from the host RNG
// The eigenvalue bounds that findminmax would compute (findminmax.cc:140-183) are supplied by
// the caller (rhmc_set_eig_bounds); they are widened by 0.95/1.05 as the reference does.
// Fields stay on the device for the whole trajectory; nothing is reallocated per trajectory.
//
// Fermion species.  The reference has one species (mass, no_flavours, no_ps).  Further species
// (e.g. the strange quark of N_f = 2+1) are added with rhmc_driver_add_species; each has its own
// pseudofermions, rational approximations and eigenvalue bounds, and every heatbath, action and
// force sums over all species.  A species of mass m_s >= the context mass m runs on the same
// links and solver with every pole shifted by m_s^2 - m^2, since M^dag M(m_s) = M^dag M(m) +
// m_s^2 - m^2 on the even sites.
#include <cmath>
#include <cstring>
#include <string>
#include <algorithm>
#include <vector>

#include <random>

#include "capi_util.h"
#include "context.h"
#include "kernels.h"
#include "solver.h"
#include "../../include/rhmc_legacy.h"

namespace rhmc {

int gauge_force(rhmc_ctx *c, int mode);
int fermion_force(rhmc_ctx *c, int nrhs, int nshift, const double *a, const double2 *x, int mode);
int mom_update(rhmc_ctx *c, double step);
int link_update(rhmc_ctx *c, double step);
int plaquette_sums(rhmc_ctx *c, double *temporal, double *spatial);
int momentum_action(rhmc_ctx *c, double *out);
int rdot(rhmc_ctx *c, const double2 *a, const double2 *b, long n, double *out);
int rational_sum(rhmc_ctx *c, int nrhs, int nshift, double a0, const double *a, const double2 *x, const double2 *b, double2 *out,
                 int add);

struct Approx {
    int order = 0;
    double a0 = 0, min_eps = 1;
    std::vector<double> a, b;
};

struct Species {
    double mass = 0;
    int no_flavours = 0, no_ps = 0;
    Approx approx[3];  // first (heatbath), md (force), last (action); normalised on [min_eps, 1]
    double eig_min = 0, eig_max = 0;  // of M^dag M at this species' mass
    bool have_bounds = false;
};

struct Driver {
    rhmc_driver_params P;
    bool configured = false;
    std::vector<Species> sp;  // sp[0]: the context mass with P.no_flavours, P.no_ps
    int cur = 0;              // the species the approx / bounds / phi / chi setters act on
    long force_evals = 0, solves = 0;
    rhmc_msolve_info sums[2] = {};  // md, metro solves (rhmc_driver_solver_stats)
    int cat = 1;                    // the sum the next solves go to (0 md, 1 metro)
    std::vector<double> pw_start;  // start vector of the power iterations (auto_bounds)
};

static void add_info(rhmc_msolve_info &a, const rhmc_msolve_info &b)
{
    a.status = b.status ? b.status : a.status;
    for (int j = 0; j < 8; j++) a.iters[j] = b.iters[j];
    a.refine_iters += b.refine_iters;
    a.reliable_updates += b.reliable_updates;
    a.seconds += b.seconds;
    a.seconds_phase_a += b.seconds_phase_a;
    a.systems_refined += b.systems_refined;
    a.iters_total += b.iters_total;
    a.iters_max = b.iters_max > a.iters_max ? b.iters_max : a.iters_max;
    a.iters_fp64 += b.iters_fp64;
    a.ms_reliable_updates += b.ms_reliable_updates;
}

// one rhmc_msolve call of the driver, its info added to the md (force) or metro sums
static int driver_msolve(rhmc_ctx *c, const rhmc_msolve_params *mp, double *x, const double *b)
{
    rhmc_msolve_info info;
    memset(&info, 0, sizeof(info));
    const int rc = rhmc_msolve(c, mp, x, b, &info);
    Driver *d = c->driver;
    add_info(d->sums[d->cat], info);
    return rc;
}

static Driver *drv(rhmc_ctx *c) { return c->driver; }

static Driver *ensure_driver(rhmc_ctx *c)
{
    if (!c->driver) {
        c->driver = new Driver();
        c->driver->sp.resize(1);
        c->driver->sp[0].mass = c->mass;
    }
    return c->driver;
}

static int nspecies(rhmc_ctx *c) { return (int)drv(c)->sp.size(); }

// workspace name of a per-species field: "drv_phi", "drv_phi.1", ...
static std::string fname(const char *base, int s) { return s == 0 ? std::string(base) : std::string(base) + "." + std::to_string(s); }

void driver_free(Driver *d) { delete d; }

static size_t SP(rhmc_ctx *c) { return 3 * (size_t)c->Vh; }

static int field(rhmc_ctx *c, const std::string &name, size_t n_spinors, double2 **out)
{
    void *p;
    CK(c->ws.get(name, n_spinors * SP(c) * sizeof(double2), &p));
    *out = (double2 *)p;
    return RHMC_OK;
}

// RationalApprox::*_inv_approx_coeff (rationalapprox.cc:134-266) for species s
static Approx rescaled(rhmc_ctx *c, int s, int which)
{
    const Species &S = drv(c)->sp[s];
    Approx r = S.approx[which];
    const double mx = S.eig_max * 1.05;
    const double ex = which == 0 ? ((double)S.no_flavours) / 8. / ((double)S.no_ps)
                                 : -((double)S.no_flavours) / 4. / ((double)S.no_ps);
    const double e = pow(mx, ex);
    r.a0 *= e;
    for (int i = 0; i < r.order; i++) {
        r.a[i] *= (mx * e);
        r.b[i] *= mx;
    }
    return r;
}

// (M^dag M(m_s) + b_i) x_i = b for the species' pseudofermions, on the context's M^dag M(m)
static int solve(rhmc_ctx *c, int s, const Approx &ap, double res, int mode, int fmt, const double2 *b, double2 *x)
{
    Driver *d = drv(c);
    const double dm2 = d->sp[s].mass * d->sp[s].mass - c->mass * c->mass;
    std::vector<double> shifts(ap.b);
    if (s != 0)
        for (double &v : shifts) v += dm2;
    rhmc_msolve_params mp;
    memset(&mp, 0, sizeof(mp));
    mp.nshift = ap.order;
    mp.shifts = shifts.data();
    mp.nrhs = d->sp[s].no_ps;
    mp.residual = res;
    mp.max_iter = d->P.max_cg;
    mp.mode = mode;
    mp.fmt = fmt;
    if (!d->P.single_rhs) {
        d->solves++;
        return driver_msolve(c, &mp, (double *)x, (const double *)b);
    }
    mp.nrhs = 1;
    for (int ps = 0; ps < d->sp[s].no_ps; ps++) {
        d->solves++;
        const int rc = driver_msolve(c, &mp, (double *)(x + (size_t)ps * ap.order * SP(c)), (const double *)(b + (size_t)ps * SP(c)));
        if (rc) return rc;
    }
    return RHMC_OK;
}

// Every pseudofermion of every species solved against its pole set: (M^dag M(m_s) + b_{s,i}) x =
// in_s, with in_s the species field fname(in_base, s).  When all species have the same number of
// poles they go through a single batched multi-shift call with a pole set per right-hand side,
// so every link load serves all of them and a lighter species' iterations carry the heavier
// one's at little extra cost; otherwise species by species.  x ("drv_x"): species s's
// [no_ps][order] solutions start at spinor xoff[s].
struct Solved {
    std::vector<Approx> ap;   // rescaled approximation per species
    std::vector<size_t> xoff; // first spinor of each species in x
    double2 *x = nullptr;
};

// Pole groups (rhmc_driver_params.pole_group = G > 0): approximation `which` is applied in
// ceil(order / G) groups of consecutive poles, each solved, used and dropped before the next, so
// only one group's shifted solutions (and solver vectors) are on the device at a time; G = 0
// keeps one group holding every pole.
static int pole_groups(rhmc_ctx *c, int which)
{
    Driver *d = drv(c);
    const int G = d->P.pole_group;
    if (G <= 0) return 1;
    int mx = 0;
    for (const Species &S : d->sp) mx = std::max(mx, S.approx[which].order);
    return (mx + G - 1) / G;
}

// poles [g G, g G + G) of ap (all of them when G == 0); the constant a0 belongs to group 0
static Approx pole_slice(const Approx &ap, int g, int G)
{
    if (G <= 0) return ap;
    Approx r;
    const int lo = std::min(g * G, ap.order), hi = std::min(lo + G, ap.order);
    r.order = hi - lo;
    r.a0 = g == 0 ? ap.a0 : 0.0;
    r.min_eps = ap.min_eps;
    r.a.assign(ap.a.begin() + lo, ap.a.begin() + hi);
    r.b.assign(ap.b.begin() + lo, ap.b.begin() + hi);
    return r;
}

// group g of the poles (species without poles in that group get order 0 and no solve)
static int solve_species(rhmc_ctx *c, int which, const char *in_base, double res, int mode, int fmt, Solved &out,
                         int g = 0)
{
    Driver *d = drv(c);
    const int ns = nspecies(c);
    out.ap.clear();
    out.xoff.clear();
    int total = 0;
    bool same = true;
    size_t xtot = 0;
    for (int s = 0; s < ns; s++) {
        out.ap.push_back(pole_slice(rescaled(c, s, which), g, d->P.pole_group));
        same = same && out.ap[s].order == out.ap[0].order;
        out.xoff.push_back(xtot);
        xtot += (size_t)d->sp[s].no_ps * out.ap[s].order;
        total += d->sp[s].no_ps;
    }
    int rc = field(c, "drv_x", xtot, &out.x);
    if (rc) return rc;
    if (ns == 1 || !same || d->P.single_rhs) {
        for (int s = 0; s < ns; s++) {
            if (out.ap[s].order == 0) continue;
            double2 *in = nullptr;
            rc = field(c, fname(in_base, s), d->sp[s].no_ps, &in);
            if (rc) return rc;
            rc = solve(c, s, out.ap[s], res, mode, fmt, in, out.x + out.xoff[s] * SP(c));
            if (rc) return rc;
        }
        return RHMC_OK;
    }
    const int order = out.ap[0].order;
    double2 *bcat = nullptr;
    rc = field(c, "drv_bcat", total, &bcat);
    if (rc) return rc;
    std::vector<double> sh((size_t)total * order);
    int r = 0;
    for (int s = 0; s < ns; s++) {
        const int nps = d->sp[s].no_ps;
        double2 *in = nullptr;
        rc = field(c, fname(in_base, s), nps, &in);
        if (rc) return rc;
        CK(cudaMemcpyAsync(bcat + (size_t)r * SP(c), in, (size_t)nps * SP(c) * sizeof(double2), cudaMemcpyDeviceToDevice,
                           c->stream));
        const double dm2 = s == 0 ? 0.0 : d->sp[s].mass * d->sp[s].mass - c->mass * c->mass;
        for (int ps = 0; ps < nps; ps++, r++)
            for (int i = 0; i < order; i++) sh[(size_t)r * order + i] = out.ap[s].b[i] + dm2;
    }
    rhmc_msolve_params mp;
    memset(&mp, 0, sizeof(mp));
    mp.nshift = order;
    mp.shifts = sh.data();
    mp.rhs_shifts = sh.data();
    mp.nrhs = total;
    mp.residual = res;
    mp.max_iter = d->P.max_cg;
    mp.mode = mode;
    mp.fmt = fmt;
    d->solves++;
    return driver_msolve(c, &mp, (double *)out.x, (const double *)bcat);
}

// findminmax (findminmax.cc:140-183) on the device, for the current links: FP64 power iterations
// for lambda_max of M^dag M at the context mass and (auto_bounds 1) for lambda_min through
// lambda_max - M^dag M, or (auto_bounds 2) lambda_min = mass^2; a species of mass m_s gets both
// shifted by m_s^2 - m^2.  The start vector is a fixed pseudo-random spinor.
static int compute_bounds(rhmc_ctx *c)
{
    Driver *d = drv(c);
    if (d->pw_start.size() != 6 * (size_t)c->Vh) {
        std::mt19937_64 rng(0x5eedULL);
        std::normal_distribution<double> nd(0.0, 1.0);
        d->pw_start.resize(6 * (size_t)c->Vh);
        for (double &v : d->pw_start) v = nd(rng);
    }
    double mx = 0.0, mn = c->mass * c->mass;
    int rc = rhmc_find_max(c, d->pw_start.data(), &mx);
    if (rc) return rc;
    if (d->P.auto_bounds == 1 && (rc = rhmc_find_min(c, d->pw_start.data(), mx, &mn))) return rc;
    for (int s = 0; s < nspecies(c); s++) {
        Species &S = d->sp[s];
        const double dm2 = S.mass * S.mass - c->mass * c->mass;
        S.eig_min = mn + dm2;
        S.eig_max = mx + dm2;
        S.have_bounds = true;
    }
    return RHMC_OK;
}

static int check_ready(rhmc_ctx *c)
{
    Driver *d = drv(c);
    if (!d || !d->configured) return fail(RHMC_ERR_STATE, "driver not configured (rhmc_driver_setup)");
    if (d->P.auto_bounds && !d->sp[0].have_bounds) {
        const int rc = compute_bounds(c);
        if (rc) return rc;
    }
    for (int s = 0; s < nspecies(c); s++) {
        const Species &S = d->sp[s];
        if (!S.have_bounds) return fail(RHMC_ERR_STATE, "species %d: eigenvalue bounds not set (rhmc_set_eig_bounds)", s);
        for (int w = 0; w < 3; w++)
            if (S.approx[w].order < 1)
                return fail(RHMC_ERR_STATE, "species %d: rational approximation %d not set (rhmc_set_approx)", s, w);
    }
    return RHMC_OK;
}

// chi = r_first(M^dag M) phi (first_inv_approx_calc) or phi = r_last(M^dag M) chi (last_...),
// for every species
static int inv_approx_calc(rhmc_ctx *c, int which, double res)
{
    int rc = check_ready(c);
    if (rc) return rc;
    Driver *d = drv(c);
    d->cat = 1;
    for (int g = 0; g < pole_groups(c, which); g++) {
        Solved sv;
        if ((rc = solve_species(c, which, which == 0 ? "drv_phi" : "drv_chi", res, d->P.metro_mode, d->P.metro_fmt, sv, g)))
            return rc;
        for (int s = 0; s < nspecies(c); s++) {
            const int nps = d->sp[s].no_ps;
            const Approx &ap = sv.ap[s];
            if (ap.order == 0) continue;
            double2 *phi = nullptr, *chi = nullptr;
            rc = field(c, fname("drv_phi", s), nps, &phi);
            if (rc) return rc;
            rc = field(c, fname("drv_chi", s), nps, &chi);
            if (rc) return rc;
            const double2 *in = which == 0 ? phi : chi;
            double2 *out = which == 0 ? chi : phi;
            // group 0: out = a0 in + its poles; later groups add their poles to out
            if ((rc = rational_sum(c, nps, ap.order, ap.a0, ap.a.data(), sv.x + sv.xoff[s] * SP(c), in, out, g > 0))) return rc;
        }
    }
    return RHMC_OK;
}

// calc_ipdot_fermion (overwrite) or its part of calc_ipdot (add): the sum over species
static int fermion_part(rhmc_ctx *c, int add)
{
    int rc = check_ready(c);
    if (rc) return rc;
    Driver *d = drv(c);
    d->cat = 0;
    for (int g = 0; g < pole_groups(c, 1); g++) {
        Solved sv;
        if ((rc = solve_species(c, 1, "drv_chi", d->P.residue_md, d->P.md_mode, d->P.md_fmt, sv, g))) return rc;
        for (int s = 0; s < nspecies(c); s++) {
            const Approx &ap = sv.ap[s];
            if (ap.order == 0) continue;
            rc = fermion_force(c, d->sp[s].no_ps, ap.order, ap.a.data(), sv.x + sv.xoff[s] * SP(c), (g == 0 && s == 0) ? add : 1);
            if (rc) return rc;
        }
    }
    d->force_evals++;
    return RHMC_OK;
}

// S_f = sum_ps chi_ps^dag r_md(M^dag M) chi_ps = sum_ps [a0 |chi|^2 + sum_i a_i Re<chi, x_i>]
// with the rescaled md approximation: the action whose derivative calc_ipdot_fermion is
// (the md pole set of fermionforce, lib/Action/fermionforce.cc:27-38)
static int fermion_action_md(rhmc_ctx *c, double *out)
{
    int rc = check_ready(c);
    if (rc) return rc;
    Driver *d = drv(c);
    d->cat = 0;
    double sum = 0.0, v;
    for (int g = 0; g < pole_groups(c, 1); g++) {
        Solved sv;
        if ((rc = solve_species(c, 1, "drv_chi", d->P.residue_md, d->P.md_mode, d->P.md_fmt, sv, g))) return rc;
        for (int s = 0; s < nspecies(c); s++) {
            const int nps = d->sp[s].no_ps;
            const Approx &ap = sv.ap[s];
            const double2 *xs = sv.x + sv.xoff[s] * SP(c);
            double2 *chi = nullptr;
            rc = field(c, fname("drv_chi", s), nps, &chi);
            if (rc) return rc;
            for (int ps = 0; ps < nps; ps++) {
                const double2 *cp = chi + ps * SP(c);
                if (g == 0) {
                    if ((rc = rdot(c, cp, cp, (long)SP(c), &v))) return rc;
                    sum += ap.a0 * v;
                }
                for (int i = 0; i < ap.order; i++) {
                    if ((rc = rdot(c, cp, xs + ((size_t)ps * ap.order + i) * SP(c), (long)SP(c), &v))) return rc;
                    sum += ap.a[i] * v;
                }
            }
        }
    }
    *out = sum;
    return RHMC_OK;
}

static int calc_ipdot_full(rhmc_ctx *c)
{
    int rc = gauge_force(c, 0);
    if (rc) return rc;
    return fermion_part(c, 1);
}

// ------------------------------------------------------------------ integrator schedules
enum Kind { KICK_FULL, KICK_FERMION, KICK_GAUGE, DRIFT };
struct Step {
    Kind k;
    double c;  // P += i c ipdot after computing the force (KICK_*), or U <- exp(i c P) U (DRIFT)
};

static const double L2MN = 0.1931833275037836;  // Omelyan et al. (minimum_norm2.cc:35)
static const double T4 = 0.08398315262876693, R4 = 0.2539785108410595, L4 = 0.6822365335719091, M4 = -0.03230286765269967;

static void sched_2MN_A(std::vector<Step> &s, int no_md, double eps)
{
    const double epsh = eps * 0.5;
    s.push_back({DRIFT, eps * L2MN});
    for (int md = 1; md < no_md; md++) {
        s.push_back({KICK_FULL, -epsh});
        s.push_back({DRIFT, eps * (1.0 - 2.0 * L2MN)});
        s.push_back({KICK_FULL, -epsh});
        s.push_back({DRIFT, eps * (2.0 * L2MN)});
    }
    s.push_back({KICK_FULL, -epsh});
    s.push_back({DRIFT, eps * (1.0 - 2.0 * L2MN)});
    s.push_back({KICK_FULL, -epsh});
    s.push_back({DRIFT, eps * L2MN});
}

static void sched_leapfrog(std::vector<Step> &s, int no_md, double eps)
{
    const double epsh = eps * 0.5;
    s.push_back({DRIFT, epsh});
    for (int md = 1; md < no_md; md++) {
        s.push_back({KICK_FULL, -eps});
        s.push_back({DRIFT, eps});
    }
    s.push_back({KICK_FULL, -eps});
    s.push_back({DRIFT, epsh});
}

static void sched_2MN_gauge(std::vector<Step> &s, int gauge_scale, double eps, double scale)
{
    const double epsh = eps * 0.5;
    s.push_back({KICK_GAUGE, -eps * (scale * L2MN)});
    for (int md = 1; md < gauge_scale; md++) {
        s.push_back({DRIFT, epsh * scale});
        s.push_back({KICK_GAUGE, -eps * ((1.0 - 2.0 * L2MN) * scale)});
        s.push_back({DRIFT, epsh * scale});
        s.push_back({KICK_GAUGE, -eps * (2.0 * L2MN * scale)});
    }
    s.push_back({DRIFT, epsh * scale});
    s.push_back({KICK_GAUGE, -eps * ((1.0 - 2.0 * L2MN) * scale)});
    s.push_back({DRIFT, epsh * scale});
    s.push_back({KICK_GAUGE, -eps * (L2MN * scale)});
}

static void sched_multistep_2MN(std::vector<Step> &s, int no_md, int gauge_scale, double eps)
{
    const double gs = 0.5 / (double)gauge_scale;
    s.push_back({KICK_FERMION, -eps * L2MN});
    for (int md = 1; md < no_md; md++) {
        sched_2MN_gauge(s, gauge_scale, eps, gs);
        s.push_back({KICK_FERMION, -eps * (1.0 - 2.0 * L2MN)});
        sched_2MN_gauge(s, gauge_scale, eps, gs);
        s.push_back({KICK_FERMION, -eps * (2.0 * L2MN)});
    }
    sched_2MN_gauge(s, gauge_scale, eps, gs);
    s.push_back({KICK_FERMION, -eps * (1.0 - 2.0 * L2MN)});
    sched_2MN_gauge(s, gauge_scale, eps, gs);
    s.push_back({KICK_FERMION, -eps * L2MN});
}

static void sched_4MN_gauge(std::vector<Step> &s, int gauge_scale, double eps, double scale)
{
    const double epsh = eps * 0.5;
    const double half = 1.0 - 2.0 * (L4 + T4), mid = 1.0 - 2.0 * (M4 + R4);
    auto tail = [&]() {
        s.push_back({DRIFT, eps * (scale * R4)});
        s.push_back({KICK_GAUGE, -eps * (L4 * scale)});
        s.push_back({DRIFT, eps * (scale * M4)});
        s.push_back({KICK_GAUGE, -epsh * (half * scale)});
        s.push_back({DRIFT, eps * (scale * mid)});
        s.push_back({KICK_GAUGE, -epsh * (half * scale)});
        s.push_back({DRIFT, eps * (scale * M4)});
        s.push_back({KICK_GAUGE, -eps * (L4 * scale)});
        s.push_back({DRIFT, eps * (scale * R4)});
    };
    s.push_back({KICK_GAUGE, -eps * (scale * T4)});
    for (int md = 1; md < gauge_scale; md++) {
        tail();
        s.push_back({KICK_GAUGE, -eps * (2 * scale * T4)});
    }
    tail();
    s.push_back({KICK_GAUGE, -eps * (scale * T4)});
}

static void sched_multistep_4MN(std::vector<Step> &s, int no_md, int gauge_scale, double eps)
{
    const double epsh = eps * 0.5;
    const double gs = 1.0 / (double)gauge_scale;
    const double half = 1.0 - 2.0 * (L4 + T4), mid = 1.0 - 2.0 * (M4 + R4);
    auto body = [&]() {
        sched_4MN_gauge(s, gauge_scale, eps, R4 * gs);
        s.push_back({KICK_FERMION, -eps * L4});
        sched_4MN_gauge(s, gauge_scale, eps, M4 * gs);
        s.push_back({KICK_FERMION, -epsh * half});
        sched_4MN_gauge(s, gauge_scale, eps, gs * mid);
        s.push_back({KICK_FERMION, -epsh * half});
        sched_4MN_gauge(s, gauge_scale, eps, M4 * gs);
        s.push_back({KICK_FERMION, -eps * L4});
        sched_4MN_gauge(s, gauge_scale, eps, R4 * gs);
    };
    s.push_back({KICK_FERMION, -eps * T4});
    for (int md = 1; md < no_md; md++) {
        body();
        s.push_back({KICK_FERMION, -eps * (2 * T4)});
    }
    body();
    s.push_back({KICK_FERMION, -eps * T4});
}

// the two sched_4MN_* tails reproduce the products of the reference, e.g. mid*gs is computed as
// gs*(1-2(mu+rho)) in the loop body and as (1-2(mu+rho))*gs in the final part; both are exact
// products of the same two doubles, so the order does not change the value.

static int run_schedule(rhmc_ctx *c, const std::vector<Step> &s)
{
    for (const Step &st : s) {
        int rc = RHMC_OK;
        switch (st.k) {
        case KICK_FULL: rc = calc_ipdot_full(c); break;
        case KICK_FERMION: rc = fermion_part(c, 0); break;
        case KICK_GAUGE: rc = gauge_force(c, 0); break;
        case DRIFT: rc = link_update(c, st.c); break;
        }
        if (rc) return rc;
        if (st.k != DRIFT) {
            rc = mom_update(c, st.c);
            if (rc) return rc;
        }
    }
    return RHMC_OK;
}

static int update_nometro(rhmc_ctx *c)
{
    int rc = check_ready(c);
    if (rc) return rc;
    const rhmc_driver_params &P = drv(c)->P;
    const double eps = 1.0 / ((double)P.no_md);
    std::vector<Step> s;
    switch (P.integrator) {
    case RHMC_INT_2MN: sched_2MN_A(s, P.no_md, eps); break;
    case RHMC_INT_MULTISTEP_2MN: sched_multistep_2MN(s, P.no_md, P.gauge_scale, eps); break;
    case RHMC_INT_MULTISTEP_4MN: sched_multistep_4MN(s, P.no_md, P.gauge_scale, eps); break;
    case RHMC_INT_LEAPFROG: sched_leapfrog(s, P.no_md, eps); break;
    default: return fail(RHMC_ERR_ARG, "unknown integrator %d", P.integrator);
    }
    return run_schedule(c, s);
}

// S = gauge + momenta + fermion part (calc_action, lib/Action/action.cc:111-156)
static int action(rhmc_ctx *c, int final_part, double *out)
{
    Driver *d = drv(c);
    double t, sp, m, f = 0.0;
    int rc = plaquette_sums(c, &t, &sp);
    if (rc) return rc;
    if ((rc = momentum_action(c, &m))) return rc;
    // initial: sum Re<phi, phi>; final: sum Re<phi, chi> with phi = r_last chi; over all species
    for (int s = 0; s < nspecies(c); s++) {
        const int nps = d->sp[s].no_ps;
        double2 *phi = nullptr, *chi = nullptr;
        double fs;
        rc = field(c, fname("drv_phi", s), nps, &phi);
        if (rc) return rc;
        rc = field(c, fname("drv_chi", s), nps, &chi);
        if (rc) return rc;
        if ((rc = rdot(c, phi, final_part ? chi : phi, (long)nps * SP(c), &fs))) return rc;
        f += fs;
    }
    *out = (c->beta / 3.0) * (t + sp) + m + f;
    return RHMC_OK;
}

static int save_conf(rhmc_ctx *c)
{
    void *p;
    const size_t bytes = 8 * 9 * (size_t)c->Vh * sizeof(double2);
    CK(c->ws.get("drv_usave", bytes, &p));
    CK(cudaMemcpyAsync(p, c->U64, bytes, cudaMemcpyDeviceToDevice, c->stream));
    return RHMC_OK;
}

static int copy_saved(rhmc_ctx *c)
{
    auto it = c->ws.buf.find("drv_usave");
    if (it == c->ws.buf.end()) return fail(RHMC_ERR_STATE, "no saved configuration");
    CK(cudaMemcpyAsync(c->U64, it->second.first, 8 * 9 * (size_t)c->Vh * sizeof(double2), cudaMemcpyDeviceToDevice,
                       c->stream));
    invalidate_links(c);
    return RHMC_OK;
}

}  // namespace rhmc

using namespace rhmc;

extern "C" {

int rhmc_driver_setup(rhmc_ctx *c, const rhmc_driver_params *p)
{
    if (!c || !p) return fail(RHMC_ERR_ARG, "null argument");
    if (p->no_ps < 1 || p->no_flavours < 1 || p->no_md < 1 || p->gauge_scale < 1 || p->max_cg < 1)
        return fail(RHMC_ERR_ARG, "no_ps, no_flavours, no_md, gauge_scale and max_cg must be positive");
    if (p->integrator < 0 || p->integrator > RHMC_INT_LEAPFROG) return fail(RHMC_ERR_ARG, "unknown integrator");
    if (p->auto_bounds < 0 || p->auto_bounds > 2) return fail(RHMC_ERR_ARG, "auto_bounds must be 0, 1 or 2");
    if (p->single_rhs != 0 && p->single_rhs != 1) return fail(RHMC_ERR_ARG, "single_rhs must be 0 or 1");
    if (p->pole_group < 0) return fail(RHMC_ERR_ARG, "pole_group must be 0 (all poles at once) or positive");
    Driver *d = ensure_driver(c);
    d->P = *p;
    memset(d->sums, 0, sizeof(d->sums));
    d->sp[0].no_flavours = p->no_flavours;
    d->sp[0].no_ps = p->no_ps;
    d->configured = true;
    return RHMC_OK;
}

int rhmc_driver_add_species(rhmc_ctx *c, double mass, int no_flavours, int no_ps, int *index)
{
    if (!c || !index) return fail(RHMC_ERR_ARG, "null argument");
    if (!(mass >= c->mass)) return fail(RHMC_ERR_ARG, "species mass %g below the context mass %g", mass, c->mass);
    if (no_flavours < 1 || no_ps < 1) return fail(RHMC_ERR_ARG, "no_flavours and no_ps must be positive");
    Driver *d = ensure_driver(c);
    if (d->sp.size() >= 8) return fail(RHMC_ERR_ARG, "at most 8 species");
    Species S;
    S.mass = mass;
    S.no_flavours = no_flavours;
    S.no_ps = no_ps;
    d->sp.push_back(S);
    *index = (int)d->sp.size() - 1;
    return RHMC_OK;
}

int rhmc_driver_select_species(rhmc_ctx *c, int index)
{
    if (!c) return fail(RHMC_ERR_ARG, "null argument");
    Driver *d = ensure_driver(c);
    if (index < 0 || index >= (int)d->sp.size()) return fail(RHMC_ERR_ARG, "no species %d", index);
    d->cur = index;
    return RHMC_OK;
}

int rhmc_set_approx(rhmc_ctx *c, int which, int order, double a0, const double *a, const double *b, double min_eps)
{
    if (!c || !a || !b || which < 0 || which > 2 || order < 1 || order > 32) return fail(RHMC_ERR_ARG, "bad argument");
    Driver *d = ensure_driver(c);
    Approx &ap = d->sp[d->cur].approx[which];
    ap.order = order;
    ap.a0 = a0;
    ap.min_eps = min_eps;
    ap.a.assign(a, a + order);
    ap.b.assign(b, b + order);
    return RHMC_OK;
}

int rhmc_set_eig_bounds(rhmc_ctx *c, double min, double max)
{
    if (!c || !(max > 0.0) || !(min > 0.0) || min > max) return fail(RHMC_ERR_ARG, "need 0 < min <= max");
    Driver *d = ensure_driver(c);
    Species &S = d->sp[d->cur];
    S.eig_min = min;
    S.eig_max = max;
    S.have_bounds = true;
    return RHMC_OK;
}

int rhmc_get_eig_bounds(rhmc_ctx *c, double *min, double *max)
{
    if (!c || !min || !max) return fail(RHMC_ERR_ARG, "null argument");
    if (!c->driver) return fail(RHMC_ERR_STATE, "driver not configured");
    const Species &S = c->driver->sp[c->driver->cur];
    if (!S.have_bounds) return fail(RHMC_ERR_STATE, "no spectral bounds yet");
    *min = S.eig_min;
    *max = S.eig_max;
    return RHMC_OK;
}

// the pseudofermions of the selected species
static int pf_io(rhmc_ctx *c, const char *name, double *host_ref, int location, int to_device)
{
    if (!c || !host_ref) return fail(RHMC_ERR_ARG, "null argument");
    if (!c->driver || !c->driver->configured) return fail(RHMC_ERR_STATE, "driver not configured");
    const int s = c->driver->cur;
    const int n = c->driver->sp[s].no_ps;
    double2 *f;
    int rc = field(c, fname(name, s), n, &f);
    if (rc) return rc;
    if (to_device) return rhmc_spinor_to_internal(c, RHMC_LINKS_F64_18, f, host_ref, n, location);
    return rhmc_spinor_from_internal(c, RHMC_LINKS_F64_18, host_ref, f, n, location);
}

int rhmc_set_phi(rhmc_ctx *c, const double *phi, int location) { return pf_io(c, "drv_phi", (double *)phi, location, 1); }
int rhmc_get_phi(rhmc_ctx *c, double *phi, int location) { return pf_io(c, "drv_phi", phi, location, 0); }
int rhmc_set_chi(rhmc_ctx *c, const double *chi, int location) { return pf_io(c, "drv_chi", (double *)chi, location, 1); }
int rhmc_get_chi(rhmc_ctx *c, double *chi, int location) { return pf_io(c, "drv_chi", chi, location, 0); }

int rhmc_first_inv_approx_calc(rhmc_ctx *c, double res) { return c ? inv_approx_calc(c, 0, res) : fail(RHMC_ERR_ARG, "null"); }
int rhmc_last_inv_approx_calc(rhmc_ctx *c, double res) { return c ? inv_approx_calc(c, 2, res) : fail(RHMC_ERR_ARG, "null"); }
int rhmc_calc_ipdot(rhmc_ctx *c) { return c ? calc_ipdot_full(c) : fail(RHMC_ERR_ARG, "null"); }
int rhmc_calc_ipdot_gauge(rhmc_ctx *c) { return c ? gauge_force(c, 0) : fail(RHMC_ERR_ARG, "null"); }
int rhmc_calc_ipdot_fermion(rhmc_ctx *c) { return c ? fermion_part(c, 0) : fail(RHMC_ERR_ARG, "null"); }
int rhmc_update_nometro(rhmc_ctx *c) { return c ? update_nometro(c) : fail(RHMC_ERR_ARG, "null"); }
int rhmc_fermion_action(rhmc_ctx *c, double *out) { return (c && out) ? fermion_action_md(c, out) : fail(RHMC_ERR_ARG, "null"); }
int rhmc_save_conf(rhmc_ctx *c) { return c ? save_conf(c) : fail(RHMC_ERR_ARG, "null"); }
int rhmc_copy_saved(rhmc_ctx *c) { return c ? copy_saved(c) : fail(RHMC_ERR_ARG, "null"); }

int rhmc_update(rhmc_ctx *c, double uniform, int *acc, double *delta_s)
{
    if (!c || !acc) return fail(RHMC_ERR_ARG, "null argument");
    Driver *d = drv(c);
    int rc;
    if (d && d->configured && d->P.auto_bounds && (rc = compute_bounds(c))) return rc;  // once per trajectory
    if ((rc = check_ready(c))) return rc;
    if ((rc = save_conf(c))) return rc;
    if ((rc = inv_approx_calc(c, 0, d->P.residue_metro))) return rc;
    double s0, s1;
    if ((rc = action(c, 0, &s0))) return rc;
    if ((rc = update_nometro(c))) return rc;
    if ((rc = inv_approx_calc(c, 2, d->P.residue_metro))) return rc;
    if ((rc = action(c, 1, &s1))) return rc;
    const double de = s1 - s0;
    if (delta_s) *delta_s = de;
    if (de < 0 || uniform < exp(-de)) {
        *acc = 1;
        return save_conf(c);
    }
    *acc = 0;
    return copy_saved(c);
}

int rhmc_driver_stats(rhmc_ctx *c, long *force_evals, long *solves)
{
    if (!c || !c->driver) return fail(RHMC_ERR_STATE, "driver not configured");
    if (force_evals) *force_evals = c->driver->force_evals;
    if (solves) *solves = c->driver->solves;
    return RHMC_OK;
}

int rhmc_driver_solver_stats(rhmc_ctx *c, int which, rhmc_msolve_info *out, int reset)
{
    if (!c || !c->driver) return fail(RHMC_ERR_STATE, "driver not configured");
    if (which != 0 && which != 1) return fail(RHMC_ERR_ARG, "which must be 0 (md solves) or 1 (metro solves)");
    if (out) *out = c->driver->sums[which];
    if (reset) memset(c->driver->sums, 0, sizeof(c->driver->sums));
    return RHMC_OK;
}

int rhmc_workspace_bytes(rhmc_ctx *c, long *bytes)
{
    if (!c || !bytes) return fail(RHMC_ERR_ARG, "null argument");
    size_t n = 0;
    for (const auto &kv : c->ws.buf) n += kv.second.second;
    *bytes = (long)n;
    return RHMC_OK;
}

int rhmc_workspace_release(rhmc_ctx *c)
{
    if (!c) return fail(RHMC_ERR_ARG, "null argument");
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "rhmc_workspace_release");
    c->graphs.release();
    // keep the buffers that carry state between calls: the pseudofermion fields and the saved
    // configuration of the Metropolis step
    for (auto it = c->ws.buf.begin(); it != c->ws.buf.end();) {
        const std::string &n = it->first;
        if (n.rfind("drv_phi", 0) == 0 || n.rfind("drv_chi", 0) == 0 || n == "drv_usave") {
            ++it;
            continue;
        }
        cudaFree(it->second.first);
        it = c->ws.buf.erase(it);
    }
    return RHMC_OK;
}

}  // extern "C"
