// conf_io.cu -- the reference's text configuration format (Conf::write_last / Conf::write and the
// stored-conf start of Conf::Conf, lib/Main/Conf/conf.cc:55-94, 141-200):
//   "nx ny nz nt beta mass no_flavours update_iteration\n"
// then for every link r = mu*V + site (sites even-first) its 3 rows, each "c0 c1 c2\n" with
// complex numbers as "(re,im)", and an empty line; numbers with 16 significant digits (the
// reference's stream precision, i.e. printf "%.16g").  On reading, the reference calls
// sunitarize and row_multiply on u_work before overwriting it with the stored link, so the
// reunitarisation it intends never happens; rhmc_read_conf applies it (Gram-Schmidt rows 0-1,
// row 2 = conj(row0 x row1) times eta, as Conf::unitarize_with_eta, conf.cc:235-251) when asked.
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "capi_util.h"
#include "context.h"
#include "kernels.h"
#include "su3.cuh"

namespace rhmc {

__global__ void unitarize_eta_kernel(Geom g, double2 *U)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 8L * g.Vh) return;
    const int mp = (int)(i / g.Vh), k = (int)(i % g.Vh);
    const int mu = mp >> 1, p = mp & 1;
    M3 u = load_link64(U, g.Vh, mu, p, k);
    const Site s = site_of(g, p, k);
    sunitarize_eta(u, (double)eta_of(g, s, mu));
    store_link64(U, g.Vh, mu, p, k, u);
}

namespace {

struct Reader {
    const char *p, *end;
    void skip() { while (p < end && isspace((unsigned char)*p)) p++; }
    bool num(double &v)
    {
        skip();
        char *e = nullptr;
        errno = 0;
        v = strtod(p, &e);
        if (e == p || errno == ERANGE) return false;
        p = e;
        return true;
    }
    bool integer(long &v)
    {
        skip();
        char *e = nullptr;
        v = strtol(p, &e, 10);
        if (e == p) return false;
        p = e;
        return true;
    }
    bool expect(char ch)
    {
        skip();
        if (p >= end || *p != ch) return false;
        p++;
        return true;
    }
    // std::complex extraction: "(re,im)", "(re)" or "re"
    bool cplx(double &re, double &im)
    {
        skip();
        im = 0.0;
        if (p < end && *p == '(') {
            p++;
            if (!num(re)) return false;
            skip();
            if (p < end && *p == ',') {
                p++;
                if (!num(im)) return false;
            }
            return expect(')');
        }
        return num(re);
    }
};

}  // namespace
}  // namespace rhmc

using namespace rhmc;

extern "C" {

int rhmc_write_conf(rhmc_ctx *c, const char *path, int no_flavours, long update_iteration)
{
    if (!c || !path) return fail(RHMC_ERR_ARG, "null argument");
    const long nl = 4 * c->V;
    std::vector<double> u((size_t)nl * 18);
    int rc = rhmc_get_gauge(c, u.data(), RHMC_HOST);
    if (rc) return rc;
    FILE *f = fopen(path, "w");
    if (!f) return fail(RHMC_ERR_ARG, "cannot open %s for writing", path);
    fprintf(f, "%d %d %d %d %.16g %.16g %d %ld\n", c->g.nx, c->g.ny, c->g.nz, c->g.nt, c->beta, c->mass, no_flavours,
            update_iteration);
    char line[512];
    for (long r = 0; r < nl; r++) {
        const double *m = u.data() + (size_t)r * 18;
        for (int i = 0; i < 3; i++) {
            const double *row = m + i * 6;
            const int n = snprintf(line, sizeof(line), "(%.16g,%.16g) (%.16g,%.16g) (%.16g,%.16g)\n%s", row[0], row[1], row[2],
                                   row[3], row[4], row[5], i == 2 ? "\n" : "");
            if (n < 0 || fwrite(line, 1, (size_t)n, f) != (size_t)n) {
                fclose(f);
                return fail(RHMC_ERR_ARG, "write to %s failed", path);
            }
        }
    }
    if (fclose(f) != 0) return fail(RHMC_ERR_ARG, "write to %s failed", path);
    return RHMC_OK;
}

int rhmc_read_conf(rhmc_ctx *c, const char *path, int reunitarize, double *beta, double *mass, int *no_flavours,
                   long *update_iteration)
{
    if (!c || !path) return fail(RHMC_ERR_ARG, "null argument");
    FILE *f = fopen(path, "rb");
    if (!f) return fail(RHMC_ERR_ARG, "cannot open %s", path);
    std::vector<char> text;
    char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) text.insert(text.end(), buf, buf + n);
    fclose(f);
    Reader rd{text.data(), text.data() + text.size()};
    long d[4], it;
    double b, m, nf;
    for (int i = 0; i < 4; i++)
        if (!rd.integer(d[i])) return fail(RHMC_ERR_ARG, "%s: bad header", path);
    if (!rd.num(b) || !rd.num(m) || !rd.num(nf) || !rd.integer(it)) return fail(RHMC_ERR_ARG, "%s: bad header", path);
    // stored_conf_not_fit (conf.cc:82-85)
    if (d[0] != c->g.nx || d[1] != c->g.ny || d[2] != c->g.nz || d[3] != c->g.nt)
        return fail(RHMC_ERR_ARG, "%s: lattice %ldx%ldx%ldx%ld does not fit %dx%dx%dx%d", path, d[0], d[1], d[2], d[3], c->g.nx, c->g.ny,
                    c->g.nz, c->g.nt);
    const long nl = 4 * c->V;
    std::vector<double> u((size_t)nl * 18);
    for (long e = 0; e < nl * 9; e++)
        if (!rd.cplx(u[2 * e], u[2 * e + 1])) return fail(RHMC_ERR_ARG, "%s: bad or missing link element %ld", path, e);
    int rc = rhmc_set_gauge(c, u.data(), RHMC_HOST);
    if (rc) return rc;
    if (reunitarize) {
        unitarize_eta_kernel<<<grid_for(8L * c->Vh, 256), 256, 0, c->stream>>>(c->g, c->U64);
        c->launches++;
        CK(cudaGetLastError());
        invalidate_links(c);
    }
    CK(cudaStreamSynchronize(c->stream));
    if (beta) *beta = b;
    if (mass) *mass = m;
    if (no_flavours) *no_flavours = (int)nf;
    if (update_iteration) *update_iteration = it;
    return RHMC_OK;
}

}  // extern "C"
