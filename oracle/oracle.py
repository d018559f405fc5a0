"""ctypes front-ends of the oracle -- TEST INFRASTRUCTURE ONLY.

``Oracle``  loads oracle/liborc.so, the C restatement (oracle/rhmc_oracle.c), any lattice size.
``RefLib``  loads oracle/_ref/libref_<tag>.so, the unmodified reference CPU sources plus the
            harness (oracle/harness/ref_harness.cc); lattice and physics parameters are the
            compile-time ones of that build (oracle/build_ref.py CONFIGS).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import this module.
All fields use the reference layouts: links/algebra (4V,3,3) complex128, spinors (Vh,3)
complex128, sites in the reference even/odd order.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _dp(a):
    assert a.flags.c_contiguous and a.dtype in (np.float64, np.complex128)
    return a.ctypes.data_as(_D)


def _fp(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _ip(a):
    assert a.flags.c_contiguous and a.dtype == np.int32
    return a.ctypes.data_as(_I)


def build_oracle(force=False):
    """Compile oracle/rhmc_oracle.c into oracle/liborc.so (no FMA contraction)."""
    src = os.path.join(HERE, "rhmc_oracle.c")
    lib = os.path.join(HERE, "liborc.so")
    if force or not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        import subprocess
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-o", lib, src, "-lm"])
    return lib


class Oracle:
    """C restatement of the reference CPU algorithms with runtime lattice sizes."""

    def __init__(self, dims, bc=0):
        self.lib = ctypes.CDLL(build_oracle())
        L = self.lib
        L.orc_init.argtypes = [ctypes.c_int] * 5
        L.orc_volume.restype = ctypes.c_long
        L.orc_tables.argtypes = [_I, _I]
        for f in ("orc_deo", "orc_doe"):
            getattr(L, f).argtypes = [_D, _D, _D]
        L.orc_mdagm.argtypes = [_D, _D, _D, ctypes.c_double, ctypes.c_double]
        L.orc_msolve.argtypes = [_D, _D, _D, ctypes.c_double, ctypes.c_int, _D, ctypes.c_double, ctypes.c_int]
        L.orc_msolve.restype = ctypes.c_int
        L.orc_polyakov.argtypes = [_D, _D, _D]
        L.orc_chiral_meas.argtypes = [_D, _D, _D, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, _D]
        L.orc_chiral_meas.restype = ctypes.c_int
        L.orc_rational_sum.argtypes = [_D, _D, _D, ctypes.c_double, _D, ctypes.c_int]
        L.orc_fermion_force_accum.argtypes = [_D, _D, _D, _D, ctypes.c_int]
        L.orc_staples.argtypes = [_D, _D]
        L.orc_ipdot_gauge_init.argtypes = [_D, _D, ctypes.c_double]
        L.orc_u_times_ta.argtypes = [_D, _D, _D]
        L.orc_ipdot_gauge.argtypes = [_D, _D, ctypes.c_double]
        L.orc_mom_update.argtypes = [_D, _D, ctypes.c_double]
        L.orc_link_update.argtypes = [_D, _D, ctypes.c_double]
        L.orc_unitarize_with_eta.argtypes = [_D]
        L.orc_gauge_action.argtypes = [_D, ctypes.c_double]
        L.orc_gauge_action.restype = ctypes.c_double
        L.orc_momentum_action.argtypes = [_D]
        L.orc_momentum_action.restype = ctypes.c_double
        L.orc_rdot.argtypes = [_D, _D]
        L.orc_rdot.restype = ctypes.c_double
        L.orc_plaquette.argtypes = [_D, _D, _D]
        self.dims = tuple(dims)
        self.bc = bc
        if L.orc_init(*dims, bc) != 0:
            raise ValueError("bad lattice dims %r" % (dims,))
        self.V = int(L.orc_volume())
        self.Vh = self.V // 2

    def _reinit(self):
        self.lib.orc_init(*self.dims, self.bc)

    # the reference packer (lib/Tools/Packer/packer.cc), between exact fields and packed floats
    def _f32(self, n):
        return np.zeros(n, np.float32)

    def pk_gauge(self):
        out = self._f32(2 * 12 * 4 * self.V)
        self.lib.ref_pk_gauge(_fp(out))
        return out

    def unpk_gauge(self, pk):
        self.lib.ref_unpk_gauge(_fp(np.ascontiguousarray(pk, np.float32)))
        return self.get_links()

    def pk_chi(self):
        out = self._f32(6 * self.Vh * self.no_ps * 2)
        self.lib.ref_pk_chi(_fp(out))
        return out

    def unpk_chi(self, pk):
        self.lib.ref_unpk_chi(_fp(np.ascontiguousarray(pk, np.float32)))
        return self.get_chi()

    def pk_fermion(self, x):
        out = self._f32(6 * self.Vh)
        self.lib.ref_pk_fermion(_fp(out), _dp(np.ascontiguousarray(x, np.complex128)))
        return out

    def pk_fermion_d(self, x):
        out = self._f32(6 * self.Vh * 2)
        self.lib.ref_pk_fermion_d(_fp(out), _dp(np.ascontiguousarray(x, np.complex128)))
        return out

    def unpk_fermion_d(self, pk):
        out = np.zeros((self.Vh, 3), np.complex128)
        self.lib.ref_unpk_fermion_d(_dp(out), _fp(np.ascontiguousarray(pk, np.float32)))
        return out

    def unpk_shifted(self, pk, order):
        self.lib.ref_unpk_shifted(_fp(np.ascontiguousarray(pk, np.float32)), order)
        return self.get_shifted(order)

    def pk_ipdot(self):
        out = self._f32(8 * 4 * self.V)
        self.lib.ref_pk_ipdot(_fp(out))
        return out

    def unpk_ipdot(self, pk):
        self.lib.ref_unpk_ipdot(_fp(np.ascontiguousarray(pk, np.float32)))
        return self.get_ipdot()

    def pk_momenta(self):
        out = self._f32(8 * 4 * self.V)
        self.lib.ref_pk_momenta(_fp(out))
        return out

    def unpk_momenta(self, pk):
        self.lib.ref_unpk_momenta(_fp(np.ascontiguousarray(pk, np.float32)))
        return self.get_momenta()

    def shift_table(self):
        t = np.zeros(8 * self.V, np.int32)
        self.lib.ref_shift_table(_ip(t))
        return t

    def tables(self):
        t = np.zeros(8 * self.V, np.int32)
        e = np.zeros(4 * self.V, np.int32)
        self.lib.orc_tables(_ip(t), _ip(e))
        return t, e

    def deo(self, u, x):
        out = np.zeros((self.Vh, 3), np.complex128)
        self.lib.orc_deo(_dp(out), _dp(np.ascontiguousarray(x)), _dp(u))
        return out

    def doe(self, u, x):
        out = np.zeros((self.Vh, 3), np.complex128)
        self.lib.orc_doe(_dp(out), _dp(np.ascontiguousarray(x)), _dp(u))
        return out

    def mdagm(self, u, x, mass, shift=0.0):
        out = np.zeros((self.Vh, 3), np.complex128)
        self.lib.orc_mdagm(_dp(out), _dp(np.ascontiguousarray(x)), _dp(u), mass, shift)
        return out

    def msolve(self, u, b, mass, shifts, res, max_cg=100000):
        shifts = np.ascontiguousarray(shifts, np.float64)
        x = np.zeros((len(shifts), self.Vh, 3), np.complex128)
        it = self.lib.orc_msolve(_dp(x), _dp(np.ascontiguousarray(b)), _dp(u), mass, len(shifts), _dp(shifts), res, max_cg)
        return x, it

    def rational_sum(self, b, x, a0, a):
        a = np.ascontiguousarray(a, np.float64)
        out = np.zeros((self.Vh, 3), np.complex128)
        self.lib.orc_rational_sum(_dp(out), _dp(np.ascontiguousarray(b)), _dp(np.ascontiguousarray(x)), a0, _dp(a), len(a))
        return out

    def fermion_force_accum(self, F, u, x, a):
        a = np.ascontiguousarray(a, np.float64)
        self.lib.orc_fermion_force_accum(_dp(F), _dp(u), _dp(np.ascontiguousarray(x)), _dp(a), len(a))
        return F

    def staples(self, u):
        st = np.zeros((4 * self.V, 3, 3), np.complex128)
        self.lib.orc_staples(_dp(st), _dp(u))
        return st

    def ipdot_gauge_init(self, u, beta):
        buf = np.zeros((4 * self.V, 3, 3), np.complex128)
        self.lib.orc_ipdot_gauge_init(_dp(buf), _dp(u), beta)
        return buf

    def u_times_ta(self, u, buf):
        out = np.zeros((4 * self.V, 3, 3), np.complex128)
        self.lib.orc_u_times_ta(_dp(out), _dp(u), _dp(buf))
        return out

    def ipdot_gauge(self, u, beta):
        out = np.zeros((4 * self.V, 3, 3), np.complex128)
        self.lib.orc_ipdot_gauge(_dp(out), _dp(u), beta)
        return out

    def mom_update(self, P, ipdot, step):
        self.lib.orc_mom_update(_dp(P), _dp(ipdot), step)
        return P

    def link_update(self, u, P, step):
        self.lib.orc_link_update(_dp(u), _dp(P), step)
        return u

    def unitarize_with_eta(self, u):
        self.lib.orc_unitarize_with_eta(_dp(u))
        return u

    def gauge_action(self, u, beta):
        return self.lib.orc_gauge_action(_dp(u), beta)

    def momentum_action(self, P):
        return self.lib.orc_momentum_action(_dp(P))

    def rdot(self, a, b):
        return self.lib.orc_rdot(_dp(np.ascontiguousarray(a)), _dp(np.ascontiguousarray(b)))

    def polyakov(self, u):
        """Conf::calc_poly (lib/Measurements/gaugemeas.cc:66-106): (re, im)."""
        re, im = np.zeros(1), np.zeros(1)
        self.lib.orc_polyakov(_dp(np.ascontiguousarray(u, np.complex128)), _dp(re), _dp(im))
        return float(re[0]), float(im[0])

    def chiral_meas(self, u, noise_e, noise_o, mass, no_flavours, res, max_cg=100000):
        """chiral_meas for one pair of noise vectors (lib/Measurements/chiralmeas.cc:44-183):
        chiral condensate, energy, baryon and pressure densities as 4 complex numbers."""
        out = np.zeros(8)
        self.lib.orc_chiral_meas(_dp(np.ascontiguousarray(u, np.complex128)),
                                 _dp(np.ascontiguousarray(noise_e, np.complex128)),
                                 _dp(np.ascontiguousarray(noise_o, np.complex128)), mass, no_flavours, res, max_cg, _dp(out))
        return out[0::2] + 1j * out[1::2]

    def plaquette(self, u):
        s = np.zeros(1)
        t = np.zeros(1)
        self.lib.orc_plaquette(_dp(u), _dp(s), _dp(t))
        return float(s[0]), float(t[0])


class RefLib:
    """The reference's own CPU code (compiled by oracle/build_ref.py) behind the harness."""

    def __init__(self, tag, seed=12345):
        path = os.path.join(HERE, "_ref", "libref_%s.so" % tag)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = L = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
        d = np.zeros(8, np.int32)
        L.ref_dims(_ip(d))
        self.dims = tuple(int(v) for v in d[:4])
        self.no_ps, self.max_order, self.no_md, self.gauge_scale = (int(v) for v in d[4:8])
        L.ref_param.restype = ctypes.c_double
        self.mass = L.ref_param(0)
        self.beta = L.ref_param(1)
        self.no_flavours = int(L.ref_param(2))
        self.residue_metro = L.ref_param(3)
        self.residue_md = L.ref_param(4)
        self.V = int(np.prod(self.dims))
        self.Vh = self.V // 2
        for name in ("ref_set_links", "ref_get_links", "ref_set_momenta", "ref_get_momenta", "ref_set_ipdot",
                     "ref_get_ipdot", "ref_set_phi", "ref_get_phi", "ref_set_chi", "ref_get_chi"):
            getattr(L, name).argtypes = [_D]
        L.ref_get_shifted.argtypes = [_D, ctypes.c_int]
        L.ref_deo.argtypes = [_D, _D]
        L.ref_doe.argtypes = [_D, _D]
        L.ref_dslash_loop.argtypes = [ctypes.c_int, _D]
        L.ref_tables.argtypes = [_I, _I]
        L.ref_set_approx.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, _D, _D]
        L.ref_set_minmax.argtypes = [ctypes.c_double, ctypes.c_double]
        L.ref_msolve.argtypes = [ctypes.c_double, ctypes.c_int, _D]
        L.ref_first_inv_approx_calc.argtypes = [ctypes.c_double]
        L.ref_last_inv_approx_calc.argtypes = [ctypes.c_double]
        L.ref_mom_update.argtypes = [ctypes.c_double]
        L.ref_link_update.argtypes = [ctypes.c_double]
        L.ref_action_end.restype = ctypes.c_double
        L.ref_plaquette.argtypes = [_D, _D]
        L.ref_polyakov.argtypes = [_D, _D]
        L.ref_chiral_meas.argtypes = [_D, _D, _D]
        L.ref_read_conf.argtypes = [_D]
        L.ref_trajectory.argtypes = [ctypes.c_int, ctypes.c_double, _I]
        L.ref_trajectory.restype = ctypes.c_double
        L.ref_findmaxeig.restype = ctypes.c_double
        L.ref_findmineig.restype = ctypes.c_double
        L.ref_findmineig.argtypes = [ctypes.c_double]
        L.ref_setup(seed)

    # field I/O
    def set_links(self, u):
        self.lib.ref_set_links(_dp(np.ascontiguousarray(u, np.complex128)))

    def get_links(self):
        u = np.zeros((4 * self.V, 3, 3), np.complex128)
        self.lib.ref_get_links(_dp(u))
        return u

    def set_momenta(self, p):
        self.lib.ref_set_momenta(_dp(np.ascontiguousarray(p, np.complex128)))

    def get_momenta(self):
        p = np.zeros((4 * self.V, 3, 3), np.complex128)
        self.lib.ref_get_momenta(_dp(p))
        return p

    def set_ipdot(self, p):
        self.lib.ref_set_ipdot(_dp(np.ascontiguousarray(p, np.complex128)))

    def get_ipdot(self):
        p = np.zeros((4 * self.V, 3, 3), np.complex128)
        self.lib.ref_get_ipdot(_dp(p))
        return p

    def set_phi(self, f):
        self.lib.ref_set_phi(_dp(np.ascontiguousarray(f, np.complex128)))

    def get_phi(self):
        f = np.zeros((self.no_ps, self.Vh, 3), np.complex128)
        self.lib.ref_get_phi(_dp(f))
        return f

    def set_chi(self, f):
        self.lib.ref_set_chi(_dp(np.ascontiguousarray(f, np.complex128)))

    def get_chi(self):
        f = np.zeros((self.no_ps, self.Vh, 3), np.complex128)
        self.lib.ref_get_chi(_dp(f))
        return f

    def get_shifted(self, order):
        f = np.zeros((self.no_ps, order, self.Vh, 3), np.complex128)
        self.lib.ref_get_shifted(_dp(f), order)
        return f

    # the reference packer (lib/Tools/Packer/packer.cc), between exact fields and packed floats
    def _f32(self, n):
        return np.zeros(n, np.float32)

    def pk_gauge(self):
        out = self._f32(2 * 12 * 4 * self.V)
        self.lib.ref_pk_gauge(_fp(out))
        return out

    def unpk_gauge(self, pk):
        self.lib.ref_unpk_gauge(_fp(np.ascontiguousarray(pk, np.float32)))
        return self.get_links()

    def pk_chi(self):
        out = self._f32(6 * self.Vh * self.no_ps * 2)
        self.lib.ref_pk_chi(_fp(out))
        return out

    def unpk_chi(self, pk):
        self.lib.ref_unpk_chi(_fp(np.ascontiguousarray(pk, np.float32)))
        return self.get_chi()

    def pk_fermion(self, x):
        out = self._f32(6 * self.Vh)
        self.lib.ref_pk_fermion(_fp(out), _dp(np.ascontiguousarray(x, np.complex128)))
        return out

    def pk_fermion_d(self, x):
        out = self._f32(6 * self.Vh * 2)
        self.lib.ref_pk_fermion_d(_fp(out), _dp(np.ascontiguousarray(x, np.complex128)))
        return out

    def unpk_fermion_d(self, pk):
        out = np.zeros((self.Vh, 3), np.complex128)
        self.lib.ref_unpk_fermion_d(_dp(out), _fp(np.ascontiguousarray(pk, np.float32)))
        return out

    def unpk_shifted(self, pk, order):
        self.lib.ref_unpk_shifted(_fp(np.ascontiguousarray(pk, np.float32)), order)
        return self.get_shifted(order)

    def pk_ipdot(self):
        out = self._f32(8 * 4 * self.V)
        self.lib.ref_pk_ipdot(_fp(out))
        return out

    def unpk_ipdot(self, pk):
        self.lib.ref_unpk_ipdot(_fp(np.ascontiguousarray(pk, np.float32)))
        return self.get_ipdot()

    def pk_momenta(self):
        out = self._f32(8 * 4 * self.V)
        self.lib.ref_pk_momenta(_fp(out))
        return out

    def unpk_momenta(self, pk):
        self.lib.ref_unpk_momenta(_fp(np.ascontiguousarray(pk, np.float32)))
        return self.get_momenta()

    def shift_table(self):
        t = np.zeros(8 * self.V, np.int32)
        self.lib.ref_shift_table(_ip(t))
        return t

    def tables(self):
        t = np.zeros(8 * self.V, np.int32)
        e = np.zeros(4 * self.V, np.int32)
        self.lib.ref_tables(_ip(t), _ip(e))
        return t, e

    def deo(self, x):
        out = np.zeros((self.Vh, 3), np.complex128)
        self.lib.ref_deo(_dp(out), _dp(np.ascontiguousarray(x, np.complex128)))
        return out

    def doe(self, x):
        out = np.zeros((self.Vh, 3), np.complex128)
        self.lib.ref_doe(_dp(out), _dp(np.ascontiguousarray(x, np.complex128)))
        return out

    def set_approx(self, which, approx):
        """approx: dict(a0, a, b, min_eps) normalised on [min_eps, 1]."""
        a = np.zeros(self.max_order)
        b = np.zeros(self.max_order)
        n = len(approx["a"])
        a[:n] = approx["a"]
        b[:n] = approx["b"]
        self.lib.ref_set_approx(which, n, approx.get("min_eps", 1e-7), approx["a0"], _dp(a), _dp(b))

    def findmaxeig(self):
        """lambda_max of M^dag M on the current links by the reference's findmaxeig."""
        return self.lib.ref_findmaxeig()

    def findmineig(self, mx):
        """lambda_min of M^dag M by the reference's findmineig (power iteration on mx - M^dag M)."""
        return self.lib.ref_findmineig(float(mx))

    def set_minmax(self, mn, mx):
        self.lib.ref_set_minmax(mn, mx)

    def msolve(self, res, shifts):
        shifts = np.ascontiguousarray(shifts, np.float64)
        self.lib.ref_msolve(res, len(shifts), _dp(shifts))
        return self.get_shifted(len(shifts))

    def plaquette(self):
        s = np.zeros(1)
        t = np.zeros(1)
        self.lib.ref_plaquette(_dp(s), _dp(t))
        return float(s[0]), float(t[0])

    def write_conf(self, directory):
        """Conf::write_last of the current links into <directory>/config; returns its text."""
        cwd = os.getcwd()
        try:
            os.chdir(directory)
            self.lib.ref_write_conf()
            with open("config", "rb") as f:
                return f.read()
        finally:
            os.chdir(cwd)

    def read_conf(self, directory):
        """The links the reference's stored-conf start reads from <directory>/config."""
        u = np.zeros((4 * self.V, 3, 3), np.complex128)
        cwd = os.getcwd()
        try:
            os.chdir(directory)
            self.lib.ref_read_conf(_dp(u))
        finally:
            os.chdir(cwd)
        return u

    def param(self, which):
        """Compile-time parameter of this build: 0 mass, 1 beta, 2 no_flavours, 3 residue_metro,
        4 residue_md, 5 max_cg."""
        self.lib.ref_param.restype = ctypes.c_double
        return float(self.lib.ref_param(which))

    def polyakov(self):
        """Conf::calc_poly (lib/Measurements/gaugemeas.cc:66-106) of the current links: (re, im)."""
        r = np.zeros(1)
        i = np.zeros(1)
        self.lib.ref_polyakov(_dp(r), _dp(i))
        return float(r[0]), float(i[0])

    def chiral_meas(self):
        """chiral_meas (lib/Measurements/chiralmeas.cc:18-194) with the reference's own Z2 noise and
        CPU CG: returns the 4 complex results (chiral condensate, energy, baryon and pressure
        densities) and the even and odd noise vectors it drew, each (Vh, 3) complex."""
        out = np.zeros(8)
        ne = np.zeros((self.Vh, 3), np.complex128)
        no = np.zeros((self.Vh, 3), np.complex128)
        self.lib.ref_chiral_meas(_dp(out), _dp(ne), _dp(no))
        return out[0::2] + 1j * out[1::2], ne, no

    def trajectory(self, integrator, uniform):
        acc = np.zeros(1, np.int32)
        de = self.lib.ref_trajectory(integrator, uniform, _ip(acc))
        return de, int(acc[0])
