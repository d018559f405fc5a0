"""Python front-end of librhmc_b200 (ctypes over the C ABI declared in include/rhmc_b200.h).

The library is the product; this module only loads it and forwards calls.  Device buffers
are passed as raw pointers (``int``) so any allocator works; the tests and bench use torch
tensors for device memory.  There is no CPU fallback: if the shared library is missing the
import of ``lib()`` raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIBPATH = os.path.join(PKG, "librhmc_b200.so")

RHMC_OK = 0
LINKS_F64_18, LINKS_F64_12, LINKS_F32_18, LINKS_F32_12, LINKS_F16_12 = 0, 1, 2, 3, 4
FMT_NAMES = {LINKS_F64_18: "f64_18", LINKS_F64_12: "f64_12", LINKS_F32_18: "f32_18", LINKS_F32_12: "f32_12",
             LINKS_F16_12: "f16_12"}


def spinor_floats(fmt, Vh):
    """Size of one internal spinor of a link format in 8-byte (FP64) or 4-byte units: 6*Vh
    doubles (FP64), 6*Vh floats (FP32) or 4*Vh floats' worth of half precision with per-site
    scales (F16_12: one 16-byte vector of three __half2 and a float scale per site)."""
    return 4 * Vh if fmt == LINKS_F16_12 else 6 * Vh
HOST, DEVICE = 0, 1

_lib = None


class RhmcError(RuntimeError):
    pass


class Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("nt", ctypes.c_int),
                ("ferm_temp_bc", ctypes.c_int), ("mass", ctypes.c_double), ("beta", ctypes.c_double),
                ("device", ctypes.c_int)]


def build(force=False):
    """Compile the library in-tree with the package Makefile (nvcc, sm_100a)."""
    import subprocess
    cmd = ["make", "-C", PKG, "-j8"]
    if force:
        subprocess.check_call(["make", "-C", PKG, "clean"])
    subprocess.check_call(cmd)
    return LIBPATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RhmcError("librhmc_b200.so not built (run __graft_entry__.build())")
        _lib = ctypes.CDLL(LIBPATH)
        _lib.rhmc_last_error.restype = ctypes.c_char_p
    return _lib


def _check(rc):
    if rc != RHMC_OK:
        raise RhmcError("rhmc error %d: %s" % (rc, lib().rhmc_last_error().decode()))
    return rc


# ------------------------------------------------------------------ launch-configuration autotuner
def autotune(enable):
    """Turns the launch-shape / RHS-packing tuning on or off; returns the previous setting."""
    return bool(lib().rhmc_autotune(int(bool(enable))))


def autotune_override(candidate):
    """Forces candidate 0..2 for every tuned launch (-1: tuned choices); returns the previous value."""
    return lib().rhmc_autotune_override(int(candidate))


def tune_cache_load(path):
    _check(lib().rhmc_tune_cache_load(os.fsencode(path)))


def tune_cache_save(path=None):
    _check(lib().rhmc_tune_cache_save(os.fsencode(path) if path else None))


def tune_report():
    """The tuned choices as a dict (the library's JSON table)."""
    import json
    L = lib()
    L.rhmc_tune_report.restype = ctypes.c_long
    L.rhmc_tune_report.argtypes = [ctypes.c_char_p, ctypes.c_long]
    n = L.rhmc_tune_report(None, 0)
    buf = ctypes.create_string_buffer(n)
    L.rhmc_tune_report(buf, n)
    return json.loads(buf.value.decode())


def tune_clear():
    _check(lib().rhmc_tune_clear())


def _vp(x):
    """Pointer argument: int (device address), numpy array (host), None."""
    if x is None:
        return ctypes.c_void_p(None)
    if isinstance(x, int):
        return ctypes.c_void_p(x)
    if isinstance(x, np.ndarray):
        assert x.flags.c_contiguous
        return ctypes.c_void_p(x.ctypes.data)
    if hasattr(x, "data_ptr"):
        return ctypes.c_void_p(x.data_ptr())
    raise TypeError(type(x))


def _loc(x):
    return HOST if isinstance(x, np.ndarray) else DEVICE


class Context:
    """One rhmc_ctx: a lattice with device-resident gauge field, momenta and ipdot."""

    def __init__(self, dims, mass=0.1, beta=5.5, ferm_temp_bc=0, device=0):
        self.dims = tuple(int(d) for d in dims)
        self.V = int(np.prod(self.dims))
        self.Vh = self.V // 2
        self.mass, self.beta = mass, beta
        p = Params(*self.dims, ferm_temp_bc, mass, beta, device)
        h = ctypes.c_void_p()
        _check(lib().rhmc_create(ctypes.byref(p), ctypes.byref(h)))
        self.h = h

    @classmethod
    def wrap(cls, handle, dims, mass, beta):
        """A view of a context owned elsewhere (e.g. the legacy entry points'); never destroyed here."""
        self = cls.__new__(cls)
        self.dims = tuple(int(d) for d in dims)
        self.V = int(np.prod(self.dims))
        self.Vh = self.V // 2
        self.mass, self.beta = mass, beta
        self.h = ctypes.c_void_p(handle)
        self.owned = False
        return self

    def close(self):
        if self.h and getattr(self, "owned", True):
            lib().rhmc_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def call(self, name, *args):
        conv = []
        for a in args:
            if isinstance(a, float):
                conv.append(ctypes.c_double(a))
            elif isinstance(a, (np.ndarray,)) or hasattr(a, "data_ptr") or a is None:
                conv.append(_vp(a))
            elif isinstance(a, ctypes._SimpleCData) or isinstance(a, ctypes.Array) or hasattr(a, "_obj"):
                conv.append(a)
            elif isinstance(a, int):
                conv.append(ctypes.c_int(a))
            else:
                conv.append(a)
        return _check(getattr(lib(), name)(self.h, *conv))

    def set_stream(self, stream_ptr):
        _check(lib().rhmc_set_stream(self.h, ctypes.c_void_p(stream_ptr)))

    def sync(self):
        self.call("rhmc_sync")

    def launch_count(self):
        n = ctypes.c_long()
        self.call("rhmc_launch_count", ctypes.byref(n))
        return n.value

    def geometry(self):
        t = np.zeros(8 * self.V, np.int32)
        e = np.zeros(4 * self.V, np.int32)
        self.call("rhmc_geometry", t, e)
        return t, e

    # fields: numpy (host) or torch (device) in the reference layout
    def set_gauge(self, u):
        self.call("rhmc_set_gauge", u, _loc(u))

    def get_gauge(self, out=None):
        if out is None:
            out = np.zeros((4 * self.V, 3, 3), np.complex128)
        self.call("rhmc_get_gauge", out, _loc(out))
        return out

    def set_momenta(self, p):
        self.call("rhmc_set_momenta", p, _loc(p))

    def get_momenta(self, out=None):
        if out is None:
            out = np.zeros((4 * self.V, 3, 3), np.complex128)
        self.call("rhmc_get_momenta", out, _loc(out))
        return out

    def set_ipdot(self, p):
        self.call("rhmc_set_ipdot", p, _loc(p))

    def get_ipdot(self, out=None):
        if out is None:
            out = np.zeros((4 * self.V, 3, 3), np.complex128)
        self.call("rhmc_get_ipdot", out, _loc(out))
        return out

    def spinor_to_internal(self, fmt, internal, ref, n=1):
        self.call("rhmc_spinor_to_internal", fmt, internal, ref, n, _loc(ref))

    def spinor_from_internal(self, fmt, ref, internal, n=1):
        self.call("rhmc_spinor_from_internal", fmt, ref, internal, n, _loc(ref))

    def dslash(self, fmt, parity_out, out, inp, n=1):
        self.call("rhmc_dslash", fmt, parity_out, out, inp, n)

    def dslash_repeat(self, fmt, even, odd, n=1, repeats=1):
        self.call("rhmc_dslash_repeat", fmt, even, odd, n, repeats)

    def dslash_host(self, parity_out, out, inp):
        self.call("rhmc_dslash_host", parity_out, out, inp)

    def dslash_sites(self, parity_out, out, inp, k_lo, k_count):
        """Half-Dslash onto output sites [k_lo, k_lo + k_count) only; out, inp: device arrays in
        the reference layout (complex (Vh, 3)), e.g. torch complex128 CUDA tensors."""
        self.call("rhmc_dslash_sites", parity_out, out, inp, ctypes.c_long(k_lo), ctypes.c_long(k_count))

    def mdagm(self, fmt, out, inp, shift=0.0, n=1):
        self.call("rhmc_mdagm", fmt, out, inp, float(shift), n)


MSOLVE_FP64, MSOLVE_MIXED, MSOLVE_FP32 = 0, 1, 2


class MsolveParams(ctypes.Structure):
    _fields_ = [("nshift", ctypes.c_int), ("shifts", ctypes.POINTER(ctypes.c_double)), ("nrhs", ctypes.c_int),
                ("residual", ctypes.c_double), ("max_iter", ctypes.c_int), ("mode", ctypes.c_int), ("fmt", ctypes.c_int),
                ("tol_phase_a", ctypes.c_double), ("ru_delta", ctypes.c_double), ("certify", ctypes.c_int),
                ("rhs_shifts", ctypes.POINTER(ctypes.c_double))]


class MsolveInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iters", ctypes.c_int * 8), ("refine_iters", ctypes.c_long),
                ("reliable_updates", ctypes.c_int), ("seconds", ctypes.c_double), ("seconds_phase_a", ctypes.c_double),
                ("systems_refined", ctypes.c_int), ("iters_total", ctypes.c_long), ("iters_max", ctypes.c_int),
                ("iters_fp64", ctypes.c_long), ("ms_reliable_updates", ctypes.c_int)]

    def as_dict(self):
        return {"status": self.status, "iters": list(self.iters), "refine_iters": self.refine_iters,
                "reliable_updates": self.reliable_updates, "seconds": self.seconds,
                "seconds_phase_a": self.seconds_phase_a, "systems_refined": self.systems_refined,
                "iters_total": self.iters_total, "iters_max": self.iters_max, "iters_fp64": self.iters_fp64,
                "ms_reliable_updates": self.ms_reliable_updates}


def _msolve_params(shifts, nrhs, residual, max_iter, mode, fmt, tol_phase_a=0.0, certify=0, ru_delta=0.0):
    """shifts: one pole set (nshift,) for every RHS, or one per RHS (nrhs, nshift)."""
    sh = np.ascontiguousarray(shifts, np.float64)
    per_rhs = sh.ndim == 2
    if per_rhs:
        assert sh.shape[0] == nrhs, "one pole set per right-hand side"
    dp = ctypes.POINTER(ctypes.c_double)
    p = MsolveParams(sh.shape[-1], sh.ctypes.data_as(dp), nrhs, residual, max_iter, mode, fmt, tol_phase_a, ru_delta, certify,
                     sh.ctypes.data_as(dp) if per_rhs else None)
    p._keep = sh
    return p


def _ctx_msolve(self, x, b, shifts, residual, nrhs=1, max_iter=100000, mode=MSOLVE_FP64, fmt=LINKS_F64_18, tol_phase_a=0.0,
                certify=0, ru_delta=0.0):
    """x, b: device FP64 internal spinors (b: nrhs, x: nrhs*nshift, RHS-major)."""
    p = _msolve_params(shifts, nrhs, residual, max_iter, mode, fmt, tol_phase_a, certify, ru_delta)
    info = MsolveInfo()
    self.call("rhmc_msolve", ctypes.byref(p), x, b, ctypes.byref(info))
    return info.as_dict()


def _ctx_msolve_host(self, b, shifts, residual, max_iter=100000, mode=MSOLVE_FP64, fmt=LINKS_F64_18, tol_phase_a=0.0,
                     certify=0):
    """b: numpy complex (Vh,3) or (nrhs,Vh,3) reference layout.  Returns (x, info) with x of shape
    (nshift,Vh,3) or (nrhs,nshift,Vh,3)."""
    b = np.ascontiguousarray(b, np.complex128)
    single = b.ndim == 2
    nrhs = 1 if single else b.shape[0]
    x = np.zeros((nrhs, np.shape(shifts)[-1], self.Vh, 3), np.complex128)
    p = _msolve_params(shifts, nrhs, residual, max_iter, mode, fmt, tol_phase_a, certify)
    info = MsolveInfo()
    self.call("rhmc_msolve_host", ctypes.byref(p), x, b, ctypes.byref(info))
    return (x[0] if single else x), info.as_dict()


def _ctx_true_residuals(self, x, b, shifts, nrhs=1):
    sh = np.ascontiguousarray(shifts, np.float64)
    out = np.zeros((nrhs, len(sh)), np.float64)
    self.call("rhmc_true_residuals", len(sh), sh, nrhs, x, b, out)
    return out


Context.msolve = _ctx_msolve
Context.msolve_host = _ctx_msolve_host
Context.true_residuals = _ctx_true_residuals


def _f(self, name, *args):
    v = ctypes.c_double()
    self.call(name, *args, ctypes.byref(v))
    return v.value


Context.gauge_force = lambda self, add=0: self.call("rhmc_gauge_force", int(add))
Context.fermion_force = lambda self, x, numerators, nrhs=1, add=0: self.call(
    "rhmc_fermion_force", nrhs, len(numerators), np.ascontiguousarray(numerators, np.float64), x, int(add))
Context.mom_update = lambda self, step: self.call("rhmc_mom_update", float(step))
Context.link_update = lambda self, step: self.call("rhmc_link_update", float(step))
Context.gauge_action = lambda self: _f(self, "rhmc_gauge_action")
Context.momentum_action = lambda self: _f(self, "rhmc_momentum_action")
Context.rdot = lambda self, a, b, n=1: _f(self, "rhmc_rdot", a, b, n)


def _plaq(self):
    s, t = ctypes.c_double(), ctypes.c_double()
    self.call("rhmc_plaquette", ctypes.byref(s), ctypes.byref(t))
    return s.value, t.value


Context.plaquette = _plaq


def _polyakov(self):
    re, im = ctypes.c_double(), ctypes.c_double()
    self.call("rhmc_polyakov", ctypes.byref(re), ctypes.byref(im))
    return re.value, im.value


def _chiral_meas(self, noise_e, noise_o, residual=1e-10, no_flavours=2, max_iter=100000):
    """chiral_meas for the given noise pairs (host (n, Vh, 3) complex or (Vh, 3)): chiral condensate,
    energy, baryon and pressure densities as 4 complex numbers."""
    ne = np.ascontiguousarray(noise_e, np.complex128)
    no = np.ascontiguousarray(noise_o, np.complex128)
    n = 1 if ne.ndim == 2 else ne.shape[0]
    out = np.zeros(8)
    self.call("rhmc_chiral_meas", n, int(no_flavours), ne, no, float(residual), int(max_iter), HOST, out)
    return out[0::2] + 1j * out[1::2]


def _write_conf(self, path, no_flavours=2, update_iteration=0):
    self.call("rhmc_write_conf", str(path).encode(), int(no_flavours), ctypes.c_long(update_iteration))


def _read_conf(self, path, reunitarize=1):
    b, m = ctypes.c_double(), ctypes.c_double()
    nf, it = ctypes.c_int(), ctypes.c_long()
    self.call("rhmc_read_conf", str(path).encode(), int(reunitarize), ctypes.byref(b), ctypes.byref(m), ctypes.byref(nf),
              ctypes.byref(it))
    return {"beta": b.value, "mass": m.value, "no_flavours": nf.value, "update_iteration": it.value}


Context.write_conf = _write_conf
Context.read_conf = _read_conf
Context.polyakov = _polyakov
Context.chiral_meas = _chiral_meas
Context.rational_sum = lambda self, out, x, b, a0, a, nrhs=1: self.call(
    "rhmc_rational_sum", nrhs, len(a), float(a0), np.ascontiguousarray(a, np.float64), x, b, out)


INT_2MN, INT_MULTISTEP_2MN, INT_MULTISTEP_4MN, INT_LEAPFROG = 0, 1, 2, 3


class DriverParams(ctypes.Structure):
    _fields_ = [("no_flavours", ctypes.c_int), ("no_ps", ctypes.c_int), ("no_md", ctypes.c_int),
                ("gauge_scale", ctypes.c_int), ("integrator", ctypes.c_int), ("max_cg", ctypes.c_int),
                ("residue_metro", ctypes.c_double), ("residue_md", ctypes.c_double),
                ("metro_mode", ctypes.c_int), ("metro_fmt", ctypes.c_int), ("md_mode", ctypes.c_int),
                ("md_fmt", ctypes.c_int), ("auto_bounds", ctypes.c_int), ("single_rhs", ctypes.c_int),
                ("pole_group", ctypes.c_int)]


def _driver_setup(self, no_flavours=2, no_ps=1, no_md=10, gauge_scale=5, integrator=INT_2MN, max_cg=100000,
                  residue_metro=1e-10, residue_md=1e-10, metro_mode=MSOLVE_FP64, metro_fmt=LINKS_F64_18,
                  md_mode=MSOLVE_FP64, md_fmt=LINKS_F64_18, auto_bounds=0, single_rhs=0, pole_group=0):
    p = DriverParams(no_flavours, no_ps, no_md, gauge_scale, integrator, max_cg, residue_metro, residue_md, metro_mode,
                     metro_fmt, md_mode, md_fmt, auto_bounds, single_rhs, pole_group)
    self.no_ps = no_ps
    self.call("rhmc_driver_setup", ctypes.byref(p))


def _set_approx(self, which, approx):
    a = np.ascontiguousarray(approx["a"], np.float64)
    b = np.ascontiguousarray(approx["b"], np.float64)
    self.call("rhmc_set_approx", which, len(a), float(approx["a0"]), a, b, float(approx.get("min_eps", 1e-7)))


def _pf_get(self, name):
    cur = getattr(self, "_cur_species", 0)
    nps = self.no_ps if cur == 0 else self._species_nps[cur]
    out = np.zeros((nps, self.Vh, 3), np.complex128)
    self.call(name, out, HOST)
    return out


def _update(self, uniform):
    acc = ctypes.c_int()
    de = ctypes.c_double()
    self.call("rhmc_update", float(uniform), ctypes.byref(acc), ctypes.byref(de))
    return de.value, acc.value


Context.driver_setup = _driver_setup
Context.set_approx = _set_approx
Context.set_eig_bounds = lambda self, mn, mx: self.call("rhmc_set_eig_bounds", float(mn), float(mx))
Context.set_phi = lambda self, phi: self.call("rhmc_set_phi", np.ascontiguousarray(phi, np.complex128), HOST)
Context.set_chi = lambda self, chi: self.call("rhmc_set_chi", np.ascontiguousarray(chi, np.complex128), HOST)
Context.get_phi = lambda self: _pf_get(self, "rhmc_get_phi")
Context.get_chi = lambda self: _pf_get(self, "rhmc_get_chi")
Context.first_inv_approx_calc = lambda self, res: self.call("rhmc_first_inv_approx_calc", float(res))
Context.last_inv_approx_calc = lambda self, res: self.call("rhmc_last_inv_approx_calc", float(res))
Context.calc_ipdot = lambda self: self.call("rhmc_calc_ipdot")
Context.calc_ipdot_gauge = lambda self: self.call("rhmc_calc_ipdot_gauge")
Context.calc_ipdot_fermion = lambda self: self.call("rhmc_calc_ipdot_fermion")
Context.update_nometro = lambda self: self.call("rhmc_update_nometro")
Context.update = _update
Context.save_conf = lambda self: self.call("rhmc_save_conf")
Context.copy_saved = lambda self: self.call("rhmc_copy_saved")


def _workspace_bytes(self):
    n = ctypes.c_long(0)
    self.call("rhmc_workspace_bytes", ctypes.byref(n))
    return n.value


def _driver_solver_stats(self, which=0, reset=False):
    """Sums of the driver's solves since the last reset: which 0 force (md), 1 heatbath/action."""
    info = MsolveInfo()
    self.call("rhmc_driver_solver_stats", int(which), ctypes.byref(info), int(bool(reset)))
    return info.as_dict()


Context.driver_solver_stats = _driver_solver_stats
Context.workspace_bytes = _workspace_bytes
Context.workspace_release = lambda self: self.call("rhmc_workspace_release")


class LegacyConfig(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("nt", ctypes.c_int),
                ("ferm_temp_bc", ctypes.c_int), ("mass", ctypes.c_double), ("beta", ctypes.c_double),
                ("no_ps", ctypes.c_int), ("max_approx_order", ctypes.c_int), ("max_cg", ctypes.c_int),
                ("device", ctypes.c_int),
                ("gauge_field_packed", ctypes.c_void_p), ("chi_packed", ctypes.c_void_p),
                ("simple_fermion_packed", ctypes.c_void_p), ("ipdot_packed", ctypes.c_void_p),
                ("momenta_packed", ctypes.c_void_p), ("shift_table", ctypes.c_void_p), ("eta", ctypes.c_void_p)]


class Legacy:
    """The reference's extern "C" GPU entry points (include/rhmc_legacy.h) over host numpy
    buffers in the packer formats; keeps the buffers alive while bound."""

    def __init__(self, dims, mass, beta, no_ps, max_approx_order, max_cg, buffers, ferm_temp_bc=0, device=0):
        self.buffers = buffers

        def ptr(k):
            return ctypes.c_void_p(buffers[k].ctypes.data) if buffers.get(k) is not None else ctypes.c_void_p(None)

        cfg = LegacyConfig(*dims, ferm_temp_bc, mass, beta, no_ps, max_approx_order, max_cg, device,
                           ptr("gauge_field_packed"), ptr("chi_packed"), ptr("simple_fermion_packed"),
                           ptr("ipdot_packed"), ptr("momenta_packed"), ptr("shift_table"), ptr("eta"))
        _check(lib().rhmc_legacy_bind(ctypes.byref(cfg)))
        L = lib()
        dp = ctypes.POINTER(ctypes.c_double)
        L.cuda_shifted_inverter.argtypes = [ctypes.c_double, dp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.cuda_shifted_inverter_d.argtypes = L.cuda_shifted_inverter.argtypes
        L.cuda_sol_sum.argtypes = [ctypes.c_int, ctypes.c_double, dp]
        L.cuda_fermion_force.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
        L.cuda_gauge_deriv.argtypes = [ctypes.c_int]
        L.cuda_exp_su3.argtypes = [ctypes.c_float]
        L.cuda_momenta_sum_multiply.argtypes = [ctypes.c_float]
        L.cuda_find_max.argtypes = [dp]
        L.cuda_find_min.argtypes = [dp, ctypes.c_double]
        L.rhmc_legacy_context.restype = ctypes.c_void_p
        self.L = L

    def context_handle(self):
        return self.L.rhmc_legacy_context()

    def shifted_inverter(self, res, shifts, psferm, double=True):
        sh = np.ascontiguousarray(shifts, np.float64)
        n = ctypes.c_int()
        f = self.L.cuda_shifted_inverter_d if double else self.L.cuda_shifted_inverter
        f(res, sh.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(sh), psferm, ctypes.byref(n))
        return n.value

    def sol_sum(self, a0, a):
        a = np.ascontiguousarray(a, np.float64)
        self.L.cuda_sol_sum(len(a), a0, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def fermion_force(self, a):
        a = np.ascontiguousarray(a, np.float32)
        self.L.cuda_fermion_force(len(a), a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))

    def find_max(self):
        v = ctypes.c_double()
        self.L.cuda_find_max(ctypes.byref(v))
        return v.value

    def find_min(self, mx):
        v = ctypes.c_double()
        self.L.cuda_find_min(ctypes.byref(v), mx)
        return v.value

    def __getattr__(self, name):  # cuda_init0, cuda_init1, cuda_end, cuda_gauge_deriv, ...
        return getattr(self.L, name)

Context.fermion_action = lambda self: _f(self, "rhmc_fermion_action")


def _add_species(self, mass, no_flavours, no_ps):
    """Adds a fermion species (rhmc_driver_add_species) and returns its index."""
    idx = ctypes.c_int()
    self.call("rhmc_driver_add_species", float(mass), int(no_flavours), int(no_ps), ctypes.byref(idx))
    self._species_nps = getattr(self, "_species_nps", {})
    self._species_nps[idx.value] = no_ps
    return idx.value


def _select_species(self, index):
    self.call("rhmc_driver_select_species", int(index))
    self._cur_species = int(index)


Context.add_species = _add_species
Context.select_species = _select_species


def _find_max(self, start):
    """Largest eigenvalue of M^dag M by FP64 power iteration (rhmc_find_max); start: host spinor."""
    v = ctypes.c_double()
    self.call("rhmc_find_max", np.ascontiguousarray(start, np.complex128), ctypes.byref(v))
    return v.value


def _find_min(self, start, mx):
    v = ctypes.c_double()
    self.call("rhmc_find_min", np.ascontiguousarray(start, np.complex128), float(mx), ctypes.byref(v))
    return v.value


Context.find_max = _find_max
Context.find_min = _find_min


def _fma_peak(self, fp64=True):
    """Measured CUDA-core FMA throughput (TFLOP/s), FP64 or FP32 (rhmc_fma_peak)."""
    v = ctypes.c_double()
    self.call("rhmc_fma_peak", int(bool(fp64)), ctypes.byref(v))
    return v.value


Context.fma_peak = _fma_peak


def _eig_bounds(self):
    """(min, max) spectral bounds of M^dag M the driver holds for the selected species."""
    mn, mx = ctypes.c_double(), ctypes.c_double()
    self.call("rhmc_get_eig_bounds", ctypes.byref(mn), ctypes.byref(mx))
    return mn.value, mx.value


Context.eig_bounds = _eig_bounds
