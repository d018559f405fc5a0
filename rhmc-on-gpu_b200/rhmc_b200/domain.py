"""Domain decomposition of the even/odd staggered operator across ranks in t-slabs (no counterpart
in the reference, which runs on one GPU, include/parameters.h:76).

Rank r of W owns the time slices [r nt/W, (r+1) nt/W) of every field (nt/W even, so a local
site's parity is its global parity).  In the reference's half-index order (t slowest,
lib/Main/Geometry/geometry.cc:5-11) a rank's sites of one parity are one contiguous range of the
global array, so scatter and gather are slices.  Locally each field lives on an extended lattice
of nt/W + 2 slices: one ghost slice below (t_ext = 0) and one above (t_ext = nt/W + 1).  Because
the ghost slice below shifts the extended coordinate by one, a global parity p is parity 1 - p of
the extended lattice.

  * Links are exchanged once per configuration: the ghost slice below receives the previous rank's
    last slice (the backward links U_mu(x - t) of the first interior slice; forward links are
    always local).  The fermion boundary sign folded into the links (conf.cc:36,49) travels with
    them.
  * Every half-Dslash exchanges one spinor face each way: a rank's first interior slice of the
    input parity goes to the previous rank's upper ghost, its last to the next rank's lower
    ghost (point-to-point isend/irecv: NCCL over NVLink between GPUs, gloo between CPU ranks).
  * Dot products are local sums followed by one all-reduce of the FP64 scalars.

The local half-Dslash is a callable on extended fields -- on the GPU the library's site-range
Dslash (rhmc_dslash_sites, FP64 links, reference spinor layout, only the interior output sites),
in the CPU tests the oracle -- so the decomposition logic is the same on both.  DDMultiShift is the
multi-shift CG of lib/Action/Inverter/inverter.cc:142-339 (the reference's recurrences, shift
freezing and stopping rule) on the decomposed operator, host-driven, one all-reduce of the two
CG scalars per iteration besides the two in the operator."""
import numpy as np
import torch


class TSlab:
    """Geometry of one rank's t-slab."""

    def __init__(self, dims, rank, world):
        nx, ny, nz, nt = dims
        if nt % world or (nt // world) % 2:
            raise ValueError("nt / world must be an even integer (nt=%d, world=%d)" % (nt, world))
        self.dims, self.rank, self.world = tuple(dims), rank, world
        self.nt_loc = nt // world
        self.t0 = rank * self.nt_loc
        self.Vs = nx * ny * nz  # sites per time slice
        self.face = self.Vs // 2  # sites of one parity per time slice
        self.Vh = self.Vs * nt // 2
        self.Vh_loc = self.face * self.nt_loc
        self.dims_ext = (nx, ny, nz, self.nt_loc + 2)
        self.Vh_ext = self.face * (self.nt_loc + 2)
        self.prev = (rank - 1) % world
        self.next = (rank + 1) % world

    def ext_parity(self, p):
        """Parity in the extended lattice of global parity p (the lower ghost slice shifts t by one)."""
        return p ^ 1

    def interior(self):
        """Half-index range of the interior in an extended field."""
        return self.face, self.face + self.Vh_loc

    def local_slice(self):
        """Half-index range of this rank's sites in a global field of one parity."""
        return self.t0 * self.face, (self.t0 + self.nt_loc) * self.face

    def scatter(self, g):
        """This rank's part (Vh_loc, 3) of a global spinor (Vh, 3)."""
        a, b = self.local_slice()
        return g[a:b]

    def extend(self, loc):
        """An extended field (Vh_ext, 3) with loc in the interior and zero ghosts."""
        e = torch.zeros((self.Vh_ext,) + tuple(loc.shape[1:]), dtype=loc.dtype, device=loc.device)
        a, b = self.interior()
        e[a:b] = loc
        return e

    def links_from_global(self, u, ghosts=True):
        """This rank's extended links (4 V_ext, 3, 3), in the extended lattice's even-first site
        order (Conf::u_work layout, include/configuration.h:9-10), from the global links
        (4 V, 3, 3): the interior, and with ghosts=True the lower ghost slice as well (which
        exchange_link_ghosts otherwise fills from the previous rank)."""
        nt = self.dims[3]
        V, Ve = 2 * self.Vh, 2 * self.Vh_ext
        out = np.zeros((4 * Ve, 3, 3), np.complex128)
        lo = ((self.t0 - 1) % nt) * self.face
        for mu in range(4):
            for q in (0, 1):  # extended parity; global parity q ^ 1
                src = mu * V + (q ^ 1) * self.Vh
                dst = mu * Ve + q * self.Vh_ext
                a, b = self.local_slice()
                out[dst + self.face:dst + self.face + self.Vh_loc] = u[src + a:src + b]
                if ghosts:
                    out[dst:dst + self.face] = u[src + lo:src + lo + self.face]
        return out


def spinor_ext_from_global(slab, x):
    """This rank's extended spinor (Vh_ext, 3), interior and both ghost slices, from a global
    spinor (Vh, 3) of one parity (what the halo exchange assembles from the neighbours)."""
    nt = slab.dims[3]
    f = slab.face
    out = np.zeros((slab.Vh_ext, 3), np.complex128)
    a, b = slab.local_slice()
    out[f:f + slab.Vh_loc] = x[a:b]
    lo = ((slab.t0 - 1) % nt) * f
    hi = ((slab.t0 + slab.nt_loc) % nt) * f
    out[:f] = x[lo:lo + f]
    out[f + slab.Vh_loc:] = x[hi:hi + f]
    return out


def library_dslash(ctx_ext, slab):
    """The local half-Dslash of a DDOperator on the GPU: ctx_ext is a library context of the
    extended lattice (slab.dims_ext) holding the extended links; only the interior output sites
    are computed (rhmc_dslash_sites), from device tensors (Vh_ext, 3) complex128."""
    a, b = slab.interior()

    def run(p_ext, out, inp):
        ctx_ext.dslash_sites(p_ext, out, inp, a, b - a)

    return run


class DDOperator:
    """The decomposed M^dag M = m^2 - D_eo D_oe on even sites (lib/Action/Inverter/inverter.cc:206-216)."""

    def __init__(self, slab, mass, local_dslash, dist=None):
        """local_dslash(p_out_ext, out_ext, in_ext) writes the half-Dslash onto parity p_out_ext of
        the extended lattice for (at least) the interior output sites; out_ext, in_ext are
        complex128 tensors (Vh_ext, 3)."""
        self.s = slab
        self.mass = mass
        self.local_dslash = local_dslash
        self.dist = dist
        self.dslash_calls = 0
        self.halo_bytes = 0

    # ------------------------------------------------------------------ communication
    def _sendrecv(self, send_prev, send_next):
        """Sends send_prev to the previous rank and send_next to the next; returns (from_next,
        from_prev), i.e. what the next rank sent down and what the previous rank sent up."""
        s = self.s
        if s.world == 1 or self.dist is None:
            return send_prev.clone(), send_next.clone()
        from_next = torch.empty_like(send_prev)
        from_prev = torch.empty_like(send_next)
        # every rank sends up then down and receives from below then from above: with two ranks
        # (previous = next) the two messages between a pair are then matched in the same order
        # on both sides, as point-to-point matching between a pair is by posting order
        ops = [self.dist.P2POp(self.dist.isend, send_next.contiguous(), s.next),
               self.dist.P2POp(self.dist.isend, send_prev.contiguous(), s.prev),
               self.dist.P2POp(self.dist.irecv, from_prev, s.prev),
               self.dist.P2POp(self.dist.irecv, from_next, s.next)]
        for r in self.dist.batch_isend_irecv(ops):
            r.wait()
        self.halo_bytes += 2 * send_prev.numel() * send_prev.element_size()
        return from_next, from_prev

    def exchange_link_ghosts(self, u_ext):
        """Fills the lower ghost slice of extended links (torch (4 V_ext, 3, 3)) with the previous
        rank's last interior slice, for every direction and parity (once per configuration)."""
        s = self.s
        Ve = 2 * s.Vh_ext
        last = torch.stack([u_ext[mu * Ve + q * s.Vh_ext + s.Vh_loc:mu * Ve + q * s.Vh_ext + s.Vh_loc + s.face]
                            for mu in range(4) for q in (0, 1)])
        _, from_prev = self._sendrecv(torch.zeros_like(last), last)
        i = 0
        for mu in range(4):
            for q in (0, 1):
                u_ext[mu * Ve + q * s.Vh_ext:mu * Ve + q * s.Vh_ext + s.face] = from_prev[i]
                i += 1
        return u_ext

    def halo(self, ext):
        """Fills both ghost slices of an extended spinor from the neighbouring ranks."""
        s = self.s
        f = s.face
        first = ext[f:2 * f]                      # t_ext = 1
        last = ext[s.Vh_loc:s.Vh_loc + f]          # t_ext = nt_loc
        from_next, from_prev = self._sendrecv(first, last)
        ext[0:f] = from_prev                       # previous rank's last slice
        ext[s.Vh_loc + f:s.Vh_loc + 2 * f] = from_next  # next rank's first slice
        return ext

    def allreduce(self, t):
        if self.dist is not None and self.s.world > 1:
            self.dist.all_reduce(t)
        return t

    def dot_re(self, a, b):
        """Re<a, b> over the whole lattice (FP64)."""
        v = torch.real(torch.vdot(a.reshape(-1), b.reshape(-1))).reshape(1).to(torch.float64)
        return float(self.allreduce(v)[0])

    def norm2(self, a):
        return self.dot_re(a, a)

    # ------------------------------------------------------------------ operator
    def dslash(self, p_out, loc_in):
        """Global half-Dslash onto parity p_out of a field of parity 1 - p_out: local parts in, local out."""
        s = self.s
        ext_in = self.halo(s.extend(loc_in))
        ext_out = torch.zeros_like(ext_in)
        self.local_dslash(s.ext_parity(p_out), ext_out, ext_in)
        self.dslash_calls += 1
        a, b = s.interior()
        return ext_out[a:b]

    def mdagm(self, x, shift=0.0):
        """(M^dag M + shift) x on the even sites."""
        return (self.mass ** 2 + shift) * x - self.dslash(0, self.dslash(1, x))


def multishift_cg(op, b, shifts, res, max_iter=100000, stop_on_frozen=False):
    """Jegerlehner's multi-shift CG as multips_shifted_invert (inverter.cc:142-339) runs it, on the
    decomposed operator: x_i = 0, r = p = p_i = b; shift i frozen when sqrt(delta zeta''_i^2) < res
    (the lagged residual, inverter.cc:275-279); stops when sqrt(|r|^2) <= res (inverter.cc:287) or,
    with stop_on_frozen, also when every shift is frozen (the GPU solver's rule,
    cuda_inverter.cu:777-785).  Returns the local parts of the solutions [nshift] and the
    iteration count."""
    shifts = [float(v) for v in shifts]
    ns = len(shifts)
    x = [torch.zeros_like(b) for _ in range(ns)]
    ps = [b.clone() for _ in range(ns)]
    r = b.clone()
    p = b.clone()
    delta = op.norm2(r)
    omega, gamma = 1.0, 0.0
    zeta_i = [1.0] * ns
    zeta_ii = [1.0] * ns
    active = [True] * ns
    it = 0
    while it < max_iter:
        s = op.mdagm(p)
        alpha = op.dot_re(p, s)
        omega_prev = omega
        omega = -delta / alpha
        zeta_iii = [0.0] * ns
        omegas = [0.0] * ns
        for i in range(ns):
            if not active[i]:
                continue
            zi, zii = zeta_i[i], zeta_ii[i]
            zeta_iii[i] = (zi * zii * omega_prev) / (omega * gamma * (zi - zii) + zi * omega_prev * (1.0 - shifts[i] * omega))
            omegas[i] = omega * zeta_iii[i] / zii
            x[i] = x[i] - omegas[i] * ps[i]
        r = r + omega * s
        lam = op.norm2(r)
        gamma = lam / delta
        p = r + gamma * p
        for i in range(ns):
            if not active[i]:
                continue
            gi = gamma * zeta_iii[i] * omegas[i] / (zeta_ii[i] * omega)
            ps[i] = zeta_iii[i] * r + gi * ps[i]
            fact = (delta * zeta_ii[i] * zeta_ii[i]) ** 0.5
            if fact < res:
                active[i] = False
            zeta_i[i] = zeta_ii[i]
            zeta_ii[i] = zeta_iii[i]
        delta = lam
        it += 1
        if lam ** 0.5 <= res or (stop_on_frozen and not any(active)):
            break
    return x, it
