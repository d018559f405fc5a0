"""Host-side lattice geometry and seeded synthetic fields in the reference layouts.

Layouts (those of coppolachan/RHMC-on-GPU's CPU classes):
  links / momenta / ipdot : complex128 (4V, 3, 3), index mu*V + site (Conf::u_work,
                            include/configuration.h:9-10)
  spinor                  : complex128 (Vh, 3) one parity (Fermion, lib/Action/fermions.h:12)
Sites are numbered even-first: num = parity*Vh + (x + y*nx + z*nx*ny + t*nx*ny*nz)//2
(lib/Main/Geometry/geometry.cc:5-11, 86).

Random inputs are numpy Philox streams keyed by a seed; they stand in for the reference's
host RNG (dSFMT), whose streams are out of scope: tests inject identical buffers into the
reference oracle and into the CUDA path.
"""
import numpy as np


def site_coords(dims):
    """(x, y, z, t) int arrays of length V, indexed by the reference even/odd site number."""
    nx, ny, nz, nt = dims
    V = nx * ny * nz * nt
    t, z, y, x = np.meshgrid(np.arange(nt), np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    x, y, z, t = (a.ravel() for a in (x, y, z, t))
    lex = x + nx * (y + ny * (z + nz * t))
    par = (x + y + z + t) & 1
    num = par * (V // 2) + lex // 2
    out = np.empty((4, V), np.int64)
    out[0, num] = x
    out[1, num] = y
    out[2, num] = z
    out[3, num] = t
    return out


def site_number(dims, x, y, z, t):
    nx, ny, nz, nt = dims
    V = nx * ny * nz * nt
    lex = x + nx * (y + ny * (z + nz * t))
    return ((x + y + z + t) & 1) * (V // 2) + lex // 2


def neighbour_table(dims):
    """int32[8V]: nnm mu=0..3 then nnp mu=0..3 (make_shift_table, lib/Tools/Packer/packer.cc:415-439)."""
    c = site_coords(dims)
    V = c.shape[1]
    tab = np.empty(8 * V, np.int32)
    for mu in range(4):
        for k, sgn in ((0, -1), (4, +1)):
            d = c.copy()
            d[mu] = (d[mu] + sgn) % dims[mu]
            tab[(k + mu) * V:(k + mu + 1) * V] = site_number(dims, *d)
    return tab


def eta_phases(dims, ferm_temp_bc=0):
    """int32[4V] staggered phases with antiperiodic time b.c. when ferm_temp_bc == 0
    (lib/Main/Geometry/geometry.cc:107-153)."""
    x, y, z, t = site_coords(dims)
    V = x.size
    eta = np.ones(4 * V, np.int32)
    eta[V:2 * V] = 1 - 2 * (x & 1)
    eta[2 * V:3 * V] = 1 - 2 * ((x + y) & 1)
    et = 1 - 2 * ((x + y + z) & 1)
    if ferm_temp_bc == 0:
        et = np.where(t == dims[3] - 1, -et, et)
    eta[3 * V:] = et
    return eta


def sunitarize(u):
    """Row-0 normalise, Gram-Schmidt row 1, row 2 = conj(row0 x row1) for a (..., 3, 3) stack
    (Su3::sunitarize, lib/Action/su3.cc:69-112)."""
    u = np.array(u, np.complex128, copy=True)
    r0 = u[..., 0, :]
    r0 /= np.sqrt(np.sum(r0.real ** 2 + r0.imag ** 2, axis=-1))[..., None]
    prod = np.sum(np.conj(r0) * u[..., 1, :], axis=-1)
    r1 = u[..., 1, :] - prod[..., None] * r0
    r1 /= np.sqrt(np.sum(r1.real ** 2 + r1.imag ** 2, axis=-1))[..., None]
    u[..., 0, :] = r0
    u[..., 1, :] = r1
    u[..., 2, 0] = np.conj(r0[..., 1] * r1[..., 2] - r0[..., 2] * r1[..., 1])
    u[..., 2, 1] = np.conj(r0[..., 2] * r1[..., 0] - r0[..., 0] * r1[..., 2])
    u[..., 2, 2] = np.conj(r0[..., 0] * r1[..., 1] - r0[..., 1] * r1[..., 0])
    return u


def haar_su3(n, rng):
    """n Haar-distributed SU(3) matrices: QR of a complex Gaussian with the phase fix of
    Mezzadri (2007), divided by det^(1/3)."""
    z = (rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r, axis1=-2, axis2=-1)
    q = q * (d / np.abs(d))[:, None, :]
    det = np.linalg.det(q)
    q = q / (det ** (1.0 / 3.0))[:, None, None]
    return q


def random_links(dims, seed=1001, ferm_temp_bc=0, kind="haar", eps=0.3):
    """Links with the staggered phases folded in, every row times eta (conf.cc:36,49),
    unitarised so that row 2 = eta * conj(row0 x row1) holds exactly.
    kind='haar' (hot start) or 'near1' (exp of a random algebra element of size eps)."""
    V = int(np.prod(dims))
    rng = np.random.Generator(np.random.Philox(seed))
    if kind == "haar":
        u = haar_su3(4 * V, rng)
    else:
        h = random_algebra(4 * V, rng) * eps
        w, v = np.linalg.eigh(h)
        u = np.einsum("nij,nj,nkj->nik", v, np.exp(1j * w), np.conj(v))
    u = sunitarize(u)
    eta = eta_phases(dims, ferm_temp_bc)
    return u * eta[:, None, None]


def random_algebra(n, rng):
    """Traceless Hermitian sum_a w_a lambda_a with w_a ~ N(0, 1/2) (Su3::gauss, gauss.cc:63-88)."""
    w = rng.standard_normal((n, 8)) * np.sqrt(0.5)
    s3 = 1.0 / np.sqrt(3.0)
    m = np.zeros((n, 3, 3), np.complex128)
    m[:, 0, 0] = w[:, 2] + s3 * w[:, 7]
    m[:, 1, 1] = -w[:, 2] + s3 * w[:, 7]
    m[:, 2, 2] = -2.0 * s3 * w[:, 7]
    m[:, 0, 1] = w[:, 0] - 1j * w[:, 1]
    m[:, 1, 0] = w[:, 0] + 1j * w[:, 1]
    m[:, 0, 2] = w[:, 3] - 1j * w[:, 4]
    m[:, 2, 0] = w[:, 3] + 1j * w[:, 4]
    m[:, 1, 2] = w[:, 5] - 1j * w[:, 6]
    m[:, 2, 1] = w[:, 5] + 1j * w[:, 6]
    return m


def random_momenta(dims, seed=3003):
    V = int(np.prod(dims))
    return random_algebra(4 * V, np.random.Generator(np.random.Philox(seed)))


def random_spinor(dims, seed=2002, n=None):
    """Complex Gaussian spinor(s) on one parity with E|z|^2 = 1 per colour component
    (Vec3::gauss, gauss.cc:25-46,90-95).  Shape (Vh, 3), or (n, Vh, 3)."""
    Vh = int(np.prod(dims)) // 2
    rng = np.random.Generator(np.random.Philox(seed))
    shape = (Vh, 3) if n is None else (n, Vh, 3)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2.0)
