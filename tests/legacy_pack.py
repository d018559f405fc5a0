"""numpy restatement of the reference's host packers (lib/Tools/Packer/packer.cc), used by the
tests to build and read the packed host buffers that the legacy GPU entry points exchange."""
import numpy as np


def _hilo(v):
    hi = v.astype(np.float32)
    lo = (v - hi.astype(np.float64)).astype(np.float32)
    return hi, lo


_ROWS01 = [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2)]


def pack_gauge(u):
    """smartpack_gauge (packer.cc:8-71): float[2*12*4V], rows 0-1 as three float4 planes per mu."""
    V = u.shape[0] // 4
    vals = np.empty((4, 3, V, 4), np.float64)
    for mu in range(4):
        b = u[mu * V:(mu + 1) * V]
        for q in range(3):
            (i0, j0), (i1, j1) = _ROWS01[2 * q], _ROWS01[2 * q + 1]
            vals[mu, q, :, 0] = b[:, i0, j0].real
            vals[mu, q, :, 1] = b[:, i0, j0].imag
            vals[mu, q, :, 2] = b[:, i1, j1].real
            vals[mu, q, :, 3] = b[:, i1, j1].imag
    hi, lo = _hilo(vals.reshape(-1))
    return np.concatenate([hi, lo])


def unpack_gauge_rows01(pk, V):
    """Rows 0 and 1 of every link of a gauge buffer, as doubles hi + lo."""
    n = 12 * 4 * V
    v = (pk[:n].astype(np.float64) + pk[n:].astype(np.float64)).reshape(4, 3, V, 4)
    u = np.zeros((4 * V, 2, 3), np.complex128)
    for mu in range(4):
        for q in range(3):
            (i0, j0), (i1, j1) = _ROWS01[2 * q], _ROWS01[2 * q + 1]
            u[mu * V:(mu + 1) * V, i0, j0] = v[mu, q, :, 0] + 1j * v[mu, q, :, 1]
            u[mu * V:(mu + 1) * V, i1, j1] = v[mu, q, :, 2] + 1j * v[mu, q, :, 3]
    return u


def pack_multifermion(f):
    """smartpack_multifermion (packer.cc:278-319): f (no_ps, Vh, 3) -> float[6*Vh*no_ps*2]."""
    nps, Vh, _ = f.shape
    V = 2 * Vh
    vals = np.zeros(3 * V * nps, np.float64)
    for ps in range(nps):
        for c in range(3):
            base = 3 * V * ps + c * V
            vals[base:base + V:2] = f[ps, :, c].real
            vals[base + 1:base + V:2] = f[ps, :, c].imag
    hi, lo = _hilo(vals)
    return np.concatenate([hi, lo])


def unpack_multifermion(pk, nps, Vh):
    """smartunpack_multifermion (packer.cc:323-366)."""
    V = 2 * Vh
    n = 3 * V * nps
    v = pk[:n].astype(np.float64) + pk[n:].astype(np.float64)
    f = np.zeros((nps, Vh, 3), np.complex128)
    for ps in range(nps):
        for c in range(3):
            base = 3 * V * ps + c * V
            f[ps, :, c] = v[base:base + V:2] + 1j * v[base + 1:base + V:2]
    return f


def pack_fermion(x):
    """smartpack_fermion (packer.cc:156-190): one (Vh, 3) spinor -> float[6*Vh], single precision
    (the hi block of pack_fermion_d); findminmax.cc:161 packs the power-iteration start with it."""
    return pack_multifermion(x[None])[:6 * x.shape[0]]


def pack_fermion_d(x):
    """smartpack_fermion_d (packer.cc:192-230): one (Vh, 3) spinor -> float[6*Vh*2]."""
    return pack_multifermion(x[None])


def _alg_vals(m, antiherm):
    V = m.shape[0] // 4
    vals = np.zeros((4, 2, V, 4), np.float64)
    for mu in range(4):
        b = m[mu * V:(mu + 1) * V]
        vals[mu, 0, :, 0] = b[:, 0, 1].real
        vals[mu, 0, :, 1] = b[:, 0, 1].imag
        vals[mu, 0, :, 2] = b[:, 0, 2].real
        vals[mu, 0, :, 3] = b[:, 0, 2].imag
        vals[mu, 1, :, 0] = b[:, 1, 2].real
        vals[mu, 1, :, 1] = b[:, 1, 2].imag
        vals[mu, 1, :, 2] = b[:, 0, 0].imag if antiherm else b[:, 0, 0].real
        vals[mu, 1, :, 3] = b[:, 1, 1].imag if antiherm else b[:, 1, 1].real
    return vals.reshape(-1).astype(np.float32)


def pack_tamatrix(ip):
    """smartpack_tamatrix (packer.cc:443-469)."""
    return _alg_vals(ip, True)


def pack_thmatrix(p):
    """smartpack_thmatrix (packer.cc:508-534)."""
    return _alg_vals(p, False)


def unpack_alg(pk, V, antiherm):
    """smartunpack_tamatrix / smartunpack_thmatrix (packer.cc:473-504, 538-569)."""
    v = pk.astype(np.float64).reshape(4, 2, V, 4)
    m = np.zeros((4 * V, 3, 3), np.complex128)
    for mu in range(4):
        s = slice(mu * V, (mu + 1) * V)
        a01 = v[mu, 0, :, 0] + 1j * v[mu, 0, :, 1]
        a02 = v[mu, 0, :, 2] + 1j * v[mu, 0, :, 3]
        a12 = v[mu, 1, :, 0] + 1j * v[mu, 1, :, 1]
        # diagonal entries built as complex(0, d) / complex(d, 0) and a22 = -a00 - a11 in complex
        # arithmetic, as the reference does, so that even the signs of zeros agree
        m00, m11 = np.zeros(V, np.complex128), np.zeros(V, np.complex128)
        if antiherm:
            m00.imag, m11.imag = v[mu, 1, :, 2], v[mu, 1, :, 3]
            m[s, 1, 0], m[s, 2, 0], m[s, 2, 1] = -np.conj(a01), -np.conj(a02), -np.conj(a12)
        else:
            m00.real, m11.real = v[mu, 1, :, 2], v[mu, 1, :, 3]
            m[s, 1, 0], m[s, 2, 0], m[s, 2, 1] = np.conj(a01), np.conj(a02), np.conj(a12)
        m[s, 0, 0], m[s, 1, 1] = m00, m11
        m[s, 2, 2] = -m00 - m11
        m[s, 0, 1], m[s, 0, 2], m[s, 1, 2] = a01, a02, a12
    return m
