"""Seeded smooth test fields shared by the CPU and GPU tests."""
import numpy as np


def smooth_field(dims, rng, modes=4, scale=1.0):
    """Real periodic field (nz, ny, nx) from a few low Fourier modes."""
    nx, ny, nz = dims
    x = np.arange(nx) / nx
    y = np.arange(ny) / ny
    z = np.arange(nz) / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    f = np.zeros(X.shape)
    for _ in range(modes):
        k = rng.integers(-2, 3, size=3)
        ph = rng.uniform(0, 2 * np.pi)
        a = rng.normal()
        f += a * np.cos(2 * np.pi * (k[0] * X + k[1] * Y + k[2] * Z) + ph)
    return scale * f


def smooth_psi(dims, seed=0, phase_scale=1.5, amp2=0.3):
    """Normalised two-component psi (nz, ny, nx, 4) float64 with smooth
    phases (neighbour phase steps well below pi) and smooth amplitudes."""
    rng = np.random.default_rng(seed)
    th1 = smooth_field(dims, rng, scale=phase_scale)
    th2 = smooth_field(dims, rng, scale=phase_scale)
    a1 = 1.0 + 0.2 * np.tanh(smooth_field(dims, rng))
    a2 = amp2 * (1.0 + 0.2 * np.tanh(smooth_field(dims, rng)))
    p1 = a1 * np.exp(1j * th1)
    p2 = a2 * np.exp(1j * th2)
    n = np.sqrt(np.abs(p1) ** 2 + np.abs(p2) ** 2)
    p1, p2 = p1 / n, p2 / n
    return np.ascontiguousarray(np.stack([p1.real, p1.imag, p2.real, p2.imag], axis=-1))


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    a = a.astype(np.complex128) if np.iscomplexobj(a) else a.astype(np.float64)
    b = b.astype(np.complex128) if np.iscomplexobj(b) else b.astype(np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def philox4x32_10_py(ctr, key):
    """Pure-Python Philox4x32-10 (Salmon et al. SC'11), independent of the C
    restatements, for cross-checking them."""
    M0, M1 = 0xD2511F53, 0xCD9E8D57
    W0, W1 = 0x9E3779B9, 0xBB67AE85
    c = list(ctr)
    k0, k1 = key
    mask = 0xFFFFFFFF
    for _ in range(10):
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        c = [((p1 >> 32) ^ c[1] ^ k0) & mask, p1 & mask, ((p0 >> 32) ^ c[3] ^ k1) & mask, p0 & mask]
        k0 = (k0 + W0) & mask
        k1 = (k1 + W1) & mask
    return c
