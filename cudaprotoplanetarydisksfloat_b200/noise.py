"""Seeded multiplicative density noise shared by the tests, the bench and the
reference hook (oracle/ref/ref_hooks.cu): Sigma_ij *= 1 + amp*u_ij with u_ij
in [-1, 1) drawn ring by ring, sector by sector from splitmix64, 24-bit
mantissa, all in float32 so every implementation produces the same bits."""
import numpy as np

_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed, n):
    """The first n outputs of splitmix64 started at `seed`."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * _G
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform_pm1(seed, n):
    """u in [-1, 1), float32, 24 random bits each."""
    z = splitmix64(seed, n)
    m = ((z >> np.uint64(40)) & np.uint64(0xFFFFFF)).astype(np.float32)
    return m / np.float32(8388608.0) - np.float32(1.0)


def perturb_density(dens, nrad, nsec, seed, amp=1e-3):
    """Apply the noise to the active rings of a (nrad+1)*nsec float32 field."""
    d = np.array(dens, dtype=np.float32, copy=True).reshape(nrad + 1, nsec)
    u = uniform_pm1(seed, nrad * nsec).reshape(nrad, nsec)
    f = np.float32(1.0) + np.float32(amp) * u
    d[:nrad] = d[:nrad] * f
    return d.reshape(-1)
