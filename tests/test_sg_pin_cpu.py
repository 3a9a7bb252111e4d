"""Pins the oracle's self-gravity to an independent evaluation.

The reference computes the disk's own gravity as a convolution on the
logarithmic polar grid (compute_selfgravity, SgMain.cu:23-162; kernels
Kernels.cu:949-1041), the method of Baruteau & Masset (2008, ApJ 678, 483):
with u = ln(r/r0), S_r = Sigma (r/r0)^(1/2) and S_t = Sigma (r/r0)^(3/2),

    g_r(u, phi)   = -G (r/r0)^(-1/2) sum S_r(u', phi') K_r(u - u', phi - phi') du dphi
                    + G Sigma du dphi / eps
    g_phi(u, phi) = -G (r/r0)^(-3/2) sum S_t(u', phi') K_t(u - u', phi - phi') du dphi
    K_r = (1 + eps^2 - cos(phi) e^-u) / B^(3/2),  K_t = sin(phi) / B^(3/2),
    B = eps^2 e^u + 2 (cosh(u) - cos(phi)),

where the radial sum runs over the disk's rings only (the reference zero-pads
the radial direction to 2 NRAD so the FFT's circular convolution adds
nothing) and the azimuthal sum is periodic.  Here the sums are evaluated
directly, term by term in float64 with numpy (no FFT), and compared with the
oracle's FFT-based accelerations: the FP64 oracle must agree to rounding,
the FP32 oracle (the reference's typing: the kernel tabulated in float) to
its float precision."""
import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import noise
from oracle.oracle import Oracle
from tests.helpers import SEED, rel_l2, small


def direct_sg(P, dens):
    """g_r, g_phi of `dens` (NRAD x NSEC) by direct summation, float64."""
    N, M = P.NRAD, P.NSEC
    R = float(P.RMIN) * np.exp(np.arange(N + 1) / N * np.log(float(P.RMAX) / float(P.RMIN)))
    rmed = 2.0 / 3.0 * (R[1:] ** 3 - R[:-1] ** 3) / (R[1:] ** 2 - R[:-1] ** 2)
    eps = float(np.float32(P.THICKNESSSMOOTHING) * np.float32(P.ASPECTRATIO))
    rstep = np.log(R[N] / R[0]) / N
    tstep = 2.0 * np.pi / M
    d = np.arange(-(N - 1), N)
    u = np.where(d >= 0, np.log(R[np.abs(d)] / R[0]), -np.log(R[np.abs(d)] / R[0]))[:, None]
    th = (2.0 * np.pi * np.arange(M) / M)[None, :]
    B = eps * eps * np.exp(u) + 2.0 * (np.cosh(u) - np.cos(th))
    Kr = (1.0 + eps * eps - np.cos(th) * np.exp(-u)) * B ** -1.5
    Kt = np.sin(th) * B ** -1.5
    x = rmed / rmed[0]
    Sr = dens * np.sqrt(x)[:, None]
    St = Sr * x[:, None]
    # circulant in phi: C[dj][j, j'] = K[dj][(j - j') mod M]
    jj = (np.arange(M)[:, None] - np.arange(M)[None, :]) % M
    Gr = np.zeros((N, M))
    Gt = np.zeros((N, M))
    for i in range(N):
        for ip in range(N):
            k = i - ip + (N - 1)
            Gr[i] -= Kr[k][jj] @ Sr[ip]
            Gt[i] -= Kt[k][jj] @ St[ip]
    accr = Gr * rstep * tstep / np.sqrt(x)[:, None] + dens * rstep * tstep / eps
    acct = Gt * rstep * tstep / (x * np.sqrt(x))[:, None]
    return accr, acct


@pytest.mark.parametrize("nrad,nsec", [(32, 64), (64, 128)])
def test_oracle_sg_matches_direct_sum(nrad, nsec):
    P, L, _ = small("sg", nrad, nsec)
    o64 = Oracle(P, L, "f64")
    f = o64.fields()
    dens = noise.perturb_density(f["dens"].reshape(-1), nrad, nsec, SEED).reshape(nrad + 1, nsec)
    o64.set_fields(dens=dens)
    accr, acct = o64.sg_accelerations()
    want_r, want_t = direct_sg(P, dens[:nrad].astype(np.float64))
    assert rel_l2(accr, want_r) <= 1e-12
    assert rel_l2(acct, want_t) <= 1e-12
    o32 = Oracle(P, L, "f32")
    o32.set_fields(dens=dens)
    r32, t32 = o32.sg_accelerations()
    # The FP32 build tabulates the kernel in float, as SgMain.cu:49-81 does.
    # g_r: near u = 0, phi = 0 the denominator's cosh(u) - cos(phi) cancels
    # to a few 1e-3, so the nearest kernel entries carry ~1e-4 relative
    # rounding; measured ~1e-5 on g_r.  g_phi of a near-axisymmetric disk is
    # the small residual (driven by the 1e-3 noise) of a large axisymmetric
    # density convolved with an antisymmetric kernel; the float table of
    # K_t = sin(phi) B^-3/2 is not exactly antisymmetric, so a part of the
    # axisymmetric density leaks into g_phi: measured ~5e-3 relative.  Both
    # are the reference's own precision, not an error of the oracle.
    assert rel_l2(r32, want_r) <= 3e-5
    assert rel_l2(t32, want_t) <= 1e-2
