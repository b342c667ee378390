"""The oracle's analytic initial condition (initFlow) against its closed form.

initFlow (source/RPCFKernels.cu:358-431) evaluates three-mode fields and
takes them to spectral space without padding.  w = A(z) (sin a1 sin b1 +
sin a2 sin b1 + sin a1 sin b2) and omega_z = B(z) (products of cosines), with
a_m = 2 pi m x / lx, b_m = 2 pi m y / ly, so the normalised 2D transform puts
+-1/4 of each product into exactly the pencils (kx, +-ky) of its wavenumbers
and the wall-normal profile into every one of them: the Chebyshev
coefficients of A (resp. B) at the nz Gauss-Lobatto points with the two wall
values set to zero.  Checked to 1e-14 of the largest coefficient.
"""
import numpy as np
import pytest

from oracle import rpcf_oracle as O


def profile(sz, f):
    z = np.cos(np.pi * np.arange(sz.nz) / (sz.nz - 1))
    vals = f(z)
    vals[0] = vals[-1] = 0.0
    S = np.zeros((1, 1, sz.mz), dtype=np.complex128)
    S[0, 0, :sz.nz] = vals
    return O.cheby_p2s(S, sz.mz, pad=False)[0, 0, :sz.nz]


@pytest.mark.parametrize("mx,my,mz,npx,npy", [(24, 24, 32, 4.0, 2.0), (48, 36, 64, 2.0, 3.0)])
def test_init_state_closed_form(mx, my, mz, npx, npy):
    sz = O.Sizes(mx, my, mz)
    aphi, beta = npx / 2, npy / 2
    lx, ly = 2 * O.PI * aphi, 2 * O.PI * beta
    V, Om = O.init_state(sz, aphi, beta)
    e = O.EPSILON_INIT
    A = profile(sz, lambda z: e * (-2.0 / 3.0) * (1.0 + np.cos(1.5 * O.PI * z)))
    B = profile(sz, lambda z: e * 2.0 * O.PI * np.sin(1.5 * O.PI * z))
    ny = sz.ny
    # (kx, ky) -> coefficient of the profile; ky < 0 is pencil ny + ky
    wv = {(1, 1): -0.25, (1, -1): 0.25, (2, 1): -0.25, (2, -1): 0.25, (1, 2): -0.25, (1, -2): 0.25}
    r, q = lx / ly, ly / lx
    oz = {(1, 1): (r + 0.5 * q) / 4, (2, 1): (0.5 * r + q) / 4, (1, 2): (2.0 * r + 0.25 * q) / 4}
    oz.update({(kx, -ky): c for (kx, ky), c in list(oz.items())})
    refV = np.zeros_like(V)
    refO = np.zeros_like(Om)
    for (kx, ky), c in wv.items():
        refV[ky % ny, kx] = c * A
    for (kx, ky), c in oz.items():
        refO[ky % ny, kx] = c * B
    assert np.max(np.abs(V - refV)) < 1e-14 * np.max(np.abs(refV))
    assert np.max(np.abs(Om - refO)) < 1e-14 * np.max(np.abs(refO))
