"""Seeded, divergence-free initial perturbation for the DNS state.

The state of the solver is (v-hat, omega_y-hat): wall-normal velocity and
wall-normal vorticity, as Chebyshev coefficients per Fourier pencil, stored in
the reference's spectral order ``[kz][kx][n]`` (spanwise mode, streamwise
mode, Chebyshev index).  The mean pencil (0,0) carries the mean streamwise
and spanwise velocity perturbations u0 / w0, as in the reference
(source/solver.cpp:332-338, source/velocity.cu:106-124).

Definition (standard axes x streamwise, y wall-normal, z spanwise):

* a vector potential A with three components, complex Fourier-Chebyshev
  coefficients ``amp(kx,kz) * 0.8**n * (xi_r + i xi_i)``, ``xi`` standard
  normal from ``numpy.random.default_rng(seed)`` drawn as one array of shape
  ``(3, 2, Nz, Kx, Ny-4)``;
* ``amp = A0 * exp(-(kx^2 + kz^2)/8)`` with integer mode indices (kz signed);
* Hermitian symmetry imposed on the kx = 0 plane; Nyquist modes and the
  (0,0) mode set to zero; Chebyshev degree of A below Ny-4 so that the
  product with ``g(y) = (1-y^2)^2`` is an exact degree < Ny polynomial;
* ``u' = curl(g A)``, so ``v-hat = i beta Psi_x - i alpha Psi_z`` and
  ``omega_y-hat = i alpha D Psi_x + i beta D Psi_z + k^2 Psi_y`` with
  ``Psi = g A``; both vanish at the walls and ``v`` has zero wall slope.
"""
from __future__ import annotations

import numpy as np


def _dct1_coeffs(vals):
    """Chebyshev coefficients from values at y_j = cos(pi j/(n-1))."""
    n = vals.shape[-1]
    N = n - 1
    j = np.arange(n)
    C = np.cos(np.pi * np.outer(j, j) / N)  # C[k, j]
    w = np.ones(n)
    w[0] = w[-1] = 0.5
    c = (vals * w) @ C.T * (2.0 / N)
    c[..., 0] *= 0.5
    c[..., -1] *= 0.5
    return c


def _cheb_eval(coef, n):
    """Values at the n Gauss-Lobatto points of sum_k coef_k T_k."""
    N = n - 1
    j = np.arange(n)[:, None]
    k = np.arange(coef.shape[-1])[None, :]
    M = np.cos(np.pi * j * k / N)
    return coef @ M.T


def _ddy(a):
    """Coefficient-space derivative (standard recurrence)."""
    n = a.shape[-1]
    b = np.zeros_like(a)
    for k in range(n - 2, -1, -1):
        nxt = b[..., k + 2] if k + 2 < n else 0.0
        b[..., k] = nxt + 2.0 * (k + 1) * a[..., k + 1]
    b[..., 0] *= 0.5
    return b


def seeded_state(Nx, Ny, Nz, n_pi_x=4.0, n_pi_y=2.0, amplitude=0.05, seed=0):
    """Return (V, O) of shape (Nz, Nx//2+1, Ny) complex128.

    Nx, Nz are the streamwise / spanwise Fourier mode counts (the reference's
    nx, ny); Ny is the number of Chebyshev modes (the reference's nz).
    """
    Kx = Nx // 2 + 1
    nA = Ny - 4
    if nA < 1:
        raise ValueError("Ny must be at least 5")
    aphi = n_pi_x / 2.0
    beta = n_pi_y / 2.0
    rng = np.random.default_rng(seed)
    xi = rng.standard_normal((3, 2, Nz, Kx, nA))
    A = xi[:, 0] + 1j * xi[:, 1]
    kx = np.arange(Kx)
    kzi = np.arange(Nz)
    kz = np.where(kzi <= Nz // 2, kzi, kzi - Nz)
    amp = amplitude * np.exp(-(kx[None, :] ** 2 + kz[:, None] ** 2) / 8.0)
    A = A * amp[None, :, :, None] * (0.8 ** np.arange(nA))[None, None, None, :]
    # Hermitian symmetry on the kx = 0 plane
    for j in range(1, Nz // 2):
        A[:, Nz - j, 0, :] = np.conj(A[:, j, 0, :])
    A[:, 0, 0, :] = 0.0
    A[:, Nz // 2, :, :] = 0.0
    A[:, :, Kx - 1, :] = 0.0
    # Psi = (1 - y^2)^2 A, exact in Ny Chebyshev modes
    y = np.cos(np.pi * np.arange(Ny) / (Ny - 1))
    g = (1.0 - y * y) ** 2
    Psi = _dct1_coeffs(_cheb_eval(A, Ny) * g)
    DPsi = _ddy(Psi)
    alpha = (kx / aphi)[None, :, None]
    bet = (np.where(kzi <= Nz // 2, kzi, kzi - Nz) / beta)[:, None, None]
    k2 = alpha ** 2 + bet ** 2
    V = 1j * bet * Psi[0] - 1j * alpha * Psi[2]
    O = 1j * alpha * DPsi[0] + 1j * bet * DPsi[2] + k2 * Psi[1]
    # the reference keeps the kz Nyquist pencil as +Nz/2 (get_ialpha_ibeta)
    V[0, 0] = 0.0
    O[0, 0] = 0.0
    return V.astype(np.complex128), O.astype(np.complex128)
