"""Physical validation cases shared by the oracle (CPU) and device tests.

* laminar base flow: a zero perturbation stays zero (plane Couette with
  rotation, plane Poiseuille);
* mean-mode Crank-Nicolson decay: u0 = cos(pi y / 2) and w0 = cos(3 pi y / 2)
  decay by the Crank-Nicolson factor (1 - a) / (1 + a), a = k^2 dt / (2 Re),
  of the diffusion equation (their Lamb vector is wall-normal, so nothing
  drives them);
* Orr-Sommerfeld: the unstable Tollmien-Schlichting mode of plane Poiseuille
  flow at Re = 10^4, alpha = 1, c = 0.23752649 + 0.00373967i (Orszag 1971),
  seeded at amplitude 1e-8 in pencil (kz, kx) = (0, 1) with Lx = 2 pi, grows
  at the rate alpha c_i.  The eigenvalue problem
      (D^2 - a^2)^2 v - i a Re [U (D^2 - a^2) - U''] v = -i a Re c (D^2 - a^2) v,
      v(+-1) = v'(+-1) = 0,
  is solved here by Chebyshev collocation at the points the reference's v
  equation uses (y_2..y_{N-2}) plus the four wall rows.
"""
import numpy as np
import scipy.linalg as sl

from oracle import rpcf_oracle as O

ORSZAG_C = 0.23752649 + 0.00373967j
OS_N, OS_RE, OS_DT, OS_STEPS, OS_EPS = 64, 1.0e4, 0.02, 250, 1e-8
OS_GRID = (24, 24, 4 * OS_N)  # mx, my, mz: Nx = Nz = 16, Ny = 65
POISEUILLE = (1.0, 0.0, -1.0)


def os_mode(N=OS_N, Re=OS_RE, alpha=1.0, prof=POISEUILLE):
    """(c, Chebyshev coefficients of v, unit norm) of the least stable mode."""
    T0, T2, T4 = O.get_T_matrix(N)
    U, _, ddU = O.get_U(N + 1, prof)
    k2 = alpha * alpha
    r = np.arange(2, N - 1)
    L2 = T2[r] - k2 * T0[r]
    L4 = T4[r] - 2 * k2 * T2[r] + k2 * k2 * T0[r]
    A = np.zeros((N + 1, N + 1), dtype=np.complex128)
    B = np.zeros_like(A)
    A[4:] = L4 - 1j * alpha * Re * (U[r, None] * L2 - ddU[r, None] * T0[r])
    B[4:] = -1j * alpha * Re * L2
    j = np.arange(N + 1)
    A[0] = 1.0
    A[1] = np.where(j % 2 == 0, 1.0, -1.0)
    A[2] = j * j
    A[3] = np.where(j % 2 == 0, -1.0, 1.0) * j * j
    w, V = sl.eig(A, B)
    ok = np.isfinite(w) & (np.abs(w) < 10)
    i = int(np.argmax(np.where(ok, w.imag, -np.inf)))
    a = V[:, i]
    return w[i], a / np.linalg.norm(a)


def os_state(sz, a, eps=OS_EPS):
    V = np.zeros((sz.ny, sz.hnx, sz.nz), dtype=np.complex128)
    V[0, 1, :] = eps * a
    return V, np.zeros_like(V)


def os_rate(V, a, eps=OS_EPS, steps=OS_STEPS, dt=OS_DT):
    """d/dt log of the mode's amplitude: alpha c_i - i alpha c_r."""
    return np.log(np.vdot(a, V[0, 1, :]) / eps) / (steps * dt)


def cn_rate(c, dt=OS_DT, alpha=1.0):
    """The same rate for the Crank-Nicolson step of d/dt = -i alpha c."""
    z = -1j * alpha * c * dt / 2
    return np.log((1 + z) / (1 - z)) / dt


def gl_coeffs(f):
    """Chebyshev coefficients of the interpolant of values f at y_j = cos(pi j / N)."""
    N = len(f) - 1
    k = np.arange(N + 1)
    c = np.where((k == 0) | (k == N), 2.0, 1.0)
    return (2.0 / N) / c * (np.cos(np.pi * np.outer(k, k) / N) @ (f / c))


MEAN_N, MEAN_RE, MEAN_DT, MEAN_STEPS = 32, 1300.0, 0.005, 50


def mean_state(sz):
    y = np.cos(np.pi * np.arange(sz.nz) / (sz.nz - 1))
    V = np.zeros((sz.ny, sz.hnx, sz.nz), dtype=np.complex128)
    Om = np.zeros_like(V)
    V[0, 0] = gl_coeffs(np.cos(np.pi * y / 2))
    Om[0, 0] = gl_coeffs(np.cos(3 * np.pi * y / 2))
    return V, Om


def mean_decay_errors(V0, O0, V, Om, Re=MEAN_RE, dt=MEAN_DT, steps=MEAN_STEPS):
    out = []
    for k2, a0, a1 in (((np.pi / 2) ** 2, V0[0, 0], V[0, 0]), ((3 * np.pi / 2) ** 2, O0[0, 0], Om[0, 0])):
        a = k2 * dt / (2 * Re)
        g = (1 - a) / (1 + a)
        out.append(np.linalg.norm(a1 - g ** steps * a0) / np.linalg.norm(a0))
    return out
