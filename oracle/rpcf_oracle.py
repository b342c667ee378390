"""CPU oracle for the v-omega Fourier-Chebyshev DNS time step.

TEST INFRASTRUCTURE ONLY.  This module restates, in plain FP64 NumPy, the
algorithm of the reference (Riveryh/gpu-spectral-channel-DNS) for the hot
path: transforms, transposes, getUVW, Lamb vector, rhsNonlinear, the CN/AB2
right-hand sides, the per-mode solves and the step/bootstrap sequence.  It is
the checker for the CUDA implementation; nothing in the product imports it.
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use it.

Parity pin: the restatement is checked against the reference's own
known-answer tests (``tests/test_coef.cpp``, ``tests/test_transform.cpp``,
``tests/test_nonlinear.cpp``, ``tests/test_getUVW.cpp``,
``tests/test_transpose.cpp``) in ``tests/test_oracle_kat.py`` and against
fixtures produced by the reference built from its own sources
(``oracle/ref_build``) in ``tests/test_oracle_vs_reference.py``.

Array conventions (logical, unpitched versions of the reference layouts):

* spectral "ZXY" field  ``S[ky, kx, k]``  shape ``(ny, hnx, mz)`` complex;
  ``k`` is the wall-normal (Chebyshev) index; entries ``[0, nz)`` hold
  coefficients, ``[0, pz)`` physical values after a padded s2p.
* physical "XYZ" field  ``P[z, y, x]``  shape ``(pz, my, mx)`` real; ``z`` is
  the wall-normal point index, ``y`` the spanwise point, ``x`` streamwise.
* XYZ complex (between the transpose and the 2D FFT) ``C[z, ky', kx]`` shape
  ``(pz, my, mx//2+1)``.

Axis names follow the reference: x streamwise, y spanwise (Fourier), z
wall-normal (Chebyshev).  Reference ``w`` is the wall-normal velocity and
``omega_z`` the wall-normal vorticity.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

PI = 4.0 * math.atan(1.0)


# --------------------------------------------------------------------------
# sizes (include/data.h:312-328, source/data.cpp:3-13)
# --------------------------------------------------------------------------
@dataclass
class Sizes:
    mx: int
    my: int
    mz: int

    @property
    def nx(self):
        return self.mx // 3 * 2

    @property
    def ny(self):
        return self.my // 3 * 2

    @property
    def nz(self):
        return self.mz // 4 + 1

    @property
    def pz(self):
        return self.mz // 2 + 1

    @property
    def hnx(self):
        return self.nx // 2 + 1


# --------------------------------------------------------------------------
# Chebyshev operator tables (source/coefficient.cu:88-159)
# --------------------------------------------------------------------------
def get_T_matrix(N):
    """T0/T2/T4[i][j] = d^{0,2,4}T_j / dy^{0,2,4} at y_i = cos(pi i / N).

    Follows source/coefficient.cu:88-147: T0 from cos(), then the derivative
    recurrence T'_j = 2 j T_{j-1} + j T'_{j-2} / (j-2) applied to T1..T4 with
    columns 0..3 seeded as in the reference.
    """
    n1 = N + 1
    i = np.arange(n1, dtype=np.float64)[:, None]
    j = np.arange(n1, dtype=np.float64)[None, :]
    # same evaluation order as the reference: cos(j*PI*i/N)
    T0 = np.cos(j * PI * i / N)
    T1 = np.zeros((n1, n1))
    T2 = np.zeros((n1, n1))
    T3 = np.zeros((n1, n1))
    T4 = np.zeros((n1, n1))
    T1[:, 1] = T0[:, 0]
    T2[:, 2] = 4 * T0[:, 0]
    T1[:, 2] = 4 * T0[:, 1]
    for jj in range(3, n1):
        T1[:, jj] = 2 * jj * T0[:, jj - 1] + jj * T1[:, jj - 2] / (jj - 2)
        T2[:, jj] = 2 * jj * T1[:, jj - 1] + jj * T2[:, jj - 2] / (jj - 2)
        T3[:, jj] = 2 * jj * T2[:, jj - 1] + jj * T3[:, jj - 2] / (jj - 2)
        T4[:, jj] = 2 * jj * T3[:, jj - 1] + jj * T4[:, jj - 2] / (jj - 2)
    return T0, T2, T4


def base_profile(y, prof):
    """U, U', U'' of the base flow U(y) = a + b y + c y^2.

    The reference hard-codes plane Couette U = (1 + y)/2
    (source/coefficient.cu:149-159, source/nonlinear.cu:402-403); that is the
    default ``prof = (0.5, 0.5, 0.0)``.  Other profiles (U = y, Poiseuille
    U = 1 - y^2) are the same formulas with other coefficients.
    """
    a, b, c = prof
    y = np.asarray(y, dtype=np.float64)
    if (a, b, c) == (0.5, 0.5, 0.0):
        U = 0.5 * (1 + y)
    else:
        U = a + b * y + c * y * y
    dU = np.full_like(y, b) + 2 * c * y
    ddU = np.full_like(y, 2 * c)
    return U, dU, ddU


def get_U(nz, prof=(0.5, 0.5, 0.0)):
    """source/coefficient.cu:149-159: U at the nz collocation points."""
    i = np.arange(nz, dtype=np.float64)
    z = np.cos(i / (nz - 1) * PI)
    return base_profile(z, prof)


def ialpha_ibeta(kx, ky, ny, aphi, beta):
    """source/RPCFKernels.cu:522-532 (get_ialpha_ibeta)."""
    ia = np.asarray(kx, dtype=np.float64) / aphi
    kyf = np.asarray(ky, dtype=np.float64)
    ib = np.where(np.asarray(ky) >= ny // 2 + 1, (kyf - ny) / beta, kyf / beta)
    return ia, ib


def coef_v(N, U, ddU, T0, T2, T4, Re, dt, kmn, alpha):
    """source/coefficient.cu:7-37 (_get_coefficient_v)."""
    n1 = N + 1
    m = np.zeros((n1, n1), dtype=np.complex128)
    r = np.arange(4, n1)
    a = T0[r - 2]
    b = T2[r - 2]
    c = T4[r - 2]
    Ui = U[r - 2][:, None]
    ddUi = ddU[r - 2][:, None]
    m[4:].real = (-c * dt * 0.5 / Re + (1 + kmn * dt / Re) * b
                  - kmn * (1 + kmn * dt * 0.5 / Re) * a)
    m[4:].imag = (alpha * dt * Ui * 0.5 * b
                  - (kmn * alpha * dt * 0.5 * Ui + alpha * dt * 0.5 * ddUi) * a)
    j = np.arange(n1)
    m[0] = 1.0
    m[1] = np.where(j % 2 == 0, 1.0, -1.0)
    m[2] = (j * j).astype(np.float64)
    m[3] = np.where(j % 2 == 0, -1.0, 1.0) * j * j
    return m


def coef_omega(N, U, T0, T2, Re, dt, kmn, alpha):
    """source/coefficient.cu:39-64 (_get_coefficient_omega)."""
    n1 = N + 1
    m = np.zeros((n1, n1), dtype=np.complex128)
    r = np.arange(2, n1)
    a = T0[r - 1]
    b = T2[r - 1]
    Ui = U[r - 1][:, None]
    m[2:].real = -b * dt * 0.5 / Re + (1 + kmn * dt * 0.5 / Re) * a
    m[2:].imag = alpha * dt * 0.5 * Ui * a
    j = np.arange(n1)
    m[0] = 1.0
    m[1] = np.where(j % 2 == 0, 1.0, -1.0)
    return m


def coef_u0(N, T0, T2, Re, dt):
    """source/coefficient.cu:66-86 (_get_coef_u0 / _get_coef_w0)."""
    n1 = N + 1
    m = np.zeros((n1, n1), dtype=np.complex128)
    r = np.arange(2, n1)
    m[2:] = -T2[r - 1] * dt * 0.5 / Re + T0[r - 1]
    j = np.arange(n1)
    m[0] = 1.0
    m[1] = np.where(j % 2 == 0, 1.0, -1.0)
    return m


# --------------------------------------------------------------------------
# Chebyshev transforms along the pencil (source/transform.cu:416-748)
# --------------------------------------------------------------------------
def cheby_s2p(S, mz, pad=True):
    """Coefficients -> Gauss-Lobatto values, in place on the pencil.

    pad=True : cheby_pre_s2p_pad + Z2Z length mz (source/transform.cu:416-453,
               679-697); nz coefficients -> pz values at cos(pi j/(pz-1)).
    pad=False: cheby_pre_s2p_noPad + Z2Z length mz/2 (:455-491, :716-732);
               nz coefficients -> nz values at cos(pi j/(nz-1)).
    """
    S = np.array(S, copy=True)
    nzl = mz // 4  # max Chebyshev index (= nz - 1)
    if pad:
        e = np.zeros(S.shape[:-1] + (mz,), dtype=np.complex128)
        e[..., 0] = S[..., 0]
        e[..., 1:nzl + 1] = 0.5 * S[..., 1:nzl + 1]
        k = np.arange(1, nzl + 1)
        e[..., mz - k] = 0.5 * S[..., k]
        S[..., :mz] = np.fft.fft(e, axis=-1)
    else:
        L = mz // 2
        e = np.zeros(S.shape[:-1] + (L,), dtype=np.complex128)
        e[..., 0] = S[..., 0]
        e[..., 1:nzl] = 0.5 * S[..., 1:nzl]
        e[..., nzl] = S[..., nzl]
        k = np.arange(1, nzl)
        e[..., L - k] = 0.5 * S[..., k]
        S[..., :L] = np.fft.fft(e, axis=-1)
    return S


def cheby_p2s(S, mz, pad=True):
    """Gauss-Lobatto values -> coefficients (DCT-I), in place on the pencil.

    source/transform.cu:494-536 (pre/post kernels) and :538-658.
    pad=True : pz values -> pz coefficients (FFT length mz).
    pad=False: nz values -> nz coefficients (FFT length mz/2).
    """
    S = np.array(S, copy=True)
    L = mz if pad else mz // 2
    p = L // 2 + 1
    e = np.zeros(S.shape[:-1] + (L,), dtype=np.complex128)
    e[..., :p] = S[..., :p]
    j = np.arange(1, p - 1)
    e[..., L - j] = S[..., j]
    F = np.fft.fft(e, axis=-1)
    F[..., :p] *= 1.0 / (p - 1)
    F[..., 0] *= 0.5
    F[..., p - 1] *= 0.5
    S[..., :L] = F
    return S


def ddz(a):
    """Chebyshev coefficient derivative, source/RPCFKernels.cu:439-520.

    b_i = sum_{j = i+1, i+3, ...}^{N-1} 2 j a_j, then b_0 halved.
    """
    N = a.shape[-1]
    b = np.zeros_like(a)
    for i in range(N):
        js = np.arange(i + 1, N, 2)
        if js.size:
            b[..., i] = np.sum(a[..., js] * (2.0 * js), axis=-1)
    b[..., 0] *= 0.5
    return b


# --------------------------------------------------------------------------
# transpose / zero padding / 2D FFT (source/transpose.cu, transform.cu)
# --------------------------------------------------------------------------
def span_map(sz: Sizes):
    """ky -> padded span index ky' (source/transpose.cu:238-241)."""
    ky = np.arange(sz.ny)
    return np.where(ky > sz.ny // 2, ky + (sz.my - sz.ny), ky)


def transpose_forward(C, sz: Sizes):
    """XYZ complex C[z, ky', kx] -> ZXY S[ky, kx, k] (transpose.cu:223-257)."""
    S = np.zeros((sz.ny, sz.hnx, sz.mz), dtype=np.complex128)
    kyp = span_map(sz)
    # tu[ky][kx][kz] = u[kz][ky'][kx] for kz < pz
    S[:, :, :sz.pz] = np.transpose(C[:sz.pz][:, kyp, :sz.hnx], (1, 2, 0))
    return S


def transpose_backward(S, sz: Sizes, C=None):
    """ZXY -> XYZ complex (transpose.cu:358-382); untouched entries kept."""
    if C is None:
        C = np.zeros((sz.pz, sz.my, sz.mx // 2 + 1), dtype=np.complex128)
    kyp = span_map(sz)
    C[:sz.pz][:, kyp, :sz.hnx] = np.transpose(S[:, :, :sz.pz], (2, 0, 1))
    return C


def set_zeros(C, sz: Sizes):
    """source/transform.cu:355-377 (zero de-aliased and Nyquist modes)."""
    C = C.copy()
    kyp = np.arange(sz.my)
    band = (kyp >= sz.ny // 2) & (kyp <= sz.my - sz.ny // 2)
    C[:, band, :] = 0.0
    C[:, ~band, sz.nx // 2:] = 0.0
    return C


def c2r_2d(C, sz: Sizes):
    """Unnormalised 2D inverse real FFT per wall-normal plane (cuFFT Z2D)."""
    return np.fft.irfft2(C, s=(sz.my, sz.mx), axes=(-2, -1)) * (sz.my * sz.mx)


def r2c_2d(P, sz: Sizes):
    """2D forward real FFT then x1/(mx*my) (cuFFT D2Z + normalizeKernel)."""
    return np.fft.rfft2(P, axes=(-2, -1)) * (1.0 / sz.mx / sz.my)


def transform_backward(S, sz: Sizes, pad=True):
    """transform_3d_one(BACKWARD) source/transform.cu:124-210."""
    S2 = cheby_s2p(S, sz.mz, pad)
    C = transpose_backward(S2, sz)
    C = set_zeros(C, sz)
    return c2r_2d(C, sz)


def transform_forward(P, sz: Sizes, pad=True):
    """transform_3d_one(FORWARD) source/transform.cu:211-315."""
    C = r2c_2d(P, sz)
    S = transpose_forward(C, sz)
    return cheby_p2s(S, sz.mz, pad)


# --------------------------------------------------------------------------
# getUVW (source/velocity.cu:90-170)
# --------------------------------------------------------------------------
def get_uvw(tw, toz, sz: Sizes, aphi, beta):
    """Recover (u, v, w, ox, oy, oz) coefficient fields from w and omega_z.

    Inputs are ZXY fields; only coefficients [0, nz) are read and written.
    Returns six ZXY arrays of shape (ny, hnx, nz).
    """
    nz = sz.nz
    w = tw[:, :, :nz].copy()
    oz = toz[:, :, :nz].copy()
    kx = np.arange(sz.hnx)[None, :]
    ky = np.arange(sz.ny)[:, None]
    ia, ib = ialpha_ibeta(kx, ky, sz.ny, aphi, beta)
    ia = np.broadcast_to(ia, (sz.ny, sz.hnx))
    ib = np.broadcast_to(ib, (sz.ny, sz.hnx))
    kmn = ia * ia + ib * ib
    with np.errstate(divide="ignore", invalid="ignore"):
        kmn1 = np.where(kmn > 0, 1.0 / kmn, 0.0)
    Dw = ddz(w)
    c_a = (1j * (ia * kmn1))[..., None]
    c_b = (1j * (ib * kmn1))[..., None]
    u = c_a * Dw - c_b * oz
    v = c_b * Dw + c_a * oz
    ox = ddz(v) + (-1j * ib)[..., None] * w
    oy = -ddz(u) + (1j * ia)[..., None] * w
    oz_out = oz.copy()
    w_out = w.copy()
    # zero wave number (velocity.cu:106-124)
    u[0, 0] = w[0, 0]
    v[0, 0] = oz[0, 0]
    w_out[0, 0] = 0.0
    ox[0, 0] = ddz(v[0, 0])
    oy[0, 0] = -ddz(u[0, 0])
    oz_out[0, 0] = 0.0
    return u, v, w_out, ox, oy, oz_out


def get_uvw_pencils(w, oz, ky, kx, sz: Sizes, aphi, beta):
    """get_uvw on a list of pencils: w, oz of shape (P, nz) at (ky[p], kx[p]).

    The same formulas as get_uvw (source/velocity.cu:90-170), pencil by
    pencil, for checks on a sample of the pencils of a large grid.
    """
    w = np.asarray(w, dtype=np.complex128)
    oz = np.asarray(oz, dtype=np.complex128)
    ky = np.asarray(ky)
    kx = np.asarray(kx)
    ia, ib = ialpha_ibeta(kx, ky, sz.ny, aphi, beta)
    kmn = ia * ia + ib * ib
    with np.errstate(divide="ignore", invalid="ignore"):
        kmn1 = np.where(kmn > 0, 1.0 / kmn, 0.0)
    Dw = ddz(w)
    c_a = (1j * (ia * kmn1))[:, None]
    c_b = (1j * (ib * kmn1))[:, None]
    u = c_a * Dw - c_b * oz
    v = c_b * Dw + c_a * oz
    ox = ddz(v) + (-1j * ib)[:, None] * w
    oy = -ddz(u) + (1j * ia)[:, None] * w
    w_out = w.copy()
    oz_out = oz.copy()
    m = (kx == 0) & (ky == 0)
    if m.any():
        u[m] = w[m]
        v[m] = oz[m]
        w_out[m] = 0.0
        ox[m] = ddz(v[m])
        oy[m] = -ddz(u[m])
        oz_out[m] = 0.0
    return u, v, w_out, ox, oy, oz_out


# --------------------------------------------------------------------------
# Lamb vector and rhsNonlinear (source/nonlinear.cu:146-242, 366-428)
# --------------------------------------------------------------------------
def lamb(u, v, w, ox, oy, oz, sz: Sizes, Ro, prof=(0.5, 0.5, 0.0)):
    k = np.arange(sz.pz, dtype=np.float64)
    y = np.cos(k / (sz.pz - 1) * PI)
    meanU = base_profile(y, prof)[0][:, None, None]
    lx = oz * v - oy * w - Ro * w
    ly = ox * w - oz * u
    lz = oy * u - ox * v + Ro * (u + meanU)
    return lx, ly, lz


def rhs_nonlinear(tlx, tly, tlz, sz: Sizes, aphi, beta):
    """Returns (H_v, H_omega) pencils of length nz; (0,0) keeps raw lambda."""
    nz = sz.nz
    lx = tlx[:, :, :nz]
    ly = tly[:, :, :nz]
    lz = tlz[:, :, :nz]
    kx = np.arange(sz.hnx)[None, :]
    ky = np.arange(sz.ny)[:, None]
    ia, ib = ialpha_ibeta(kx, ky, sz.ny, aphi, beta)
    ia = np.broadcast_to(ia, (sz.ny, sz.hnx))[..., None]
    ib = np.broadcast_to(ib, (sz.ny, sz.hnx))[..., None]
    kmn = ia * ia + ib * ib
    Dlx = ddz(lx)
    Dly = ddz(ly)
    hv = kmn * lz + 1j * ia * Dlx + 1j * ib * Dly
    ho = 1j * ia * ly - 1j * ib * lx
    hv[0, 0] = lx[0, 0]
    ho[0, 0] = ly[0, 0]
    return hv, ho


# --------------------------------------------------------------------------
# analytic initial condition (initFlow, source/RPCFKernels.cu:358-431)
# --------------------------------------------------------------------------
EPSILON_INIT = 0.005  # source/RPCFKernels.cu:132


def init_fields(sz: Sizes, aphi, beta):
    """init_flow_kernel (source/RPCFKernels.cu:311-356) for the two fields
    that enter the state: w (:182-194) and omega_z (:212-223).

    Points: x = i/px*lx, y = j/py*ly (lx = 2 pi aphi, ly = 2 pi beta,
    source/data.cpp:5-6), z = cos(pi k/(nz-1)) for the nz planes k, both
    fields zero on the wall planes k = 0, nz-1.  Returns two XYZ arrays of
    shape (pz, my, mx); planes nz..pz-1 are zero (not read by the no-padding
    transform).
    """
    lx = 2 * PI * aphi
    ly = 2 * PI * beta
    nz = sz.nz
    xx = (np.arange(sz.mx) * 1.0) / sz.mx * lx
    yy = (np.arange(sz.my) * 1.0) / sz.my * ly
    zz = np.cos(PI * np.arange(nz) / (nz - 1))
    z, y, x = np.meshgrid(zz, yy, xx, indexing="ij")
    e = EPSILON_INIT
    sa1, sa2 = np.sin(2 * PI * x / lx), np.sin(4.0 * PI * x / lx)
    ca1, ca2 = np.cos(2 * PI * x / lx), np.cos(4.0 * PI * x / lx)
    sb1, sb2 = np.sin(2 * PI * y / ly), np.sin(4 * PI * y / ly)
    cb1, cb2 = np.cos(2.0 * PI * y / ly), np.cos(4.0 * PI * y / ly)
    w = e * (-2.0 / 3.0) * (1.0 + np.cos(1.5 * PI * z)) * (sa1 * sb1 + sa2 * sb1 + sa1 * sb2)
    oz = e * 2.0 * PI * np.sin(1.5 * PI * z) * (
        lx / ly * (ca1 * cb1 + 0.5 * ca2 * cb1 + 2.0 * ca1 * cb2)
        + ly / lx * (0.5 * ca1 * cb1 + ca2 * cb1 + 0.25 * ca1 * cb2))
    W = np.zeros((sz.pz, sz.my, sz.mx))
    OZ = np.zeros_like(W)
    W[1:nz - 1] = w[1:nz - 1]
    OZ[1:nz - 1] = oz[1:nz - 1]
    return W, OZ


def init_state(sz: Sizes, aphi, beta):
    """initFlow's state: the no-padding forward transforms of w and omega_z
    (source/RPCFKernels.cu:397-406), copied to rhs_v / rhs_omega_y.
    Returns (V, O), each (ny, hnx, nz) complex."""
    W, OZ = init_fields(sz, aphi, beta)
    V = transform_forward(W, sz, pad=False)[..., :sz.nz]
    O = transform_forward(OZ, sz, pad=False)[..., :sz.nz]
    return V, O


# --------------------------------------------------------------------------
# full problem / time step
# --------------------------------------------------------------------------
@dataclass
class Params:
    mx: int
    my: int
    mz: int
    n_pi_x: float = 4.0
    n_pi_y: float = 2.0
    Re: float = 1300.0
    Ro: float = 0.0
    dt: float = 0.005
    prof: tuple = (0.5, 0.5, 0.0)


@dataclass
class Problem:
    """State and step of the reference's solver, restated in NumPy.

    State between steps (source/solver.cpp:35-101, source/rhs.cpp):
      V[ky,kx,:nz]   v-hat (reference rhs_v); pencil (0,0) holds u0.
      O[ky,kx,:nz]   omega_y-hat (reference rhs_omega_y); (0,0) holds w0.
      Nv_p, No_p     previous-step nonlinear terms at the nz collocation
                     points (reference nonlinear_v_p, nonlinear_omega_y_p).
      lx0_p, lz0_p   previous-step mean-mode lambda (lambx0_p, lambz0_p).
    """
    p: Params
    sz: Sizes = field(init=False)

    def __post_init__(self):
        p = self.p
        self.sz = Sizes(p.mx, p.my, p.mz)
        sz = self.sz
        self.aphi = p.n_pi_x / 2
        self.beta = p.n_pi_y / 2
        N = sz.nz - 1
        self.T0, self.T2, self.T4 = get_T_matrix(N)
        self.U, self.dU, self.ddU = get_U(sz.nz, p.prof)
        kx = np.arange(sz.hnx)[None, :]
        ky = np.arange(sz.ny)[:, None]
        ia, ib = ialpha_ibeta(kx, ky, sz.ny, self.aphi, self.beta)
        self.ia = np.broadcast_to(ia, (sz.ny, sz.hnx)).copy()
        self.ib = np.broadcast_to(ib, (sz.ny, sz.hnx)).copy()
        self.kmn = self.ia ** 2 + self.ib ** 2
        self._inv_v = None
        self._inv_o = None
        self.solver = "inverse"

    # -- operators (source/solver.cpp:260-320) -----------------------------
    def operators(self, ky, kx):
        """The v and omega collocation matrices of pencils (ky[i], kx[i]).

        source/solver.cpp:275-313: pencil (0,0) carries the mean-mode
        operator (_get_coef_u0 = _get_coef_w0) in both slots.
        """
        sz, p = self.sz, self.p
        N = sz.nz - 1
        n = len(ky)
        Av = np.zeros((n, sz.nz, sz.nz), dtype=np.complex128)
        Ao = np.zeros_like(Av)
        for i, (y, x) in enumerate(zip(ky, kx)):
            if x == 0 and y == 0:
                Av[i] = coef_u0(N, self.T0, self.T2, p.Re, p.dt)
                Ao[i] = Av[i]
                continue
            Av[i] = coef_v(N, self.U, self.ddU, self.T0, self.T2, self.T4, p.Re, p.dt,
                           self.kmn[y, x], self.ia[y, x])
            Ao[i] = coef_omega(N, self.U, self.T0, self.T2, p.Re, p.dt, self.kmn[y, x],
                               self.ia[y, x])
        return Av, Ao

    def build_inverses(self):
        sz = self.sz
        ky, kx = np.meshgrid(np.arange(sz.ny), np.arange(sz.hnx), indexing="ij")
        Av, Ao = self.operators(ky.ravel(), kx.ravel())
        shape = (sz.ny, sz.hnx, sz.nz, sz.nz)
        self.A_v, self.A_o = Av.reshape(shape), Ao.reshape(shape)
        self._inv_v = np.linalg.inv(self.A_v)
        self._inv_o = np.linalg.inv(self.A_o)

    @property
    def inv_v(self):
        if self._inv_v is None:
            self.build_inverses()
        return self._inv_v

    @property
    def inv_o(self):
        if self._inv_o is None:
            self.build_inverses()
        return self._inv_o

    def solve(self, which, rhs):
        """solveEq (source/solver.cpp:107-123) on every pencil of ``rhs``.

        ``solver`` selects how: "inverse" multiplies by the stored explicit
        inverses, as the reference does (source/matrix_op.cpp:68-78);
        "lu" solves the stored matrices by LU with partial pivoting;
        "batched" / "batched-lu" form the matrices a block of pencils at a
        time without keeping them and invert / LU-solve them (the
        arithmetic of "inverse" / "lu" for grids whose 2 H Ny^2 matrix
        entries do not fit in memory).  The spread
        between "inverse" and "lu" is the oracle's own rounding floor.
        """
        if self.solver == "inverse":
            inv = self.inv_v if which == "v" else self.inv_o
            return np.einsum("yxij,yxj->yxi", inv, rhs)
        if self.solver == "lu":
            if self._inv_v is None and getattr(self, "A_v", None) is None:
                self.build_inverses()
            A = self.A_v if which == "v" else self.A_o
            return np.linalg.solve(A, rhs[..., None])[..., 0]
        if self.solver not in ("batched", "batched-lu"):
            raise ValueError("solver must be inverse, lu, batched or batched-lu")
        sz = self.sz
        ky, kx = np.meshgrid(np.arange(sz.ny), np.arange(sz.hnx), indexing="ij")
        ky, kx = ky.ravel(), kx.ravel()
        flat = rhs.reshape(-1, sz.nz)
        out = np.empty_like(flat)
        blk = max(1, (1 << 25) // (sz.nz * sz.nz))
        for a in range(0, len(ky), blk):
            Av, Ao = self.operators(ky[a:a + blk], kx[a:a + blk])
            A = Av if which == "v" else Ao
            if self.solver == "batched":
                out[a:a + blk] = np.einsum("pij,pj->pi", np.linalg.inv(A), flat[a:a + blk])
            else:
                out[a:a + blk] = np.linalg.solve(A, flat[a:a + blk, :, None])[..., 0]
        return out.reshape(rhs.shape)

    # -- state -------------------------------------------------------------
    def set_state(self, V, O):
        """V, O: (ny, hnx, nz) complex; pencil (0,0) carries u0 / w0."""
        self.V = np.array(V, dtype=np.complex128)
        self.O = np.array(O, dtype=np.complex128)
        self.Nv_p = None
        self.No_p = None
        self.lx0_p = None
        self.lz0_p = None

    def spectral_fields(self):
        """getUVW on the current state: six (ny, hnx, nz) arrays."""
        sz = self.sz
        tw = np.zeros((sz.ny, sz.hnx, sz.mz), dtype=np.complex128)
        toz = np.zeros_like(tw)
        tw[:, :, :sz.nz] = self.V
        toz[:, :, :sz.nz] = self.O
        return get_uvw(tw, toz, sz, self.aphi, self.beta)

    def physical_fields(self, fields=None):
        sz = self.sz
        if fields is None:
            fields = self.spectral_fields()
        out = []
        for f in fields:
            S = np.zeros((sz.ny, sz.hnx, sz.mz), dtype=np.complex128)
            S[:, :, :sz.nz] = f
            out.append(transform_backward(S, sz, pad=True))
        return out

    def nonlinear(self):
        """getNonlinear + worker post-processing (rhs.cpp:83-127).

        Returns (Nv, No) at the nz collocation points for every pencil;
        pencil (0,0) holds raw lambda_x / lambda_y(span) values.
        """
        sz, p = self.sz, self.p
        u, v, w, ox, oy, oz = self.physical_fields()
        lx, ly, lz = lamb(u, v, w, ox, oy, oz, sz, p.Ro, p.prof)
        tlz = transform_forward(lz, sz, pad=True)
        tly = transform_forward(ly, sz, pad=True)
        tlx = transform_forward(lx, sz, pad=True)
        hv, ho = rhs_nonlinear(tlx, tly, tlz, sz, self.aphi, self.beta)
        Hv = np.zeros((sz.ny, sz.hnx, sz.mz), dtype=np.complex128)
        Ho = np.zeros_like(Hv)
        Hv[:, :, :sz.nz] = hv
        Ho[:, :, :sz.nz] = ho
        Nv = cheby_s2p(Hv, sz.mz, pad=False)[:, :, :sz.nz]
        No = cheby_s2p(Ho, sz.mz, pad=False)[:, :, :sz.nz]
        return Nv, No

    def bootstrap(self):
        """The "extra previous step" of source/main_loop.cpp:39-52.

        Its only lasting effect is that the AB2 history of the first real
        step equals the nonlinear term of the initial field.
        """
        Nv, No = self.nonlinear()
        self.Nv_p, self.No_p = Nv, No
        self.lx0_p = Nv[0, 0].copy()
        self.lz0_p = No[0, 0].copy()

    def linear_v(self, V):
        """_get_linear_v (linear.cpp:86-125) for all pencils; rows 4..N."""
        p = self.p
        nz = self.sz.nz
        dt, Re = p.dt, p.Re
        kmn = self.kmn[..., None]
        ia = self.ia[..., None]
        r = np.arange(4, nz)
        T0 = self.T0[r - 2]
        T2 = self.T2[r - 2]
        T4 = self.T4[r - 2]
        Ui = self.U[r - 2]
        ddUi = self.ddU[r - 2]
        P0 = V @ T0.T
        P2 = V @ T2.T
        P4 = V @ T4.T
        re = (P4 * dt * 0.5 / Re + (1 - kmn * dt / Re) * P2
              - kmn * (1 - kmn * dt * 0.5 / Re) * P0)
        im = (-ia * dt * 0.5 * Ui * P2
              + (kmn * ia * dt * 0.5 * Ui + ia * dt * 0.5 * ddUi) * P0)
        out = np.zeros_like(V)
        out[..., 4:] = re + 1j * im
        return out

    def linear_omega(self, O, Vnew, Vold):
        """_get_linear_omega_y (linear.cpp:127-171) rows 2..N, no AB2."""
        p = self.p
        nz = self.sz.nz
        dt, Re = p.dt, p.Re
        kmn = self.kmn[..., None]
        ia = self.ia[..., None]
        ib = self.ib[..., None]
        r = np.arange(2, nz)
        T0 = self.T0[r - 1]
        T2 = self.T2[r - 1]
        Ui = self.U[r - 1]
        dUi = self.dU[r - 1]
        Q0 = O @ T0.T
        Q2 = O @ T2.T
        S0 = (Vold + Vnew) @ T0.T
        out = np.zeros_like(O)
        out[..., 2:] = (Q2 * 0.5 / Re * dt + (1 - kmn * dt * 0.5 / Re) * Q0
                        + 1j * (-ia * dt * 0.5 * Ui * Q0)
                        + 1j * (-0.5 * ib * dUi * dt) * S0)
        return out

    def linear_u0(self, u0, l0, l0_p):
        """_get_linear_u0 (linear.cpp:173-200)."""
        p = self.p
        nz = self.sz.nz
        r = np.arange(2, nz)
        M = self.T0[r - 1] + p.dt * 0.5 / p.Re * self.T2[r - 1]
        out = np.zeros_like(u0)
        out[2:] = M @ u0 - (l0[r - 1] * 1.5 - l0_p[r - 1] * 0.5) * p.dt
        return out

    def step(self):
        """One nextStep (source/solver.cpp:35-101)."""
        p = self.p
        nz = self.sz.nz
        dt = p.dt
        if self.Nv_p is None:
            raise RuntimeError("call bootstrap() before the first step")
        Nv, No = self.nonlinear()
        lx0 = Nv[0, 0].copy()
        lz0 = No[0, 0].copy()
        Vold = self.V.copy()
        # get_rhs_v (rhs.cpp:185-219)
        rv = self.linear_v(self.V)
        k = np.arange(4, nz)
        rv[..., 4:] += (Nv[..., k - 2] * 1.5 - self.Nv_p[..., k - 2] * 0.5) * dt
        rv[0, 0] = self.linear_u0(self.V[0, 0], lx0, self.lx0_p)
        ro00 = self.linear_u0(self.O[0, 0], lz0, self.lz0_p)
        # solveEq v (solver.cpp:107-123)
        Vnew = self.solve("v", rv)
        # get_rhs_omega (linear.cpp:52-84)
        ro = self.linear_omega(self.O, Vnew, Vold)
        i = np.arange(2, nz)
        ro[..., 2:] += (No[..., i - 1] * 1.5 - self.No_p[..., i - 1] * 0.5) * dt
        ro[0, 0] = ro00
        Onew = self.solve("o", ro)
        self.V, self.O = Vnew, Onew
        self.Nv_p, self.No_p = Nv, No
        self.lx0_p, self.lz0_p = lx0, lz0
        self.last_rhs_v, self.last_rhs_o = rv, ro
