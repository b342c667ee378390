"""Pin the CPU oracle to the reference's own known-answer tests.

Each test restates one check of the reference's ``tests/`` directory (those
tests are not compiled by the reference's build, so their analytic fields are
re-derived here) and runs it against ``oracle/rpcf_oracle.py`` at a tolerance
far tighter than the reference's ``isEqual`` (1e-8 abs or 1e-4 rel,
source/operation.cpp:98-111).
"""
import math

import numpy as np
import pytest

from oracle import rpcf_oracle as O

SIZES = [(48, 48, 128), (24, 24, 32), (36, 48, 64)]


def grid(sz, lx, ly, npts=None):
    pz = sz.pz if npts is None else npts
    k = np.arange(pz)
    z = np.cos(k / (pz - 1) * O.PI)[:, None, None]
    y = (ly * np.arange(sz.my) / sz.my)[None, :, None]
    x = (lx * np.arange(sz.mx) / sz.mx)[None, None, :]
    return x, y, z


def test_T_matrix_known_values():
    """tests/test_coef.cpp:8-32."""
    T0, T2, T4 = O.get_T_matrix(100)
    assert T4[16, 100] / 1e9 == pytest.approx(1.846564249235145, rel=1e-12)
    assert T4[42, 95] / 1e7 == pytest.approx(8.842927487588026, rel=1e-12)
    assert T4[0, 4] == pytest.approx(192.0, rel=1e-14)
    assert T4[100, 5] == pytest.approx(-1920.0, rel=1e-14)
    assert np.all(T4[:, :4] == 0.0)
    # T0/T2 are exact Chebyshev values/second derivatives at the points
    y = np.cos(np.pi * np.arange(101) / 100)
    assert np.allclose(T0[:, 3], 4 * y ** 3 - 3 * y, atol=1e-13)
    assert np.allclose(T2[:, 3], 24 * y, atol=1e-11)


@pytest.mark.parametrize("mx,my,mz", SIZES)
def test_transform_round_trip(mx, my, mz):
    """tests/test_transform.cpp:13-151, 218-255 (padded and no-pad)."""
    sz = O.Sizes(mx, my, mz)
    lx, ly = 2 * O.PI * 2.0, 2 * O.PI * 1.0
    x, y, z = grid(sz, lx, ly)
    u = (1 - z * z) * np.sin(y) * np.cos(x)
    oy = -2 * z * np.sin(y) * np.cos(x)
    oz = -(1 - z * z) * np.cos(y) * np.cos(x)
    for f in (u, oy, oz):
        S = O.transform_forward(f, sz, pad=True)
        back = O.transform_backward(S, sz, pad=True)
        assert np.max(np.abs(back - f)) < 1e-12
        # padded forward then no-pad backward: values on the nz points
        back_np = O.transform_backward(S, sz, pad=False)
        x2, y2, z2 = grid(sz, lx, ly, npts=sz.nz)
        if f is u:
            ex = (1 - z2 * z2) * np.sin(y2) * np.cos(x2)
        elif f is oy:
            ex = -2 * z2 * np.sin(y2) * np.cos(x2)
        else:
            ex = -(1 - z2 * z2) * np.cos(y2) * np.cos(x2)
        assert np.max(np.abs(back_np[:sz.nz] - ex)) < 1e-12


def test_spectra_of_parabola():
    """tests/test_transform.cpp:154-190: 1 - z^2 = 0.5 T0 - 0.5 T2."""
    sz = O.Sizes(48, 48, 128)
    x, y, z = grid(sz, 4 * O.PI, 2 * O.PI)
    f = np.broadcast_to(1 - z * z, (sz.pz, sz.my, sz.mx)).copy()
    S = O.transform_forward(f, sz, pad=True)
    ex = np.zeros((sz.ny, sz.hnx, sz.pz), dtype=complex)
    ex[0, 0, 0] = 0.5
    ex[0, 0, 2] = -0.5
    assert np.max(np.abs(S[:, :, :sz.pz] - ex)) < 1e-14


def test_transpose_index_tags():
    """tests/test_transpose.cpp:8-90: tags 100 i + j + 0.01 k survive."""
    sz = O.Sizes(48, 48, 128)
    C = np.zeros((sz.pz, sz.my, sz.mx // 2 + 1), dtype=complex)
    kyp = O.span_map(sz)
    for j in range(sz.ny):
        for i in range(sz.hnx):
            C[:, kyp[j], i] = 100 * i + j + 0.01 * np.arange(sz.pz)
    S = O.transpose_forward(C, sz)
    i = np.arange(sz.hnx)[None, :, None]
    j = np.arange(sz.ny)[:, None, None]
    k = np.arange(sz.pz)[None, None, :]
    assert np.array_equal(S[:, :, :sz.pz].real, (100 * i + j + 0.01 * k) * np.ones_like(S[:, :, :sz.pz].real))
    C2 = O.transpose_backward(S, sz)
    assert np.array_equal(C2[:, kyp, :sz.hnx], C[:, kyp, :sz.hnx])


def test_lamb_closed_form():
    """tests/test_nonlinear.cpp:103-143, 188-225 (Ro = 0)."""
    sz = O.Sizes(48, 48, 128)
    x, y, z = grid(sz, 4 * O.PI, 2 * O.PI)
    shp = (sz.pz, sz.my, sz.mx)
    u = np.broadcast_to((1 - z * z) * np.sin(y) * np.cos(x), shp)
    zero = np.zeros(shp)
    oy = np.broadcast_to(-2 * z * np.sin(y) * np.cos(x), shp)
    oz = np.broadcast_to(-(1 - z * z) * np.cos(y) * np.cos(x), shp)
    lx, ly, lz = O.lamb(u, zero, zero, zero, oy, oz, sz, Ro=0.0)
    assert np.max(np.abs(lx)) == 0.0
    ex_ly = (1 - z * z) ** 2 * np.cos(y) * np.sin(y) * np.cos(x) ** 2
    ex_lz = -2.0 * z * (1 - z * z) * np.sin(y) ** 2 * np.cos(x) ** 2
    assert np.max(np.abs(ly - ex_ly)) < 1e-15
    assert np.max(np.abs(lz - ex_lz)) < 1e-15


def test_rhs_nonlinear_closed_form():
    """tests/test_nonlinear.cpp:527-603 (check_nonlinear_complex)."""
    sz = O.Sizes(48, 48, 128)
    aphi, beta = 2.0, 1.0
    x, y, z = grid(sz, 2 * O.PI * aphi, 2 * O.PI * beta)
    shp = (sz.pz, sz.my, sz.mx)
    u = np.broadcast_to((1 - z * z) * np.sin(y) * np.cos(x), shp)
    zero = np.zeros(shp)
    oy = np.broadcast_to(-2 * z * np.sin(y) * np.cos(x), shp)
    oz = np.broadcast_to(-(1 - z * z) * np.cos(y) * np.cos(x), shp)
    lx, ly, lz = O.lamb(u, zero, zero, zero, oy, oz, sz, Ro=0.0)
    tlz = O.transform_forward(lz, sz)
    tly = O.transform_forward(ly, sz)
    tlx = O.transform_forward(lx, sz)
    hv, ho = O.rhs_nonlinear(tlx, tly, tlz, sz, aphi, beta)
    Sv = tlx.copy()
    So = tly.copy()
    Sv[:, :, :sz.nz] = hv
    So[:, :, :sz.nz] = ho
    pv = O.transform_backward(Sv, sz)
    po = O.transform_backward(So, sz)
    ex_v = (-(1 - z * z) * (2 * z) * (np.cos(2 * x) - np.cos(2 * y)
                                      - 2 * np.cos(2 * y) * np.cos(2 * x))
            + 2 * (1 - z * z) * (-2 * z) * np.cos(2 * y) * np.cos(x) ** 2)
    ex_o = -(1 - z * z) ** 2 * np.cos(y) * np.sin(y) * 2 * np.cos(x) * np.sin(x)
    assert np.max(np.abs(pv - ex_v)) < 1e-11
    assert np.max(np.abs(po - ex_o)) < 1e-11


def test_get_uvw_closed_form():
    """tests/test_getUVW.cpp:15-206."""
    sz = O.Sizes(48, 48, 128)
    aphi, beta = 2.0, 1.0
    x, y, z = grid(sz, 2 * O.PI * aphi, 2 * O.PI * beta)
    shp = (sz.pz, sz.my, sz.mx)
    ex = {
        "u": np.sin(x) + 0 * y * z,
        "v": np.cos(y) + 0 * x * z,
        "w": -z * np.cos(x) + z * np.sin(y),
        "ox": -z * np.cos(y) + 0 * x,
        "oy": z * np.sin(x) + 0 * y,
        "oz": np.zeros(shp),
    }
    ex = {k: np.broadcast_to(v, shp) for k, v in ex.items()}
    tw = O.transform_forward(ex["w"], sz)
    toz = O.transform_forward(ex["oz"], sz)
    fields = O.get_uvw(tw, toz, sz, aphi, beta)
    for name, f in zip(["u", "v", "w", "ox", "oy", "oz"], fields):
        S = np.zeros((sz.ny, sz.hnx, sz.mz), dtype=complex)
        S[:, :, :sz.nz] = f
        back = O.transform_backward(S, sz)
        # two coefficient derivatives amplify rounding by ~N^4
        assert np.max(np.abs(back - ex[name])) < 1e-10, name
