"""ctypes binding of libdnsb200.so (include/dns_b200.h).

The library is the only compute path: if it is missing, or no CUDA device is
present, creating a context raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdnsb200.so")

FORWARD, BACKWARD = 0, 1
PADDING, NO_PADDING = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
HOST, DEVICE = 0, 1

# every entry point declared in include/dns_b200.h
EXPORTS = [
    "dns_status_string", "dns_last_error", "dns_abi_version", "dns_params_default",
    "dns_read_parameter_file", "dns_create", "dns_destroy", "dns_geometry", "dns_get_stream",
    "dns_synchronize", "dns_memory_bytes", "dns_set_state", "dns_get_state",
    "dns_get_history", "dns_set_history", "dns_bootstrap", "dns_step", "dns_step_profiled",
    "dns_kernel_name",
    "dns_transform_3d_one", "dns_transform", "dns_cuda_transpose", "dns_cheby_s2p",
    "dns_cheby_p2s", "dns_get_uvw", "dns_compute_lamb", "dns_rhs_nonlinear", "dns_solve_eq",
    "dns_init_aux_matrix", "dns_transform_3d_one_noalloc",
    "dns_write_recovery", "dns_read_recovery", "dns_write_fields", "dns_init_flow",
    "dns_solve_wall", "dns_step_many", "dns_slab_ranges", "dns_slab_segments", "dns_check_state",
    "dns_slab_create", "dns_slab_exchange_bytes", "dns_slab_local", "dns_slab_part", "dns_create_batch",
    "dns_nonlinear", "dns_rhs_v", "dns_rhs_omega", "dns_rhs_mean", "dns_operator_matrices",
    "dns_operator_tables", "dns_set_wait_limit", "dns_set_variant", "dns_get_variant",
    "dns_autotune", "dns_solve_residual",
]

PASS_Y3, PASS_Y1, PASS_ZB, PASS_ZF, PASS_Y2, PASS_X, NUM_PASSES, MAX_VARIANTS = 0, 1, 2, 3, 4, 5, 6, 4
Y3_FFT, Y3_TENSOR, Y3_BLOCK = 0, 1, 2
Y1_WARP, Y1_BLOCK = 0, 1
Z_TENSOR_COPY, Z_WARP, Z_BLOCK = 0, 1, 2
Y2_RING3_12K, Y2_RING3_12K_EF, Y2_RING2_8K_EF, Y2_RING3_8K_EF = 0, 1, 2, 3
X_WARP3, X_WARP6, X_BLOCK = 0, 1, 2
# names of the tunable passes and their variants (bench and test reports)
PASS_NAMES = {PASS_Y3: "y3_uvw_s2p", PASS_Y1: "y1_p2s_rhs", PASS_ZB: "zb_span_inverse", PASS_ZF: "zf_span_forward",
              PASS_Y2: "y2_solve", PASS_X: "x_c2r_lamb_r2c"}
VARIANT_NAMES = {
    PASS_Y3: {Y3_FFT: "warp_fft", Y3_TENSOR: "tensor_core_3xtf32", Y3_BLOCK: "block_fft"},
    PASS_Y1: {Y1_WARP: "warp_fft", Y1_BLOCK: "block_fft"},
    PASS_ZB: {Z_TENSOR_COPY: "warp_fft_tensor_copy", Z_WARP: "warp_fft", Z_BLOCK: "block_fft"},
    PASS_ZF: {Z_TENSOR_COPY: "warp_fft_tensor_copy", Z_WARP: "warp_fft", Z_BLOCK: "block_fft"},
    PASS_Y2: {Y2_RING3_12K: "ring_3x12k", Y2_RING3_12K_EF: "ring_3x12k_evict_first",
              Y2_RING2_8K_EF: "ring_2x8k_evict_first", Y2_RING3_8K_EF: "ring_3x8k_evict_first"},
    PASS_X: {X_WARP3: "warp_fft_3_warps", X_WARP6: "warp_fft_6_warps", X_BLOCK: "block_fft"},
}

SLAB_PENCILS, SLAB_PLANES = 0, 1
SLAB_Y3, SLAB_XZ, SLAB_Y1 = 0, 1, 2
SLAB_V, SLAB_OMEGA, SLAB_NV, SLAB_NOMEGA = 0, 1, 2, 3


class SlabSegment(C.Structure):
    _fields_ = [("peer", C.c_int), ("kz0", C.c_int), ("nkz", C.c_int), ("local_row0", C.c_int),
                ("y0", C.c_int), ("ny", C.c_int)]


class DnsParams(C.Structure):
    _fields_ = [
        ("mx", C.c_int), ("my", C.c_int), ("mz", C.c_int),
        ("n_pi_x", C.c_double), ("n_pi_y", C.c_double),
        ("Re", C.c_double), ("Ro", C.c_double), ("dt", C.c_double),
        ("U0", C.c_double), ("U1", C.c_double), ("U2", C.c_double),
        ("precision", C.c_int), ("device", C.c_int),
    ]


class DnsRunParams(C.Structure):
    _fields_ = [
        ("start_type", C.c_int), ("start_step", C.c_int), ("end_step", C.c_int),
        ("save_internal", C.c_int), ("save_recovery_internal", C.c_int),
        ("output_file_prefix", C.c_char * 512), ("recovery_file_prefix", C.c_char * 512),
    ]


class DnsError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"dns status {status}: {msg}")
        self.status = status


_lib = None


def load_library(path: str | None = None):
    """Load libdnsb200.so (building it first if the sources are newer)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing: run build.py (nvcc, sm_100a) first")
    lib = C.CDLL(p)
    vp = C.c_void_p
    sz = C.c_size_t
    i = C.c_int
    lib.dns_status_string.restype = C.c_char_p
    lib.dns_status_string.argtypes = [i]
    lib.dns_last_error.restype = C.c_char_p
    lib.dns_last_error.argtypes = []
    lib.dns_abi_version.restype = i
    lib.dns_kernel_name.restype = C.c_char_p
    lib.dns_kernel_name.argtypes = [i]
    sigs = {
        "dns_params_default": [C.POINTER(DnsParams)],
        "dns_read_parameter_file": [C.c_char_p, C.POINTER(DnsParams), C.POINTER(DnsRunParams)],
        "dns_create": [C.POINTER(DnsParams), C.POINTER(vp)],
        "dns_destroy": [vp],
        "dns_geometry": [vp, C.POINTER(C.c_int)],
        "dns_get_stream": [vp, C.POINTER(vp)],
        "dns_synchronize": [vp],
        "dns_memory_bytes": [vp, C.POINTER(sz)],
        "dns_set_state": [vp, vp, vp, sz, i],
        "dns_get_state": [vp, vp, vp, sz, i],
        "dns_get_history": [vp, vp, vp, sz, i],
        "dns_write_recovery": [vp, C.c_char_p],
        "dns_read_recovery": [vp, C.c_char_p],
        "dns_write_fields": [vp, C.c_char_p, C.c_char_p],
        "dns_init_flow": [vp],
        "dns_set_history": [vp, vp, vp, sz, i],
        "dns_bootstrap": [vp],
        "dns_step": [vp, i],
        "dns_step_profiled": [vp, i, C.POINTER(C.c_double)],
        "dns_transform_3d_one": [vp, i, vp, sz, vp, sz, i],
        "dns_transform_3d_one_noalloc": [vp, i, vp, sz, vp, sz, i],
        "dns_transform": [vp, i, i, C.POINTER(vp), sz, C.POINTER(vp), sz],
        "dns_cuda_transpose": [vp, i, vp, sz, vp, sz],
        "dns_cheby_s2p": [vp, vp, sz, i],
        "dns_cheby_p2s": [vp, vp, sz, i],
        "dns_get_uvw": [vp, C.POINTER(vp), sz],
        "dns_compute_lamb": [vp, C.POINTER(vp), C.POINTER(vp), sz],
        "dns_rhs_nonlinear": [vp, vp, vp, vp, sz],
        "dns_solve_eq": [vp, vp, vp, i, sz, i],
        "dns_nonlinear": [vp, vp, vp, vp, vp, sz, i],
        "dns_rhs_v": [vp, vp, vp, vp, vp, sz, i],
        "dns_rhs_omega": [vp, vp, vp, vp, vp, vp, sz, i],
        "dns_rhs_mean": [vp, vp, vp, vp, vp, vp, vp, i],
        "dns_operator_matrices": [vp, vp, vp, i],
        "dns_operator_tables": [vp, vp, vp, vp, vp, vp, vp],
        "dns_set_wait_limit": [vp, C.c_longlong],
        "dns_set_variant": [vp, i, i],
        "dns_get_variant": [vp, i, C.POINTER(C.c_int)],
        "dns_autotune": [vp, C.POINTER(C.c_double)],
        "dns_solve_residual": [vp, vp, vp, vp, vp, sz, i, C.POINTER(C.c_double)],
        "dns_init_aux_matrix": [vp, vp, vp, i],
        "dns_solve_wall": [vp, vp, vp, sz, i],
        "dns_step_many": [C.POINTER(vp), i, i],
        "dns_check_state": [vp],
        "dns_slab_ranges": [i, i, i, i, i, C.POINTER(C.c_int)],
        "dns_slab_segments": [i, i, i, i, i, i, C.POINTER(SlabSegment), i, C.POINTER(C.c_int)],
        "dns_slab_create": [C.POINTER(DnsParams), i, i, C.POINTER(vp)],
        "dns_create_batch": [C.POINTER(DnsParams), i, C.POINTER(vp)],
        "dns_slab_exchange_bytes": [vp, i, C.POINTER(sz), C.POINTER(sz)],
        "dns_slab_local": [vp, i, vp, i, i],
        "dns_slab_part": [vp, i, i, vp, vp],
    }
    for name, args in sigs.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = i
    if path is None:
        _lib = lib
    return lib


def _check(lib, st):
    if st != 0:
        raise DnsError(st, lib.dns_last_error().decode(errors="replace"))


def make_params(mx, my, mz, n_pi_x=4.0, n_pi_y=2.0, Re=1300.0, Ro=0.0, dt=0.005,
                U=(0.5, 0.5, 0.0), precision=PREC_FP64, device=0) -> DnsParams:
    p = DnsParams()
    p.mx, p.my, p.mz = mx, my, mz
    p.n_pi_x, p.n_pi_y = n_pi_x, n_pi_y
    p.Re, p.Ro, p.dt = Re, Ro, dt
    p.U0, p.U1, p.U2 = U
    p.precision = precision
    p.device = device
    return p


def read_parameter_file(path):
    lib = load_library()
    p = DnsParams()
    r = DnsRunParams()
    _check(lib, lib.dns_read_parameter_file(path.encode(), C.byref(p), C.byref(r)))
    return p, r


def _ptrs(seq):
    arr = (C.c_void_p * len(seq))(*[C.c_void_p(int(x)) for x in seq])
    return arr


def slab_ranges(mx, my, mz, nranks, rank):
    """(slot0, slot1, y0, y1, pencils) of one rank of a slab decomposition."""
    lib = load_library()
    out = (C.c_int * 5)()
    _check(lib, lib.dns_slab_ranges(mx, my, mz, nranks, rank, out))
    return tuple(out)


def slab_segments(mx, my, mz, nranks, rank, role):
    """The exchange segments of one rank as dicts (peer, kz0, nkz, local_row0, y0, ny)."""
    lib = load_library()
    n = C.c_int()
    _check(lib, lib.dns_slab_segments(mx, my, mz, nranks, rank, role, None, 0, C.byref(n)))
    arr = (SlabSegment * max(n.value, 1))()
    _check(lib, lib.dns_slab_segments(mx, my, mz, nranks, rank, role, arr, n.value, C.byref(n)))
    return [{f: getattr(arr[k], f) for f, _ in SlabSegment._fields_} for k in range(n.value)]


def step_many(contexts, n=1):
    """n steps of each of several independent runs, concurrently (one stream
    per run); asynchronous like Context.step."""
    ctxs = list(contexts)
    if not ctxs:
        raise ValueError("no contexts")
    lib = ctxs[0].lib
    _check(lib, lib.dns_step_many(_ptrs([c.h.value for c in ctxs]), len(ctxs), int(n)))


class Context:
    """One DNS problem on one GPU (a ``dns_ctx``)."""

    def __init__(self, params: DnsParams):
        self.lib = load_library()
        h = C.c_void_p()
        _check(self.lib, self.lib.dns_create(C.byref(params), C.byref(h)))
        self.h = h
        self.params = params
        g = (C.c_int * 8)()
        _check(self.lib, self.lib.dns_geometry(self.h, g))
        self.Nx, self.Ny, self.Nz, self.Kx, self.Px, self.Py, self.Pz, self.H = list(g)

    def close(self):
        if getattr(self, "h", None):
            self.lib.dns_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- helpers -----------------------------------------------------------
    def _call(self, name, *args):
        _check(self.lib, getattr(self.lib, name)(self.h, *args))

    @property
    def stream(self):
        s = C.c_void_p()
        self._call("dns_get_stream", C.byref(s))
        return s.value

    def memory_bytes(self):
        b = C.c_size_t()
        self._call("dns_memory_bytes", C.byref(b))
        return b.value

    def synchronize(self):
        self._call("dns_synchronize")

    # -- state (numpy host arrays, shape (Nz, Kx, Ny) complex128) -----------
    @property
    def shape(self):
        """Shape of the state and history arrays: (Nz, Kx, Ny), a batch (n, Nz, Kx, Ny)."""
        return (self.Nz, self.Kx, self.Ny)

    def _pencils(self, a):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        if a.shape != self.shape:
            raise ValueError(f"expected shape {self.shape}, got {a.shape}")
        return a

    def set_state(self, V, O):
        V = self._pencils(V)
        O = self._pencils(O)
        self._call("dns_set_state", V.ctypes.data, O.ctypes.data, self.Ny * 16, HOST)

    def get_state(self):
        V = np.empty(self.shape, dtype=np.complex128)
        O = np.empty_like(V)
        self._call("dns_get_state", V.ctypes.data, O.ctypes.data, self.Ny * 16, HOST)
        return V, O

    def get_history(self):
        V = np.empty(self.shape, dtype=np.complex128)
        O = np.empty_like(V)
        self._call("dns_get_history", V.ctypes.data, O.ctypes.data, self.Ny * 16, HOST)
        return V, O

    def set_history(self, Nv, No):
        Nv = self._pencils(Nv)
        No = self._pencils(No)
        self._call("dns_set_history", Nv.ctypes.data, No.ctypes.data, self.Ny * 16, HOST)

    def write_recovery(self, path):
        """The reference's recovery file (write_recover_data)."""
        self._call("dns_write_recovery", os.fsencode(path))

    def read_recovery(self, path):
        """Restore state and AB2 history from a recovery file."""
        self._call("dns_read_recovery", os.fsencode(path))

    def write_fields(self, velocity_path=None, vorticity_path=None):
        """The reference's output_velocity files (physical u, v, w and vorticity)."""
        self._call("dns_write_fields", None if velocity_path is None else os.fsencode(velocity_path),
                   None if vorticity_path is None else os.fsencode(vorticity_path))

    def init_flow(self):
        """The reference's analytic initial state (initFlow); bootstrap next."""
        self._call("dns_init_flow")

    def set_state_device(self, v_ptr, o_ptr, pitch):
        self._call("dns_set_state", C.c_void_p(v_ptr), C.c_void_p(o_ptr), pitch, DEVICE)

    def get_state_device(self, v_ptr, o_ptr, pitch):
        self._call("dns_get_state", C.c_void_p(v_ptr), C.c_void_p(o_ptr), pitch, DEVICE)

    def bootstrap(self):
        self._call("dns_bootstrap")

    def check_state(self):
        """Raise DnsError (DNS_ERR_NONFINITE) if the state holds NaN or Inf."""
        self._call("dns_check_state")

    def step(self, n=1):
        self._call("dns_step", int(n))

    def step_profiled(self, n=1):
        """Run n un-graphed steps; returns {kernel name: mean ms per launch}."""
        ms = (C.c_double * 6)()
        self._call("dns_step_profiled", int(n), ms)
        return {self.lib.dns_kernel_name(k).decode(): ms[k] for k in range(6)}

    # -- reference-layout entry points (device pointers as ints) -----------
    def transform_3d_one(self, direction, phys, pitch, spec, tpitch, pad=PADDING):
        self._call("dns_transform_3d_one", int(direction), C.c_void_p(phys), pitch,
                   C.c_void_p(spec), tpitch, int(pad))

    def transform_3d_one_noalloc(self, direction, phys, pitch, spec, tpitch, pad=PADDING):
        """transform_3d_one without device allocation at call time (see the
        header): same results, work buffer in a 16 MiB static device array."""
        self._call("dns_transform_3d_one_noalloc", int(direction), C.c_void_p(phys), pitch,
                   C.c_void_p(spec), tpitch, int(pad))

    def transform(self, direction, phys, pitch, spec, tpitch):
        self._call("dns_transform", int(direction), len(phys), _ptrs(phys), pitch, _ptrs(spec), tpitch)

    def cuda_transpose(self, direction, xyz, pitch, zxy, tpitch):
        self._call("dns_cuda_transpose", int(direction), C.c_void_p(xyz), pitch, C.c_void_p(zxy), tpitch)

    def cheby_s2p(self, zxy, tpitch, pad=PADDING):
        self._call("dns_cheby_s2p", C.c_void_p(zxy), tpitch, int(pad))

    def cheby_p2s(self, zxy, tpitch, pad=PADDING):
        self._call("dns_cheby_p2s", C.c_void_p(zxy), tpitch, int(pad))

    def get_uvw(self, fields, tpitch):
        self._call("dns_get_uvw", _ptrs(fields), tpitch)

    def compute_lamb(self, fin, fout, pitch):
        self._call("dns_compute_lamb", _ptrs(fin), _ptrs(fout), pitch)

    def rhs_nonlinear(self, lx, ly, lz, tpitch):
        self._call("dns_rhs_nonlinear", C.c_void_p(lx), C.c_void_p(ly), C.c_void_p(lz), tpitch)

    def solve_eq(self, inv, rhs, N, tpitch, where=DEVICE):
        self._call("dns_solve_eq", C.c_void_p(inv), C.c_void_p(rhs), int(N), tpitch, int(where))

    def nonlinear(self, v, omega, nv, nomega, tpitch, where=DEVICE):
        """getNonlinear + no-pad s2p: state -> nonlinear terms at the points."""
        self._call("dns_nonlinear", C.c_void_p(v), C.c_void_p(omega), C.c_void_p(nv),
                   C.c_void_p(nomega), tpitch, int(where))

    def rhs_v(self, rhs_v, rhs_v_p, nv, nv_p, tpitch, where=DEVICE):
        self._call("dns_rhs_v", C.c_void_p(rhs_v), C.c_void_p(rhs_v_p), C.c_void_p(nv),
                   C.c_void_p(nv_p), tpitch, int(where))

    def rhs_omega(self, rhs_omega, nomega, nomega_p, rhs_v, rhs_v_p, tpitch, where=DEVICE):
        self._call("dns_rhs_omega", C.c_void_p(rhs_omega), C.c_void_p(nomega), C.c_void_p(nomega_p),
                   C.c_void_p(rhs_v), C.c_void_p(rhs_v_p), tpitch, int(where))

    def rhs_mean(self, u0, lx0, lx0_p, w0, lz0, lz0_p, where=DEVICE):
        self._call("dns_rhs_mean", C.c_void_p(u0), C.c_void_p(lx0), C.c_void_p(lx0_p),
                   C.c_void_p(w0), C.c_void_p(lz0), C.c_void_p(lz0_p), int(where))

    def set_variant(self, pass_, variant):
        self._call("dns_set_variant", int(pass_), int(variant))

    def get_variant(self, pass_):
        v = C.c_int()
        self._call("dns_get_variant", int(pass_), C.byref(v))
        return v.value

    def autotune(self):
        """Time every available kernel variant, keep the fastest; returns
        {pass: {variant: ms}} for the available variants."""
        ms = (C.c_double * (NUM_PASSES * MAX_VARIANTS))()
        self._call("dns_autotune", ms)
        return {p: {v: ms[p * MAX_VARIANTS + v] for v in range(MAX_VARIANTS) if ms[p * MAX_VARIANTS + v] >= 0}
                for p in range(NUM_PASSES)}

    def set_wait_limit(self, cycles=1 << 31):
        """Bound of the staging waits (SM cycles); negative: give up at once."""
        self._call("dns_set_wait_limit", int(cycles))

    def operator_matrices(self, a_v, a_o, where=DEVICE):
        self._call("dns_operator_matrices", C.c_void_p(a_v), C.c_void_p(a_o), int(where))

    def operator_tables(self):
        """(T0, T2, T4, U, dU, ddU) as numpy arrays."""
        import numpy as np
        n = self.Ny
        T = [np.zeros((n, n)) for _ in range(3)]
        U = [np.zeros(n) for _ in range(3)]
        self._call("dns_operator_tables", *[a.ctypes.data_as(C.c_void_p) for a in T + U])
        return (*T, *U)

    def solve_wall(self, v, omega, tpitch, where=DEVICE):
        """solveEq of both wall-normal systems with the banded factors, in place.

        Device pointers (ints) with where=DEVICE; with where=HOST, numpy
        arrays of shape (Nz, Kx, L >= Ny) complex128, overwritten."""
        if where == HOST:
            for a in (v, omega):
                if not (isinstance(a, np.ndarray) and a.dtype == np.complex128 and a.ndim == 3
                        and a.shape[:2] == (self.Nz, self.Kx) and a.shape[2] * 16 == tpitch
                        and a.flags.c_contiguous):
                    raise ValueError("host arrays must be C-contiguous (Nz, Kx, tpitch/16) complex128")
            self._call("dns_solve_wall", v.ctypes.data, omega.ctypes.data, tpitch, HOST)
        else:  # device pointers; 0 or None leaves that system alone
            self._call("dns_solve_wall", C.c_void_p(v or None), C.c_void_p(omega or None), tpitch, DEVICE)

    def solve_residual(self, bv, bo, xv, xo, tpitch, where=DEVICE):
        """(max per-pencil ||Ax-b||/||b|| of v, omega; the same over all
        pencils; max backward error of v, omega)."""
        out = (C.c_double * 6)()
        arrs = (bv, bo, xv, xo)
        if where == HOST:  # numpy arrays (Nz, Kx, tpitch/16) complex128
            for a in arrs:
                if not (isinstance(a, np.ndarray) and a.dtype == np.complex128 and a.ndim == 3
                        and a.shape[:2] == (self.Nz, self.Kx) and a.shape[2] * 16 == tpitch
                        and a.flags.c_contiguous):
                    raise ValueError("host arrays must be C-contiguous (Nz, Kx, tpitch/16) complex128")
            ptrs = [C.c_void_p(a.ctypes.data) for a in arrs]
        else:
            ptrs = [C.c_void_p(int(a)) for a in arrs]
        self._call("dns_solve_residual", *ptrs, tpitch, int(where), out)
        return tuple(out)

    def init_aux_matrix(self, inv_v, inv_o, where=DEVICE):
        if where == HOST:
            self._call("dns_init_aux_matrix", inv_v.ctypes.data, inv_o.ctypes.data, HOST)
        else:
            self._call("dns_init_aux_matrix", C.c_void_p(inv_v), C.c_void_p(inv_o), DEVICE)


class SlabContext(Context):
    """One rank of a slab-decomposed step (``dns_slab_create``): the pencils
    of its operator slots and the wall-normal planes of its range.  A step
    is ``part(SLAB_Y3)``, exchange 0, ``part(SLAB_XZ)``, exchange 1,
    ``part(SLAB_Y1)``; the exchanges are the caller's (``slab.py``)."""

    def __init__(self, params: DnsParams, nranks: int, rank: int):
        self.lib = load_library()
        h = C.c_void_p()
        _check(self.lib, self.lib.dns_slab_create(C.byref(params), int(nranks), int(rank), C.byref(h)))
        self.h = h
        self.params = params
        g = (C.c_int * 8)()
        _check(self.lib, self.lib.dns_geometry(self.h, g))
        self.Nx, self.Ny, self.Nz, self.Kx, self.Px, self.Py, self.Pz, self.H = list(g)
        self.nranks, self.rank = int(nranks), int(rank)
        self.ranges = slab_ranges(params.mx, params.my, params.mz, nranks, rank)
        self.np = self.ranges[4]
        segs = slab_segments(params.mx, params.my, params.mz, nranks, rank, SLAB_PENCILS)
        self.runs = sorted({(sg["kz0"], sg["nkz"], sg["local_row0"]) for sg in segs}, key=lambda t: t[2])
        # global pencil index p = kz Kx + kx of each local row
        self.pencils = np.concatenate([np.arange(kz0 * self.Kx, (kz0 + nkz) * self.Kx)
                                       for kz0, nkz, _ in self.runs]).astype(np.int64)

    def exchange_bytes(self, exchange):
        """(send bytes per peer, recv bytes per peer) of exchange 0 or 1."""
        snd = (C.c_size_t * self.nranks)()
        rcv = (C.c_size_t * self.nranks)()
        self._call("dns_slab_exchange_bytes", int(exchange), snd, rcv)
        return list(snd), list(rcv)

    def set_local(self, which, a):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        if a.shape != (self.np, self.Ny):
            raise ValueError(f"expected shape {(self.np, self.Ny)}, got {a.shape}")
        self._call("dns_slab_local", int(which), C.c_void_p(a.ctypes.data), HOST, 1)

    def get_local(self, which):
        a = np.empty((self.np, self.Ny), dtype=np.complex128)
        self._call("dns_slab_local", int(which), C.c_void_p(a.ctypes.data), HOST, 0)
        return a

    def scatter_state(self, V, O):
        """This rank's pencils of whole-grid (Nz, Kx, Ny) arrays."""
        self.set_local(SLAB_V, np.asarray(V).reshape(self.H, self.Ny)[self.pencils])
        self.set_local(SLAB_OMEGA, np.asarray(O).reshape(self.H, self.Ny)[self.pencils])

    def gather_state(self, V, O):
        """Write this rank's pencils into whole-grid (Nz, Kx, Ny) arrays."""
        V.reshape(self.H, self.Ny)[self.pencils] = self.get_local(SLAB_V)
        O.reshape(self.H, self.Ny)[self.pencils] = self.get_local(SLAB_OMEGA)

    def part(self, part, send_ptr, recv_ptr, boot=False):
        """Enqueue one part on the context's stream (asynchronous)."""
        self._call("dns_slab_part", int(part), int(bool(boot)), C.c_void_p(send_ptr or None),
                   C.c_void_p(recv_ptr or None))


class BatchContext(Context):
    """A batch of independent runs of one grid (``dns_create_batch``): every
    pass one launch for all runs; Re, Ro and dt may differ between runs.
    State and history arrays have shape (n, Nz, Kx, Ny)."""

    def __init__(self, params_list):
        self.lib = load_library()
        plist = list(params_list)
        arr = (DnsParams * len(plist))(*plist)
        h = C.c_void_p()
        _check(self.lib, self.lib.dns_create_batch(arr, len(plist), C.byref(h)))
        self.h = h
        self.params = plist[0]
        self.n = len(plist)
        g = (C.c_int * 8)()
        _check(self.lib, self.lib.dns_geometry(self.h, g))
        self.Nx, self.Ny, self.Nz, self.Kx, self.Px, self.Py, self.Pz, self.H = list(g)

    @property
    def shape(self):
        return (self.n, self.Nz, self.Kx, self.Ny)
