"""dns_transform_3d_one_noalloc against dns_transform_3d_one.

The no-allocation variant exists for callers that cannot have the library
cudaMalloc at call time (an application that has reserved almost all device
memory for its own arena, or a loop that cannot take cudaMalloc's implicit
device synchronisation).  It keeps its work buffer in a 16 MiB static device
array and processes wall-normal planes in slabs.  Two calls in a row, with
different inputs, must each match the allocating entry point (the buffer
keeps the previous call's contents).  This file is collected last on purpose.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("mx,my,mz", [(192, 192, 256), (48, 48, 128)])
@pytest.mark.parametrize("pad", [0, 1])
def test_noalloc_matches_allocating_transform(pkg, mx, my, mz, pad):
    ctx = pkg.Context(pkg.make_params(mx, my, mz, Re=3000.0, Ro=0.02, dt=0.001))
    ny, hnx, nz, pz = my // 3 * 2, mx // 3 + 1, mz // 4 + 1, mz // 2 + 1
    pitch = (mx + 2) * 8
    tpitch = mz * 16
    rng = np.random.default_rng(123 + pad)
    for call in range(2):  # two calls in a row, different inputs
        S = rng.standard_normal((ny, hnx, nz)) + 1j * rng.standard_normal((ny, hnx, nz))
        outs = []
        for noalloc in (False, True):
            spec = torch.zeros((ny, hnx, mz), dtype=torch.complex128)
            spec[:, :, :nz] = torch.from_numpy(S)
            spec = spec.cuda()
            phys = torch.zeros((pz, my, mx + 2), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            f = ctx.transform_3d_one_noalloc if noalloc else ctx.transform_3d_one
            f(pkg.BACKWARD, phys.data_ptr(), pitch, spec.data_ptr(), tpitch, pad)
            ctx.synchronize()
            back = phys.cpu().numpy()[..., :mx].copy()
            spec2 = torch.zeros((ny, hnx, mz), dtype=torch.complex128, device="cuda")
            torch.cuda.synchronize()
            f(pkg.FORWARD, phys.data_ptr(), pitch, spec2.data_ptr(), tpitch, pad)
            ctx.synchronize()
            outs.append((back, spec2.cpu().numpy()))
        npl = pz if pad == 0 else nz
        ncoef = pz if pad == 0 else nz
        assert _rel(outs[1][0][:npl], outs[0][0][:npl]) < 1e-13, call
        assert _rel(outs[1][1][..., :ncoef], outs[0][1][..., :ncoef]) < 1e-13, call
    ctx.close()


def test_noalloc_rejects_oversized_grid(pkg):
    # one wall-normal plane of a 1536 x 1536 padded grid needs 1536 * 776 * 16 B > 16 MiB
    ctx = None
    try:
        ctx = pkg.Context(pkg.make_params(1536, 1536, 16, Re=1000.0, dt=0.001))
    except pkg.DnsError:
        pytest.skip("could not create the large context")
    try:
        with pytest.raises(pkg.DnsError) as ei:
            ctx.transform_3d_one_noalloc(pkg.BACKWARD, 1, 1538 * 8, 1, 16 * 16)
        assert "16 MiB" in str(ei.value)
    finally:
        ctx.close()
