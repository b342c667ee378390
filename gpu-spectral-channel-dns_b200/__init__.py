"""B200-native v-omega Fourier-Chebyshev DNS time step.

Host-side mirror of the reference's interface over the C ABI of
``libdnsb200.so`` (declared in ``include/dns_b200.h``).  All compute runs in
the CUDA library; this package only moves buffers and parameters.
"""
from .abi import (  # noqa: F401
    BACKWARD, DEVICE, FORWARD, HOST, NO_PADDING, PADDING, PREC_FP64, PREC_MIXED,
    Context, BatchContext, DnsError, DnsParams, EXPORTS, LIB_PATH, load_library, make_params,
    read_parameter_file, step_many, SLAB_PENCILS, SLAB_PLANES, slab_ranges, slab_segments,
    PASS_Y3, PASS_Y1, PASS_ZB, PASS_ZF, PASS_Y2, PASS_X, X_WARP3, X_WARP6, X_BLOCK, NUM_PASSES, MAX_VARIANTS, Y3_FFT, Y3_TENSOR, Y3_BLOCK,
    Y1_WARP, Y1_BLOCK, Z_TENSOR_COPY, Z_WARP, Z_BLOCK, Y2_RING3_12K, Y2_RING3_12K_EF, Y2_RING2_8K_EF, Y2_RING3_8K_EF,
    PASS_NAMES, VARIANT_NAMES, SlabContext, SLAB_Y3, SLAB_XZ, SLAB_Y1, SLAB_V, SLAB_OMEGA, SLAB_NV,
    SLAB_NOMEGA,
)
from .seed import seeded_state  # noqa: F401
