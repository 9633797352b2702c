"""rs_b200: B200-native Reed-Solomon encode/reconstruct with the tape-reed-solomon API.

The directory name contains a hyphen, so import it through `load_package()` in
`__graft_entry__` (or tests/conftest.py), which registers it as `reed_solomon_b200`.
"""
from .coder import (  # noqa: F401
    ENCODE,
    ERROR_NAMES,
    MATRIX_ONLY,
    NO_GRAPH,
    RECONSTRUCT,
    RECONSTRUCT_DATA,
    Batch,
    PreparedDecoder,
    PreparedDecoder16,
    Queue,
    ReedSolomon,
    ReedSolomon16,
    RsError,
    device_check,
    frame_stripe_count,
    kernel_launch_count,
    mul_slice,
    mul_slice_dev,
    mul_slice_xor,
    outer_shape,
    outer_shard_bytes,
)
from ._lib import LIB_PATH, load  # noqa: F401
from .server import Server  # noqa: F401
