"""ctypes binding of librsb200.so (the C ABI declared in include/rs_b200.h).

The shared library is built in-tree by build_lib.py. There is no CPU fallback: if
the library is missing, or no CUDA device is usable, calls raise.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librsb200.so")

_sz = ctypes.c_size_t
_vp = ctypes.c_void_p
_int = ctypes.c_int
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u16p = ctypes.POINTER(ctypes.c_uint16)
_szp = ctypes.POINTER(ctypes.c_size_t)
_intp = ctypes.POINTER(ctypes.c_int)
_pp = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes); every symbol include/rs_b200.h declares.
SIGNATURES = {
    "rs_strerror": (ctypes.c_char_p, [_int]),
    "rs_abi_version": (ctypes.c_uint32, []),
    "rs_device_check": (_int, []),
    "rs_kernel_launch_count": (ctypes.c_uint64, []),
    "rs_set_fft_variant": (_int, [_sz, _int]),
    "rs_fft_variant_count": (_int, []),
    "rs_set_fft_lanes": (_int, [_sz, _int]),
    "rs_set_host_copy_threads": (_int, [_int]),
    "rs_set_host_staging": (_int, [_int]),
    "rs_set_matrix_variant": (_int, [_int]),
    "rs_set_fft16_pass": (_int, [_int]),
    "rs_set_matrix_bits": (_int, [_int]),
    "rs_matrix_variant_count": (_int, []),
    "rs_generator_rows": (_int, [_int, _sz, _sz, _u16p, _sz]),
    "rs_decode_rows": (_int, [_int, _sz, _sz, _u8p, _u16p, _sz, _szp]),
    "rs8_new": (_int, [_sz, _sz, _pp]),
    "rs8_clone": (_int, [_vp, _pp]),
    "rs8_free": (None, [_vp]),
    "rs8_data_shard_count": (_sz, [_vp]),
    "rs8_parity_shard_count": (_sz, [_vp]),
    "rs8_total_shard_count": (_sz, [_vp]),
    "rs8_equal": (_int, [_vp, _vp]),
    "rs8_parity_matrix": (_int, [_vp, _u8p, _sz]),
    "rs8_encode": (_int, [_vp, _pp, _sz, _sz]),
    "rs8_encode_sep": (_int, [_vp, _pp, _sz, _pp, _sz, _sz]),
    "rs8_encode_rows": (_int, [_vp, _vp, _sz, _sz, _vp, _sz]),
    "rs8_encode_batch": (_int, [_vp, _vp, _sz, _vp, _sz, _sz, _sz]),
    "rs8_verify": (_int, [_vp, _pp, _sz, _sz, _intp]),
    "rs8_reconstruct": (_int, [_vp, _pp, _szp, _u8p, _sz, _int]),
    "rs8_reconstruct_rows": (_int, [_vp, _vp, _sz, _sz, _u8p, _sz]),
    "rs8_prepare_decode": (_int, [_vp, _u8p, _sz, _pp]),
    "rs8_dec_reconstruct": (_int, [_vp, _pp, _szp, _u8p, _sz, _int]),
    "rs8_dec_clone": (_int, [_vp, _pp]),
    "rs8_dec_free": (None, [_vp]),
    "rs8_encode_route": (ctypes.c_char_p, [_vp, _sz]),
    "rs8_set_route": (_int, [_vp, _int]),
    "rs8_encode_dev": (_int, [_vp, _pp, _sz, _sz, _vp]),
    "rs8_encode_sep_dev": (_int, [_vp, _pp, _sz, _pp, _sz, _sz, _vp]),
    "rs8_encode_rows_dev": (_int, [_vp, _vp, _sz, _vp, _vp]),
    "rs8_encode_batch_dev": (_int, [_vp, _vp, _sz, _vp, _sz, _sz, _sz, _vp]),
    "rs8_verify_dev": (_int, [_vp, _pp, _sz, _sz, _intp, _vp]),
    "rs8_reconstruct_dev": (_int, [_vp, _pp, _szp, _u8p, _sz, _int, _vp]),
    "rs8_reconstruct_batch_dev": (_int, [_vp, _vp, _sz, _sz, _sz, _u8p, _int, _intp, _vp]),
    "rs8_reconstruct_batch_noalloc": (_int, [_vp, _vp, _sz, _sz, _sz, _u8p, _int, _intp, _vp]),
    "rs8_reconstruct_batch_noalloc_limit": (_sz, [_sz, _sz, _sz]),
    "rs_batch_create": (_int, [_vp, _sz, _int, _intp, _pp]),
    "rs_batch_create_configured": (_int, [_vp, _sz, _int, _intp, _intp, _pp]),
    "rs_batch_choose": (_int, [_vp, _sz, _vp, _intp]),
    "rs_tuning_config_count": (_int, []),
    "rs_tuning_config": (_int, [_int, _intp, _intp, _intp]),
    "rs_tuning_features": (_int, []),
    "rs_batch_launch": (_int, [_vp, _vp]),
    "rs_batch_stats": (_int, [_vp, _szp, _szp, _szp, ctypes.POINTER(ctypes.c_uint64)]),
    "rs_batch_free": (None, [_vp]),
    "rs_queue_create": (_int, [_sz, _sz, ctypes.c_uint64, _pp]),
    "rs_queue_start": (_int, [_vp]),
    "rs_queue_push": (_int, [_vp, _vp, _sz, _intp]),
    "rs_queue_progress": (_int, [_vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "rs_queue_finish": (_int, [_vp]),
    "rs_queue_wait": (_int, [_vp]),
    "rs_queue_free": (None, [_vp]),
    "rs_server_create": (_int, [_vp, _pp]),
    "rs_server_submit": (_int, [_vp, _vp, _sz, _intp]),
    "rs_server_poll": (_int, [_vp, _vp, _sz, _szp, _int]),
    "rs_server_set_fft_route": (_int, [_vp, _sz, _int, _int]),
    "rs_server_stats_get": (_int, [_vp, _vp]),
    "rs_server_free": (None, [_vp]),
    "rs16_new": (_int, [_sz, _sz, _pp]),
    "rs16_clone": (_int, [_vp, _pp]),
    "rs16_free": (None, [_vp]),
    "rs16_data_shard_count": (_sz, [_vp]),
    "rs16_parity_shard_count": (_sz, [_vp]),
    "rs16_total_shard_count": (_sz, [_vp]),
    "rs16_equal": (_int, [_vp, _vp]),
    "rs16_parity_matrix": (_int, [_vp, _u16p, _sz]),
    "rs16_encode": (_int, [_vp, _pp, _sz, _sz]),
    "rs16_encode_sep": (_int, [_vp, _pp, _sz, _pp, _sz, _sz]),
    "rs16_verify": (_int, [_vp, _pp, _sz, _sz, _intp]),
    "rs16_reconstruct": (_int, [_vp, _pp, _szp, _u8p, _sz, _int]),
    "rs16_reconstruct_rows": (_int, [_vp, _vp, _sz, _sz, _u8p, _sz]),
    "rs16_prepare_decode": (_int, [_vp, _u8p, _sz, _pp]),
    "rs16_dec_reconstruct": (_int, [_vp, _pp, _szp, _u8p, _sz, _int]),
    "rs16_dec_clone": (_int, [_vp, _pp]),
    "rs16_dec_free": (None, [_vp]),
    "rs16_encode_route": (ctypes.c_char_p, [_vp]),
    "rs16_encode_route_for": (ctypes.c_char_p, [_vp, _sz, _sz]),
    "rs16_set_route": (_int, [_vp, _int]),
    "rs16_encode_dev": (_int, [_vp, _pp, _sz, _sz, _vp]),
    "rs16_encode_batch_dev": (_int, [_vp, _vp, _sz, _vp, _sz, _sz, _sz, _vp]),
    "rs16_reconstruct_dev": (_int, [_vp, _pp, _szp, _u8p, _sz, _int, _vp]),
    "rs_frame_stripe_count": (_sz, [_sz, _sz, _sz]),
    "rs8_frame_encode_dev": (_int, [_vp, _vp, _sz, _sz, _vp, _sz, _vp]),
    "rs8_frame_decode_dev": (_int, [_vp, _vp, _sz, _sz, _u8p, _vp, _sz, _intp, _vp]),
    "rs16_frame_encode_dev": (_int, [_vp, _vp, _sz, _sz, _vp, _sz, _vp]),
    "rs16_frame_decode_dev": (_int, [_vp, _vp, _sz, _sz, _u8p, _vp, _sz, _intp, _vp]),
    "rs_outer_shape": (_int, [_sz, _szp, _szp]),
    "rs_outer_shard_bytes": (_int, [_sz, _sz, _szp]),
    "rs_mlp_create": (_int, [_int, _int, _int, ctypes.c_uint64, _pp]),
    "rs_mlp_free": (None, [_vp]),
    "rs_mlp_dims": (_int, [_vp, _intp, _intp, _intp]),
    "rs_mlp_save": (_int, [_vp, ctypes.c_char_p]),
    "rs_mlp_load": (_int, [ctypes.c_char_p, _pp]),
    "rs_mlp_param_count": (_sz, [_vp]),
    "rs_mlp_get_params": (_int, [_vp, _vp, _sz]),
    "rs_mlp_set_params": (_int, [_vp, _vp, _sz]),
    "rs_mlp_predict": (_int, [_vp, _vp, _int, _vp]),
    "rs_mlp_gradients": (_int, [_vp, _vp, _vp, _vp, _int, ctypes.c_float, _vp, _sz,
                                ctypes.POINTER(ctypes.c_float)]),
    "rs_mlp_train_step": (_int, [_vp, _vp, _vp, _vp, _int, ctypes.c_float, ctypes.c_float,
                                 ctypes.POINTER(ctypes.c_float)]),
    "gf8_mul_slice": (_int, [_vp, _sz, _vp, _sz, ctypes.c_uint8, _int]),
    "gf8_mul_slice_dev": (_int, [_vp, _vp, _sz, ctypes.c_uint8, _int, _vp]),
}

_lib = None


def load():
    """Load librsb200.so, raising if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "librsb200.so is not built (run reed-solomon_b200/build_lib.py); "
                "there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib
