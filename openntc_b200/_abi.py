"""ctypes mirror of include/ontc.h (the C ABI of libontc.so).

Struct layouts here must stay byte-identical to the C header; tests check sizes and
offsets against the C compiler's view.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

MAX_MIPS = 12
MAX_CHANNELS = 16
MAX_LEVELS = 6
MAX_SOURCES = 16

SUCCESS, INVALID_DIMENSION, ALLOCATION_FAILURE, INVALID_MANIFEST, FILE_NOT_FOUND, \
    INVALID_FILE, FILE_WRITE_FAILURE, INVALID_STATE, CUDA_FAILURE = range(9)
RESULT_NAMES = ["Success", "InvalidDimension", "AllocationFailure", "InvalidManifest", "FileNotFound",
                "InvalidFile", "FileWriteFailure", "InvalidState", "CudaFailure"]

BPP_0_2, BPP_0_5, BPP_1_0, BPP_2_25 = range(4)
QUALITY_LOW, QUALITY_MEDIUM, QUALITY_HIGH, QUALITY_ULTRA = range(4)
MANIFEST_LOADED, TRAIN_IN_PROGRESS, TRAIN_COMPLETE, TRAIN_ERROR = 0, 1, 2, -1
PRECISION_BF16, PRECISION_FP32, PRECISION_BF16X3 = 0, 1, 2
DECODE_INT8 = 0  # ONTC_DECODE_INT8: SampleMaterial integer semantics
DECODE_FP32, DECODE_BF16, DECODE_FP8 = 1, 2, 3  # float-model decoders (ontc_decoder_create_float)
SCREEN_DISCARD_OUTSIDE = 1  # ONTC_SCREEN_DISCARD_OUTSIDE
SCREEN_MATERIAL = 2  # ONTC_SCREEN_MATERIAL
# ontc_material_params: MaterialParams (ntc_decode.hlsli:507-522), 17 floats then `present`
MATERIAL_FIELDS = ["albedo", 3, "alpha", 1, "displacement", 1, "emissive", 1, "gloss", 1, "metallic", 1,
                   "normal", 3, "ao", 1, "roughness", 1, "specular", 3, "transmission", 1]
MATERIAL_WORDS = 18


class Calibration(C.Structure):
    _fields_ = [("max_abs_a1", C.c_float), ("max_abs_a2", C.c_float), ("s_a1", C.c_float), ("s_a2", C.c_float)]


class Constants(C.Structure):
    _fields_ = [
        ("g0_grid_dim", C.c_int32 * 8), ("g1_grid_dim", C.c_int32 * 8),
        ("g0_offset", C.c_uint32 * 8), ("g1_offset", C.c_uint32 * 8),
        ("g0_bits_per_channel", C.c_int32), ("g1_bits_per_channel", C.c_int32),
        ("g0_channels", C.c_int32), ("g1_channels", C.c_int32),
        ("dim", C.c_int32), ("mip_count", C.c_int32),
        ("rcp_s_a1", C.c_float), ("rcp_s_a2", C.c_float),
        ("channel_count", C.c_int32), ("pad0", C.c_int32 * 3),
        ("channel_semantics", C.c_uint32 * 16),
    ]


class CompressedData(C.Structure):
    _fields_ = [
        ("g0", C.POINTER(C.c_uint32) * MAX_LEVELS), ("g1", C.POINTER(C.c_uint32) * MAX_LEVELS),
        ("decoder", C.c_void_p),
        ("g0_size", C.c_size_t * MAX_LEVELS), ("g1_size", C.c_size_t * MAX_LEVELS),
        ("g0_offset", C.c_size_t * MAX_LEVELS), ("g1_offset", C.c_size_t * MAX_LEVELS),
        ("g0_total_size", C.c_size_t), ("g1_total_size", C.c_size_t), ("decoder_size", C.c_size_t),
        ("g0_grid_dim", C.c_int32 * MAX_LEVELS), ("g1_grid_dim", C.c_int32 * MAX_LEVELS),
        ("g0_bits_per_channel", C.c_int32), ("g1_bits_per_channel", C.c_int32),
        ("g0_channels", C.c_int32), ("g1_channels", C.c_int32),
        ("dim", C.c_int32), ("mip_count", C.c_int32), ("level_count", C.c_int32), ("channel_count", C.c_int32),
        ("channel_semantics", C.c_int32 * MAX_CHANNELS),
        ("profile", C.c_int32),
        ("caldata", Calibration),
    ]


class TrainProgress(C.Structure):
    _fields_ = [("phase", C.c_int32), ("result", C.c_int32), ("batches_complete", C.c_int32), ("total_batches", C.c_int32)]


class EvalResults(C.Structure):
    _fields_ = [("mse", C.c_double), ("psnr", C.c_double)]


class TextureData(C.Structure):
    _fields_ = [
        ("tex_count", C.c_int32), ("mip_count", C.c_int32),
        ("channels", C.c_int32 * MAX_SOURCES), ("semantics", C.c_int32 * MAX_SOURCES),
        ("mips", (C.POINTER(C.c_uint8) * MAX_MIPS) * MAX_SOURCES),
    ]


class TrainOptions(C.Structure):
    _fields_ = [("steps_override", C.c_int32), ("has_lock_step", C.c_int32), ("lock_step", C.c_int32),
                ("precision", C.c_int32), ("noise_mode", C.c_int32), ("latent_adam", C.c_int32),
                ("calibration", C.c_int32), ("reserved", C.c_int32)]


LATENT_ADAM_DEFERRED, LATENT_ADAM_DENSE = 0, 1


NOISE_COUNTER, NOISE_UPSTREAM = 0, 1


class KernelTime(C.Structure):
    _fields_ = [("launches", C.c_int64), ("total_ms", C.c_double), ("bytes", C.c_double), ("flops", C.c_double)]


KCLASS_UNITS_FP32, KCLASS_UNITS_BF16, KCLASS_ADAM, KCLASS_CATCHUP = 0, 1, 2, 3
KCLASS_SIDE_CATCHUP, KCLASS_SIDE_UPDATE, KCLASS_UNITS_BF16X3, KCLASS_COUNT = 4, 5, 6, 7


class DebugStep(C.Structure):
    _fields_ = [("lod", C.c_int32), ("n_grids", C.c_int32), ("ox", C.c_int32 * 8), ("oy", C.c_int32 * 8),
                ("noise", C.c_int32), ("seed", C.c_uint32), ("step", C.c_int32), ("level", C.c_int32),
                ("lr_grid", C.c_float), ("lr_dec", C.c_float), ("b1", C.c_float), ("b2", C.c_float),
                ("gb1", C.c_float), ("gb2", C.c_float), ("grid_update", C.c_int32), ("pad", C.c_int32)]


DBG_G0, DBG_G1, DBG_G0_M, DBG_G0_V, DBG_G1_M, DBG_G1_V, DBG_G0_GRAD, DBG_G1_GRAD, DBG_NOISE0, DBG_NOISE1 = range(10)
DBG_W, DBG_W_M, DBG_W_V, DBG_W_GRAD = 10, 11, 12, 13

# name -> (restype, argtypes); every symbol include/ontc.h and include/ontc_debug.h declare.
P = C.c_void_p
SIGNATURES = {
    "ontc_create": (P, []),
    "ontc_destroy": (None, [P]),
    "ontc_init": (C.c_int, [P, C.c_int32, P]),
    "ontc_set_min_dimension": (C.c_int, [P, C.c_int32]),
    "ontc_load_manifest": (C.c_int, [P, C.c_char_p]),
    "ontc_unload_manifest": (None, [P]),
    "ontc_begin_training": (None, [P, C.c_int32, C.c_int32]),
    "ontc_set_train_options": (C.c_int, [P, C.POINTER(TrainOptions)]),
    "ontc_train": (None, [P, C.c_int32, C.POINTER(TrainProgress)]),
    "ontc_train_until_complete": (None, [P, C.POINTER(TrainProgress)]),
    "ontc_eval": (None, [P, C.POINTER(EvalResults)]),
    "ontc_eval_decoded": (None, [P, C.POINTER(EvalResults)]),
    "ontc_calibrate": (None, [P, C.c_float, C.POINTER(Calibration)]),
    "ontc_get_compressed_data": (None, [P, C.POINTER(CompressedData)]),
    "ontc_get_texture_data": (None, [P, C.POINTER(TextureData)]),
    "ontc_get_mip_dim": (C.c_int32, [P, C.c_int32]),
    "ontc_feature_level_for_lod": (C.c_int32, [P, C.c_int32]),
    "ontc_get_last_error": (C.c_int, [P]),
    "ontc_steps_for_quality": (C.c_int32, [C.c_int32]),
    "ontc_get_step_losses": (C.c_int, [P, C.POINTER(C.c_double), C.c_int32]),
    "ontc_fill_constants": (None, [C.POINTER(CompressedData), C.POINTER(Constants)]),
    "ontc_dump": (C.c_int, [C.c_char_p, C.POINTER(CompressedData)]),
    "ontc_load": (C.c_int, [C.c_char_p, C.POINTER(P), C.POINTER(CompressedData)]),
    "ontc_file_free": (None, [P]),
    "ontc_profile_to_string": (C.c_char_p, [C.c_int32]),
    "ontc_profile_from_string": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32)]),
    "ontc_semantic_to_string": (C.c_char_p, [C.c_int32]),
    "ontc_semantic_from_name": (C.c_int32, [C.c_char_p]),
    "ontc_channel_count_for_semantic": (C.c_int32, [C.c_int32]),
    "ontc_kernel_launch_count": (C.c_int64, [P]),
    "ontc_texels_trained": (C.c_int64, [P]),
    "ontc_version": (C.c_char_p, []),
    "ontc_profile_kernels": (C.c_int, [P, C.c_int32]),
    "ontc_kernel_times": (C.c_int, [P, C.POINTER(KernelTime), C.c_int32]),
    "ontc_debug_tensor": (C.c_int64, [P, C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_int32]),
    "ontc_debug_last_step": (C.c_int, [P, C.POINTER(DebugStep)]),
    "ontc_debug_gradients": (C.c_int, [P, C.POINTER(DebugStep), C.POINTER(C.c_double)]),
    "ontc_debug_tile_costs": (C.c_int, [P, C.POINTER(C.c_float), C.c_int32]),
    "ontc_debug_quantize_pack": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p]),
    "ontc_debug_lanczos_down": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "ontc_debug_lanczos_weights": (C.c_int, [C.c_void_p]),
    "ontc_debug_package": (C.c_int, [P, C.c_int32, C.c_void_p]),
    "ontc_debug_shape": (C.c_int, [P, C.c_void_p]),
    "ontc_debug_disjoint_cover": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]),
    "ontc_debug_cover_op": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32]),
    "ontc_lanczos_down_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "ontc_debug_wait_timeout": (C.c_int, [C.c_int32]),
    "ontc_debug_exact_gradients": (C.c_int, [P, C.c_int32]),
    "ontc_debug_fail_device_alloc": (C.c_int64, [C.c_int64]),
    "ontc_debug_load_image": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_void_p]),
    "ontc_debug_complete": (C.c_int, [P, C.c_void_p]),
    "ontc_debug_decode_features": (C.c_int, [P, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "ontc_train_batch": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(TrainProgress)]),
    "ontc_decoder_create": (C.c_int, [C.POINTER(CompressedData), C.c_int32, C.c_void_p, C.POINTER(C.c_void_p)]),
    "ontc_decoder_destroy": (None, [P]),
    "ontc_decode": (C.c_int, [P, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "ontc_decode_host": (C.c_int, [P, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "ontc_decoder_status": (C.c_int, [P]),
    "ontc_decode_material": (C.c_int, [P, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "ontc_decoder_create_float": (C.c_int, [P, C.c_int32, C.c_void_p, C.POINTER(C.c_void_p)]),
    "ontc_sample_screen": (C.c_int, [P, C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_int32, C.c_void_p]),
}


def declared_symbols(header: Path) -> list[str]:
    """Function names declared in a C header (one declaration per line starting a type)."""
    import re
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(ontc_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def bind(lib: C.CDLL) -> C.CDLL:
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib
