"""ctypes binding of libqsmgpu.so (the C ABI declared in include/qsmgpu.h).

The library is loaded from ``qsm.rs_b200/lib/libqsmgpu.so`` (built in-tree by
``qsm.rs_b200/build.py``).  There is no fallback: if the library is missing the
import fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "lib", "libqsmgpu.so"))

QSM_OK = 0
STATUS_NAMES = {
    0: "QSM_OK",
    1: "QSM_ERR_INVALID_ARGUMENT",
    2: "QSM_ERR_DIMENSION_MISMATCH",
    3: "QSM_ERR_UNSUPPORTED_SIZE",
    4: "QSM_ERR_ALLOC",
    5: "QSM_ERR_CUDA",
    6: "QSM_ERR_INVALID_CONFIG",
    7: "QSM_ERR_NO_DEVICE",
    8: "QSM_ERR_IO",
}

PRECISION_F64 = 0
PRECISION_MIXED = 1
PLANS_COMPILED = 0
PLANS_RUNTIME = 1

c_double_p = C.POINTER(C.c_double)
c_u8_p = C.POINTER(C.c_uint8)
PROGRESS_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_size_t, C.c_size_t)


class QsmGrid(C.Structure):
    _fields_ = [("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
                ("vsx", C.c_double), ("vsy", C.c_double), ("vsz", C.c_double)]


class QsmTvParams(C.Structure):
    _fields_ = [("lambda_", C.c_double), ("rho", C.c_double), ("tol", C.c_double), ("max_iter", C.c_size_t)]


class QsmTkdParams(C.Structure):
    _fields_ = [("threshold", C.c_double)]


class QsmTikhonovParams(C.Structure):
    _fields_ = [("lambda_", C.c_double), ("reg", C.c_int)]


class QsmSharpParams(C.Structure):
    _fields_ = [("threshold", C.c_double), ("radius", C.c_double)]


class QsmVsharpParams(C.Structure):
    _fields_ = [("threshold", C.c_double), ("max_radius", C.c_double), ("min_radius", C.c_double)]


class QsmResharpParams(C.Structure):
    _fields_ = [("radius", C.c_double), ("tik_reg", C.c_double), ("tol", C.c_double), ("max_iter", C.c_size_t)]


class QsmIsmvParams(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_size_t), ("radius", C.c_double)]


class QsmRtsParams(C.Structure):
    _fields_ = [("delta", C.c_double), ("mu", C.c_double), ("rho", C.c_double), ("tol", C.c_double),
                ("max_iter", C.c_size_t), ("lsmr_iter", C.c_size_t)]


class QsmNltvParams(C.Structure):
    _fields_ = [("lambda_", C.c_double), ("mu", C.c_double), ("tol", C.c_double), ("max_iter", C.c_size_t),
                ("newton_iter", C.c_size_t)]


class QsmLinearFitParams(C.Structure):
    _fields_ = [("estimate_offset", C.c_int), ("reliability_threshold_percentile", C.c_double)]


class QsmNiftiHeader(C.Structure):
    _fields_ = [("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t), ("nt", C.c_size_t),
                ("voxel_size", C.c_double * 3), ("affine", C.c_double * 16), ("scl_slope", C.c_double),
                ("scl_inter", C.c_double), ("raw_slope", C.c_double), ("datatype", C.c_int), ("ndim", C.c_int),
                ("big_endian", C.c_int), ("gzip", C.c_int), ("vox_offset", C.c_size_t)]


class QsmIlsqrParams(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_size_t)]


class QsmTgvParams(C.Structure):
    _fields_ = [("alpha1", C.c_float), ("alpha0", C.c_float), ("iterations", C.c_size_t), ("erosions", C.c_size_t),
                ("step_size", C.c_float), ("fieldstrength", C.c_float), ("te", C.c_float), ("tol", C.c_float)]


class QsmVolume(C.Structure):
    _fields_ = [("local_field", C.c_void_p), ("mask", C.c_void_p), ("out_chi", C.c_void_p), ("grid", QsmGrid),
                ("bdir", C.c_double * 3)]


class QsmScanMetadata(C.Structure):
    _fields_ = [("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
                ("vsx", C.c_double), ("vsy", C.c_double), ("vsz", C.c_double),
                ("field_strength", C.c_double), ("b0_direction", C.c_double * 3)]


class QsmInversionConfig(C.Structure):
    _fields_ = [("algorithm", C.c_int), ("tkd", QsmTkdParams), ("tsvd", QsmTkdParams),
                ("tikhonov", QsmTikhonovParams), ("tv", QsmTvParams), ("ilsqr", QsmIlsqrParams),
                ("rts", QsmRtsParams), ("nltv", QsmNltvParams)]


class QsmBgRemovalConfig(C.Structure):
    _fields_ = [("algorithm", C.c_int), ("vsharp", QsmVsharpParams), ("sharp", QsmSharpParams),
                ("resharp", QsmResharpParams), ("ismv", QsmIsmvParams)]


# (name, restype, argtypes)
_SIGS = [
    ("qsm_ctx_create", C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("qsm_ctx_destroy", C.c_int, [C.c_void_p]),
    ("qsm_ctx_set_precision", C.c_int, [C.c_void_p, C.c_int]),
    ("qsm_ctx_get_precision", C.c_int, [C.c_void_p]),
    ("qsm_ctx_set_plan_mode", C.c_int, [C.c_void_p, C.c_int]),
    ("qsm_ctx_get_plan_mode", C.c_int, [C.c_void_p]),
    ("qsm_ctx_set_krylov_precision", C.c_int, [C.c_void_p, C.c_int]),
    ("qsm_ctx_get_krylov_precision", C.c_int, [C.c_void_p]),
    ("qsm_ctx_set_input_check", C.c_int, [C.c_void_p, C.c_int]),
    ("qsm_ctx_set_autotune", C.c_int, [C.c_void_p, C.c_int]),
    ("qsm_ctx_force_launch_shape", C.c_int, [C.c_void_p, C.c_int]),
    ("qsm_ctx_autotune_count", C.c_size_t, [C.c_void_p]),
    ("qsm_ctx_autotune_entry", C.c_int, [C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t, C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_size_t,
                                         C.POINTER(C.c_size_t)]),
    ("qsm_ctx_inject_alloc_failure", C.c_int, [C.c_void_p, C.c_longlong]),
    ("qsm_ctx_release_workspace", C.c_int, [C.c_void_p]),
    ("qsm_last_error", C.c_char_p, [C.c_void_p]),
    ("qsm_ctx_kernel_launches", C.c_uint64, [C.c_void_p]),
    ("qsm_ctx_stream", C.c_void_p, [C.c_void_p]),
    ("qsm_version", C.c_char_p, []),
    ("qsm_ctx_set_profiling", C.c_int, [C.c_void_p, C.c_int]),
    ("qsm_ctx_profile_reset", C.c_int, [C.c_void_p]),
    ("qsm_ctx_profile_count", C.c_size_t, [C.c_void_p]),
    ("qsm_ctx_profile_entry", C.c_int, [C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t,
                                        C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    ("qsm_grid_supported", C.c_int, [C.POINTER(QsmGrid)]),
    ("qsm_tv_params_default", None, [C.POINTER(QsmTvParams)]),
    ("qsm_ilsqr_params_default", None, [C.POINTER(QsmIlsqrParams)]),
    ("qsm_rts_params_default", None, [C.POINTER(QsmRtsParams)]),
    ("qsm_nltv_params_default", None, [C.POINTER(QsmNltvParams)]),
    ("qsm_nltv", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), c_double_p, C.POINTER(QsmNltvParams),
                           PROGRESS_FN, C.c_void_p, c_double_p]),
    ("qsm_nltv_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), c_double_p,
                                  C.POINTER(QsmNltvParams), PROGRESS_FN, C.c_void_p, C.c_void_p]),
    ("qsm_rts", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), c_double_p, C.POINTER(QsmRtsParams),
                          PROGRESS_FN, C.c_void_p, c_double_p]),
    ("qsm_rts_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), c_double_p,
                                 C.POINTER(QsmRtsParams), PROGRESS_FN, C.c_void_p, C.c_void_p]),
    ("qsm_tv_admm_unrolled_vjp_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), c_double_p,
                                                  C.c_double, C.c_double, C.c_size_t, C.c_size_t, C.c_void_p,
                                                  C.c_void_p, C.c_void_p, c_double_p]),
    ("qsm_dipole_forward_device", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), c_double_p, C.c_void_p]),
    ("qsm_tv_admm_batch", C.c_int, [C.c_void_p, C.POINTER(QsmVolume), C.c_size_t, C.POINTER(QsmTvParams),
                                    PROGRESS_FN, C.c_void_p, C.POINTER(C.c_size_t)]),
    ("qsm_tv_admm_batch_device", C.c_int, [C.c_void_p, C.POINTER(QsmVolume), C.c_size_t, C.POINTER(QsmTvParams),
                                           PROGRESS_FN, C.c_void_p, C.POINTER(C.c_size_t)]),
    ("qsm_batch_partition", C.c_int, [C.POINTER(QsmGrid), C.POINTER(C.c_size_t), C.c_size_t, C.c_size_t,
                                      C.POINTER(C.c_uint32), C.POINTER(C.c_double)]),
    ("qsm_tkd_batch_device", C.c_int, [C.c_void_p, C.POINTER(QsmVolume), C.c_size_t, C.POINTER(QsmTkdParams)]),
    ("qsm_apply_reference", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.c_size_t, C.c_int, c_double_p]),
    ("qsm_run_tgv", C.c_int, [C.c_void_p, C.POINTER(c_double_p), C.c_size_t, C.c_size_t, c_u8_p,
                              C.POINTER(QsmScanMetadata), C.POINTER(QsmTgvParams), C.c_int, PROGRESS_FN,
                              C.c_void_p, c_double_p]),
    ("qsm_ismv_params_default", None, [C.POINTER(QsmIsmvParams)]),
    ("qsm_ismv", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), C.POINTER(QsmIsmvParams),
                           PROGRESS_FN, C.c_void_p, c_double_p, c_u8_p]),
    ("qsm_ismv_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), C.POINTER(QsmIsmvParams),
                                  PROGRESS_FN, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("qsm_resharp_params_default", None, [C.POINTER(QsmResharpParams)]),
    ("qsm_resharp", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), C.POINTER(QsmResharpParams),
                              PROGRESS_FN, C.c_void_p, c_double_p, c_u8_p]),
    ("qsm_resharp_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid),
                                     C.POINTER(QsmResharpParams), PROGRESS_FN, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("qsm_cg_kspace_normal_device", C.c_int, [C.c_void_p, C.POINTER(QsmGrid), C.c_void_p, C.c_void_p, C.c_double,
                                              C.c_void_p, C.c_void_p, C.c_double, C.c_size_t, PROGRESS_FN,
                                              C.c_void_p, C.c_void_p]),
    ("qsm_tgv_params_default", None, [C.POINTER(QsmTgvParams)]),
    ("qsm_tgv_qsm", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), C.POINTER(QsmTgvParams),
                              c_double_p, PROGRESS_FN, C.c_void_p, c_double_p]),
    ("qsm_tgv_qsm_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid),
                                     C.POINTER(QsmTgvParams), c_double_p, PROGRESS_FN, C.c_void_p, C.c_void_p]),
    ("qsm_tgv_oblique_stencil", C.c_int, [c_double_p, c_double_p, C.POINTER(C.c_float)]),
    ("qsm_prctile_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, c_double_p, C.c_size_t,
                                     c_double_p]),
    ("qsm_ilsqr", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), c_double_p,
                            C.POINTER(QsmIlsqrParams), PROGRESS_FN, C.c_void_p, c_double_p, c_double_p, c_double_p,
                            c_double_p]),
    ("qsm_ilsqr_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), c_double_p,
                                   C.POINTER(QsmIlsqrParams), PROGRESS_FN, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    ("qsm_ilsqr_lsqr_operator_device", C.c_int, [C.c_void_p, C.POINTER(QsmGrid), c_double_p, C.c_void_p,
                                                 C.c_void_p, C.c_void_p]),
    ("qsm_tkd_params_default", None, [C.POINTER(QsmTkdParams)]),
    ("qsm_tikhonov_params_default", None, [C.POINTER(QsmTikhonovParams)]),
    ("qsm_sharp_params_default", None, [C.POINTER(QsmSharpParams)]),
    ("qsm_vsharp_params_default", None, [C.POINTER(QsmVsharpParams)]),
    ("qsm_tv_admm", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), c_double_p,
                              C.POINTER(QsmTvParams), PROGRESS_FN, C.c_void_p, c_double_p]),
    ("qsm_tv_admm_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), c_double_p,
                                     C.POINTER(QsmTvParams), PROGRESS_FN, C.c_void_p, C.c_void_p]),
    ("qsm_tv_last_iterations", C.c_size_t, [C.c_void_p]),
    ("qsm_tkd", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), c_double_p,
                          C.POINTER(QsmTkdParams), c_double_p]),
    ("qsm_tkd_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), c_double_p,
                                 C.POINTER(QsmTkdParams), C.c_void_p]),
    ("qsm_tkd_device_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), c_double_p,
                                         C.POINTER(QsmTkdParams), C.c_void_p, C.c_void_p]),
    ("qsm_tsvd", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), c_double_p,
                           C.POINTER(QsmTkdParams), c_double_p]),
    ("qsm_tsvd_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), c_double_p,
                                  C.POINTER(QsmTkdParams), C.c_void_p]),
    ("qsm_tikhonov", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), c_double_p,
                               C.POINTER(QsmTikhonovParams), c_double_p]),
    ("qsm_tikhonov_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid), c_double_p,
                                      C.POINTER(QsmTikhonovParams), C.c_void_p]),
    ("qsm_dipole_forward", C.c_int, [C.c_void_p, c_double_p, C.POINTER(QsmGrid), c_double_p, c_double_p]),
    ("qsm_laplacian_unwrap", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), c_double_p]),
    ("qsm_laplacian_unwrap_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid),
                                              C.c_void_p]),
    ("qsm_smv", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), C.c_double, c_double_p, c_u8_p]),
    ("qsm_sharp", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), C.POINTER(QsmSharpParams),
                            c_double_p, c_u8_p]),
    ("qsm_vsharp", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), C.POINTER(QsmVsharpParams),
                             PROGRESS_FN, C.c_void_p, c_double_p, c_u8_p]),
    ("qsm_vsharp_with_radii", C.c_int, [C.c_void_p, c_double_p, c_u8_p, C.POINTER(QsmGrid), c_double_p,
                                        C.c_size_t, C.c_double, PROGRESS_FN, C.c_void_p, c_double_p, c_u8_p]),
    ("qsm_vsharp_with_radii_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(QsmGrid),
                                               c_double_p, C.c_size_t, C.c_double, PROGRESS_FN, C.c_void_p,
                                               C.c_void_p, C.c_void_p]),
    ("qsm_inversion_config_default", None, [C.POINTER(QsmInversionConfig)]),
    ("qsm_bg_removal_config_default", None, [C.POINTER(QsmBgRemovalConfig)]),
    ("qsm_run_dipole_inversion", C.c_int, [C.c_void_p, c_double_p, C.c_size_t, c_u8_p,
                                           C.POINTER(QsmScanMetadata), C.POINTER(QsmInversionConfig),
                                           PROGRESS_FN, C.c_void_p, c_double_p]),
    ("qsm_run_bg_removal", C.c_int, [C.c_void_p, c_double_p, C.c_size_t, c_u8_p, C.POINTER(QsmScanMetadata),
                                     C.POINTER(QsmBgRemovalConfig), PROGRESS_FN, C.c_void_p, c_double_p,
                                     c_u8_p]),
    ("qsm_fft3d_real", C.c_int, [C.c_void_p, c_double_p, C.POINTER(QsmGrid), c_double_p]),
    ("qsm_nifti_parse_header", C.c_int, [c_u8_p, C.c_size_t, C.POINTER(QsmNiftiHeader), C.c_char_p, C.c_size_t]),
    ("qsm_nifti_load", C.c_int, [c_u8_p, C.c_size_t, C.c_int, c_double_p, C.c_size_t, C.POINTER(QsmNiftiHeader),
                                 C.c_char_p, C.c_size_t]),
    ("qsm_nifti_save", C.c_int, [c_double_p, C.c_size_t, C.c_size_t, C.c_size_t, c_double_p, c_double_p, C.c_int,
                                 c_u8_p, C.c_size_t, C.POINTER(C.c_size_t), C.c_char_p, C.c_size_t]),
    ("qsm_nifti_read_dims", C.c_int, [C.c_char_p, C.POINTER(C.c_size_t), C.c_char_p, C.c_size_t]),
    ("qsm_nifti_read_file_header", C.c_int, [C.c_char_p, C.POINTER(QsmNiftiHeader), C.c_char_p, C.c_size_t]),
    ("qsm_nifti_read_file", C.c_int, [C.c_char_p, C.c_int, c_double_p, C.c_size_t, C.POINTER(QsmNiftiHeader),
                                      C.c_char_p, C.c_size_t]),
    ("qsm_nifti_save_file", C.c_int, [C.c_char_p, c_double_p, C.c_size_t, C.c_size_t, C.c_size_t, c_double_p,
                                      c_double_p, C.c_char_p, C.c_size_t]),
    ("qsm_nifti_load_device", C.c_int, [C.c_void_p, c_u8_p, C.c_size_t, C.c_int, C.c_void_p, C.c_size_t,
                                        C.POINTER(QsmNiftiHeader)]),
    ("qsm_nifti_save_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t, c_double_p,
                                        c_double_p, C.c_int, c_u8_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    ("qsm_linear_fit_params_default", None, [C.POINTER(QsmLinearFitParams)]),
    ("qsm_calculate_b0_weighted", C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p, C.c_size_t, c_u8_p,
                                            C.c_size_t, C.c_int, c_double_p]),
    ("qsm_calculate_b0_weighted_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, c_double_p, C.c_size_t,
                                                   C.c_void_p, C.c_size_t, C.c_int, C.c_void_p]),
    ("qsm_multi_echo_linear_fit", C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p, C.c_size_t, c_u8_p,
                                            C.c_size_t, C.POINTER(QsmLinearFitParams), c_double_p, c_double_p,
                                            c_double_p, c_u8_p]),
    ("qsm_multi_echo_linear_fit_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, c_double_p, C.c_size_t,
                                                   C.c_void_p, C.c_size_t, C.POINTER(QsmLinearFitParams),
                                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
]

EXPORTED_SYMBOLS = [s[0] for s in _SIGS]

_lib = None


def load():
    """Load libqsmgpu.so and declare every signature; raises if the build is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libqsmgpu.so not found at {LIB_PATH}; build it with `python qsm.rs_b200/build.py` "
            "(the CUDA library is required: there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in _SIGS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
