"""ctypes binding of ``libomega_b200.so`` (the C-ABI of include/omega_b200.h).

The library is loaded from ``omega_b200/lib``; there is no fallback: if it is
missing or fails to load, every projector call raises.  Build it with
``python -m omega_b200.build``.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libomega_b200.so")

OMB_ABI_VERSION = 5
OMB_PET_SINOGRAM = 0
OMB_CT_PANEL = 1
OMB_PET_LISTMODE = 2
OMB_PET_INDEXED = 3
OMB_READ_FP32 = 0
OMB_READ_BF16 = 1
OMB_BP_FLOAT_ATOMIC = 0
OMB_BP_FIXED64 = 1
OMB_BP_RAY = 2

_c_float_p = ctypes.POINTER(ctypes.c_float)
_c_i64_p = ctypes.POINTER(ctypes.c_int64)


class GeometryDesc(ctypes.Structure):
    """Mirror of ``omb_geometry_desc`` (explicit natural layout, no packing)."""
    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("abi_version", ctypes.c_uint32),
        ("modality", ctypes.c_int32),
        ("fp_type", ctypes.c_int32),
        ("bp_type", ctypes.c_int32),
        ("nx", ctypes.c_uint32),
        ("ny", ctypes.c_uint32),
        ("nz", ctypes.c_uint32),
        ("dx", ctypes.c_float),
        ("dy", ctypes.c_float),
        ("dz", ctypes.c_float),
        ("bx", ctypes.c_float),
        ("by", ctypes.c_float),
        ("bz", ctypes.c_float),
        ("n_rows_d", ctypes.c_uint32),
        ("n_cols_d", ctypes.c_uint32),
        ("n_proj", ctypes.c_int64),
        ("n_subsets", ctypes.c_int32),
        ("subset_type", ctypes.c_int32),
        ("n_meas", _c_i64_p),
        ("xy", _c_float_p),
        ("n_xy", ctypes.c_int64),
        ("z", _c_float_p),
        ("n_z", ctypes.c_int64),
        ("dpitch_x", ctypes.c_float),
        ("dpitch_y", ctypes.c_float),
        ("global_factor", ctypes.c_float),
        ("epps", ctypes.c_float),
        ("tof_bins", ctypes.c_int32),
        ("sigma_x", ctypes.c_float),
        ("tof_centers", _c_float_p),
        ("dL", ctypes.c_float),
        ("d_scale4", ctypes.c_float * 3),
        ("d_size5", ctypes.c_float * 2),
        ("d_scale5", ctypes.c_float * 3),
        ("kerroin", ctypes.c_float),
        ("fixed64_workspace", ctypes.c_int32),
        ("tr_index", ctypes.POINTER(ctypes.c_uint16)),
        ("ax_index", ctypes.POINTER(ctypes.c_uint16)),
        ("n_rays_xy", ctypes.c_int32),
        ("n_rays_z", ctypes.c_int32),
        ("tube_width", ctypes.c_float),
        ("tube_radius", ctypes.c_float),
        ("orth_xy", ctypes.c_int32),
        ("orth_z", ctypes.c_int32),
        ("vol_bmin", ctypes.c_float),
        ("vol_bmax", ctypes.c_float),
        ("vol_vmax", ctypes.c_float),
        ("vol_v", ctypes.POINTER(ctypes.c_float)),
        ("n_vol_v", ctypes.c_int64),
    ]


class ReconParams(ctypes.Structure):
    """Mirror of ``omb_recon_params``."""
    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("algorithm", ctypes.c_int32),
        ("n_iter", ctypes.c_int32),
        ("beta", ctypes.c_float),
        ("tv_smoothing", ctypes.c_float),
        ("tau", ctypes.c_float),
        ("sigma", ctypes.c_float),
        ("theta", ctypes.c_float),
        ("power_iterations", ctypes.c_int32),
        ("positivity", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
        ("tau_used", ctypes.c_float),
        ("rdp_gamma", ctypes.c_float),
        ("prior", ctypes.c_int32),
        ("prior_window", ctypes.c_void_p),
        ("prior_g", ctypes.c_int32 * 3),
        ("huber_delta", ctypes.c_float),
        ("relaxation", ctypes.c_void_p),
        ("momentum", ctypes.c_void_p),
        ("upper_bound", ctypes.c_float),
        ("nlm_type", ctypes.c_int32),
        ("nlm_patch", ctypes.c_int32 * 3),
        ("nlm_h", ctypes.c_float),
        ("nlm_gaussian", ctypes.c_void_p),
        ("nlm_ref", ctypes.c_void_p),
        ("ggmrf", ctypes.c_float * 3),
        ("nlm_adaptive", ctypes.c_int32),
        ("nlm_adaptive_s", ctypes.c_float),
        ("precond", ctypes.c_int32),
        ("mrp_no_norm", ctypes.c_int32),
        ("ggmrf_weights", ctypes.c_void_p),
        ("hyper_weights", ctypes.c_void_p),
        ("hyper_delta", ctypes.c_float),
        ("wmean_weights", ctypes.c_void_p),
        ("wmean_type", ctypes.c_int32),
        ("tv_variant", ctypes.c_int32),
        ("tv_sigma", ctypes.c_float),
        ("tv_c", ctypes.c_float),
        ("tv_ref", ctypes.c_void_p),
        ("wmean_wsum", ctypes.c_float),
        ("tv_prox", ctypes.c_int32),
        ("sigma2", ctypes.c_float),
        ("l2_ball", ctypes.c_int32),
        ("diff_type", ctypes.c_int32),
        ("precond_ref", ctypes.c_void_p),
        ("precond_alpha", ctypes.c_void_p),
        ("precond_grad", ctypes.c_int32),
        ("grad_v", ctypes.c_float * 2),
        ("grad_iters", ctypes.c_int32 * 2),
        ("precond_curv", ctypes.c_int32),
        ("precond_meas", ctypes.c_int32),
        ("pkma_relax", ctypes.c_int32),
        ("filter_h", ctypes.c_void_p),
        ("filter_hinv", ctypes.c_void_p),
        ("filter_nf", ctypes.c_int32),
        ("filter_rows", ctypes.c_int32),
        ("filter_iters", ctypes.c_int32),
        ("tau_filt", ctypes.c_float),
        ("tgv", ctypes.c_int32),
        ("alpha0_tgv", ctypes.c_float),
        ("alpha1_tgv", ctypes.c_float),
        ("img_filter_h", ctypes.c_void_p),
        ("img_filter_nf", ctypes.c_int32),
        ("tau_used2", ctypes.c_float),
        ("ad_dt", ctypes.c_float),
        ("ad_k", ctypes.c_float),
        ("ad_niter", ctypes.c_int32),
        ("ad_flux", ctypes.c_int32),
        ("ad_diffusion", ctypes.c_int32),
        ("rdp_edge", ctypes.c_int32),
        ("lfilter_weights", ctypes.c_void_p),
        ("fmh_weights", ctypes.c_void_p),
    ]


OMB_RECON_OSEM = 1
OMB_RECON_PDHG_TV = 2
OMB_RECON_OSL_OSEM = 3
OMB_RECON_ROSEM = 4
OMB_RECON_RAMLA = 5
OMB_RECON_BSREM = 6
OMB_RECON_ROSEM_MAP = 7
OMB_RECON_PKMA = 8
OMB_RECON_MRAMLA = 9
OMB_RECON_MBSREM = 10
OMB_PRIOR_RDP = 1
OMB_PRIOR_QUAD = 2
OMB_PRIOR_HUBER = 3
OMB_PRIOR_NLM = 4
OMB_PRIOR_MRP = 5
OMB_PRIOR_TV = 6
OMB_TV_PLAIN, OMB_TV_SATV, OMB_TV_W1, OMB_TV_ANAT1, OMB_TV_ANAT2, OMB_TV_APLS = range(6)
OMB_PRIOR_GGMRF = 7
OMB_PRIOR_HYPERBOLIC = 8
OMB_PRIOR_WMEAN = 9
OMB_PRIOR_AD = 10
OMB_PRIOR_LFILTER = 11
OMB_PRIOR_FMH = 12


class Tuning(ctypes.Structure):
    """Mirror of ``omb_tuning``."""
    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("siddon_blocks_per_sm", ctypes.c_int32),
        ("siddon_frames_per_walk", ctypes.c_int32),
        ("bdd_fp_columns", ctypes.c_int32),
        ("bdd_bp_zrun", ctypes.c_int32),
        ("bdd_fp_block_rows", ctypes.c_int32),
        ("bdd_bp_block_rows", ctypes.c_int32),
        ("siddon_frame_layout", ctypes.c_int32),
        ("siddon_fp_steps", ctypes.c_int32),
        ("bdd_fp_staged", ctypes.c_int32),
        ("bdd_bp_staged", ctypes.c_int32),
        ("siddon_bp_matrix", ctypes.c_int32),
    ]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_[1:]}


_v, _i32, _i64, _f = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float

# (name, restype, argtypes) of every exported entry point of include/*.h
EXPORTS = [
    ("omb_abi_version", ctypes.c_int, []),
    ("omb_last_error", ctypes.c_char_p, []),
    ("omb_create", ctypes.c_int, [ctypes.POINTER(GeometryDesc), ctypes.POINTER(ctypes.c_void_p)]),
    ("omb_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("omb_measurement_count", ctypes.c_int64, [ctypes.c_void_p, ctypes.c_int32]),
    ("omb_image_count", ctypes.c_int64, [ctypes.c_void_p]),
    ("omb_forward", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_backward", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ("omb_forward_frames", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                          ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    ("omb_backward_frames", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                           ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    ("omb_osem_subset", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_sensitivity", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_osem_subset_frames", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                              ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_loglik", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_float,
                                  ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_reduce_workspace_bytes", ctypes.c_size_t, [ctypes.c_int64]),
    ("omb_backward_fixed64_noalloc", ctypes.c_int, [ctypes.POINTER(GeometryDesc), ctypes.c_int32, ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_pdhg_iteration", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_pdhg_dual", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                     ctypes.c_float, ctypes.c_void_p]),
    ("omb_pdhg_primal", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_float, ctypes.c_int32, ctypes.c_void_p]),
    ("omb_power_method", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                        ctypes.c_void_p]),
    ("omb_power_workspace_bytes", ctypes.c_size_t, []),
    ("omb_set_read_precision", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    ("omb_take_device_error", ctypes.c_int, []),
    ("omb_osl_subset", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]),
    ("omb_rosem_subset", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p]),
    ("omb_ramla_subset", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_float, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p]),
    ("omb_pkma_subset", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_int32,
                                       ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]),
    ("omb_mbsrem_subset", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_int32,
                                         ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    ("omb_precond_image", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_map_step", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_void_p]),
    ("omb_wmean_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_void_p, ctypes.c_float, ctypes.c_int32, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_int32, ctypes.c_void_p]),
    ("omb_hyperbolic_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                               ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                               ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_void_p]),
    ("omb_ggmrf_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_void_p]),
    ("omb_tv_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_void_p]),
    ("omb_tv_gradient_ex", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                                          ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_row_filter", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64,
                                      ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ("omb_image_filter", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ("omb_proxtv_dual", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_void_p]),
    ("omb_proxtv_divergence", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    ("omb_proxtgv_step", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                                        ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_void_p]),
    ("omb_ad_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                                       ctypes.c_void_p]),
    ("omb_mrp_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_float, ctypes.c_float, ctypes.c_int32, ctypes.c_void_p]),
    ("omb_lfilter_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                                            ctypes.c_void_p]),
    ("omb_fmh_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                                        ctypes.c_void_p]),
    ("omb_nlm_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                        ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p, ctypes.c_float,
                                        ctypes.c_float, ctypes.c_float, ctypes.c_int32, ctypes.c_float,
                                        ctypes.POINTER(ctypes.c_float), ctypes.c_int32, ctypes.c_float,
                                        ctypes.c_void_p]),
    ("omb_psf_convolve", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_void_p]),
    ("omb_rdp_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                        ctypes.c_void_p]),
    ("omb_rdp_gradient_ex", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                        ctypes.c_int32, ctypes.c_void_p]),
    ("omb_reconstruct", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ReconParams), ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_set_randoms", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    ("omb_set_corrections", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                           ctypes.c_int64, ctypes.c_void_p]),
    ("omb_get_tuning", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Tuning)]),
    ("omb_set_tuning", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Tuning)]),
    ("omb_autotune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(Tuning),
                                    ctypes.c_void_p]),
    ("omb_system_matrix_nnz", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]),
    ("omb_intersection_count", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64),
                                              ctypes.c_void_p]),
    ("omb_batch_create", ctypes.c_int, [ctypes.POINTER(GeometryDesc), ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    ("omb_batch_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("omb_batch_image_offset", ctypes.c_int64, [ctypes.c_void_p, ctypes.c_int32]),
    ("omb_batch_measurement_offset", ctypes.c_int64, [ctypes.c_void_p, ctypes.c_int32]),
    ("omb_batch_forward", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("omb_batch_backward", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    # learned warm start (include/omega_b200_unet.h)
    ("omb_unet_conv", ctypes.c_int, [_i32, _i32, _v, _v, _v, _v, _v, _i32, _i32, _i32, _i32, _i32, _v]),
    ("omb_unet_conv_tc", ctypes.c_int, [_i32, _i32, _v, _v, _v, _v, _v, _i32, _i32, _i32, _i32, _i32, _v]),
    ("omb_unet_take_error", ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)]),
    ("omb_unet_conv_wgrad", ctypes.c_int, [_i32, _i32, _v, _v, _v, _i32, _i32, _i32, _i32, _v]),
    ("omb_unet_conv_wgrad_tc", ctypes.c_int, [_i32, _i32, _v, _v, _v, _i32, _i32, _i32, _i32, _v]),
    ("omb_unet_bias_grad", ctypes.c_int, [_i32, _v, _v, _i64, _v]),
    ("omb_unet_flip_weights", ctypes.c_int, [_v, _v, _i32, _i32, _v]),
    ("omb_unet_avgpool", ctypes.c_int, [_v, _v, _i32, _i32, _i32, _i32, _i32, _i32, _v]),
    ("omb_unet_up_concat", ctypes.c_int, [_v, _v, _v, _i32, _i32, _i32, _i32, _i32, _i32, _v]),
    ("omb_unet_up_concat_bwd", ctypes.c_int, [_v, _v, _v, _i32, _i32, _i32, _i32, _i32, _i32, _v]),
    ("omb_unet_relu_mask", ctypes.c_int, [_v, _v, _i64, _v]),
    ("omb_unet_make_input", ctypes.c_int, [_v, _i64, _v, _v, _f, _v, _i32, _i32, _i32, _i32, _i32, _v]),
    ("omb_unet_head_fwd", ctypes.c_int, [_v, _v, _v, _v, _v, _i64, _v]),
    ("omb_unet_head_bwd", ctypes.c_int, [_v, _v, _v, _i64, _v, _v, _v, _v, _v, _v, _i32, _i32, _i32, _i32, _i32,
                                         _v]),
    ("omb_unet_head_out", ctypes.c_int, [_v, _v, _v, _i64, _f, _i32, _i32, _i32, _i32, _i32, _v]),
    ("omb_unet_adam", ctypes.c_int, [_v, _v, _v, _v, _v, _i64, _f, _f, _f, _i32, _f, _v]),
    ("omb_unet_to_bf16", ctypes.c_int, [_v, _v, _i64, _v]),
]

_lib = None
_lock = threading.Lock()


class NativeError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, fn, status, msg):
        super().__init__(f"{fn} failed with status {status}: {msg}")
        self.status = status


def lib():
    """The loaded library (raises if it cannot be loaded: no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"omega_b200 native library not found at {LIB_PATH}; "
                                   "build it with `python -m omega_b200.build`")
            L = ctypes.CDLL(LIB_PATH)
            for name, res, args in EXPORTS:
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            if L.omb_abi_version() != OMB_ABI_VERSION:
                raise RuntimeError("omega_b200 native library ABI version mismatch")
            _lib = L
    return _lib


def check(fn_name, status):
    if status != 0:
        msg = lib().omb_last_error().decode(errors="replace")
        raise NativeError(fn_name, status, msg)


def check_device(what):
    """Reads and clears the device error word of the staged type-5 kernels
    (synchronises the device).  A nonzero word means a bounded wait on a
    staged copy ran out: the results of the calls since the last read are
    void, and this raises NativeError."""
    v = lib().omb_take_device_error()
    if v < 0:
        check("omb_take_device_error", v)
    if v:
        raise NativeError(what, v, "a staged kernel's bounded wait ran out; the results since the last check "
                                   "are void")


def call(fn_name, *args):
    """Calls an int-returning entry point and raises NativeError on failure."""
    st = getattr(lib(), fn_name)(*args)
    check(fn_name, st)
    return st


def f32_ptr(a: np.ndarray):
    return a.ctypes.data_as(_c_float_p)


def i64_ptr(a: np.ndarray):
    return a.ctypes.data_as(_c_i64_p)
