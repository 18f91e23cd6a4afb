"""ctypes binding of libmoist2d_sm100a.so (the CUDA library). There is no CPU fallback: if the
library or a CUDA device is missing, calls raise."""
import ctypes as C
import os

from .abi import (moist_adjoint_grad, moist_adjoint_seed, moist_bubble, moist_init_profile, moist_params,
                  moist_state_host)

_HERE = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.path.join(_HERE, "libmoist2d_sm100a.so")
_lib = None

EXPORTS = ("moist_abi_version", "moist_status_string", "moist_ctx_create", "moist_ctx_destroy",
           "moist_last_error", "moist_nan_field", "moist_upload_state", "moist_download_state",
           "moist_rk3_step", "moist_compute_step", "moist_cloud_microphysics",
           "moist_rain_sedimentation", "moist_implicit_correction", "moist_eval_helper",
           "moist_budget", "moist_stream", "moist_synchronize", "moist_time_steps",
           "moist_rk3_step_host", "moist_step_profile", "moist_set_device",
           "moist_implicit_correction_noalloc", "moist_tracer_pass_counts", "moist_batch_create",
           "moist_batch_destroy", "moist_batch_member", "moist_batch_upload", "moist_batch_download",
           "moist_batch_step", "moist_batch_time_steps", "moist_batch_last_error", "moist_batch_nan_member",
           "moist_batch_profile", "moist_adjoint_run", "moist_batch_adjoint_run",
           "moist_autotune", "moist_batch_autotune", "moist_history_diagnostics", "moist_io_last_error",
           "moist_history_create", "moist_history_append", "moist_history_append_host",
           "moist_history_close", "moist_restart_read", "moist_surface_fluxes", "moist_gray_radiation",
           "moist_set_wait_limit", "moist_uniform", "moist_init_state", "moist_init_warm_bubble",
           "moist_init_sounding", "moist_sounding_bubble_row", "moist_ensemble_member_draw",
           "moist_tracer_pass_trace", "moist_set_adjoint_tapes", "moist_batch_set_adjoint_tapes")


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO_PATH):
            raise RuntimeError("libmoist2d_sm100a.so is not built (run __graft_entry__.build() or "
                               "make -C moist2d_b200/csrc); there is no CPU fallback")
        L = C.CDLL(SO_PATH)
        P, S, V, I, D = C.POINTER(moist_params), C.POINTER(moist_state_host), C.c_void_p, C.c_int, C.c_double
        Ctx = C.c_void_p
        L.moist_abi_version.restype = I
        L.moist_status_string.argtypes = [I]
        L.moist_status_string.restype = C.c_char_p
        L.moist_ctx_create.argtypes = [P, I, I, C.POINTER(Ctx)]
        L.moist_ctx_destroy.argtypes = [Ctx]
        L.moist_last_error.argtypes = [Ctx]
        L.moist_last_error.restype = C.c_char_p
        L.moist_nan_field.argtypes = [Ctx]
        L.moist_upload_state.argtypes = [Ctx, S]
        L.moist_download_state.argtypes = [Ctx, S]
        L.moist_rk3_step.argtypes = [Ctx, I]
        L.moist_compute_step.argtypes = [Ctx, C.POINTER(V), S, D, I]
        L.moist_cloud_microphysics.argtypes = [Ctx]
        L.moist_rain_sedimentation.argtypes = [Ctx, V]
        L.moist_surface_fluxes.argtypes = [Ctx]
        L.moist_gray_radiation.argtypes = [Ctx]
        L.moist_implicit_correction.argtypes = [P, I, I, V, V, V, V, D]
        L.moist_eval_helper.argtypes = [P, I, I, I, C.POINTER(D), C.POINTER(D)]
        L.moist_budget.argtypes = [Ctx, C.POINTER(D)]
        L.moist_stream.argtypes = [Ctx]
        L.moist_stream.restype = V
        L.moist_synchronize.argtypes = [Ctx]
        L.moist_time_steps.argtypes = [Ctx, I, C.POINTER(C.c_float)]
        L.moist_rk3_step_host.argtypes = [Ctx, S, I]
        L.moist_set_device.argtypes = [I]
        L.moist_tracer_pass_counts.argtypes = [Ctx, C.POINTER(I), I]
        L.moist_set_wait_limit.argtypes = [Ctx, C.c_longlong]
        L.moist_tracer_pass_trace.argtypes = [Ctx, I, I, C.POINTER(C.c_longlong), C.POINTER(I), C.POINTER(I)]
        L.moist_implicit_correction_noalloc.argtypes = [P, I, I, I, V, V, V, V, D, V, C.c_char_p,
                                                        C.c_size_t]
        L.moist_step_profile.argtypes = [Ctx, I, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                         C.POINTER(C.c_longlong)]
        B = C.c_void_p
        L.moist_batch_create.argtypes = [P, I, I, I, C.POINTER(B)]
        L.moist_batch_destroy.argtypes = [B]
        L.moist_batch_member.argtypes = [B, I]
        L.moist_batch_member.restype = Ctx
        L.moist_batch_upload.argtypes = [B, I, S]
        L.moist_batch_download.argtypes = [B, I, S]
        L.moist_batch_step.argtypes = [B, I]
        L.moist_batch_time_steps.argtypes = [B, I, C.POINTER(C.c_float)]
        L.moist_batch_last_error.argtypes = [B]
        L.moist_batch_last_error.restype = C.c_char_p
        L.moist_batch_nan_member.argtypes = [B]
        L.moist_batch_profile.argtypes = [B, I, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.moist_adjoint_run.argtypes = [Ctx, I, I, C.POINTER(moist_adjoint_seed), C.POINTER(moist_adjoint_grad)]
        L.moist_autotune.argtypes = [Ctx, I, C.c_char_p, C.c_size_t]
        L.moist_history_diagnostics.argtypes = [Ctx, C.POINTER(V), C.POINTER(D)]
        L.moist_batch_autotune.argtypes = [B, I, C.c_char_p, C.c_size_t]
        L.moist_batch_adjoint_run.argtypes = [B, I, I, C.POINTER(moist_adjoint_seed), C.POINTER(moist_adjoint_grad), I]
        L.moist_set_adjoint_tapes.argtypes = [Ctx, I]
        L.moist_batch_set_adjoint_tapes.argtypes = [B, I]
        H = C.c_void_p
        L.moist_io_last_error.restype = C.c_char_p
        L.moist_history_create.argtypes = [C.c_char_p, P, I, C.POINTER(H)]
        L.moist_history_append.argtypes = [H, D, Ctx]
        L.moist_history_append_host.argtypes = [H, D, S, C.POINTER(V)]
        L.moist_history_close.argtypes = [H]
        L.moist_restart_read.argtypes = [C.c_char_p, P, I, S]
        U32 = C.c_uint32
        Bp = C.POINTER(moist_bubble)
        L.moist_uniform.argtypes = [U32, U32, C.c_int64, C.POINTER(C.c_uint64), C.POINTER(D)]
        L.moist_init_state.argtypes = [P, I, C.POINTER(moist_init_profile), U32, S]
        L.moist_init_warm_bubble.argtypes = [P, I, U32, S]
        L.moist_init_sounding.argtypes = [P, I, Bp, I, S]
        L.moist_sounding_bubble_row.argtypes = [U32, I, D, D, D, D, D, D, Bp]
        L.moist_ensemble_member_draw.argtypes = [U32, I, C.POINTER(I), I, C.POINTER(I), I, D, D, D, D, D, D,
                                                 C.POINTER(I), C.POINTER(I), Bp]
        _lib = L
    return _lib
