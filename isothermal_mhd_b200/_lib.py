"""ctypes binding of libimhd.so (the C ABI declared in include/imhd.h).

The library is built in-tree by ``isothermal_mhd_b200.build``.  Loading fails
loudly when it is missing; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libimhd.so")

IMHD_OK = 0
IMHD_E_PHYSICS = 4
ERRORS = {1: "IMHD_E_ARG", 2: "IMHD_E_CUDA", 3: "IMHD_E_NOMEM", 4: "IMHD_E_PHYSICS", 5: "IMHD_E_STATE"}
S_FLOOR, S_NAN, S_ZERO_SPEED, S_FORCE, S_WAIT, S_PROTECT = 1, 2, 4, 8, 16, 32
# interface reconstruction (imhd_config.recon): characteristic PLM / PPM (the
# reference's default, vanleer_mod.f90:1488-1818) or primitive-variable PLM / PPM
# (primitive_reconstruction, :1144-1485)
RECON = {"plm": 0, "ppm": 1, "plm-prim": 2, "ppm-prim": 3}

# Every symbol declared in include/imhd.h (checked by tests/test_capi_symbols.py).
EXPORTS = (
    "imhd_default_config", "imhd_create", "imhd_upload", "imhd_download", "imhd_set_force",
    "imhd_step", "imhd_max_speed", "imhd_diagnostics", "imhd_status", "imhd_wave_speeds",
    "imhd_destroy", "imhd_last_error", "imhd_launch_count", "imhd_set_stream", "imhd_profile",
    "imhd_stage_times", "imhd_step_static", "imhd_fourier_field", "imhd_init_uniform",
    "imhd_batch_create", "imhd_batch_upload", "imhd_batch_set_force", "imhd_batch_download", "imhd_batch_schedule",
    "imhd_batch_run", "imhd_batch_clock", "imhd_batch_init_uniform", "imhd_batch_fourier_field", "imhd_batch_set_stream",
    "imhd_batch_launch_count", "imhd_batch_destroy",
    "imhd_server_default_config", "imhd_server_start", "imhd_server_submit", "imhd_server_poll",
    "imhd_server_stats", "imhd_server_stop", "imhd_server_destroy",
    "imhd_write_xyzcube", "imhd_write_state_dump", "imhd_write_cuts", "imhd_write_restart", "imhd_read_restart",
    "imhd_init_turb", "imhd_generate_force", "imhd_turb_seeds", "imhd_get_force",
    "imhd_force_sums", "imhd_set_force_sums",
    "imhd_set_geometry", "imhd_pack_planes", "imhd_unpack_planes", "imhd_batch_tuning",
)
NSTAGES = 13
STAGES = ("force_sums", "pred_flux", "pred_emf", "pred_update", "corr_flux_x", "corr_flux_y", "corr_flux_z",
          "corr_emf", "final_update", "force_kick", "passive_pred", "passive_corr", "finalize")


class ImhdConfig(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("precision", ctypes.c_int), ("riemann", ctypes.c_int), ("recon", ctypes.c_int),
        ("npass", ctypes.c_int),
        ("sound_speed", ctypes.c_double), ("cour", ctypes.c_double),
        ("edot", ctypes.c_double), ("dt_turb", ctypes.c_double),
        ("ng", ctypes.c_int), ("ng_pass", ctypes.c_int), ("device", ctypes.c_int),
        ("protect", ctypes.c_int),
    ]


class ImhdServerConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int), ("precision", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_double),
        ("max_resident_cells", ctypes.c_longlong), ("steps_per_round", ctypes.c_int),
    ]


class ImhdRequest(ctypes.Structure):
    _fields_ = [
        ("box", ImhdConfig), ("steps", ctypes.c_longlong), ("t_end", ctypes.c_double), ("dt0", ctypes.c_double),
        ("rho", ctypes.c_double), ("b0", ctypes.c_double * 3), ("nmodes", ctypes.c_int),
        ("kvec", ctypes.POINTER(ctypes.c_int)), ("amp_velocity", ctypes.POINTER(ctypes.c_double)),
        ("scale_velocity", ctypes.c_double), ("amp_force", ctypes.POINTER(ctypes.c_double)),
        ("scale_force", ctypes.c_double), ("forcing", ctypes.c_int),
    ]


REQ_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}
SERVER_NSTATS = 16


class ImhdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load libimhd.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m isothermal_mhd_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        dp = ctypes.POINTER(ctypes.c_double)
        L.imhd_default_config.argtypes = [ctypes.POINTER(ImhdConfig)]
        L.imhd_default_config.restype = None
        L.imhd_create.argtypes = [ctypes.POINTER(ImhdConfig), ctypes.POINTER(vp)]
        L.imhd_create.restype = i
        L.imhd_upload.argtypes = [vp, dp, dp, dp]
        L.imhd_upload.restype = i
        L.imhd_download.argtypes = [vp, dp, dp, dp]
        L.imhd_download.restype = i
        L.imhd_set_force.argtypes = [vp, dp]
        L.imhd_set_force.restype = i
        L.imhd_step.argtypes = [vp, d, i, dp]
        L.imhd_step.restype = i
        L.imhd_max_speed.argtypes = [vp, dp]
        L.imhd_max_speed.restype = i
        L.imhd_diagnostics.argtypes = [vp, dp]
        L.imhd_diagnostics.restype = i
        L.imhd_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(ctypes.c_longlong), i]
        L.imhd_status.restype = i
        L.imhd_wave_speeds.argtypes = [vp, dp, dp]
        L.imhd_wave_speeds.restype = i
        L.imhd_destroy.argtypes = [vp]
        L.imhd_destroy.restype = None
        L.imhd_last_error.argtypes = []
        L.imhd_last_error.restype = ctypes.c_char_p
        L.imhd_launch_count.argtypes = [vp]
        L.imhd_launch_count.restype = ctypes.c_longlong
        L.imhd_set_stream.argtypes = [vp, vp]
        L.imhd_set_stream.restype = i
        L.imhd_profile.argtypes = [vp, i]
        L.imhd_profile.restype = i
        L.imhd_stage_times.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_longlong), i, i]
        L.imhd_stage_times.restype = i
        L.imhd_step_static.argtypes = [i, i, i, i, i, i, d, d, vp, vp, d, dp, vp]
        L.imhd_step_static.restype = i
        ip = ctypes.POINTER(ctypes.c_int)
        L.imhd_fourier_field.argtypes = [vp, i, ip, dp, i, d]
        L.imhd_fourier_field.restype = i
        L.imhd_init_uniform.argtypes = [vp, d, dp]
        L.imhd_init_uniform.restype = i
        L.imhd_batch_init_uniform.argtypes = [vp, i, d, dp]
        L.imhd_batch_init_uniform.restype = i
        L.imhd_batch_create.argtypes = [ctypes.POINTER(ImhdConfig), i, ctypes.POINTER(vp)]
        L.imhd_batch_create.restype = i
        for name in ("imhd_batch_upload", "imhd_batch_download"):
            getattr(L, name).argtypes = [vp, i, dp, dp, dp]
            getattr(L, name).restype = i
        L.imhd_batch_set_force.argtypes = [vp, i, dp]
        L.imhd_batch_set_force.restype = i
        L.imhd_batch_schedule.argtypes = [vp, i, d, d, ctypes.c_longlong, d, i]
        L.imhd_batch_schedule.restype = i
        L.imhd_batch_run.argtypes = [vp, i]
        L.imhd_batch_run.restype = i
        L.imhd_batch_clock.argtypes = [vp, i, dp, ctypes.POINTER(ctypes.c_longlong), dp, ip]
        L.imhd_batch_clock.restype = i
        L.imhd_batch_fourier_field.argtypes = [vp, i, i, ip, dp, i, d]
        L.imhd_batch_fourier_field.restype = i
        L.imhd_batch_set_stream.argtypes = [vp, vp]
        L.imhd_batch_set_stream.restype = i
        L.imhd_batch_launch_count.argtypes = [vp]
        L.imhd_batch_launch_count.restype = ctypes.c_longlong
        L.imhd_batch_destroy.argtypes = [vp]
        L.imhd_batch_destroy.restype = None
        L.imhd_server_default_config.argtypes = [ctypes.POINTER(ImhdServerConfig)]
        L.imhd_server_default_config.restype = None
        L.imhd_server_start.argtypes = [ctypes.POINTER(ImhdServerConfig), ctypes.POINTER(vp)]
        L.imhd_server_start.restype = i
        L.imhd_server_submit.argtypes = [vp, ctypes.POINTER(ImhdRequest), ctypes.POINTER(ctypes.c_longlong)]
        L.imhd_server_submit.restype = i
        L.imhd_server_poll.argtypes = [vp, ctypes.c_longlong, ip, dp, dp, dp, dp]
        L.imhd_server_poll.restype = i
        L.imhd_server_stats.argtypes = [vp, dp, i]
        L.imhd_server_stats.restype = i
        L.imhd_server_stop.argtypes = [vp, i]
        L.imhd_server_stop.restype = i
        L.imhd_server_destroy.argtypes = [vp]
        L.imhd_server_destroy.restype = None
        cp = ctypes.c_char_p
        L.imhd_write_xyzcube.argtypes = [vp, cp, i]
        L.imhd_write_xyzcube.restype = i
        L.imhd_write_state_dump.argtypes = [vp, cp, i]
        L.imhd_write_state_dump.restype = i
        L.imhd_write_cuts.argtypes = [vp, cp, i, i, i, i]
        L.imhd_write_cuts.restype = i
        L.imhd_write_restart.argtypes = [vp, cp, d, i, i, i, i, i]
        L.imhd_write_restart.restype = i
        L.imhd_read_restart.argtypes = [vp, cp, i, dp, ip, ip, ip, ip]
        L.imhd_read_restart.restype = i
        L.imhd_init_turb.argtypes = [vp, i, i, i, i]
        L.imhd_init_turb.restype = i
        L.imhd_generate_force.argtypes = [vp]
        L.imhd_generate_force.restype = i
        L.imhd_turb_seeds.argtypes = [vp, ip, ip, ip]
        L.imhd_turb_seeds.restype = i
        L.imhd_get_force.argtypes = [vp, dp]
        L.imhd_get_force.restype = i
        L.imhd_force_sums.argtypes = [vp, dp]
        L.imhd_force_sums.restype = i
        L.imhd_set_force_sums.argtypes = [vp, dp]
        L.imhd_set_force_sums.restype = i
        L.imhd_set_geometry.argtypes = [vp, d, i, i]
        L.imhd_set_geometry.restype = i
        L.imhd_pack_planes.argtypes = [vp, i, i, vp]
        L.imhd_pack_planes.restype = i
        L.imhd_unpack_planes.argtypes = [vp, i, i, vp]
        L.imhd_unpack_planes.restype = i
        L.imhd_batch_tuning.argtypes = [vp, i, ip, ip, ip, ip]
        L.imhd_batch_tuning.restype = i
        _lib = L
    return _lib


def check(rc):
    if rc != IMHD_OK:
        raise ImhdError(rc, lib().imhd_last_error().decode(errors="replace"))
