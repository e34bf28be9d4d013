"""ctypes binding of libmaragpu.so (the C ABI in include/mara_gpu.h).

The library is built in-tree (``make -C ctf_b200/csrc``).  There is no fallback: if the
shared library is missing and cannot be built, importing the binding raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libmaragpu.so")
CSRC = os.path.join(HERE, "csrc")

# The FP64 kernels built with FMA contraction on (a comparator, not the parity path).
LIB_FMAD_PATH = os.path.join(HERE, "_lib", "libmaragpu_fmad.so")

_lock = threading.Lock()
_lib = None
_lib_fmad = None


class MgpuConfig(ctypes.Structure):
    _fields_ = [("fluid", ctypes.c_int), ("gamma", ctypes.c_double), ("recon", ctypes.c_int),
                ("theta", ctypes.c_double), ("is_mode", ctypes.c_int), ("sz10A", ctypes.c_double),
                ("riemann", ctypes.c_int), ("rk", ctypes.c_int), ("pfloor", ctypes.c_double),
                ("ereset", ctypes.c_int), ("preset", ctypes.c_double), ("dreset", ctypes.c_double),
                ("precision", ctypes.c_int), ("learned_c2p", ctypes.c_int), ("godunov", ctypes.c_int),
                ("layout", ctypes.c_int)]


class MgpuStats(ctypes.Structure):
    _fields_ = [("max_lambda", ctypes.c_double), ("dt", ctypes.c_double), ("errors", ctypes.c_int),
                ("committed", ctypes.c_int), ("c2p_calls", ctypes.c_ulonglong),
                ("c2p_iters", ctypes.c_ulonglong), ("c2p_attempt", ctypes.c_ulonglong * 6),
                ("face_c2p_calls", ctypes.c_ulonglong), ("face_c2p_iters", ctypes.c_ulonglong),
                ("hlld_ok", ctypes.c_ulonglong), ("hlld_hllc", ctypes.c_ulonglong),
                ("pcm_retry", ctypes.c_ulonglong), ("c2p_failed", ctypes.c_ulonglong),
                ("advances", ctypes.c_ulonglong),
                ("failed_advances", ctypes.c_ulonglong), ("failed_zones", ctypes.c_ulonglong)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "c2p_attempt"}
        d["c2p_attempt"] = list(self.c2p_attempt)
        return d


class MgpuEnsembleLaunch(ctypes.Structure):
    _fields_ = [("zone_tile", ctypes.c_int), ("face_tile", ctypes.c_int), ("zone_ctas_per_sm", ctypes.c_int),
                ("face_ctas_per_sm", ctypes.c_int), ("c2p_ctas_per_sm", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


# exported symbol -> (restype, argtypes)
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
SIGNATURES = {
    "mgpu_default_config": (ctypes.c_int, [ctypes.POINTER(MgpuConfig)]),
    "mgpu_create": (ctypes.c_int, [ctypes.POINTER(MgpuConfig), ctypes.POINTER(_vp)]),
    "mgpu_destroy": (ctypes.c_int, [_vp]),
    "mgpu_set_stream": (ctypes.c_int, [_vp, _vp]),
    "mgpu_last_error": (ctypes.c_char_p, [_vp]),
    "mgpu_set_domain": (ctypes.c_int, [_vp, _dp, _dp, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "mgpu_num_zones": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "mgpu_upload_prim": (ctypes.c_int, [_vp, _dp]),
    "mgpu_download_prim": (ctypes.c_int, [_vp, _dp]),
    "mgpu_upload_prim_device": (ctypes.c_int, [_vp, _vp]),
    "mgpu_download_prim_device": (ctypes.c_int, [_vp, _vp]),
    "mgpu_upload_prim_range": (ctypes.c_int, [_vp, _dp, ctypes.c_longlong, ctypes.c_longlong]),
    "mgpu_download_prim_range": (ctypes.c_int, [_vp, _dp, ctypes.c_longlong, ctypes.c_longlong]),
    "mgpu_advance": (ctypes.c_int, [_vp, ctypes.c_double, _ip]),
    "mgpu_advance_host": (ctypes.c_int, [_vp, _dp, ctypes.c_double, _dp, _ip]),
    "mgpu_set_pipeline": (ctypes.c_int, [_vp, ctypes.c_int]),
    "mgpu_get_pipeline": (ctypes.c_int, [_vp, _ip, _ip]),
    "mgpu_pipeline_schedule": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _ip, ctypes.c_int]),
    "mgpu_pipeline_bounds": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _ip, ctypes.c_int]),
    "mgpu_advance_async": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double]),
    "mgpu_synchronize": (ctypes.c_int, [_vp]),
    "mgpu_get_timestep": (ctypes.c_int, [_vp, ctypes.c_double, _dp]),
    "mgpu_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(MgpuStats)]),
    "mgpu_set_primitive": (ctypes.c_int, [_vp, _dp]),
    "mgpu_measure_divB": (ctypes.c_int, [_vp, _dp, _dp]),
    "mgpu_max_lorentz_factor": (ctypes.c_int, [_vp, _dp]),
    "mgpu_measure_divB_state": (ctypes.c_int, [_vp, _dp, _dp]),
    "mgpu_profile_enable": (ctypes.c_int, [_vp, ctypes.c_int]),
    "mgpu_profile_disable": (ctypes.c_int, [_vp]),
    "mgpu_profile_read": (ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_longlong)]),
    "mgpu_set_c2p_network": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float), ctypes.c_longlong]),
    "mgpu_mlp_param_count": (ctypes.c_int, []),
    "mgpu_c2p_harvest": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]),
    "mgpu_mlp_work_floats": (ctypes.c_longlong, [ctypes.c_longlong]),
    "mgpu_mlp_loss_grad": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_longlong, _vp, _vp, _dp]),
    "mgpu_mlp_train": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_float, ctypes.c_int, _vp, _dp]),
    "mgpu_mlp_forward": (ctypes.c_int, [_vp, _vp, ctypes.c_longlong, _vp]),
    "mgpu_mlp_forward_tc": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float), _vp, ctypes.c_longlong, _vp]),
    "mgpu_mlp_tc_image_bytes": (ctypes.c_int, []),
    "mgpu_mlp_build_tc_image": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float), _vp]),
    "mgpu_advance_noalloc": (ctypes.c_int, [ctypes.POINTER(MgpuConfig), _dp, _dp, _ip, ctypes.c_int, _vp, _vp,
                                            ctypes.c_double, _ip, _dp, _vp, ctypes.c_char_p, ctypes.c_int]),
    "mgpu_advance_phase": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double]),
    "mgpu_reduction_targets": (ctypes.c_int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "mgpu_set_external_guards": (ctypes.c_int, [_vp, _ip, _ip]),
    "mgpu_halo_bytes": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]),
    "mgpu_halo_pack": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "mgpu_halo_unpack": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "mgpu_new_ou_field": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                         _vp, ctypes.POINTER(ctypes.c_longlong)]),
    "mgpu_set_driving": (ctypes.c_int, [_vp, _vp, ctypes.c_longlong]),
    "mgpu_driving_advance": (ctypes.c_int, [_vp, ctypes.c_double]),
    "mgpu_driving_resample": (ctypes.c_int, [_vp]),
    "mgpu_driving_serialize": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_longlong)]),
    "mgpu_driving_power": (ctypes.c_int, [_vp, _dp]),
    "mgpu_ou_field_advance": (ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_double]),
    "mgpu_ensemble_create": (ctypes.c_int, [ctypes.POINTER(MgpuConfig), ctypes.c_int, ctypes.c_int, _ip, _dp, _dp,
                                            ctypes.POINTER(_vp)]),
    "mgpu_ensemble_destroy": (ctypes.c_int, [_vp]),
    "mgpu_ensemble_last_error": (ctypes.c_char_p, [_vp]),
    "mgpu_ensemble_set_stream": (ctypes.c_int, [_vp, _vp]),
    "mgpu_ensemble_num_zones": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]),
    "mgpu_ensemble_total_interior": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "mgpu_ensemble_upload_prim": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "mgpu_ensemble_download_prim": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "mgpu_ensemble_upload_prim_device": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "mgpu_ensemble_download_prim_device": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "mgpu_ensemble_get_launch": (ctypes.c_int, [_vp, ctypes.POINTER(MgpuEnsembleLaunch)]),
    "mgpu_ensemble_set_launch": (ctypes.c_int, [_vp, ctypes.POINTER(MgpuEnsembleLaunch)]),
    "mgpu_ensemble_advance": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_int]),
    "mgpu_ensemble_synchronize": (ctypes.c_int, [_vp]),
    "mgpu_ensemble_errors": (ctypes.c_int, [_vp, _ip]),
    "mgpu_ensemble_get_stats": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(MgpuStats)]),
    "mgpu_ensemble_get_timesteps": (ctypes.c_int, [_vp, ctypes.c_double, _dp]),
    "mgpu_ensemble_profile_enable": (ctypes.c_int, [_vp, ctypes.c_int]),
    "mgpu_ensemble_profile_disable": (ctypes.c_int, [_vp]),
    "mgpu_ensemble_profile_read": (ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_longlong),
                                                  ctypes.POINTER(ctypes.c_longlong)]),
    "mgpu_ensemble_time_advance": (ctypes.c_int, [_vp, ctypes.POINTER(MgpuEnsembleLaunch), _dp, ctypes.c_int, _dp]),
    "mgpu_ensemble_autotune": (ctypes.c_int, [_vp, _dp, ctypes.c_int, ctypes.POINTER(MgpuEnsembleLaunch), _dp]),
    "mgpu_probe_prim_to_cons": (ctypes.c_int, [ctypes.c_double, _vp, ctypes.c_longlong, _vp, _vp]),
    "mgpu_probe_c2p": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double, _vp, _vp, ctypes.c_longlong,
                                      _vp, _vp, _vp]),
    "mgpu_probe_flux": (ctypes.c_int, [ctypes.c_double, ctypes.c_int, _vp, ctypes.c_longlong, _vp, _vp]),
    "mgpu_probe_riemann": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_double, ctypes.c_double, _vp,
                                          _vp, ctypes.c_longlong, _vp, _vp, _vp, _vp]),
    "mgpu_probe_reconstruct": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, _vp,
                                              ctypes.c_longlong, _vp]),
    "mgpu_measure_mean_cons": (ctypes.c_int, [_vp, _dp]),
    "mgpu_measure_mean_prim": (ctypes.c_int, [_vp, _dp]),
    "mgpu_measure_mean_energies": (ctypes.c_int, [_vp, _dp]),
    "mgpu_measure_mean_velocity": (ctypes.c_int, [_vp, _dp]),
    "mgpu_measure_mean_max_temperature": (ctypes.c_int, [_vp, _dp, _dp]),
    "mgpu_measure_mean_max_magnetic_field": (ctypes.c_int, [_vp, _dp, _dp]),
    "mgpu_measure_mean_max_sonic_mach": (ctypes.c_int, [_vp, _dp, _dp]),
    "mgpu_measure_mean_min_alfvenic_mach": (ctypes.c_int, [_vp, _dp, _dp]),
    "mgpu_diffuse": (ctypes.c_int, [_vp, ctypes.c_double, _ip]),
    "mgpu_diffuse_host": (ctypes.c_int, [_vp, _dp, ctypes.c_double, _ip]),
    "mgpu_set_failmask": (ctypes.c_int, [_vp, ctypes.c_int]),
    "mgpu_reconfigure": (ctypes.c_int, [_vp, ctypes.POINTER(MgpuConfig)]),
    "mgpu_halo_pack_on": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "mgpu_halo_unpack_on": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]),
}


def build(force: bool = False) -> str:
    """Compile libmaragpu.so for sm_100a with nvcc (no GPU needed)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", CSRC, "-j4"], check=True)
    return LIB_PATH


def _bind(path: str) -> ctypes.CDLL:
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def load(variant: str = "") -> ctypes.CDLL:
    """Load the library (building it first if it is absent); raises if that fails.

    variant "fmad" loads libmaragpu_fmad.so, whose FP64 kernels are compiled with FMA
    contraction on: the comparator of an FP64 build that uses fused multiply-adds.  It is not
    the parity path (the plain FP64 path rounds every multiply and add as the reference
    does)."""
    global _lib, _lib_fmad
    with _lock:
        if variant == "fmad":
            if _lib_fmad is None:
                if not os.path.exists(LIB_FMAD_PATH):
                    build(force=True)
                _lib_fmad = _bind(LIB_FMAD_PATH)
            return _lib_fmad
        if variant:
            raise ValueError(f"no library variant {variant!r}")
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            _lib = _bind(LIB_PATH)
        return _lib
