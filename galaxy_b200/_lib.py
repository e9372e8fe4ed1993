"""Loader of libgalaxy_b200.so and ctypes signatures of the C ABI (include/galaxy_b200.h).

There is no CPU fallback: if the library is missing or cannot load, every entry
point raises instead of computing anything elsewhere.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgalaxy_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "galaxy_b200.h")

GX_OK = 0
ERRORS = {
    -1: "GX_ERR_INVALID_ARG",
    -2: "GX_ERR_CUDA",
    -3: "GX_ERR_NO_DEVICE",
    -4: "GX_ERR_BUDGET",
    -5: "GX_ERR_STATE",
    -6: "GX_ERR_DEVICE_CHECK",
    -7: "GX_ERR_NOT_FOUND",
    -8: "GX_ERR_CAPACITY",
    -9: "GX_ERR_CANCELLED",
}

ERRORS_BY_NAME = {v: k for k, v in ERRORS.items()}

GX_PREC_F32, GX_PREC_F64 = 0, 1
GX_MULTIPOLE_MONO, GX_MULTIPOLE_QUAD = 0, 1
GX_FLAG_NO_KAHAN, GX_FLAG_STATS, GX_FLAG_STAGE_TIMES, GX_FLAG_MORTON63 = 1, 2, 4, 8


class GxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("precision", C.c_uint32),
        ("multipole", C.c_uint32),
        ("flags", C.c_uint32),
        ("device", C.c_int32),
        ("walk_block", C.c_uint32),
        ("walk_ctas_per_sm", C.c_uint32),
        ("walk_group", C.c_uint32),
        ("radix_bits", C.c_uint32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("n", C.c_uint64),
        ("leaf_interactions", C.c_uint64),
        ("far_interactions", C.c_uint64),
        ("nodes_opened", C.c_uint64),
        ("f64_rechecks", C.c_uint64),
        ("warp_node_visits", C.c_uint64),
        ("ms_bbox_morton", C.c_float),
        ("ms_sort", C.c_float),
        ("ms_build", C.c_float),
        ("ms_walk", C.c_float),
        ("ms_total", C.c_float),
        ("ms_sph", C.c_float),
        ("ms_sph_density", C.c_float),
    ]


GX_EOS_ISOTHERMAL, GX_EOS_ADIABATIC = 0, 1


class SphParams(C.Structure):
    _fields_ = [
        ("n_ngb", C.c_double),
        ("h_tol_rel", C.c_double),
        ("eos", C.c_int),
        ("warm_start", C.c_int),
        ("c_s", C.c_double),
        ("gamma", C.c_double),
        ("alpha", C.c_double),
        ("beta", C.c_double),
        ("visc_eps2", C.c_double),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("walk_block", C.c_uint32),
        ("walk_ctas_per_sm", C.c_uint32),
        ("walk_group", C.c_uint32),
        ("radix_bits", C.c_uint32),
        ("ms", C.c_float),
        ("sort_ms", C.c_float),
    ]


GX_TUNE_MAX_CANDIDATES = 24


class BatchStats(C.Structure):
    _fields_ = [
        ("systems", C.c_uint64),
        ("particles", C.c_uint64),
        ("steps", C.c_uint64),
        ("bytes_in_use", C.c_uint64),
        ("budget_bytes", C.c_uint64),
        ("ms_last_step", C.c_float),
    ]


class SnapOpts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("every", C.c_uint64),
        ("path_prefix", C.c_char_p),
        ("rng_seed", C.c_uint64),
        ("config_hash", C.c_uint64),
        ("units", C.c_char_p),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("steps", C.c_uint64),
        ("particle_steps", C.c_uint64),
        ("completed", C.c_uint64),
        ("queued", C.c_uint64),
        ("live", C.c_uint64),
        ("max_live", C.c_uint64),
        ("bytes_in_use", C.c_uint64),
        ("busy_s", C.c_double),
        ("wall_s", C.c_double),
        ("step_ms_p50", C.c_double),
        ("step_ms_p99", C.c_double),
        ("step_ms_mean", C.c_double),
        ("particle_steps_per_s_device", C.c_double),
        ("queue_s_p50", C.c_double),
        ("queue_s_p99", C.c_double),
    ]


_lib = None

_vp, _sz, _d, _u64, _i = C.c_void_p, C.c_size_t, C.c_double, C.c_uint64, C.c_int

SIGNATURES = {
    "gx_create": (_i, [_d, _d, _d, C.POINTER(Options), C.POINTER(_vp)]),
    "gx_destroy": (None, [_vp]),
    "gx_last_error": (C.c_char_p, [_vp]),
    "gx_device_info": (_i, [_i, C.c_char_p, _sz, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i), C.POINTER(_sz)]),
    "gx_device_synchronize": (_i, [_i]),
    "gx_selftest_bounded_wait": (_i, [_i, C.c_uint32, C.POINTER(C.c_uint32)]),
    "gx_accelerations": (_i, [_vp, _sz, _vp, _vp, _vp]),
    "gx_accelerations_device": (_i, [_vp, _sz, _vp, _vp, _vp]),
    "gx_accelerations_active": (_i, [_vp, _sz, _vp, _vp, _sz, _vp, _vp]),
    "gx_rebuild_gravity_cache": (_i, [_vp, _sz, _vp, _vp]),
    "gx_gravity_active_cached": (_i, [_vp, _sz, _vp, _vp, _sz, _vp, _vp]),
    "gx_potential_energy": (_i, [_vp, _sz, _vp, _vp, C.POINTER(_d)]),
    "gx_direct_sum_f64": (_i, [_vp, _sz, _vp, _vp, _sz, _vp, _vp]),
    "gx_upload": (_i, [_vp, _sz, _vp, _vp, _vp]),
    "gx_step": (_i, [_vp, _d]),
    "gx_step_many": (_i, [_vp, _d, _u64]),
    "gx_step_many_async": (_i, [_vp, _d, _u64]),
    "gx_synchronize": (_i, [_vp]),
    "gx_snapshot": (_i, [_vp, _vp, _vp]),
    "gx_resident_accelerations": (_i, [_vp, _vp]),
    "gx_time": (_i, [_vp, C.POINTER(_d)]),
    "gx_len": (_i, [_vp, C.POINTER(_sz)]),
    "gx_launches": (_i, [_vp, C.POINTER(_u64)]),
    "gx_diagnostics": (_i, [_vp, _i, _vp]),
    "gx_get_stats": (_i, [_vp, C.POINTER(Stats)]),
    "gx_step_many_timed": (_i, [_vp, _d, _u64, C.POINTER(C.c_float)]),
    "gx_autotune": (_i, [_vp, C.c_uint32, C.POINTER(Tuning), C.POINTER(Tuning), C.POINTER(C.c_uint32)]),
    "gx_tuning_lookup": (_i, [_i, _sz, C.POINTER(Options), _i, C.POINTER(Tuning)]),
    "gx_kdk_step_host": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, C.POINTER(_i), _d]),
    "gx_host_alloc": (_i, [_sz, C.POINTER(_vp)]),
    "gx_host_free": (None, [_vp]),
    "gx_sort_noalloc": (_i, [_vp, _vp, _vp, _sz, _vp]),
    "gx_stage_morton": (_i, [_vp, _sz, _vp, _vp, _vp, _vp]),
    "gx_stage_sort": (_i, [_vp, _sz, _vp, _vp, _vp]),
    "gx_stage_build": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gx_batch_create": (_i, [_sz, C.POINTER(Options), C.POINTER(_vp)]),
    "gx_batch_destroy": (None, [_vp]),
    "gx_batch_last_error": (C.c_char_p, [_vp]),
    "gx_system_add": (_i, [_vp, _sz, _vp, _vp, _vp, _d, _d, _d, _d, C.POINTER(_u64)]),
    "gx_system_remove": (_i, [_vp, _u64]),
    "gx_system_bytes": (_i, [_vp, _sz, C.POINTER(_sz)]),
    "gx_batch_step": (_i, [_vp, _u64]),
    "gx_system_snapshot": (_i, [_vp, _u64, _vp, _vp, C.POINTER(_d)]),
    "gx_system_len": (_i, [_vp, _u64, C.POINTER(_sz)]),
    "gx_batch_stats_get": (_i, [_vp, C.POINTER(BatchStats)]),
    "gx_batch_set_graph": (_i, [_vp, _i]),
    "gx_batch_autotune": (_i, [_vp, C.c_uint32, C.POINTER(Tuning), C.POINTER(Tuning), C.POINTER(C.c_uint32)]),
    "gx_server_create": (_i, [_sz, C.POINTER(Options), C.POINTER(_vp)]),
    "gx_server_destroy": (None, [_vp]),
    "gx_server_last_error": (C.c_char_p, [_vp]),
    "gx_server_submit": (_i, [_vp, _sz, _vp, _vp, _vp, _d, _d, _d, _d, _u64, C.POINTER(_u64)]),
    "gx_server_status": (_i, [_vp, _u64, C.POINTER(_i), C.POINTER(_u64)]),
    "gx_server_wait": (_i, [_vp, _u64, _d]),
    "gx_server_result": (_i, [_vp, _u64, _vp, _vp, C.POINTER(_d)]),
    "gx_server_release": (_i, [_vp, _u64]),
    "gx_server_submit_snapshots": (_i, [_vp, _sz, _vp, _vp, _vp, _d, _d, _d, _d, _u64, C.POINTER(SnapOpts),
                                        C.POINTER(_u64)]),
    "gx_server_snapshots_written": (_i, [_vp, _u64, C.POINTER(_u64)]),
    "gx_server_cancel": (_i, [_vp, _u64]),
    "gx_server_set_metrics_log": (_i, [_vp, C.c_char_p]),
    "gx_glxysnap_write": (_i, [C.c_char_p, _d, _u64, _d, _u64, _u64, C.c_char_p, _sz, _vp, _vp, _vp]),
    "gx_server_stats_get": (_i, [_vp, C.POINTER(ServerStats)]),
    "gx_ic_plummer": (_i, [_sz, _u64, _d, _d, _d, _vp, _vp, _vp]),
    "gx_ic_collision": (_i, [_sz, _u64, _d, _d, _d, _d, _vp, _vp, _vp]),
    "gx_ic_disk_galaxy": (_i, [_sz, _u64, _vp, _vp, _vp]),
    "gx_sph_default_params": (None, [C.POINTER(SphParams)]),
    "gx_sph_enable": (_i, [_vp, C.POINTER(SphParams)]),
    "gx_upload_species": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp]),
    "gx_gas_count": (_i, [_vp, C.POINTER(_sz)]),
    "gx_snapshot_gas_density": (_i, [_vp, _vp, _vp, _vp]),
    "gx_snapshot_gas_accel": (_i, [_vp, _vp, _vp]),
    "gx_snapshot_accel": (_i, [_vp, _vp]),
    "gx_min_stable_dt": (_i, [_vp, _d, C.POINTER(_d)]),
    "gx_snapshot_gas_dt": (_i, [_vp, _d, _vp]),
    "gx_sph_accelerations": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gx_sph_accel_and_dudt": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gx_sph_accelerations_active": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _sz, _vp, _vp]),
    "gx_sph_accel_and_dudt_active": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _sz, _vp, _vp, _vp]),
    "gx_sph_sf_fields": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gx_sph_max_stable_dt": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _d, _vp, C.POINTER(_d)]),
    "gx_sph_coupled_pairs": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _sz, C.POINTER(_sz)]),
    "gx_sph_density": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp]),
    "gx_sph_hydro": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gx_sph_cfl": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _d, _vp, C.POINTER(_d)]),
}


def lib():
    """The loaded library (raises if it is absent: there is no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                               "(galaxy_b200 has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, handle=None, err_fn="gx_last_error") -> None:
    if rc != GX_OK:
        msg = getattr(lib(), err_fn)(handle)
        raise GxError(rc, msg.decode() if msg else "")


def header_symbols() -> list[str]:
    """Every function the public header declares."""
    import re

    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(gx_[a-z0-9_]+)\s*\(", text)))
