"""ctypes view of include/natray.h: the structures, and the loaded library.

The library is the in-tree libnatray.so. It loads on a machine without a GPU (parameters and
world construction are CPU only); simulation calls on such a machine fail with NTR_E_NODEVICE.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libnatray.so"

MAX_SHOTS = 4
MAX_PATCHES = 576
N_SEC = 32
LOG_CAP = 256
OUTLINE = 33
HIT_FIELDS = 13
ACC_FIELDS = 19
CELL_FIELDS = 11
AIR_FIELDS = 5
LAYER_MODES = 6
WORLD_MAGIC = 0x5752544E
WORLD_VERSION = 1

STATUS = {0: "NTR_OK", 1: "NTR_E_INVALID", 2: "NTR_E_NOMEM", 3: "NTR_E_OVERFLOW", 4: "NTR_E_UNCONVERGED",
          5: "NTR_E_TIMEOUT", 6: "NTR_E_CUDA", 7: "NTR_E_NODEVICE", 8: "NTR_E_BUSY"}

SECTIONS = ["PARTICLES", "MEM_X", "MEM_V", "MEM_MASS", "MEM_WATER", "MEM_LAYER", "MEM_PUSH", "TRIS", "ALIVE",
            "VTRI_OFF", "VTRI", "BULLETS", "PATCHES", "OUTLINES", "SECTIONS", "BULLET_HIT", "POSE_LOG",
            "BLOCKS_PREV", "BLOCK_ACTIVE", "AIR", "SPRAY", "LANDED", "TOUCH"]
SEC = {n: i for i, n in enumerate(SECTIONS)}
NTR_SEC_COUNT = len(SECTIONS)

BUFS = ["PARTICLES", "STATE", "MEM_POS", "TRIS", "ALIVE", "VTRI_OFF", "VTRI", "SPRAY", "TOUCH", "LANDED",
        "BLOCK_LIST", "SORTED", "BLOCK_START", "ACC", "CF", "AIR", "BLOCK_NB"]
BUF = {n: i for i, n in enumerate(BUFS)}


class Shot(C.Structure):
    _fields_ = [("bullet", C.c_uint32), ("speed", C.c_float), ("caliber_mm", C.c_float), ("mass_g", C.c_float),
                ("spin_rpm", C.c_float), ("range_m", C.c_float), ("muzzle_yaw_deg", C.c_float),
                ("azimuth_deg", C.c_float), ("elevation_deg", C.c_float), ("impact_offset_cm", C.c_float),
                ("impact_side_cm", C.c_float), ("delay_ms", C.c_float)]


class SimParams(C.Structure):
    _fields_ = [("n_shots", C.c_uint32), ("shots", Shot * MAX_SHOTS), ("balloon_diameter_cm", C.c_float),
                ("balloon_height", C.c_float), ("rubber_modulus_mpa", C.c_float),
                ("rubber_rest_diameter_cm", C.c_float), ("rubber_break_stretch", C.c_float),
                ("rubber_thickness_mm", C.c_float), ("gravity", C.c_float), ("spray_amount", C.c_float),
                ("mist_amount", C.c_float), ("resolution", C.c_uint32), ("mesh_level", C.c_uint32),
                ("dt_max", C.c_float), ("seed", C.c_uint64), ("block_cap", C.c_uint32), ("spray_cap", C.c_uint32),
                ("max_iters", C.c_uint32), ("solve_tol", C.c_float)]


class GpuParams(C.Structure):
    _fields_ = [("origin", C.c_float * 4), ("dims", C.c_uint32 * 4), ("bdims", C.c_uint32 * 4),
                ("gravity", C.c_float * 4), ("fluid", C.c_float * 4), ("wet", C.c_float * 4),
                ("limits", C.c_uint32 * 4), ("solve", C.c_float * 4), ("mem", C.c_uint32 * 4),
                ("rubber", C.c_float * 4), ("rubber2", C.c_float * 4), ("knot", C.c_float * 4)]


class State(C.Structure):
    _fields_ = [("t_ns", C.c_uint32), ("dt_ns", C.c_uint32), ("step", C.c_uint32), ("n_blocks", C.c_uint32),
                ("max_speed", C.c_float), ("n_blocks_prev", C.c_uint32), ("overflow", C.c_uint32),
                ("solve_iters", C.c_uint32), ("rz", C.c_float), ("alpha", C.c_float), ("b_norm", C.c_float),
                ("r_norm", C.c_float), ("free_dt_ns", C.c_uint32), ("iters_max", C.c_uint32),
                ("unconverged", C.c_uint32), ("beta", C.c_float), ("spray_count", C.c_uint32),
                ("mem_dt", C.c_float), ("cap_dt", C.c_float), ("mem_dt_seen", C.c_float), ("dt_flow", C.c_float),
                ("air_dt", C.c_float), ("air_dt_seen", C.c_float), ("mem_ticket", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class WorldHeader(C.Structure):
    _fields_ = [("magic", C.c_uint32), ("version", C.c_uint32), ("n_particles", C.c_uint32),
                ("n_verts", C.c_uint32), ("n_tris", C.c_uint32), ("n_vtri", C.c_uint32), ("n_shots", C.c_uint32),
                ("n_blocks_prev", C.c_uint32), ("n_spray", C.c_uint32), ("wet_res", C.c_uint32),
                ("spray_cap", C.c_uint32), ("block_cap", C.c_uint32), ("iters", C.c_uint32),
                ("substeps", C.c_uint32), ("air_substeps", C.c_uint32), ("unconverged", C.c_uint32),
                ("started", C.c_uint32), ("max_iters", C.c_uint32), ("t", C.c_double), ("t_start", C.c_double),
                ("t0", C.c_double), ("dx", C.c_double), ("params", GpuParams), ("state", State),
                ("offset", C.c_uint64 * NTR_SEC_COUNT), ("bytes", C.c_uint64 * NTR_SEC_COUNT)]


class SimInfo(C.Structure):
    _fields_ = [("n_particles", C.c_uint32), ("n_verts", C.c_uint32), ("n_tris", C.c_uint32),
                ("n_shots", C.c_uint32), ("dims", C.c_uint32 * 3), ("block_cap", C.c_uint32),
                ("spray_cap", C.c_uint32), ("iters", C.c_uint32), ("substeps", C.c_uint32),
                ("air_substeps", C.c_uint32), ("dx", C.c_double), ("spacing", C.c_double),
                ("grid_origin", C.c_float * 3), ("pad", C.c_float), ("t", C.c_double), ("t_start", C.c_double),
                ("t0", C.c_double), ("device_bytes", C.c_uint64)]


PROFILE_SAMPLES = 402


class Profile(C.Structure):
    _fields_ = [("n_samples", C.c_uint32), ("pad", C.c_uint32), ("neck_angle", C.c_double), ("z_neck", C.c_double),
                ("neck_r", C.c_double), ("volume", C.c_double), ("z_centroid", C.c_double), ("stretch", C.c_double),
                ("r_max", C.c_double), ("samples", (C.c_double * 3) * PROFILE_SAMPLES)]


BATCH_MAX = 128


class Tuning(C.Structure):
    _fields_ = [("solve_ctas", C.c_uint32), ("cell_ctas_per_sm", C.c_uint32), ("block_ctas_per_sm", C.c_uint32),
                ("pad", C.c_uint32)]


class BatchSlot(C.Structure):
    _fields_ = [("in_use", C.c_uint32), ("finished", C.c_uint32), ("steps_done", C.c_uint32),
                ("steps_target", C.c_uint32), ("device_bytes", C.c_uint64), ("state", State)]


class BatchInfo(C.Structure):
    _fields_ = [("max_scenes", C.c_uint32), ("in_use", C.c_uint32), ("active", C.c_uint32), ("captures", C.c_uint32),
                ("held_bytes", C.c_uint64), ("budget_bytes", C.c_uint64), ("free_bytes", C.c_uint64),
                ("steps", C.c_uint64), ("instantiations", C.c_uint32), ("pad", C.c_uint32)]


MAX_SHOTS = 4
SHOWN = {"PARTICLES": 0, "SPRAY": 1, "MEM_POS": 2, "ALIVE": 3, "WET": 4, "SPRAY_W": 5}
SHOWN_COUNT = 6


class CacheParams(C.Structure):
    _fields_ = [("page_bytes", C.c_uint64), ("pages", C.c_uint32), ("n_arrivals", C.c_uint32), ("t_end", C.c_double),
                ("arrivals", C.c_double * MAX_SHOTS)]


class KeyInfo(C.Structure):
    _fields_ = [("t", C.c_double), ("offset", C.c_uint64), ("bytes", C.c_uint64), ("page", C.c_uint32),
                ("spray", C.c_uint32), ("live", C.c_uint32), ("pad", C.c_uint32)]


class CacheInfo(C.Structure):
    _fields_ = [("keys", C.c_uint32), ("done", C.c_uint32), ("full", C.c_uint32), ("shown_spray", C.c_uint32),
                ("used_bytes", C.c_uint64), ("pool_bytes", C.c_uint64), ("shown_id", C.c_uint64), ("end", C.c_double),
                ("next_t", C.c_double), ("shown", C.c_double)]


class Flight(C.Structure):
    _fields_ = [("x", C.c_double * 3), ("u", C.c_double * 3), ("n", C.c_double * 3), ("h", C.c_double * 3),
                ("roll", C.c_double), ("t_read", C.c_double), ("t_hit", C.c_double), ("v_impact", C.c_double),
                ("sg_air", C.c_double), ("yaw_impact_deg", C.c_double), ("twist", C.c_double),
                ("muzzle_x", C.c_double * 3), ("muzzle_u", C.c_double * 3)]


class StatsBullet(C.Structure):
    _fields_ = [("state", C.c_uint32), ("sections", C.c_uint32), ("x", C.c_float * 3), ("speed", C.c_float),
                ("yaw_deg", C.c_float), ("spin_rev_s", C.c_float), ("kinetic_j", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("water", C.c_uint32), ("n_particles", C.c_uint32), ("lo", C.c_float * 3), ("hi", C.c_float * 3),
                ("mean", C.c_double * 3), ("vmean", C.c_double * 3), ("vmax", C.c_float), ("fastest", C.c_float * 3),
                ("volume_l", C.c_double), ("inside_l", C.c_double), ("mem_lo", C.c_float * 3),
                ("mem_hi", C.c_float * 3), ("free_verts", C.c_uint32), ("on_water", C.c_uint32), ("torn", C.c_uint32),
                ("n_tension", C.c_uint32), ("fill_min", C.c_float), ("fill_mean", C.c_float),
                ("rubber_vmax", C.c_float), ("pad0", C.c_float), ("tension", C.c_double * 3),
                ("tension_tri", C.c_uint32 * 3), ("pad1", C.c_uint32), ("stretch", (C.c_float * 2) * 3),
                ("air_cells", C.c_uint32), ("vapour_cells", C.c_uint32), ("gauge_lo", C.c_float),
                ("gauge_hi", C.c_float), ("air_umax", C.c_float), ("pad2", C.c_float), ("water_j", C.c_double),
                ("bullets_j", C.c_double), ("vapour_cm3", C.c_double), ("vapour_j", C.c_double),
                ("n_bullets", C.c_uint32), ("pad3", C.c_uint32), ("bullets", StatsBullet * MAX_SHOTS)]


# Every entry point include/natray.h declares, with its ctypes signature.
_P = C.c_void_p
_SIGS = {
    "ntr_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "ntr_version": (C.c_char_p, []),
    "ntr_free": (None, [_P]),
    "ntr_params_default": (C.c_int, [C.POINTER(SimParams)]),
    "ntr_params_set": (C.c_int, [C.POINTER(SimParams), C.c_char_p, C.c_char_p]),
    "ntr_params_preset": (C.c_int, [C.POINTER(SimParams), C.c_char_p]),
    "ntr_world_build": (C.c_int, [C.POINTER(SimParams), C.POINTER(_P), C.POINTER(C.c_size_t)]),
    "ntr_shot_flights": (C.c_int, [C.POINTER(SimParams), C.POINTER(Flight), C.c_uint32, C.POINTER(C.c_uint32)]),
    "ntr_inflate": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.POINTER(Profile)]),
    "ntr_sim_create": (C.c_int, [C.POINTER(SimParams), C.c_int, C.POINTER(_P)]),
    "ntr_sim_create_from_world": (C.c_int, [_P, C.c_size_t, C.c_int, C.POINTER(_P)]),
    "ntr_sim_destroy": (C.c_int, [_P]),
    "ntr_sim_step": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32)]),
    "ntr_sim_advance": (C.c_int, [_P, C.c_double, C.c_uint32, C.POINTER(C.c_uint32)]),
    "ntr_sim_read_state": (C.c_int, [_P, C.POINTER(State)]),
    "ntr_sim_info_get": (C.c_int, [_P, C.POINTER(SimInfo)]),
    "ntr_sim_buffer": (C.c_int, [_P, C.c_int, C.POINTER(_P), C.POINTER(C.c_size_t)]),
    "ntr_sim_download": (C.c_int, [_P, C.c_int, _P, C.c_size_t]),
    "ntr_sim_snapshot": (C.c_int, [_P, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "ntr_sim_restore": (C.c_int, [_P, _P, C.c_size_t]),
    "ntr_sim_set_precision": (C.c_int, [_P, C.c_int]),
    "ntr_sim_set_batch_steps": (C.c_int, [_P, C.c_uint32]),
    "ntr_sim_stats": (C.c_int, [_P, C.POINTER(Stats)]),
    "ntr_sim_pack_particles": (C.c_int, [_P, _P, C.c_size_t, _P]),
    "ntr_sim_profile": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "ntr_sim_last_launches": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    "ntr_sim_work": (C.c_int, [_P, C.POINTER(C.c_uint64), C.c_int]),
    "ntr_sim_test_barrier": (C.c_int, [_P, C.c_uint32, C.c_uint32]),
    "ntr_sim_conservation": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "ntr_sort_by_block_noalloc": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P, _P]),
    "ntr_sim_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "ntr_sim_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "ntr_sim_autotune": (C.c_int, [_P, C.c_uint32, C.POINTER(Tuning), C.POINTER(C.c_double)]),
    "ntr_probe_shared_atomics": (C.c_int, [C.c_int, C.c_uint32, C.POINTER(C.c_double)]),
    "ntr_batch_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "ntr_batch_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "ntr_batch_autotune": (C.c_int, [_P, C.c_uint32, C.POINTER(Tuning), C.POINTER(C.c_double)]),
    "ntr_batch_create": (C.c_int, [C.c_int, C.c_uint32, C.c_uint64, C.POINTER(_P)]),
    "ntr_batch_destroy": (C.c_int, [_P]),
    "ntr_batch_admit": (C.c_int, [_P, _P, C.c_size_t, C.c_uint32, C.POINTER(C.c_uint32)]),
    "ntr_batch_step": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "ntr_batch_profile": (C.c_int, [_P, C.c_uint32, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "ntr_batch_poll": (C.c_int, [_P, C.c_uint32, C.POINTER(BatchSlot)]),
    "ntr_batch_snapshot": (C.c_int, [_P, C.c_uint32, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "ntr_batch_retire": (C.c_int, [_P, C.c_uint32]),
    "ntr_batch_info_get": (C.c_int, [_P, C.POINTER(BatchInfo)]),
    "ntr_batch_enqueue": (C.c_int, [_P, _P, C.c_size_t, C.c_uint32, C.POINTER(C.c_uint64)]),
    "ntr_world_device_bytes": (C.c_int, [_P, C.c_size_t, C.POINTER(C.c_uint64)]),
    "ntr_batch_ticket": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_uint32)]),
    "ntr_cache_params_default": (C.c_int, [C.POINTER(SimParams), C.POINTER(CacheParams)]),
    "ntr_key_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]),
    "ntr_key_next_time": (C.c_double, [C.c_double, C.POINTER(C.c_double), C.c_uint32, C.c_double, C.c_uint64,
                                       C.c_uint64]),
    "ntr_cache_create": (C.c_int, [_P, C.POINTER(CacheParams), C.POINTER(_P)]),
    "ntr_cache_rebuild": (C.c_int, [_P, _P]),
    "ntr_cache_destroy": (C.c_int, [_P]),
    "ntr_cache_bake": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "ntr_cache_store": (C.c_int, [_P]),
    "ntr_cache_show": (C.c_int, [_P, C.c_double, C.POINTER(C.c_int)]),
    "ntr_cache_info_get": (C.c_int, [_P, C.POINTER(CacheInfo)]),
    "ntr_cache_last_times": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ntr_cache_key": (C.c_int, [_P, C.c_uint32, C.POINTER(KeyInfo)]),
    "ntr_cache_key_buffer": (C.c_int, [_P, C.c_uint32, C.POINTER(_P), C.POINTER(C.c_size_t)]),
    "ntr_cache_buffer": (C.c_int, [_P, C.c_int, C.POINTER(_P), C.POINTER(C.c_size_t)]),
    "ntr_cache_download": (C.c_int, [_P, C.c_uint32, _P, C.c_size_t]),
}

_lib = None


def lib() -> C.CDLL:
    """The native library, loaded once. Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m natray_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class NatrayError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def check(status: int) -> None:
    if status != 0:
        buf = C.create_string_buffer(1024)
        lib().ntr_last_error(buf, 1024)
        raise NatrayError(status, buf.value.decode(errors="replace"))


def declared_symbols() -> list[str]:
    """Entry points declared in include/natray.h (parsed from the header)."""
    import re
    text = (PKG.parent / "include" / "natray.h").read_text()
    return sorted(set(re.findall(r"NTR_API\s+[\w\s\*]+?\b(ntr_\w+)\s*\(", text)))


os.environ.setdefault("CUDA_MODULE_LOADING", "LAZY")
