"""ctypes declarations of the C ABI in ``include/ropephysics_b200.h``.

``load()`` opens the in-tree ``librp_b200.so`` and declares every exported
function. There is no fallback: if the library is missing the import fails
with the build command to run.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librp_b200.so")

i32, i64, f32, f64, u8 = C.c_int32, C.c_int64, C.c_float, C.c_double, C.c_uint8
P = C.POINTER


class Material(C.Structure):
    _fields_ = [("youngs", f64), ("poisson", f64), ("density", f64), ("radius", f64)]


class RodDesc(C.Structure):
    _fields_ = [
        ("num_particles", i32), ("num_frames", i32), ("num_stretch", i32), ("num_bend", i32),
        ("material", Material),
        ("x", P(f64)), ("v", P(f64)), ("inv_mass", P(f64)), ("mass", P(f64)),
        ("ext_force", P(f64)), ("kin_velocity", P(f64)),
        ("q", P(f64)), ("omega", P(f64)), ("inertia", P(f64)), ("inv_inertia", P(f64)),
        ("ext_torque", P(f64)),
        ("s_p0", P(i32)), ("s_p1", P(i32)), ("s_seg", P(i32)), ("s_rest", P(f64)),
        ("s_compliance", P(f64)),
        ("b_a", P(i32)), ("b_b", P(i32)), ("b_rest", P(f64)), ("b_compliance", P(f64)),
        ("b_rest_darboux", P(f64)),
    ]


class Primitive(C.Structure):
    _fields_ = [("type", i32), ("reserved", i32), ("a", f64 * 3), ("b", f64 * 3),
                ("normal", f64 * 3), ("half_extents", f64 * 3), ("rotation", f64 * 4),
                ("radius", f64), ("friction", f64)]


class World(C.Structure):
    _fields_ = [("primitives", P(Primitive)), ("num_primitives", i32), ("self_collision", i32),
                ("self_friction", f64), ("self_skip", i32), ("hash_table_size", i32),
                ("contact_margin_radii", f64)]


class StepParams(C.Structure):
    _fields_ = [("dt", f32), ("substeps", i32), ("iterations", i32), ("gravity", f32 * 3),
                ("linear_damping", f32), ("angular_damping", f32), ("contact_interval", i32)]


class Drive(C.Structure):
    _fields_ = [("particle", i32), ("reserved", i32), ("axis", f32 * 3), ("amplitude", f32),
                ("frequency", f32), ("phase", f32)]


MAX_WAYPOINTS = 8


class WaypointDrive(C.Structure):
    _fields_ = [("particle", i32), ("count", i32), ("steps_per_control", i32), ("reserved", i32),
                ("dt", C.c_double), ("start", C.c_double * 2), ("height", C.c_double),
                ("legs", C.c_double * MAX_WAYPOINTS), ("waypoints", (C.c_double * 2) * MAX_WAYPOINTS)]


class HarnessBoard(C.Structure):
    _fields_ = [("peg_a", C.c_double * 2), ("peg_b", C.c_double * 2), ("clip", C.c_double * 2),
                ("peg_radius", C.c_double), ("clip_half_gap", C.c_double), ("clip_height", C.c_double),
                ("cable_radius", C.c_double), ("lay_slack", C.c_double)]


class HarnessOutcome(C.Structure):
    _fields_ = [("score", C.c_double), ("side_a", C.c_double), ("side_b", C.c_double),
                ("clip_miss", C.c_double), ("below_a", C.c_uint8), ("above_b", C.c_uint8),
                ("through_clip", C.c_uint8), ("success", C.c_uint8), ("reserved", C.c_uint8 * 4)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("params", StepParams), ("precision", i32),
                ("max_steps_in_flight", i32)]


class Request(C.Structure):
    _fields_ = [("rods", P(P(RodDesc))), ("num_rods", i32), ("steps", i32), ("worlds", P(World)),
                ("num_worlds", i32), ("reserved", i32), ("world_of_rod", P(i32)), ("drives", P(Drive)),
                ("youngs_scale", P(f32)), ("friction_scale", P(f32))]


class RequestInfo(C.Structure):
    _fields_ = [("state", i32), ("num_rods", i32), ("num_particles", i64), ("resident_bytes", i64),
                ("segment_substeps", i64), ("submit_s", f64), ("admit_s", f64), ("done_s", f64)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", i64), ("admitted", i64), ("completed", i64), ("queued", i64),
                ("running", i64), ("steps_launched", i64), ("segment_substeps", i64),
                ("resident_bytes", i64), ("peak_resident_bytes", i64), ("budget_bytes", i64),
                ("now_s", f64), ("busy_s", f64)]


vp = C.c_void_p
pp = P(vp)

# name: (restype, argtypes) -- one entry per declaration in the header
SIGNATURES = {
    "rp_abi_version": (i32, []),
    "rp_cuda_available": (i32, []),
    "rp_device_name": (i32, [C.c_char_p, C.c_size_t]),
    "rp_diagnostic": (i32, [C.c_char_p, C.c_size_t]),
    "rp_max_fused_segments": (i32, []),
    "rp_last_error": (C.c_char_p, []),
    "rp_measure_fp32_peak": (i32, [i32, P(f64), P(f64)]),
    "rp_rod_create_straight": (i32, [i32, f64, P(Material), P(f64), P(f64), pp]),
    "rp_rod_create_centerline": (i32, [P(f64), i32, P(Material), P(f64), f64, pp]),
    "rp_rod_create_from_desc": (i32, [P(RodDesc), pp]),
    "rp_rod_destroy": (None, [vp]),
    "rp_rod_view": (i32, [vp, P(RodDesc)]),
    "rp_rod_clamp_end": (i32, [vp, i32, P(i32)]),
    "rp_rod_pin_particle": (i32, [vp, i32]),
    "rp_rod_set_rest_from_current": (i32, [vp]),
    "rp_rod_coloring": (i32, [P(RodDesc), i32, P(i32), P(i32), P(i32)]),
    "rp_color_constraints": (i32, [i32, P(i32), P(i32), P(i32), P(i32), P(i32)]),
    "rp_self_collision_index_gap": (i32, [P(RodDesc), P(World), P(i32)]),
    "rp_batch_create": (i32, [P(RodDesc), i32, i32, P(World), pp]),
    "rp_batch_create_mixed": (i32, [P(P(RodDesc)), i32, P(World), i32, P(i32), i32, pp]),
    "rp_batch_destroy": (None, [vp]),
    "rp_batch_step": (i32, [vp, P(StepParams)]),
    "rp_batch_step_many": (i32, [vp, P(StepParams), i32]),
    "rp_batch_step_static_scratch": (i32, [vp, P(StepParams)]),
    "rp_batch_autotune": (i32, [vp, P(StepParams), i32]),
    "rp_batch_get_tuning": (i32, [vp, P(C.c_int32), P(C.c_int32), P(C.c_int32)]),
    "rp_batch_set_tuning": (i32, [vp, i32, i32, i32]),
    "rp_batch_synchronize": (i32, [vp]),
    "rp_batch_set_stream": (i32, [vp, vp]),
    "rp_batch_set_precision": (i32, [vp, i32]),
    "rp_batch_set_graph": (i32, [vp, i32]),
    "rp_batch_download": (i32, [vp, i32, P(RodDesc)]),
    "rp_batch_download_positions": (i32, [vp, P(f32), i64]),
    "rp_batch_download_frames": (i32, [vp, P(f32), i64]),
    "rp_batch_upload": (i32, [vp, P(RodDesc)]),
    "rp_batch_set_loads": (i32, [vp, i32, P(RodDesc)]),
    "rp_batch_upload_rod": (i32, [vp, i32, P(RodDesc)]),
    "rp_batch_set_kinematic_velocities": (i32, [vp, P(f32), i64]),
    "rp_batch_set_material_scales": (i32, [vp, P(f32), P(f32), i32]),
    "rp_batch_set_drives": (i32, [vp, P(Drive), i32]),
    "rp_batch_set_time": (i32, [vp, f64]),
    "rp_batch_set_waypoint_drives": (i32, [vp, P(WaypointDrive), i32]),
    "rp_batch_evaluate_harness": (i32, [vp, P(HarnessBoard), P(HarnessOutcome), i32]),
    "rp_batch_read_state_async": (i32, [vp, i32, vp, i64]),
    "rp_batch_write_state_async": (i32, [vp, i32, vp, i64]),
    "rp_batch_set_copy_stream": (i32, [vp, vp]),
    "rp_batch_read_state_overlapped": (i32, [vp, i32, vp, i64]),
    "rp_batch_write_state_overlapped": (i32, [vp, i32, vp, i64]),
    "rp_batch_read_contact_states": (i32, [vp, P(u8), i64, P(i64)]),
    "rp_batch_read_self_contacts": (i32, [vp, i32, P(i32), i32, P(i32)]),
    "rp_batch_arm_hold_observer": (i32, [vp, P(i32), i32, i32, f64]),
    "rp_batch_arm_hold_observer_at": (i32, [vp, P(i32), P(f64), i32, i32, f64]),
    "rp_batch_read_hold_verdicts": (i32, [vp, P(f64), P(u8), P(u8), i32]),
    "rp_batch_num_rods": (i32, [vp]),
    "rp_batch_num_segments": (i32, [vp, i32]),
    "rp_batch_num_particles": (i32, [vp, i32]),
    "rp_batch_particle_offset": (i64, [vp, i32]),
    "rp_batch_num_frames": (i32, [vp, i32]),
    "rp_batch_frame_offset": (i64, [vp, i32]),
    "rp_batch_strategy": (i32, [vp]),
    "rp_batch_stretch_colors": (i32, [vp]),
    "rp_batch_bend_colors": (i32, [vp]),
    "rp_batch_shared_bytes_per_block": (C.c_size_t, [vp]),
    "rp_batch_launches_per_step": (i32, [vp, P(StepParams)]),
    "rp_batch_self_contact_overflow": (i64, [vp]),
    "rp_batch_kernel_launches": (i64, [vp]),
    "rp_batch_error_count": (i64, [vp]),
    "rp_server_create": (i32, [P(ServerConfig), pp]),
    "rp_server_destroy": (None, [vp]),
    "rp_server_submit": (i32, [vp, P(Request), P(C.c_uint64)]),
    "rp_server_info": (i32, [vp, C.c_uint64, P(RequestInfo)]),
    "rp_server_wait": (i32, [vp, C.c_uint64, f64]),
    "rp_server_result": (i32, [vp, C.c_uint64, P(f32), i64]),
    "rp_server_release": (i32, [vp, C.c_uint64]),
    "rp_server_get_stats": (i32, [vp, P(ServerStats)]),
    "rp_server_drain": (i32, [vp, f64]),
    "rp_traj_open": (i32, [C.c_char_p, i32, vp, f32, f32, pp]),
    "rp_traj_append": (i32, [vp, vp, f32]),
    "rp_traj_close": (i32, [vp, P(i32)]),
}

_lib = None


def load():
    """Open the native library once and declare its functions."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m ropephysics_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def header_symbols(header: str) -> list:
    """Function names declared in the C header (for the export check)."""
    import re
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rp_[a-z0-9_]+)\s*\(", text)))
