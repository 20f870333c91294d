"""ctypes binding of libsundog.so (declarations in include/sundog_api.h).

The library is loaded from this package's lib/ directory (built in-tree by
sundog_b200.build). There is no fallback: if the shared library is missing
or fails to load, load() raises.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SUNDOG_B200_LIB") or os.path.join(HERE, "lib", "libsundog.so")

c_d3 = ctypes.c_double * 3


class XformStep(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("a", ctypes.c_double),
                ("b", ctypes.c_double), ("c", ctypes.c_double)]


class PhysicsBody(ctypes.Structure):
    _fields_ = [("dynamic", ctypes.c_int32), ("density", ctypes.c_double),
                ("has_velocity", ctypes.c_int32),
                ("has_angular_velocity", ctypes.c_int32),
                ("velocity", ctypes.c_double * 3),
                ("angular_velocity", ctypes.c_double * 3),
                ("friction", ctypes.c_double), ("restitution", ctypes.c_double),
                ("thickness", ctypes.c_double)]


class RenderOptions(ctypes.Structure):
    _fields_ = [("out_path", ctypes.c_char_p), ("stats_path", ctypes.c_char_p),
                ("aov_albedo_path", ctypes.c_char_p),
                ("aov_normal_path", ctypes.c_char_p),
                ("scene_name", ctypes.c_char_p),
                ("spp", ctypes.c_int32), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32), ("seed", ctypes.c_int64),
                ("denoise", ctypes.c_int32), ("transparent_shadows", ctypes.c_int32),
                ("clamp", ctypes.c_double), ("physics_time", ctypes.c_double),
                ("quiet", ctypes.c_int32)]


class DeviceInfo(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 256),
                ("cc_major", ctypes.c_int32), ("cc_minor", ctypes.c_int32),
                ("driver_version", ctypes.c_int32), ("runtime_version", ctypes.c_int32),
                ("total_mem_mb", ctypes.c_uint64),
                ("optix_header_version", ctypes.c_uint32),
                ("rtcore_version", ctypes.c_uint32)]


class RenderExt(ctypes.Structure):
    _fields_ = [("film_rgba", ctypes.c_void_p), ("aov_albedo", ctypes.c_void_p),
                ("aov_normal", ctypes.c_void_p), ("chunk_spp", ctypes.c_int32),
                ("repeat", ctypes.c_int32), ("guiding", ctypes.c_int32),
                ("sample_offset", ctypes.c_int32), ("frame_spp", ctypes.c_int32),
                ("engine", ctypes.c_int32), ("shard_count", ctypes.c_int32),
                ("shard_index", ctypes.c_int32)]


class RenderResult(ctypes.Structure):
    _fields_ = [("rays_traced", ctypes.c_uint64), ("paths", ctypes.c_uint64),
                ("render_ms", ctypes.c_double), ("build_ms", ctypes.c_double),
                ("load_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("mrays_per_sec", ctypes.c_double), ("samples_per_sec", ctypes.c_double),
                ("kernel_launches", ctypes.c_uint64), ("kernel_ms", ctypes.c_double)]


class SessionStats(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("spp", ctypes.c_int32), ("chunk_spp", ctypes.c_int32),
                ("grid", ctypes.c_int32), ("block", ctypes.c_int32),
                ("device_bytes", ctypes.c_uint64), ("bvh_nodes", ctypes.c_uint64),
                ("triangles", ctypes.c_uint64), ("instances", ctypes.c_uint64),
                ("tlas_depth", ctypes.c_int32), ("blas_depth", ctypes.c_int32),
                ("load_ms", ctypes.c_double), ("build_ms", ctypes.c_double),
                ("setup_ms", ctypes.c_double)]


class TraceCounts(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_uint64), ("box_tests", ctypes.c_uint64),
                ("tri_tests", ctypes.c_uint64), ("quadric_tests", ctypes.c_uint64),
                ("blas_entries", ctypes.c_uint64), ("trav_iters", ctypes.c_uint64),
                ("trav_lanes", ctypes.c_uint64), ("loop_iters", ctypes.c_uint64),
                ("loop_lanes", ctypes.c_uint64)]


class StageTimes(ctypes.Structure):
    _fields_ = [("start_ms", ctypes.c_double), ("trace_ms", ctypes.c_double),
                ("shade_a_ms", ctypes.c_double), ("shadow_ms", ctypes.c_double),
                ("shade_b_ms", ctypes.c_double), ("iterations", ctypes.c_uint64),
                ("radiance_rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("launches", ctypes.c_uint64)]


class GuidingConfig(ctypes.Structure):
    _fields_ = [("train_spp", ctypes.c_int32), ("pass_spp", ctypes.c_int32),
                ("steps_per_pass", ctypes.c_int32), ("batch", ctypes.c_int32),
                ("learning_rate", ctypes.c_float), ("mix", ctypes.c_float),
                ("seed", ctypes.c_uint64), ("record_cap", ctypes.c_uint64)]


class GuidingStats(ctypes.Structure):
    _fields_ = [("records", ctypes.c_uint64), ("passes", ctypes.c_int32),
                ("train_steps", ctypes.c_int32), ("train_ms", ctypes.c_double),
                ("bake_ms", ctypes.c_double), ("last_loss", ctypes.c_double),
                ("box_lo", ctypes.c_float * 3), ("box_hi", ctypes.c_float * 3)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("max_jobs", ctypes.c_int32), ("tile", ctypes.c_int32),
                ("pass_spp", ctypes.c_int32), ("engine", ctypes.c_int32),
                ("iteration_paths", ctypes.c_uint64), ("reserve_bytes", ctypes.c_uint64),
                ("scene_cache_bytes", ctypes.c_uint64)]


class JobStatus(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32), ("spp", ctypes.c_int32),
                ("paths_done", ctypes.c_uint64), ("paths_total", ctypes.c_uint64),
                ("queued_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("error", ctypes.c_char * 256)]


class ServerStatistics(ctypes.Structure):
    _fields_ = [("jobs_submitted", ctypes.c_uint64), ("jobs_done", ctypes.c_uint64),
                ("jobs_failed", ctypes.c_uint64), ("jobs_cancelled", ctypes.c_uint64),
                ("iterations", ctypes.c_uint64), ("rays", ctypes.c_uint64),
                ("paths", ctypes.c_uint64), ("busy_ms", ctypes.c_double),
                ("wall_ms", ctypes.c_double), ("active_jobs", ctypes.c_int32),
                ("queued_jobs", ctypes.c_int32), ("scenes_resident", ctypes.c_uint64),
                ("scene_bytes", ctypes.c_uint64)]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = range(5)

# Parameter count of the guiding network (include/sundog_api.h).
GUIDE_PARAMS = 14576

# Every symbol include/sundog_api.h declares (the first 27 are the drop-in
# surface of the reference ABI).
DROP_IN_SYMBOLS = [
    "sundog_last_error", "sundog_scene_create", "sundog_scene_destroy",
    "sundog_set_render", "sundog_set_camera", "sundog_set_background_solid",
    "sundog_set_background_gradient", "sundog_set_background_envmap",
    "sundog_set_physics", "sundog_add_texture_solid", "sundog_add_texture_checker",
    "sundog_add_texture_grid", "sundog_add_texture_image",
    "sundog_add_material_lambert", "sundog_add_material_metal",
    "sundog_add_material_dielectric", "sundog_add_material_emissive",
    "sundog_add_material_water", "sundog_add_material_plastic", "sundog_add_mesh",
    "sundog_add_object", "sundog_add_flame", "sundog_add_point_light",
    "sundog_add_distant_light", "sundog_scene_validate", "sundog_probe",
    "sundog_render",
]
ADDITIVE_SYMBOLS = [
    "sundog_set_flame_steps", "sundog_render_ex", "sundog_scene_debug_json",
    "sundog_selftest", "sundog_session_create", "sundog_session_render",
    "sundog_session_read", "sundog_session_info", "sundog_session_destroy",
    "sundog_session_trace_counts", "sundog_transfer_bytes",
    "sundog_session_render_tile_noalloc", "sundog_guiding_defaults",
    "sundog_session_set_guiding", "sundog_session_guiding_stats", "sundog_guide_init_params",
    "sundog_guide_outputs", "sundog_guide_gradients", "sundog_session_guide_params",
    "sundog_session_guide_records", "sundog_server_defaults", "sundog_server_create",
    "sundog_server_submit", "sundog_server_status", "sundog_server_wait",
    "sundog_server_cancel", "sundog_server_stats", "sundog_server_destroy",
    "sundog_session_copy_film", "sundog_session_trace_counts_split",
    "sundog_session_set_stage_timing", "sundog_session_stage_times", "sundog_session_table",
    "sundog_set_device_memory_cache", "sundog_release_device_memory", "sundog_session_read_pq12",
    "sundog_set_bvh_builder", "sundog_session_denoise", "sundog_server_create_on_device",
    "sundog_device_count",
]

_lib = None


def declare_scene_abi(lib):
    """Prototypes of the scene-construction half of the ABI (sundog_last_error
    ... sundog_scene_validate, plus sundog_set_flame_steps) on a loaded
    library. The CPU oracle applies them to its build of the reference's own
    scene code, which exports the same functions."""
    vp, ip, dp, cp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char_p
    d3 = ctypes.POINTER(ctypes.c_double)
    lib.sundog_last_error.restype = cp
    lib.sundog_scene_create.restype = vp
    lib.sundog_scene_create.argtypes = [cp]
    lib.sundog_scene_destroy.argtypes = [vp]
    lib.sundog_scene_destroy.restype = None
    lib.sundog_set_render.argtypes = [vp, ip, ip, ip, ip, dp, ctypes.c_int64, dp, ip]
    lib.sundog_set_camera.argtypes = [vp, d3, d3, d3, dp, dp, dp]
    lib.sundog_set_background_solid.argtypes = [vp, d3]
    lib.sundog_set_background_gradient.argtypes = [vp, d3, d3]
    lib.sundog_set_background_envmap.argtypes = [vp, cp, dp, dp, ip]
    lib.sundog_set_physics.argtypes = [vp, d3, dp, dp, dp, dp, ip, ip, dp, dp]
    lib.sundog_add_texture_solid.argtypes = [vp, d3]
    lib.sundog_add_texture_checker.argtypes = [vp, d3, d3, d3]
    lib.sundog_add_texture_grid.argtypes = [vp, d3, d3, d3, dp]
    lib.sundog_add_texture_image.argtypes = [vp, cp, ip]
    lib.sundog_add_material_lambert.argtypes = [vp, d3, ip]
    lib.sundog_add_material_metal.argtypes = [vp, d3, ip, dp]
    lib.sundog_add_material_dielectric.argtypes = [vp, dp, d3, d3, ip, dp]
    lib.sundog_add_material_emissive.argtypes = [vp, d3, ip, dp, ip]
    lib.sundog_add_material_water.argtypes = [vp, dp, d3, dp, dp, d3]
    lib.sundog_add_material_plastic.argtypes = [vp, d3, ip, dp]
    lib.sundog_add_mesh.argtypes = [vp, cp, ip, cp]
    lib.sundog_add_object.argtypes = [vp, ip, ip, ip, ip, ip, ctypes.POINTER(XformStep), ip,
                                      ip, ctypes.POINTER(PhysicsBody)]
    lib.sundog_add_flame.argtypes = [vp, d3, dp, dp, dp, dp, dp, ctypes.c_int64, dp]
    lib.sundog_add_point_light.argtypes = [vp, d3, d3, dp]
    lib.sundog_add_distant_light.argtypes = [vp, d3, d3]
    lib.sundog_scene_validate.argtypes = [vp]
    lib.sundog_set_flame_steps.argtypes = [vp, ip, ip]
    return lib


def load(path=None):
    """Load libsundog.so once and declare every prototype."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.isfile(p):
        raise RuntimeError("libsundog.so not built at %s (run sundog_b200.build.build())" % p)
    lib = ctypes.CDLL(p, mode=ctypes.RTLD_GLOBAL)
    declare_scene_abi(lib)
    vp, ip, dp, cp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char_p
    lib.sundog_probe.argtypes = [ctypes.POINTER(DeviceInfo)]
    lib.sundog_render.argtypes = [vp, ctypes.POINTER(RenderOptions)]
    lib.sundog_render_ex.argtypes = [vp, ctypes.POINTER(RenderOptions),
                                     ctypes.POINTER(RenderExt), ctypes.POINTER(RenderResult)]
    lib.sundog_scene_debug_json.argtypes = [vp, cp, ctypes.c_size_t,
                                            ctypes.POINTER(ctypes.c_size_t)]
    lib.sundog_selftest.argtypes = [ip, vp, ip, vp, ctypes.c_size_t]
    lib.sundog_selftest_sizes.argtypes = [ip, ctypes.POINTER(ctypes.c_size_t),
                                          ctypes.POINTER(ctypes.c_size_t)]
    lib.sundog_session_create.restype = vp
    lib.sundog_session_create.argtypes = [vp, ctypes.POINTER(RenderOptions),
                                          ctypes.POINTER(RenderExt)]
    lib.sundog_session_render.argtypes = [vp, vp, ip, ctypes.POINTER(RenderResult)]
    lib.sundog_session_read.argtypes = [vp, vp, vp, vp]
    lib.sundog_session_info.argtypes = [vp, ctypes.POINTER(SessionStats)]
    lib.sundog_session_copy_film.argtypes = [vp, vp, vp]
    lib.sundog_session_trace_counts.argtypes = [vp, ctypes.POINTER(TraceCounts)]
    lib.sundog_session_trace_counts_split.argtypes = [vp, ctypes.POINTER(TraceCounts),
                                                      ctypes.POINTER(TraceCounts)]
    lib.sundog_session_table.argtypes = [vp, ip, vp, ctypes.c_size_t,
                                         ctypes.POINTER(ctypes.c_size_t)]
    lib.sundog_session_read_pq12.argtypes = [vp, dp, vp]
    lib.sundog_session_denoise.argtypes = [vp, vp]
    lib.sundog_set_bvh_builder.argtypes = [ip]
    lib.sundog_set_device_memory_cache.argtypes = [ip]
    lib.sundog_release_device_memory.argtypes = []
    lib.sundog_session_set_stage_timing.argtypes = [vp, ip]
    lib.sundog_session_stage_times.argtypes = [vp, ctypes.POINTER(StageTimes)]
    lib.sundog_transfer_bytes.argtypes = [ctypes.POINTER(ctypes.c_uint64)] * 2
    lib.sundog_transfer_bytes.restype = None
    lib.sundog_session_render_tile_noalloc.argtypes = [vp, ip, ip, ip, ip, ip, ip, vp,
                                                       ctypes.POINTER(ctypes.c_uint64), vp]
    lib.sundog_session_destroy.argtypes = [vp]
    lib.sundog_session_destroy.restype = None
    lib.sundog_guiding_defaults.argtypes = [ctypes.POINTER(GuidingConfig)]
    lib.sundog_guiding_defaults.restype = None
    lib.sundog_session_set_guiding.argtypes = [vp, ip, ctypes.POINTER(GuidingConfig)]
    lib.sundog_session_guiding_stats.argtypes = [vp, ctypes.POINTER(GuidingStats)]
    lib.sundog_guide_init_params.argtypes = [ctypes.c_uint64, vp]
    lib.sundog_guide_outputs.argtypes = [vp, vp, ip, vp]
    lib.sundog_guide_gradients.argtypes = [vp, vp, ip, vp, vp, vp]
    lib.sundog_session_guide_params.argtypes = [vp, vp]
    lib.sundog_session_guide_records.argtypes = [vp, vp, ctypes.c_uint64,
                                                 ctypes.POINTER(ctypes.c_uint64)]
    lib.sundog_server_defaults.argtypes = [ctypes.POINTER(ServerConfig)]
    lib.sundog_server_defaults.restype = None
    lib.sundog_server_create.argtypes = [ctypes.POINTER(ServerConfig)]
    lib.sundog_server_create.restype = vp
    lib.sundog_server_create_on_device.argtypes = [ctypes.POINTER(ServerConfig), ip]
    lib.sundog_server_create_on_device.restype = vp
    lib.sundog_device_count.argtypes = []
    lib.sundog_server_submit.argtypes = [vp, vp, ctypes.POINTER(RenderOptions), vp]
    lib.sundog_server_submit.restype = ctypes.c_int64
    lib.sundog_server_status.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(JobStatus)]
    lib.sundog_server_wait.argtypes = [vp, ctypes.c_int64, dp, ctypes.POINTER(JobStatus)]
    lib.sundog_server_cancel.argtypes = [vp, ctypes.c_int64]
    lib.sundog_server_stats.argtypes = [vp, ctypes.POINTER(ServerStatistics)]
    lib.sundog_server_destroy.argtypes = [vp]
    lib.sundog_server_destroy.restype = None
    if path is None:
        _lib = lib
    return lib


def last_error(lib=None):
    lib = lib or load()
    return (lib.sundog_last_error() or b"unknown error").decode("utf-8", "replace")


class SundogError(RuntimeError):
    """A libsundog call returned an error code; the message is the library's."""


def check(rc, what, lib=None):
    if rc != 0:
        raise SundogError("%s: %s" % (what, last_error(lib)))
    return rc


def options(out=None, stats=None, aov_albedo=None, aov_normal=None, scene_name="(scene)",
            spp=-1, width=-1, height=-1, seed=-1, denoise=-1, transparent_shadows=-1,
            clamp=float("nan"), physics_time=float("nan"), quiet=True):
    """sundog_render_options with the ABI's "unset" sentinels as defaults."""
    enc = lambda s: s.encode() if s else None
    return RenderOptions(out_path=enc(out), stats_path=enc(stats),
                         aov_albedo_path=enc(aov_albedo), aov_normal_path=enc(aov_normal),
                         scene_name=enc(scene_name), spp=spp, width=width, height=height,
                         seed=seed, denoise=denoise, transparent_shadows=transparent_shadows,
                         clamp=clamp, physics_time=physics_time, quiet=1 if quiet else 0)
