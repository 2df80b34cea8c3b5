"""ctypes mirrors of the C ABI types declared in include/slosh_cuda.h.

Each structure follows the plugin type it stands in for (SloshDemo/Plugins/Slosh/Source/SloshCore/
Public/SloshTypes.h): SloshSettings <- FSloshSolverSettings (:113-160), Particle <- FSloshParticleGPU
(:84-91), Collider <- FSloshColliderGPU (:32-44), Manipulator <- FSloshManipulatorGPU (:66-80),
EmitRequest <- FSloshEmitRequest (:169-181), FrameInput <- FSloshFrameInput (:184-194),
Results <- FSloshResults (:208-231).
"""
import ctypes as C

import numpy as np

MAX_COLLIDERS = 64
MAX_MANIPULATORS = 32
NUM_STATS = 16
MAX_MG_LEVELS = 8

# slosh_status
OK = 0
ERR_INVALID_ARG = 1
ERR_OUT_OF_MEMORY = 2
WARN_POOL_OVERFLOW = 3
ERR_NOT_CONVERGED = 4
ERR_DEVICE_TIMEOUT = 5
ERR_CUDA = 6
ERR_NO_DEVICE = 7
ERR_CAPACITY = 8
WARNINGS = (WARN_POOL_OVERFLOW, ERR_NOT_CONVERGED)

TRANSFER_FLIP, TRANSFER_APIC = 0, 1
MANIP_DRAIN, MANIP_DIRECTIONAL, MANIP_RADIAL, MANIP_SWIRL, MANIP_DRAG = 0, 1, 2, 3, 4
SHAPE_SPHERE, SHAPE_BOX, SHAPE_CAPSULE, SHAPE_EVERYWHERE = 0, 1, 2, 3
SOLVER_RBGS, SOLVER_MGPCG = 0, 1
COLLIDER_SPHERE, COLLIDER_BOX, COLLIDER_CAPSULE = 0, 1, 2
EMIT_FILL_CELLS, EMIT_SPHERE, EMIT_BOX = 0, 1, 2
PRECISION_FP32, PRECISION_FP16_STORAGE, PRECISION_BF16_STORAGE = 0, 1, 2
WARM_START_ZERO, WARM_START_PREVIOUS, WARM_START_LEARNED = 0, 1, 2

# slosh_buffer_id
BUF = dict(
    PARTICLES=0, VEL=1, VEL_OLD=2, FACE_FLAGS=3, FACE_WEIGHT=4, CELL_TYPE=5, CELL_COUNT=6, PRESSURE=7,
    DIVERGENCE=8, CELL_DIAG=9, DENSITY_Q=10, DENSITY_RHS=11, BRICK_TABLE=12, SLOT_BRICK=13, FREE_SLOTS=14,
    ACTIVE_BRICKS=15, NEW_SLOTS=16, BRICK_TOUCH=17, STATS=18, SORT_COUNTS=19, SORT_OFFSETS=20, SORT_PERM=21,
    PARTICLE_COUNT=22, ACCUM=23, VEL_EXTRAP=24, COUPLING=25,
    SURFACE_FIELD=26, SURFACE_BRICKS=27, SURFACE_POSITIONS=28, SURFACE_NORMALS=29, SURFACE_TANGENTS=30,
    SURFACE_INDICES=31,
)
BUF_DTYPE = dict(
    PARTICLES=None, VEL=np.float32, VEL_OLD=np.float32, FACE_FLAGS=np.uint32, FACE_WEIGHT=np.float32,
    CELL_TYPE=np.uint32, CELL_COUNT=np.int32, PRESSURE=np.float32, DIVERGENCE=np.float32, CELL_DIAG=np.float32,
    DENSITY_Q=np.float32, DENSITY_RHS=np.float32, BRICK_TABLE=np.uint32, SLOT_BRICK=np.uint32,
    FREE_SLOTS=np.uint32, ACTIVE_BRICKS=np.uint32, NEW_SLOTS=np.uint32, BRICK_TOUCH=np.uint32, STATS=np.uint32,
    SORT_COUNTS=np.uint32, SORT_OFFSETS=np.uint32, SORT_PERM=np.uint32, PARTICLE_COUNT=np.uint32,
    ACCUM=np.int32, VEL_EXTRAP=np.float32, COUPLING=np.int32,
    SURFACE_FIELD=np.uint16, SURFACE_BRICKS=np.uint32, SURFACE_POSITIONS=np.float32, SURFACE_NORMALS=np.float32,
    SURFACE_TANGENTS=np.float32, SURFACE_INDICES=np.uint32,
)


class Settings(C.Structure):
    _fields_ = [
        ("grid_dim", C.c_int32 * 3), ("cell_size", C.c_float), ("particle_capacity", C.c_uint32),
        ("transfer_mode", C.c_uint32), ("flip_ratio", C.c_float), ("density", C.c_float),
        ("kinematic_viscosity", C.c_float), ("boundary_friction", C.c_float), ("adhesion", C.c_float),
        ("adhesion_distance", C.c_float), ("density_correction", C.c_float), ("density_deadband", C.c_float),
        ("two_sided_density_projection", C.c_uint32), ("density_relaxation", C.c_float),
        ("density_projection_iterations", C.c_int32), ("density_projection_interval", C.c_int32),
        ("sparse_bricks", C.c_uint32), ("sparse_max_active_fraction", C.c_float),
        ("sparse_storage_budget", C.c_float), ("particle_radius_cells", C.c_float), ("gravity", C.c_float * 3),
        ("pressure_solver", C.c_uint32), ("pressure_iterations", C.c_int32), ("sor_weight", C.c_float),
        ("pcg_iterations", C.c_int32), ("mg_coarse_iterations", C.c_int32), ("sort_interval", C.c_int32),
        ("smooth_coupling_force", C.c_uint32), ("ghost_fluid", C.c_uint32), ("viscosity_iterations", C.c_int32),
        ("extrapolation_layers", C.c_int32), ("min_substeps", C.c_int32), ("max_substeps", C.c_int32),
        ("max_frame_dt", C.c_float), ("cfl", C.c_float), ("max_speed", C.c_float),
        ("tolerance", C.c_float), ("max_iterations", C.c_int32), ("precision_mode", C.c_uint32),
        ("warm_start", C.c_uint32), ("mg_correction_scale", C.c_float), ("mg_smoothing_sweeps", C.c_int32),
        ("pcg_flexible", C.c_uint32), ("mg_smoother_weight", C.c_float),
    ]


class Particle(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("age", C.c_float), ("vel", C.c_float * 3), ("c", C.c_uint32 * 5)]


class Collider(C.Structure):
    _fields_ = [
        ("center", C.c_float * 3), ("type", C.c_uint32), ("rotation", C.c_float * 4), ("extent", C.c_float * 3),
        ("flags", C.c_uint32), ("linear_velocity", C.c_float * 3), ("pad0", C.c_float),
        ("angular_velocity", C.c_float * 3), ("pad1", C.c_float),
    ]


class Manipulator(C.Structure):
    _fields_ = [
        ("center", C.c_float * 3), ("kind", C.c_uint32), ("rotation", C.c_float * 4), ("extent", C.c_float * 3),
        ("shape", C.c_uint32), ("axis", C.c_float * 3), ("strength", C.c_float), ("falloff", C.c_float),
        ("param0", C.c_float), ("param1", C.c_float), ("pad", C.c_uint32),
    ]


class EmitRequest(C.Structure):
    _fields_ = [
        ("shape", C.c_uint32), ("center", C.c_float * 3), ("extent", C.c_float * 3), ("velocity", C.c_float * 3),
        ("rotation", C.c_float * 4), ("velocity_spread", C.c_float), ("speed_jitter", C.c_float),
        ("cell_min", C.c_int32 * 3), ("cell_dims", C.c_int32 * 3), ("count", C.c_uint32),
        ("fill_jitter", C.c_float),
    ]


class SurfaceParams(C.Structure):
    _fields_ = [
        ("field_resolution", C.c_float), ("surface_smoothing", C.c_float), ("particle_radius_scale", C.c_float),
        ("iso_level", C.c_float), ("build_mesh", C.c_uint32), ("max_vertices", C.c_uint32), ("max_indices", C.c_uint32),
    ]


class SurfaceInfo(C.Structure):
    _fields_ = [
        ("field_dim", C.c_int32 * 3), ("brick_dim", C.c_int32 * 3), ("voxel_size", C.c_float),
        ("vertices_requested", C.c_uint32), ("num_vertices", C.c_uint32), ("indices_requested", C.c_uint32),
        ("num_indices", C.c_uint32),
    ]


class FrameInput(C.Structure):
    _fields_ = [
        ("settings", Settings), ("colliders", C.POINTER(Collider)), ("num_colliders", C.c_uint32),
        ("emits", C.POINTER(EmitRequest)), ("num_emits", C.c_uint32),
        ("manipulators", C.POINTER(Manipulator)), ("num_manipulators", C.c_uint32),
        ("delta_time", C.c_float), ("reset", C.c_uint32), ("paused", C.c_uint32),
    ]


class ColliderFeedback(C.Structure):
    _fields_ = [
        ("pressure_force", C.c_float * 3), ("pressure_torque", C.c_float * 3),
        ("mean_fluid_velocity", C.c_float * 3), ("submerged_centroid_offset", C.c_float * 3),
        ("wetted_faces", C.c_int32), ("submerged_cells", C.c_int32), ("solid_cells", C.c_int32),
    ]


class Results(C.Structure):
    _fields_ = [
        ("max_particle_speed", C.c_float), ("fluid_cells", C.c_int32), ("max_divergence", C.c_float),
        ("mean_divergence", C.c_float), ("mean_interior_density", C.c_float), ("interior_cells", C.c_int32),
        ("active_brick_fraction", C.c_float), ("pool_usage", C.c_float), ("pool_overflow_bricks", C.c_int32),
        ("clamped_particles", C.c_int32), ("clamped_in_solid", C.c_int32), ("clamped_centroid", C.c_float * 3),
        ("grid_memory_mb", C.c_float), ("particle_memory_mb", C.c_float),
        ("allocated_particle_capacity", C.c_int32), ("live_particles", C.c_int32),
        ("drained_particles", C.c_int64), ("substeps", C.c_int32), ("sim_frame", C.c_uint64),
        ("num_colliders", C.c_uint32), ("colliders", ColliderFeedback * MAX_COLLIDERS),
        ("last_solve_iterations", C.c_int32), ("last_solve_rel_residual", C.c_float),
        ("last_solve_true_rel_residual", C.c_float), ("raw_stats", C.c_uint32 * NUM_STATS),
    ]


class Layout(C.Structure):
    _fields_ = [
        ("grid_dim", C.c_int32 * 3), ("brick_dim", C.c_int32 * 3), ("num_bricks", C.c_uint32),
        ("num_pool_bricks", C.c_uint32), ("pool_cells", C.c_uint32), ("total_faces", C.c_uint32),
        ("sort_brick_dim", C.c_int32 * 3), ("num_sort_keys", C.c_uint32), ("num_mg_levels", C.c_uint32),
        ("mg_dim", (C.c_int32 * 3) * MAX_MG_LEVELS), ("num_particles", C.c_uint32),
        ("particle_capacity", C.c_uint32), ("current_vel", C.c_uint32),
    ]


assert C.sizeof(Particle) == 48
assert C.sizeof(Collider) == 80
assert C.sizeof(Manipulator) == 80

# numpy view of the 48-byte particle record
PARTICLE_DTYPE = np.dtype([("pos", "<f4", 3), ("age", "<f4"), ("vel", "<f4", 3), ("c", "<u4", 5)])
assert PARTICLE_DTYPE.itemsize == 48


def settings_default(lib):
    """Reference defaults (SloshTypes.h:113-160) through the library's own default function."""
    s = Settings()
    lib(C.byref(s))
    return s


def frame_input(settings, emits=(), colliders=(), manipulators=(), delta_time=1.0 / 120.0, reset=False,
                paused=False):
    """Builds a FrameInput; the returned object keeps its arrays alive."""
    fi = FrameInput()
    fi.settings = settings
    ea = (EmitRequest * max(len(emits), 1))(*emits) if emits else None
    ca = (Collider * max(len(colliders), 1))(*colliders) if colliders else None
    ma = (Manipulator * max(len(manipulators), 1))(*manipulators) if manipulators else None
    fi.emits = C.cast(ea, C.POINTER(EmitRequest)) if ea is not None else None
    fi.num_emits = len(emits)
    fi.colliders = C.cast(ca, C.POINTER(Collider)) if ca is not None else None
    fi.num_colliders = len(colliders)
    fi.manipulators = C.cast(ma, C.POINTER(Manipulator)) if ma is not None else None
    fi.num_manipulators = len(manipulators)
    fi.delta_time = delta_time
    fi.reset = 1 if reset else 0
    fi.paused = 1 if paused else 0
    fi._keep = (ea, ca, ma)
    return fi


class UnetConfig(C.Structure):
    """slosh_unet_config_t: the learned warm-start network's grid, batch, seed and Adam settings."""
    _fields_ = [("dim", C.c_uint32 * 3), ("batch", C.c_uint32), ("seed", C.c_uint32), ("learning_rate", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float)]


class ConvTest(C.Structure):
    """slosh_conv_test_t: one convolution's host arrays for slosh_unet_conv_test."""
    _fields_ = [("dim", C.c_uint32 * 3), ("batch", C.c_uint32), ("nblocks", C.c_uint32), ("cin", C.c_uint32 * 2),
                ("cout", C.c_uint32), ("x", C.c_void_p * 2), ("w", C.c_void_p), ("bias", C.c_void_p), ("dy", C.c_void_p),
                ("y", C.c_void_p), ("dx", C.c_void_p * 2), ("dw", C.c_void_p), ("db", C.c_void_p)]


class AutotuneResult(C.Structure):
    """slosh_autotune_result_t: per candidate CTAs-per-SM count, the device ms per substep."""
    _fields_ = [("num_candidates", C.c_uint32), ("ctas_per_sm", C.c_uint32 * 8), ("ms_per_substep", C.c_float * 8),
                ("best_ctas_per_sm", C.c_uint32), ("brick_ctas", C.c_uint32)]
