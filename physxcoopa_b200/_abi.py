"""ctypes / numpy mirrors of the plain-old-data types in include/physxcoopa_b200.h.

The numpy dtypes reproduce the reference's in-memory layouts (physxcoopa/cloth/cloth.h:83-160,
physxcoopa/hair/strand.h:79-87) byte for byte, so arrays built here can be handed to the C-ABI
(and to the reference's own code) without conversion.
"""
import ctypes as C

import numpy as np

f32 = C.c_float
u32 = C.c_uint32
i32 = C.c_int32

PARTICLE = np.dtype([("position", "<f4", 3), ("prev_position", "<f4", 3),
                     ("velocity", "<f4", 3), ("inv_mass", "<f4")])
CONSTRAINT = np.dtype([("a", "<u4"), ("b", "<u4"), ("rest_length", "<f4"), ("lambda", "<f4")])
BATCH = np.dtype([("begin", "<u4"), ("end", "<u4")])
TETHER = np.dtype([("particle", "<u4"), ("anchor", "<u4"), ("max_length", "<f4")])
ANCHOR = np.dtype([("particle", "<u4"), ("body_index", "<u4"), ("body_generation", "<u4"),
                   ("local_position", "<f4", 3), ("world_position", "<f4", 3),
                   ("prev_world_position", "<f4", 3)])
STRAND = np.dtype([("first", "<u4"), ("count", "<u4"), ("root_position", "<f4", 3),
                   ("root_orientation", "<f4", 4), ("prev_root_position", "<f4", 3),
                   ("prev_root_orientation", "<f4", 4)])
COLLIDER = np.dtype([("type", "<i4"), ("enabled", "<i4"), ("position", "<f4", 3),
                     ("orientation", "<f4", 4), ("local_center", "<f4", 3),
                     ("local_rotation", "<f4", 4), ("radius", "<f4"), ("half_extents", "<f4", 3),
                     ("capsule_radius", "<f4"), ("capsule_half_height", "<f4"),
                     ("capsule_axis", "<i4"), ("sweep", "<f4", 3), ("end_orientation", "<f4", 4),
                     ("bounds_min", "<f4", 3), ("bounds_max", "<f4", 3),
                     ("geometry", "<u4"), ("geometry_scale", "<f4")])
BODY_POSE = np.dtype([("position", "<f4", 3), ("orientation", "<f4", 4), ("generation", "<u4"),
                      ("alive", "<u4")])
GRAVITY_SOURCE = np.dtype([("centre", "<f4", 3), ("strength", "<f4"), ("radius", "<f4"),
                           ("range", "<f4")])
FRAME_RESULT = np.dtype([("bounds_min", "<f4", 3), ("bounds_max", "<f4", 3),
                         ("max_speed", "<f4"), ("time", "<f4")])

assert PARTICLE.itemsize == 40 and CONSTRAINT.itemsize == 16 and ANCHOR.itemsize == 48
assert STRAND.itemsize == 64 and COLLIDER.itemsize == 152 and TETHER.itemsize == 12
assert BODY_POSE.itemsize == 36

SHAPE_SPHERE, SHAPE_BOX, SHAPE_CAPSULE, SHAPE_TRIANGLE_MESH, SHAPE_CONVEX_HULL = range(5)

(PXB_OK, PXB_ERR_INVALID_ARGUMENT, PXB_ERR_UNSUPPORTED, PXB_ERR_CUDA, PXB_ERR_OUT_OF_MEMORY,
 PXB_ERR_INVALID_HANDLE, PXB_ERR_DEVICE_STATUS, PXB_ERR_TOO_LARGE) = range(8)
STATUS_NAMES = {0: "PXB_OK", 1: "PXB_ERR_INVALID_ARGUMENT", 2: "PXB_ERR_UNSUPPORTED",
                3: "PXB_ERR_CUDA", 4: "PXB_ERR_OUT_OF_MEMORY", 5: "PXB_ERR_INVALID_HANDLE",
                6: "PXB_ERR_DEVICE_STATUS", 7: "PXB_ERR_TOO_LARGE"}


class ClothParams(C.Structure):
    """pxb_cloth_params == cloth::ClothParams (cloth.h:167-256) + the shear-compliance extension."""
    _fields_ = [("stretch_compliance", f32), ("bend_compliance", f32), ("damping", f32),
                ("thickness", f32), ("friction", f32), ("gravity_scale", f32),
                ("max_velocity", f32), ("external_acceleration", f32 * 3), ("wind", f32 * 3),
                ("wind_turbulence", f32), ("air_drag", f32), ("air_lift", f32),
                ("self_collision", i32), ("self_distance", f32), ("tether_scale", f32),
                ("substeps", u32), ("iterations", u32), ("sleep_threshold", f32),
                ("sleep_time", f32), ("layer", u32), ("has_shear_compliance", i32),
                ("shear_compliance", f32)]

    @classmethod
    def defaults(cls):
        """The reference's ClothParams defaults (cloth.h:171-255)."""
        p = cls()
        p.stretch_compliance = 0.0
        p.bend_compliance = 5e-5
        p.damping = 0.05
        p.thickness = 0.03
        p.friction = 0.5
        p.gravity_scale = 1.0
        p.max_velocity = 100.0
        p.wind_turbulence = 0.0
        p.air_drag = 0.02
        p.air_lift = 0.02
        p.self_collision = 0
        p.self_distance = 0.0
        p.tether_scale = 1.02
        p.substeps = 0
        p.iterations = 0
        p.sleep_threshold = 0.05
        p.sleep_time = 0.5
        p.layer = 0
        p.has_shear_compliance = 0
        p.shear_compliance = 0.0
        return p


class StrandParams(C.Structure):
    """pxb_strand_params == hair::StrandParams (strand.h:93-148)."""
    _fields_ = [("stretch_compliance", f32), ("global_shape", f32),
                ("global_shape_falloff", f32), ("local_shape", f32), ("damping", f32),
                ("thickness", f32), ("friction", f32), ("gravity_scale", f32),
                ("max_velocity", f32), ("external_acceleration", f32 * 3), ("wind", f32 * 3),
                ("wind_turbulence", f32), ("air_drag", f32), ("substeps", u32),
                ("iterations", u32), ("sleep_threshold", f32), ("sleep_time", f32),
                ("layer", u32)]

    @classmethod
    def defaults(cls):
        """The reference's StrandParams defaults (strand.h:96-147)."""
        p = cls()
        p.stretch_compliance = 0.0
        p.global_shape = 0.22
        p.global_shape_falloff = 1.6
        p.local_shape = 0.35
        p.damping = 0.08
        p.thickness = 0.01
        p.friction = 0.4
        p.gravity_scale = 1.0
        p.max_velocity = 50.0
        p.wind_turbulence = 0.1
        p.air_drag = 0.6
        p.substeps = 0
        p.iterations = 0
        p.sleep_threshold = 0.02
        p.sleep_time = 0.6
        p.layer = 0
        return p


P = C.c_void_p


class MeshClothDesc(C.Structure):
    """pxb_mesh_cloth_desc: a cloth built from an arbitrary triangle mesh."""
    _fields_ = [("vertices", C.c_void_p), ("n_vertices", C.c_uint32), ("indices", C.c_void_p),
                ("n_indices", C.c_uint32), ("total_mass", f32), ("bend", C.c_int32), ("params", ClothParams)]


class HeightGridDesc(C.Structure):
    """pxb_height_grid_desc: geometry::HeightGrid's samples."""
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("cell_x", f32), ("cell_y", f32),
                ("heights", C.c_void_p), ("n_heights", C.c_uint32)]


class ClothPlan(C.Structure):
    """pxb_cloth_plan: the device layout pxb_cloth_add would choose."""
    _fields_ = [("n_ranks", C.c_int32), ("rows_per_rank", C.c_int32), ("threads", C.c_int32),
                ("smem_bytes", C.c_int32), ("n_colours", C.c_int32), ("n_segments", C.c_int32),
                ("layout_slots", C.c_int32), ("constraint_slots", C.c_int32),
                ("self_collision", C.c_int32), ("self_smem_bytes", C.c_int32), ("topology", C.c_int32),
                ("lean", C.c_int32), ("phases", C.c_int32)]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class MlpWeights(C.Structure):
    """pxb_mlp_weights: the warm-start network (row-major weights, out x in)."""
    _fields_ = [("w1", (f32 * 24) * 64), ("b1", f32 * 64), ("w2", (f32 * 64) * 64), ("b2", f32 * 64),
                ("w3", (f32 * 64) * 3), ("b3", f32 * 3), ("in_mean", f32 * 24), ("in_scale", f32 * 24),
                ("out_scale", f32 * 3)]

    @classmethod
    def from_numpy(cls, w1, b1, w2, b2, w3, b3, in_mean=None, in_scale=None, out_scale=None):
        m = cls()
        for name, arr in (("w1", w1), ("b1", b1), ("w2", w2), ("b2", b2), ("w3", w3), ("b3", b3),
                          ("in_mean", np.zeros(24) if in_mean is None else in_mean),
                          ("in_scale", np.ones(24) if in_scale is None else in_scale),
                          ("out_scale", np.ones(3) if out_scale is None else out_scale)):
            dst = np.ctypeslib.as_array(getattr(m, name))
            dst[...] = np.asarray(arr, np.float32).reshape(dst.shape)
        return m

    def as_numpy(self):
        return {name: np.ctypeslib.as_array(getattr(self, name)).copy() for name, _ in self._fields_}


class MlpTrainDesc(C.Structure):
    """pxb_mlp_train_desc."""
    _fields_ = [("epochs", u32), ("batch", u32), ("learning_rate", f32), ("seed", C.c_uint64)]


class WarmStartDesc(C.Structure):
    """pxb_warm_start_desc."""
    _fields_ = [("warm_iterations", u32), ("residual_threshold", f32), ("thresholds", P),
                ("continue_iterations", u32)]


WARM_RESULT = np.dtype([("residual", "<f4"), ("fallbacks", "<u4"), ("substeps", "<u4"),
                        ("extra_iterations", "<u4")])


class HullDesc(C.Structure):
    """pxb_hull_desc (geometry::ConvexHull's arrays)."""
    _fields_ = [("vertices", P), ("n_vertices", u32), ("face_planes", P), ("n_faces", u32),
                ("face_starts", P), ("face_vertices", P)]


class MeshDesc(C.Structure):
    """pxb_mesh_desc (geometry::TriangleMesh's vertices, indices and face normals)."""
    _fields_ = [("vertices", P), ("n_vertices", u32), ("indices", P), ("n_indices", u32),
                ("normals", P)]


class ClothDesc(C.Structure):
    """pxb_cloth_desc: a cloth as plain pointers into caller memory."""
    _fields_ = [("particles", P), ("n_particles", u32), ("stretch", P), ("n_stretch", u32),
                ("stretch_batches", P), ("n_stretch_batches", u32), ("bend", P),
                ("n_bend", u32), ("bend_batches", P), ("n_bend_batches", u32), ("tethers", P),
                ("n_tethers", u32), ("anchors", P), ("n_anchors", u32), ("triangles", P),
                ("n_triangle_indices", u32), ("columns", u32), ("rows", u32),
                ("params", ClothParams), ("time", f32), ("stretch_batch_compliance", P),
                ("bend_batch_compliance", P)]


class StrandSetDesc(C.Structure):
    """pxb_strand_set_desc."""
    _fields_ = [("particles", P), ("n_particles", u32), ("stretch", P), ("n_stretch", u32),
                ("stretch_batches", P), ("n_stretch_batches", u32), ("rest_local", P),
                ("rest_offset", P), ("strands", P), ("n_strands", u32),
                ("params", StrandParams), ("time", f32)]


class GridClothDesc(C.Structure):
    """pxb_grid_cloth_desc == cloth::GridClothDesc (cloth_builder.h:52-64) + seeded jitter."""
    _fields_ = [("columns", u32), ("rows", u32), ("width", f32), ("height", f32),
                ("center", f32 * 3), ("orientation", f32 * 4), ("total_mass", f32),
                ("shear", i32), ("params", ClothParams), ("jitter", f32),
                ("jitter_seed", C.c_uint64)]


class ClothStepDesc(C.Structure):
    """pxb_cloth_step_desc."""
    _fields_ = [("cloths", P), ("n_cloths", u32), ("colliders", P), ("collider_offsets", P),
                ("gravity", f32 * 3), ("sources", P), ("source_offsets", P),
                ("substeps", u32), ("iterations", u32), ("h", f32)]


class ClothFrameDesc(C.Structure):
    """pxb_cloth_frame_desc: one PhysicsWorld::step_cloths_ frame."""
    _fields_ = [("cloths", P), ("n_cloths", u32), ("bodies", P), ("n_bodies", u32), ("colliders", P),
                ("collider_offsets", P), ("collider_moving", P), ("gravity", f32 * 3), ("sources", P),
                ("source_offsets", P), ("fixed_dt", f32), ("cloth_substeps", u32), ("cloth_iterations", u32),
                ("dt", f32)]


class StrandFrameDesc(C.Structure):
    """pxb_strand_frame_desc: one PhysicsWorld::step_strands_ frame."""
    _fields_ = [("sets", P), ("n_sets", u32), ("colliders", P), ("collider_offsets", P), ("collider_moving", P),
                ("gravity", f32 * 3), ("sources", P), ("source_offsets", P), ("fixed_dt", f32),
                ("cloth_substeps", u32), ("cloth_iterations", u32), ("dt", f32)]


class StrandStepDesc(C.Structure):
    """pxb_strand_step_desc."""
    _fields_ = [("sets", P), ("n_sets", u32), ("colliders", P), ("collider_offsets", P),
                ("gravity", f32 * 3), ("sources", P), ("source_offsets", P),
                ("substeps", u32), ("iterations", u32), ("h", f32)]


def ptr(a):
    """Data pointer of a numpy array (None for an empty/None array)."""
    if a is None or a.size == 0:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data
