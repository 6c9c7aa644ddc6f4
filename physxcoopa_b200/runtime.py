"""ctypes host over the C-ABI library (include/physxcoopa_b200.h).

`Context` mirrors the reference's cloth entry points at PhysicsWorld granularity
(add_cloth / remove_cloth / step, physxcoopa/world.h:552-596, 1749-1847) and the drop-in
`solve_cloth` contract (physxcoopa/cloth/cloth_solver.h:158-467) on host arrays.
`HostCloth` wraps the library's setup-time builders (make_grid_cloth / pin_static /
build_tethers, physxcoopa/cloth/cloth_builder.h).

There is no fallback: if the shared library is missing, loading raises.
"""
import ctypes as C
import os

import numpy as np

from . import _abi as A
from .arrays import ClothArrays, HeightGrid, Hull, StrandArrays

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libphysxcoopa_b200.so")

P = C.c_void_p
u32 = C.c_uint32
u64 = C.c_uint64
f32 = C.c_float
f32p = C.POINTER(C.c_float)

# Every symbol the header declares, with its argument types.
SIGNATURES = {
    "pxb_context_create": ([C.c_int, C.POINTER(P)], C.c_int),
    "pxb_context_destroy": ([P], C.c_int),
    "pxb_last_error": ([P], C.c_char_p),
    "pxb_context_stream": ([P, C.POINTER(P)], C.c_int),
    "pxb_context_synchronize": ([P], C.c_int),
    "pxb_context_launch_count": ([P], u64),
    "pxb_cloth_params_default": ([C.POINTER(A.ClothParams)], None),
    "pxb_cloth_add": ([P, C.POINTER(A.ClothDesc), C.POINTER(u64)], C.c_int),
    "pxb_cloth_remove": ([P, u64], C.c_int),
    "pxb_cloths_gather_positions_device": ([P, P, u32, P, C.c_size_t], C.c_int),
    "pxb_mlp_set_weights": ([P, C.POINTER(A.MlpWeights)], C.c_int),
    "pxb_mlp_get_weights": ([P, C.POINTER(A.MlpWeights)], C.c_int),
    "pxb_mlp_infer": ([P, P, u32, P], C.c_int),
    "pxb_mlp_train": ([P, P, P, u64, C.POINTER(A.MlpTrainDesc), C.POINTER(f32)], C.c_int),
    "pxb_mlp_loss_gradients": ([P, P, P, u64, C.POINTER(f32), C.POINTER(A.MlpWeights)], C.c_int),
    "pxb_cloths_step_warm": ([P, C.POINTER(A.ClothStepDesc), C.POINTER(A.WarmStartDesc)], C.c_int),
    "pxb_cloths_read_warm_results": ([P, P, u32, P], C.c_int),
    "pxb_cloths_record": ([P, C.POINTER(A.ClothStepDesc), u32, P, P, u64, C.POINTER(u64)], C.c_int),
    "pxb_cloth_plan_layout": ([C.POINTER(A.ClothDesc), C.POINTER(A.ClothPlan), C.c_char_p, u32], C.c_int),
    "pxb_cloth_set_params": ([P, u64, C.POINTER(A.ClothParams)], C.c_int),
    "pxb_cloth_write_particles": ([P, u64, P, u32], C.c_int),
    "pxb_cloth_read_particles": ([P, u64, P, u32], C.c_int),
    "pxb_cloth_read_lambdas": ([P, u64, P, u32, P, u32], C.c_int),
    "pxb_cloth_set_anchor_targets": ([P, u64, P, u32], C.c_int),
    "pxb_cloth_read_anchors": ([P, u64, P, u32], C.c_int),
    "pxb_cloth_read_time": ([P, u64, f32p], C.c_int),
    "pxb_cloths_step": ([P, C.POINTER(A.ClothStepDesc)], C.c_int),
    "pxb_cloths_step_graph": ([P, C.POINTER(A.ClothStepDesc)], C.c_int),
    "pxb_cloths_read_results": ([P, P, u32, P], C.c_int),
    "pxb_cloths_read_positions": ([P, P, u32, P, C.c_size_t], C.c_int),
    "pxb_cloths_read_positions_async": ([P, P, u32, P, C.c_size_t], C.c_int),
    "pxb_cloths_wait_positions": ([P], C.c_int),
    "pxb_cloths_read_results_async": ([P, P, u32, P], C.c_int),
    "pxb_solve_cloth_host": ([P, C.POINTER(A.ClothDesc), P, P, P, P, P, u32, f32p, u32, u32, f32,
                              f32p, f32p], C.c_int),
    "pxb_project_particles": ([P, P, f32, P, P, u32, P, P, P, P], C.c_int),
    "pxb_cloths_step_frame": ([P, C.POINTER(A.ClothFrameDesc), P], C.c_int),
    "pxb_cloths_state_hash": ([P, P, u32, u64, C.POINTER(u64)], C.c_int),
    "pxb_cloths_read_render_buffer": ([P, P, u32, P, C.c_size_t], C.c_int),
    "pxb_cloths_read_sleep_state": ([P, P, u32, P, P], C.c_int),
    "pxb_strands_step_frame": ([P, C.POINTER(A.StrandFrameDesc), P], C.c_int),
    "pxb_strands_read_sleep_state": ([P, P, u32, P, P], C.c_int),
    "pxb_host_cloth_pin_to_body": ([P, u32, u32, f32p, f32p, f32p, f32, C.POINTER(u32)], C.c_int),
    "pxb_geometry_create_hull": ([P, C.POINTER(A.HullDesc), C.POINTER(u32)], C.c_int),
    "pxb_geometry_create_mesh": ([P, C.POINTER(A.MeshDesc), C.POINTER(u32)], C.c_int),
    "pxb_geometry_create_height_grid": ([P, C.POINTER(A.HeightGridDesc), C.POINTER(u32)], C.c_int),
    "pxb_geometry_destroy": ([P, u32], C.c_int),
    "pxb_host_cloth_make_grid": ([C.POINTER(A.GridClothDesc), C.POINTER(P)], C.c_int),
    "pxb_host_cloth_make_mesh": ([C.POINTER(A.MeshClothDesc), C.POINTER(P)], C.c_int),
    "pxb_host_cloth_destroy": ([P], C.c_int),
    "pxb_host_cloth_pin_static": ([P, f32p, f32, C.POINTER(u32)], C.c_int),
    "pxb_host_cloth_build_tethers": ([P], C.c_int),
    "pxb_host_cloth_build_tethers_device": ([P, P], C.c_int),
    "pxb_build_tethers_device": ([P, P, u32, P, u32, P, u32, f32, P, u32, C.POINTER(u32)], C.c_int),
    "pxb_host_cloth_view": ([P, C.POINTER(A.ClothDesc)], C.c_int),
    "pxb_host_cloth_mutable": ([P, C.POINTER(P), C.POINTER(P), C.POINTER(P)], C.c_int),
    "pxb_measure_smem_bandwidth": ([P, C.POINTER(C.c_double)], C.c_int),
    "pxb_check_quotients": ([P, u64, u64, C.POINTER(u64)], C.c_int),
    "pxb_check_quotient_significands": ([P, u32, u32, C.POINTER(u64)], C.c_int),
    "pxb_check_projections": ([P, u64, u64, C.POINTER(u64), C.POINTER(f32)], C.c_int),
    "pxb_context_set_cloth_variant": ([P, C.c_int32], C.c_int),
    "pxb_context_set_launch_mode": ([P, C.c_int32], C.c_int),
    "pxb_context_set_lean_arrays": ([P, C.c_int32], C.c_int),
    "pxb_context_set_thread_fit": ([P, C.c_int32], C.c_int),
    "pxb_context_set_lean_mid": ([P, C.c_int32], C.c_int),
    "pxb_context_get_tuning": ([P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                C.POINTER(C.c_int32), C.POINTER(C.c_double)], C.c_int),
    "pxb_context_set_wait_test": ([P, u32, u32], C.c_int),
    "pxb_strands_add": ([P, C.POINTER(A.StrandSetDesc), C.POINTER(u64)], C.c_int),
    "pxb_strands_remove": ([P, u64], C.c_int),
    "pxb_strands_set_params": ([P, u64, C.POINTER(A.StrandParams)], C.c_int),
    "pxb_strands_set_roots": ([P, u64, P, u32, P, u32], C.c_int),
    "pxb_strands_write_particles": ([P, u64, P, u32], C.c_int),
    "pxb_strands_read_particles": ([P, u64, P, u32], C.c_int),
    "pxb_strands_read_lambdas": ([P, u64, P, u32], C.c_int),
    "pxb_strands_read_strands": ([P, u64, P, u32], C.c_int),
    "pxb_strands_read_time": ([P, u64, f32p], C.c_int),
    "pxb_strands_step": ([P, C.POINTER(A.StrandStepDesc)], C.c_int),
    "pxb_strands_read_results": ([P, P, u32, P], C.c_int),
    "pxb_solve_strands_host": ([P, C.POINTER(A.StrandSetDesc), P, P, P, u32, f32p, u32, u32, f32, f32p,
                                f32p], C.c_int),
    "pxb_host_strands_make": ([u32, P, P, P, P, C.POINTER(A.StrandParams), C.POINTER(P)], C.c_int),
    "pxb_host_strands_destroy": ([P], C.c_int),
    "pxb_host_strands_view": ([P, C.POINTER(A.StrandSetDesc)], C.c_int),
    "pxb_strand_params_default": ([C.POINTER(A.StrandParams)], None),
    "pxb_cloths_autotune": ([P, C.POINTER(A.ClothStepDesc), u32, C.POINTER(C.c_int32), P], C.c_int),
}

_lib = None


class PxbError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{A.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def library():
    """Loads libphysxcoopa_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m physxcoopa_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def _vec(x, n=3):
    return (C.c_float * n)(*[float(v) for v in x])


def plan_cloth(c: ClothArrays) -> dict:
    """The device layout pxb_cloth_add would give this cloth (no GPU needed); raises PxbError
    with the library's message for a cloth it would refuse."""
    d = c.desc()
    out = A.ClothPlan()
    err = C.create_string_buffer(512)
    st = library().pxb_cloth_plan_layout(C.byref(d), C.byref(out), err, 512)
    if st:
        raise PxbError(st, err.value.decode())
    return out.as_dict()


class HostCloth:
    """A cloth built by the library's host builders (cloth_builder.h), in library memory."""

    def __init__(self, columns, rows, width, height, center=(0, 0, 0), orientation=(0, 0, 0, 1),
                 total_mass=1.0, shear=True, params=None, jitter=0.0, seed=0):
        d = A.GridClothDesc()
        d.columns, d.rows, d.width, d.height = columns, rows, width, height
        d.center = _vec(center)
        d.orientation = _vec(orientation, 4)
        d.total_mass = total_mass
        d.shear = 1 if shear else 0
        d.params = params if params is not None else A.ClothParams.defaults()
        d.jitter = jitter
        d.jitter_seed = seed
        self._h = P()
        st = library().pxb_host_cloth_make_grid(C.byref(d), C.byref(self._h))
        if st:
            raise PxbError(st, "make_grid failed")

    @classmethod
    def from_mesh(cls, vertices, indices, total_mass=1.0, bend=True, params=None):
        """A cloth over an arbitrary triangle mesh (pxb_host_cloth_make_mesh): one particle per
        vertex, stretch along the distinct edges, bend across shared edges, both lists coloured
        into particle-disjoint batches."""
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        ix = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        d = A.MeshClothDesc()
        d.vertices = v.ctypes.data
        d.n_vertices = len(v)
        d.indices = ix.ctypes.data if len(ix) else None
        d.n_indices = len(ix)
        d.total_mass = total_mass
        d.bend = 1 if bend else 0
        d.params = params if params is not None else A.ClothParams.defaults()
        self = cls.__new__(cls)
        self._h = P()
        st = library().pxb_host_cloth_make_mesh(C.byref(d), C.byref(self._h))
        if st:
            self._h = None
            raise PxbError(st, "make_mesh failed")
        return self

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pxb_host_cloth_destroy(self._h)
            self._h = None

    def pin_static(self, point, radius):
        n = u32()
        st = library().pxb_host_cloth_pin_static(self._h, _vec(point), radius, C.byref(n))
        if st:
            raise PxbError(st, "pin_static failed")
        return n.value

    def pin_to_body(self, body_index, body_generation, body_position, body_orientation, point, radius):
        """cloth::pin_to_body: anchors the particles within `radius` of `point` to the body."""
        out = u32()
        st = library().pxb_host_cloth_pin_to_body(self._h, body_index, body_generation, _vec(body_position),
                                                   _vec(body_orientation, 4), _vec(point), radius, C.byref(out))
        if st:
            raise PxbError(st, "pin_to_body")
        return int(out.value)

    def build_tethers(self):
        st = library().pxb_host_cloth_build_tethers(self._h)
        if st:
            raise PxbError(st, "build_tethers failed")

    def mutable_particles(self):
        """The builder's particle array as a writable numpy view (pxb_host_cloth_mutable); valid
        until the next builder call."""
        pp, pa, pr = P(), P(), P()
        st = library().pxb_host_cloth_mutable(self._h, C.byref(pp), C.byref(pa), C.byref(pr))
        if st:
            raise PxbError(st, "host_cloth_mutable")
        v = A.ClothDesc()
        library().pxb_host_cloth_view(self._h, C.byref(v))
        buf = (C.c_char * (v.n_particles * A.PARTICLE.itemsize)).from_address(pp.value)
        return np.frombuffer(buf, A.PARTICLE)

    def build_tethers_device(self, ctx):
        """cloth::build_tethers on the device (pxb_host_cloth_build_tethers_device)."""
        ctx._check(library().pxb_host_cloth_build_tethers_device(ctx.h, self._h), "build_tethers_device")

    def arrays(self) -> ClothArrays:
        v = A.ClothDesc()
        library().pxb_host_cloth_view(self._h, C.byref(v))
        return ClothArrays.from_desc(v)


def make_strands(polylines, params=None, root_orientations=None, particle_masses=None) -> StrandArrays:
    """hair::make_strands (strand_builder.h:58-127) through the library's host builder."""
    counts = np.array([len(p) for p in polylines], np.uint32)
    pts = (np.ascontiguousarray(np.concatenate([np.asarray(p, np.float32).reshape(-1, 3) for p in polylines]),
                                np.float32) if len(polylines) else np.zeros((0, 3), np.float32))
    rot = None if root_orientations is None else np.ascontiguousarray(root_orientations, np.float32)
    mass = None if particle_masses is None else np.ascontiguousarray(particle_masses, np.float32)
    params = params if params is not None else A.StrandParams.defaults()
    h = P()
    lib = library()
    st = lib.pxb_host_strands_make(len(counts), A.ptr(counts), A.ptr(pts), A.ptr(rot), A.ptr(mass),
                                   C.byref(params), C.byref(h))
    if st:
        raise PxbError(st, "make_strands failed")
    try:
        v = A.StrandSetDesc()
        lib.pxb_host_strands_view(h, C.byref(v))

        def grab(addr, n, dtype):
            if n == 0 or not addr:
                return np.zeros(0, dtype)
            return np.frombuffer(bytes((C.c_char * (n * dtype.itemsize)).from_address(addr)), dtype).copy()
        n = v.n_particles
        f = np.dtype("<f4")
        p = A.StrandParams()
        C.pointer(p)[0] = v.params
        parts = grab(v.particles, n, A.PARTICLE)
        pos = parts["position"]
        # StrandSet::bounds = compute_bounds(set) at build (strand_builder.h:125, strand.h:195-202)
        bounds = (np.concatenate([pos.min(axis=0), pos.max(axis=0)]).astype(np.float32) if n else
                  np.array([3.4028235e38] * 3 + [-3.4028235e38] * 3, np.float32))
        return StrandArrays(particles=parts,
                            stretch=grab(v.stretch, v.n_stretch, A.CONSTRAINT),
                            stretch_batches=grab(v.stretch_batches, v.n_stretch_batches, A.BATCH),
                            rest_local=grab(v.rest_local, 3 * n, f).reshape(-1, 3),
                            rest_offset=grab(v.rest_offset, 3 * n, f).reshape(-1, 3),
                            strands=grab(v.strands, v.n_strands, A.STRAND), params=p, time=0.0,
                            bounds=bounds)
    finally:
        lib.pxb_host_strands_destroy(h)


def make_grid_cloth(columns, rows, width, height, **kw) -> ClothArrays:
    pins = kw.pop("pins", ())
    tethers = kw.pop("tethers", False)
    h = HostCloth(columns, rows, width, height, **kw)
    for point, radius in pins:
        h.pin_static(point, radius)
    if tethers:
        h.build_tethers()
    return h.arrays()


def _flatten(per_cloth, dtype, n):
    """A list of per-cloth record arrays -> (flat array, offsets) or (None, None)."""
    if per_cloth is None:
        return None, None
    if isinstance(per_cloth, np.ndarray) and per_cloth.dtype == dtype:
        per_cloth = [per_cloth] * n
    lens = [0 if a is None else len(a) for a in per_cloth]
    offs = np.zeros(n + 1, np.uint32)
    offs[1:] = np.cumsum(lens)
    if offs[-1] == 0:
        return None, None
    flat = np.ascontiguousarray(np.concatenate([a for a in per_cloth if a is not None and len(a)]))
    return flat, offs


class Context:
    """One device, one stream (pxb_context)."""

    def __init__(self, device=0):
        self.lib = library()
        self.h = P()
        st = self.lib.pxb_context_create(device, C.byref(self.h))
        if st:
            raise PxbError(st, "pxb_context_create failed (is a CUDA device visible?)")
        self._keep = []
        self._slots = {}
        self.cloth_variant = 0  # the context's kernel variant and launch form, as last set
        self.launch_mode = 1

    def close(self):
        if self.h:
            self.lib.pxb_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st:
            raise PxbError(st, f"{what}: {self.lib.pxb_last_error(self.h).decode()}")

    @property
    def stream(self):
        s = P()
        self._check(self.lib.pxb_context_stream(self.h, C.byref(s)), "stream")
        return s.value

    def synchronize(self):
        self._check(self.lib.pxb_context_synchronize(self.h), "synchronize")

    def measure_smem_bandwidth(self):
        """Achievable device-wide shared-memory bandwidth, bytes/s (roofline denominator)."""
        v = C.c_double()
        self._check(self.lib.pxb_measure_smem_bandwidth(self.h, C.byref(v)), "measure_smem_bandwidth")
        return v.value

    def check_quotients(self, samples, seed=0):
        """pxb_check_quotients: (reciprocal mismatches, quotient mismatches); both should be 0."""
        out = (u64 * 2)()
        self._check(self.lib.pxb_check_quotients(self.h, samples, seed, out), "check_quotients")
        return int(out[0]), int(out[1])

    def check_projections(self, samples, seed=0):
        """pxb_check_projections: (mismatching projections, first mismatching input or None)."""
        out = u64()
        fb = (f32 * 8)()
        self._check(self.lib.pxb_check_projections(self.h, samples, seed, C.byref(out), fb), "check_projections")
        return int(out.value), (list(fb) if out.value else None)

    def check_quotient_significands(self, b_first=0, b_count=1 << 23):
        """pxb_check_quotient_significands: quotients differing from IEEE division over divisor
        significands [b_first, b_first + b_count) and every numerator significand."""
        out = u64()
        self._check(self.lib.pxb_check_quotient_significands(self.h, b_first, b_count, C.byref(out)),
                    "check_quotient_significands")
        return int(out.value)

    @property
    def launch_count(self):
        return int(self.lib.pxb_context_launch_count(self.h))

    # --- warm-start network ---------------------------------------------------------------
    def set_mlp(self, weights):
        self._check(self.lib.pxb_mlp_set_weights(self.h, C.byref(weights)), "mlp_set_weights")

    def get_mlp(self):
        w = A.MlpWeights()
        self._check(self.lib.pxb_mlp_get_weights(self.h, C.byref(w)), "mlp_get_weights")
        return w

    def mlp_infer(self, features):
        x = np.ascontiguousarray(features, np.float32).reshape(-1, 24)
        out = np.zeros((len(x), 3), np.float32)
        self._check(self.lib.pxb_mlp_infer(self.h, A.ptr(x), len(x), A.ptr(out)), "mlp_infer")
        return out

    def mlp_train(self, features, targets, epochs=20, batch=8192, learning_rate=3e-3, seed=0):
        """Fits and installs the network (pxb_mlp_train); returns the last epoch's mean loss."""
        x = np.ascontiguousarray(features, np.float32).reshape(-1, 24)
        y = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
        d = A.MlpTrainDesc(epochs, batch, learning_rate, seed)
        loss = f32()
        self._check(self.lib.pxb_mlp_train(self.h, A.ptr(x), A.ptr(y), len(x), C.byref(d), C.byref(loss)),
                    "mlp_train")
        return loss.value

    def mlp_loss_gradients(self, features, targets):
        x = np.ascontiguousarray(features, np.float32).reshape(-1, 24)
        y = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
        loss = f32()
        g = A.MlpWeights()
        self._check(self.lib.pxb_mlp_loss_gradients(self.h, A.ptr(x), A.ptr(y), len(x), C.byref(loss), C.byref(g)),
                    "mlp_loss_gradients")
        return loss.value, g.as_numpy()

    def step_warm(self, ids, colliders=None, gravity=(0, 0, -9.81), sources=None, substeps=4,
                  iterations=10, h=1.0 / 60.0, warm_iterations=4, threshold=1e-4, thresholds=None,
                  continue_iterations=False):
        """One warm-started step (pxb_cloths_step_warm); warm_iterations=0 is the plain solve
        with its residual measured."""
        d, keep = self.make_step(ids, colliders, gravity, sources, substeps, iterations, h)
        return self.step_warm_desc(d, warm_iterations, threshold, thresholds, keep, continue_iterations)

    def step_warm_desc(self, d, warm_iterations=4, threshold=1e-4, thresholds=None, keep=None,
                       continue_iterations=False):
        w = A.WarmStartDesc()
        w.warm_iterations = warm_iterations
        w.continue_iterations = 1 if continue_iterations else 0
        w.residual_threshold = threshold
        th = None if thresholds is None else np.ascontiguousarray(thresholds, np.float32)
        w.thresholds = A.ptr(th)
        self._check(self.lib.pxb_cloths_step_warm(self.h, C.byref(d), C.byref(w)), "cloths_step_warm")
        del keep

    def read_warm_results(self, ids):
        ids = np.ascontiguousarray(ids, np.uint64)
        out = np.zeros(len(ids), A.WARM_RESULT)
        self._check(self.lib.pxb_cloths_read_warm_results(self.h, A.ptr(ids), len(ids), A.ptr(out)),
                    "read_warm_results")
        return out

    def record(self, ids, colliders=None, gravity=(0, 0, -9.81), sources=None, substeps=4,
               iterations=10, h=1.0 / 60.0, substep=0, capacity=None):
        """Training rows from one plain step (pxb_cloths_record): (features n x 24, targets n x 3)."""
        if capacity is None:
            capacity = sum(self._layout_slots(i) for i in ids)
        d, keep = self.make_step(ids, colliders, gravity, sources, substeps, iterations, h)
        x = np.zeros((max(capacity, 1), 24), np.float32)
        y = np.zeros((max(capacity, 1), 3), np.float32)
        n = u64()
        self._check(self.lib.pxb_cloths_record(self.h, C.byref(d), substep, A.ptr(x), A.ptr(y), capacity,
                                               C.byref(n)), "cloths_record")
        del keep
        return x[:n.value], y[:n.value]

    def _layout_slots(self, cid):
        return self._slots.get(cid, 0)

    # --- registry ------------------------------------------------------------------------
    def add_cloth(self, c: ClothArrays) -> int:
        d = c.desc()
        out = u64()
        self._check(self.lib.pxb_cloth_add(self.h, C.byref(d), C.byref(out)), "add_cloth")
        self._slots[out.value] = c.rows * 4 * ((c.columns + 3) // 4)
        return out.value

    def remove_cloth(self, cid):
        self._check(self.lib.pxb_cloth_remove(self.h, cid), "remove_cloth")

    def set_params(self, cid, params):
        self._check(self.lib.pxb_cloth_set_params(self.h, cid, C.byref(params)), "set_params")

    def write_particles(self, cid, particles):
        p = np.ascontiguousarray(particles, A.PARTICLE)
        self._check(self.lib.pxb_cloth_write_particles(self.h, cid, A.ptr(p), len(p)), "write_particles")

    def read_particles(self, cid, n):
        out = np.zeros(n, A.PARTICLE)
        self._check(self.lib.pxb_cloth_read_particles(self.h, cid, A.ptr(out), n), "read_particles")
        return out

    def read_lambdas(self, cid, n_stretch, n_bend):
        s = np.zeros(n_stretch, np.float32)
        b = np.zeros(n_bend, np.float32)
        self._check(self.lib.pxb_cloth_read_lambdas(self.h, cid, A.ptr(s) if n_stretch else None,
                                                    n_stretch, A.ptr(b) if n_bend else None, n_bend),
                    "read_lambdas")
        return s, b

    def set_anchor_targets(self, cid, world):
        w = np.ascontiguousarray(world, np.float32).reshape(-1, 3)
        self._check(self.lib.pxb_cloth_set_anchor_targets(self.h, cid, A.ptr(w), len(w)),
                    "set_anchor_targets")

    def read_anchors(self, cid, n):
        out = np.zeros(n, A.ANCHOR)
        self._check(self.lib.pxb_cloth_read_anchors(self.h, cid, A.ptr(out), n), "read_anchors")
        return out

    def read_time(self, cid):
        t = f32()
        self._check(self.lib.pxb_cloth_read_time(self.h, cid, C.byref(t)), "read_time")
        return t.value

    # --- stepping ------------------------------------------------------------------------
    def make_step(self, ids, colliders=None, gravity=(0, 0, -9.81), sources=None, substeps=4,
                  iterations=10, h=1.0 / 60.0):
        """Builds (and keeps alive) a pxb_cloth_step_desc; reuse it to step repeatedly."""
        ids = np.ascontiguousarray(ids, np.uint64)
        n = len(ids)
        cols, coff = _flatten(colliders, A.COLLIDER, n)
        src, soff = _flatten(sources, A.GRAVITY_SOURCE, n)
        d = A.ClothStepDesc()
        d.cloths = A.ptr(ids)
        d.n_cloths = n
        d.colliders = A.ptr(cols)
        d.collider_offsets = A.ptr(coff)
        d.gravity = _vec(gravity)
        d.sources = A.ptr(src)
        d.source_offsets = A.ptr(soff)
        d.substeps, d.iterations, d.h = substeps, iterations, h
        keep = (ids, cols, coff, src, soff)
        return d, keep

    def step_desc(self, d):
        self._check(self.lib.pxb_cloths_step(self.h, C.byref(d)), "cloths_step")

    def step_graph_desc(self, d):
        """pxb_cloths_step_graph: the step replayed from a captured CUDA graph."""
        self._check(self.lib.pxb_cloths_step_graph(self.h, C.byref(d)), "cloths_step_graph")

    def step(self, ids, colliders=None, gravity=(0, 0, -9.81), sources=None, substeps=4,
             iterations=10, h=1.0 / 60.0):
        d, keep = self.make_step(ids, colliders, gravity, sources, substeps, iterations, h)
        self.step_desc(d)
        del keep

    def set_wait_test(self, grid_wait_polls=1 << 22, unreachable=False):
        """pxb_context_set_wait_test: bound of a grid-barrier wait, and whether no grid barrier
        can complete (to drive the expiry path in a test)."""
        self._check(self.lib.pxb_context_set_wait_test(self.h, grid_wait_polls, 1 if unreachable else 0),
                    "set_wait_test")

    def set_lean_arrays(self, enable):
        """pxb_context_set_lean_arrays: cloths added afterwards may (1) or may not (0) take the
        one-CTA float-array layout."""
        self._check(self.lib.pxb_context_set_lean_arrays(self.h, 1 if enable else 0), "set_lean_arrays")

    def set_lean_mid(self, enable):
        """pxb_context_set_lean_mid: sheets added afterwards that an SM would hold one of when held
        whole take the lean layout where it holds two or more (1), or stay whole (0)."""
        self._check(self.lib.pxb_context_set_lean_mid(self.h, 1 if enable else 0), "set_lean_mid")

    def set_thread_fit(self, mode):
        """pxb_context_set_thread_fit: 1 splits an SM's threads between the CTAs of one-CTA grid
        cloths that shared memory lets it hold, 0 gives each its own thread count."""
        self._check(self.lib.pxb_context_set_thread_fit(self.h, mode), "set_thread_fit")

    TUNE_CLASS_KINDS = ("whole in shared memory", "whole in shared memory, extended stages",
                        "general topology in HBM", "lean float4", "lean float4, extended stages",
                        "lean float arrays", "lean float arrays, extended stages")

    def tuning(self):
        """pxb_context_get_tuning: the block-size variant, launch mode, thread fit, and per layout
        class that the last plain step launched, its variant and its layout slots."""
        v, m, f = C.c_int32(), C.c_int32(), C.c_int32()
        cv = (C.c_int32 * 21)()
        cw = (C.c_double * 21)()
        self._check(self.lib.pxb_context_get_tuning(self.h, C.byref(v), C.byref(m), C.byref(f), cv, cw), "tuning")
        classes = [{"kind": self.TUNE_CLASS_KINDS[c // 3], "ctas_per_sm_by_smem": ("1", "2", "3+")[c % 3],
                    "block_cap": (512, 768, 1024)[cv[c]], "slots": int(cw[c])}
                   for c in range(21) if cw[c] > 0]
        return {"variant": v.value, "launch_mode": m.value, "thread_fit": f.value, "classes": classes}

    def set_launch_mode(self, mode):
        """pxb_context_set_launch_mode: 1 persistent work-queue kernels, 0 one CTA per cloth."""
        self._check(self.lib.pxb_context_set_launch_mode(self.h, mode), "set_launch_mode")
        self.launch_mode = mode

    def set_cloth_variant(self, variant):
        self._check(self.lib.pxb_context_set_cloth_variant(self.h, variant), "set_cloth_variant")
        self.cloth_variant = variant

    def autotune(self, d, trials=3):
        """Times the kernel variants in both launch forms on step desc `d` (state restored);
        returns (best = variant + 3 * launch mode, ms list of six)."""
        best = C.c_int32()
        ms = (C.c_float * 6)()
        self._check(self.lib.pxb_cloths_autotune(self.h, C.byref(d), trials, C.byref(best), ms),
                    "autotune")
        self.cloth_variant, self.launch_mode = best.value % 3, best.value // 3
        return best.value, list(ms)

    def read_results(self, ids):
        ids = np.ascontiguousarray(ids, np.uint64)
        out = np.zeros(len(ids), A.FRAME_RESULT)
        self._check(self.lib.pxb_cloths_read_results(self.h, A.ptr(ids), len(ids), A.ptr(out)),
                    "read_results")
        return out

    def read_positions_async(self, ids, out):
        """pxb_cloths_read_positions_async into `out` (float32, ideally pinned); completes at
        wait_positions()."""
        ids = np.ascontiguousarray(ids, np.uint64)
        self._check(self.lib.pxb_cloths_read_positions_async(self.h, A.ptr(ids), len(ids), out.ctypes.data, out.size),
                    "read_positions_async")

    def read_results_async(self, ids, out):
        """pxb_cloths_read_results_async into `out` (A.FRAME_RESULT records, ideally pinned);
        completes at wait_positions()."""
        ids = np.ascontiguousarray(ids, np.uint64)
        self._check(self.lib.pxb_cloths_read_results_async(self.h, A.ptr(ids), len(ids), out.ctypes.data),
                    "read_results_async")

    def wait_positions(self):
        self._check(self.lib.pxb_cloths_wait_positions(self.h), "wait_positions")

    def read_positions(self, ids, out=None):
        ids = np.ascontiguousarray(ids, np.uint64)
        if out is None:
            raise ValueError("pass an output float32 array (3 floats per particle)")
        self._check(self.lib.pxb_cloths_read_positions(self.h, A.ptr(ids), len(ids), out.ctypes.data,
                                                       out.size), "read_positions")
        return out

    def gather_positions_device(self, ids, out_ptr, capacity):
        """pxb_cloths_gather_positions_device: positions into device memory at out_ptr
        (capacity floats), with no allocation; enqueued on the context stream."""
        ids = np.ascontiguousarray(ids, np.uint64)
        self._check(self.lib.pxb_cloths_gather_positions_device(self.h, A.ptr(ids), len(ids), out_ptr, capacity),
                    "gather_positions_device")

    def project_particles(self, collider, thickness, points, motion_start=None):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        n = len(pts)
        st = None if motion_start is None else np.ascontiguousarray(motion_start, np.float32).reshape(-1, 3)
        assert st is None or len(st) == n
        col = np.ascontiguousarray(np.asarray(collider, A.COLLIDER).reshape(1))
        out = np.zeros_like(pts)
        nrm = np.zeros_like(pts)
        dep = np.zeros(n, np.float32)
        hit = np.zeros(n, np.int32)
        self._check(self.lib.pxb_project_particles(self.h, A.ptr(col), thickness, A.ptr(pts), A.ptr(st), n,
                                                   A.ptr(out), A.ptr(nrm), A.ptr(dep), A.ptr(hit)),
                    "project_particles")
        return hit, out, nrm, dep

    # --- whole frames (PhysicsWorld::step_cloths_) ------------------------------------------
    def step_frame(self, ids, bodies=None, colliders=None, collider_moving=None, gravity=(0, 0, -9.81),
                   sources=None, fixed_dt=1.0 / 60.0, cloth_substeps=4, cloth_iterations=10, dt=1.0 / 60.0):
        """pxb_cloths_step_frame: anchors from body poses, sleep gate, solve, sleep bookkeeping.
        Returns each cloth's awake flag after the frame."""
        ids = np.ascontiguousarray(ids, np.uint64)
        n = len(ids)
        cols, coff = _flatten(colliders, A.COLLIDER, n)
        src, soff = _flatten(sources, A.GRAVITY_SOURCE, n)
        bod = None if bodies is None else np.ascontiguousarray(bodies, A.BODY_POSE).reshape(-1)
        mov = None if collider_moving is None else np.ascontiguousarray(collider_moving, np.uint8)
        d = A.ClothFrameDesc()
        d.cloths, d.n_cloths = A.ptr(ids), n
        d.bodies, d.n_bodies = A.ptr(bod), 0 if bod is None else len(bod)
        d.colliders, d.collider_offsets, d.collider_moving = A.ptr(cols), A.ptr(coff), A.ptr(mov)
        d.gravity = _vec(gravity)
        d.sources, d.source_offsets = A.ptr(src), A.ptr(soff)
        d.fixed_dt, d.cloth_substeps, d.cloth_iterations, d.dt = fixed_dt, cloth_substeps, cloth_iterations, dt
        awake = np.zeros(n, np.uint8)
        self._check(self.lib.pxb_cloths_step_frame(self.h, C.byref(d), A.ptr(awake)), "step_frame")
        return awake

    def step_strands_frame(self, ids, colliders=None, collider_moving=None, gravity=(0, 0, -9.81), sources=None,
                           fixed_dt=1.0 / 60.0, cloth_substeps=4, cloth_iterations=10, dt=1.0 / 60.0):
        """pxb_strands_step_frame: root-moved wake, sleep gate, solve, sleep bookkeeping. Returns
        each set's awake flag after the frame."""
        ids = np.ascontiguousarray(ids, np.uint64)
        n = len(ids)
        cols, coff = _flatten(colliders, A.COLLIDER, n)
        src, soff = _flatten(sources, A.GRAVITY_SOURCE, n)
        mov = None if collider_moving is None else np.ascontiguousarray(collider_moving, np.uint8)
        d = A.StrandFrameDesc()
        d.sets, d.n_sets = A.ptr(ids), n
        d.colliders, d.collider_offsets, d.collider_moving = A.ptr(cols), A.ptr(coff), A.ptr(mov)
        d.gravity = _vec(gravity)
        d.sources, d.source_offsets = A.ptr(src), A.ptr(soff)
        d.fixed_dt, d.cloth_substeps, d.cloth_iterations, d.dt = fixed_dt, cloth_substeps, cloth_iterations, dt
        awake = np.zeros(n, np.uint8)
        self._check(self.lib.pxb_strands_step_frame(self.h, C.byref(d), A.ptr(awake)), "strands_step_frame")
        return awake

    def read_strand_sleep_state(self, ids):
        ids = np.ascontiguousarray(ids, np.uint64)
        awake = np.zeros(len(ids), np.uint8)
        timer = np.zeros(len(ids), np.float32)
        self._check(self.lib.pxb_strands_read_sleep_state(self.h, A.ptr(ids), len(ids), A.ptr(awake), A.ptr(timer)),
                    "strands_read_sleep_state")
        return awake, timer

    def state_hash(self, ids, seed=1469598103934665603):
        """pxb_cloths_state_hash: world_state_hash's cloth part, continued from `seed`."""
        ids = np.ascontiguousarray(ids, np.uint64)
        out = u64()
        self._check(self.lib.pxb_cloths_state_hash(self.h, A.ptr(ids), len(ids), seed, C.byref(out)), "state_hash")
        return int(out.value)

    def read_render_buffer(self, ids, n_particles):
        """pxb_cloths_read_render_buffer: (n, 6) float32, position and unit vertex normal."""
        ids = np.ascontiguousarray(ids, np.uint64)
        out = np.zeros((int(n_particles), 6), np.float32)
        self._check(self.lib.pxb_cloths_read_render_buffer(self.h, A.ptr(ids), len(ids), A.ptr(out), out.size),
                    "read_render_buffer")
        return out

    def read_sleep_state(self, ids):
        ids = np.ascontiguousarray(ids, np.uint64)
        awake = np.zeros(len(ids), np.uint8)
        timer = np.zeros(len(ids), np.float32)
        self._check(self.lib.pxb_cloths_read_sleep_state(self.h, A.ptr(ids), len(ids), A.ptr(awake), A.ptr(timer)),
                    "read_sleep_state")
        return awake, timer

    # --- collider geometry ----------------------------------------------------------------
    def create_hull(self, hull) -> int:
        """pxb_geometry_create_hull: returns the id a ConvexHull collider names."""
        d = hull.desc()
        out = u32()
        self._check(self.lib.pxb_geometry_create_hull(self.h, C.byref(d), C.byref(out)), "create_hull")
        return int(out.value)

    def create_mesh(self, mesh) -> int:
        """pxb_geometry_create_mesh: returns the id a TriangleMesh collider names."""
        d = mesh.desc()
        out = u32()
        self._check(self.lib.pxb_geometry_create_mesh(self.h, C.byref(d), C.byref(out)), "create_mesh")
        return int(out.value)

    def create_height_grid(self, grid) -> int:
        """pxb_geometry_create_height_grid: returns the id a TriangleMesh collider over
        TriangleMesh::from_height_grid(grid) names."""
        d = grid.desc()
        out = u32()
        self._check(self.lib.pxb_geometry_create_height_grid(self.h, C.byref(d), C.byref(out)),
                    "create_height_grid")
        return int(out.value)

    def create_geometry(self, g) -> int:
        """Registers a Hull, a Mesh or a HeightGrid."""
        if isinstance(g, Hull):
            return self.create_hull(g)
        if isinstance(g, HeightGrid):
            return self.create_height_grid(g)
        return self.create_mesh(g)

    def destroy_geometry(self, gid):
        self._check(self.lib.pxb_geometry_destroy(self.h, gid), "destroy_geometry")

    # --- strand sets ----------------------------------------------------------------------
    def add_strands(self, s: StrandArrays) -> int:
        d = s.desc()
        out = u64()
        self._check(self.lib.pxb_strands_add(self.h, C.byref(d), C.byref(out)), "add_strands")
        return out.value

    def remove_strands(self, sid):
        self._check(self.lib.pxb_strands_remove(self.h, sid), "remove_strands")

    def set_strand_params(self, sid, params):
        self._check(self.lib.pxb_strands_set_params(self.h, sid, C.byref(params)), "set_strand_params")

    def set_strand_roots(self, sid, positions, orientations=None):
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        rot = None if orientations is None else np.ascontiguousarray(orientations, np.float32).reshape(-1, 4)
        self._check(self.lib.pxb_strands_set_roots(self.h, sid, A.ptr(pos), len(pos), A.ptr(rot),
                                                   0 if rot is None else len(rot)), "set_strand_roots")

    def read_strand_particles(self, sid, n):
        out = np.zeros(n, A.PARTICLE)
        self._check(self.lib.pxb_strands_read_particles(self.h, sid, A.ptr(out), n), "read_strand_particles")
        return out

    def write_strand_particles(self, sid, particles):
        p = np.ascontiguousarray(particles, A.PARTICLE)
        self._check(self.lib.pxb_strands_write_particles(self.h, sid, A.ptr(p), len(p)), "write_strand_particles")

    def read_strand_lambdas(self, sid, n):
        out = np.zeros(n, np.float32)
        self._check(self.lib.pxb_strands_read_lambdas(self.h, sid, A.ptr(out) if n else None, n),
                    "read_strand_lambdas")
        return out

    def read_strand_time(self, sid):
        t = f32()
        self._check(self.lib.pxb_strands_read_time(self.h, sid, C.byref(t)), "read_strand_time")
        return t.value

    def make_strand_step(self, ids, colliders=None, gravity=(0, 0, -9.81), sources=None, substeps=4,
                         iterations=4, h=1.0 / 60.0):
        ids = np.ascontiguousarray(ids, np.uint64)
        n = len(ids)
        cols, coff = _flatten(colliders, A.COLLIDER, n)
        src, soff = _flatten(sources, A.GRAVITY_SOURCE, n)
        d = A.StrandStepDesc()
        d.sets = A.ptr(ids)
        d.n_sets = n
        d.colliders = A.ptr(cols)
        d.collider_offsets = A.ptr(coff)
        d.gravity = _vec(gravity)
        d.sources = A.ptr(src)
        d.source_offsets = A.ptr(soff)
        d.substeps, d.iterations, d.h = substeps, iterations, h
        return d, (ids, cols, coff, src, soff)

    def step_strands(self, ids, colliders=None, gravity=(0, 0, -9.81), sources=None, substeps=4,
                     iterations=4, h=1.0 / 60.0):
        d, keep = self.make_strand_step(ids, colliders, gravity, sources, substeps, iterations, h)
        self._check(self.lib.pxb_strands_step(self.h, C.byref(d)), "strands_step")
        del keep

    def step_strands_desc(self, d):
        self._check(self.lib.pxb_strands_step(self.h, C.byref(d)), "strands_step")

    def read_strand_results(self, ids):
        ids = np.ascontiguousarray(ids, np.uint64)
        out = np.zeros(len(ids), A.FRAME_RESULT)
        self._check(self.lib.pxb_strands_read_results(self.h, A.ptr(ids), len(ids), A.ptr(out)),
                    "read_strand_results")
        return out

    def solve_strands_host(self, s: StrandArrays, colliders=None, gravity=(0, 0, -9.81), substeps=4,
                           iterations=4, h=1.0 / 60.0):
        """The drop-in solve_strands on host arrays: advances `s` in place."""
        d = s.desc()
        cols = colliders if colliders is not None else np.zeros(0, A.COLLIDER)
        t = f32(s.time)
        b = (C.c_float * 6)()
        self._check(self.lib.pxb_solve_strands_host(self.h, C.byref(d), A.ptr(s.particles), A.ptr(s.stretch),
                                                    A.ptr(cols), len(cols), _vec(gravity), substeps,
                                                    iterations, h, C.byref(t), b), "solve_strands_host")
        s.time = t.value
        s.bounds = np.array(b[:], np.float32)
        return s

    def solve_cloth_host(self, c: ClothArrays, colliders=None, gravity=(0, 0, -9.81), substeps=4,
                         iterations=10, h=1.0 / 60.0):
        """The drop-in solve_cloth on host arrays: advances `c` in place."""
        d = c.desc()
        cols = colliders if colliders is not None else np.zeros(0, A.COLLIDER)
        t = f32(c.time)
        b = (C.c_float * 6)()
        self._check(self.lib.pxb_solve_cloth_host(
            self.h, C.byref(d), A.ptr(c.particles), A.ptr(c.stretch), A.ptr(c.bend),
            A.ptr(c.anchors), A.ptr(cols), len(cols), _vec(gravity), substeps, iterations, h,
            C.byref(t), b), "solve_cloth_host")
        c.time = t.value
        c.bounds = np.array(b[:], np.float32)
        return c
