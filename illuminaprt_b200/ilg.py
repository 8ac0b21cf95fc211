"""Python binding of the C ABI in include/ilg.h (ctypes over libilg.so).

The names mirror the reference's space interface (Core/Space/Space.h:23-46):
``GpuSpace.initialise`` / ``build`` / ``intersects`` / ``occluded`` stand for
ISpace::Initialise / Build / Intersects(ray, isect) / Intersects(ray), batched
over arrays of rays. Errors raise ``IlgError`` carrying the library's status
code and message (the reference throws ``Exception*``; here it is a Python
exception). There is no CPU fallback: without the CUDA library or a GPU,
construction fails loudly.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

ILG_OK, ILG_EINVAL, ILG_ENOMEM, ILG_ECUDA, ILG_ETIMEOUT, ILG_EOVERFLOW, ILG_ESTATE = range(7)
ILG_DEVICE_PTRS = 0x1
ILG_WATERTIGHT = 0x2
ILG_RENDER_COUNT = 0x4
ILG_RENDER_HASH_CACHE = 0x8
ILG_RENDER_PERSISTENT = 0x20

STATUS_NAMES = {0: "ILG_OK", 1: "ILG_EINVAL", 2: "ILG_ENOMEM", 3: "ILG_ECUDA", 4: "ILG_ETIMEOUT",
                5: "ILG_EOVERFLOW", 6: "ILG_ESTATE"}

# Every symbol the public headers declare; tests check the library exports them.
EXPORTED = ["ilg_create", "ilg_destroy", "ilg_last_error", "ilg_set_mesh", "ilg_build", "ilg_get_stats",
            "ilg_intersect", "ilg_intersect_counted", "ilg_occluded", "ilg_sync", "ilg_stream",
            "ilg_set_materials", "ilg_set_quad_lights", "ilg_render", "ilg_intersect_noalloc",
            "ilg_mlp_init", "ilg_mlp_get_params", "ilg_mlp_set_params", "ilg_mlp_infer", "ilg_mlp_grads",
            "ilg_mlp_train_step", "ilg_render_batch", "ilg_intersect_excluding", "ilg_occluded_excluding",
            "ilg_camera_frame_of", "ilg_render_region", "ilg_mlp_get_grid", "ilg_mlp_set_grid",
            "ilg_mlp_get_grid_grads", "ilg_accumulate", "ilg_accumulate_reset", "ilg_tonemap",
            "ilg_render_counts", "ilg_save", "ilg_load", "ilg_hash_cache_reset", "ilg_last_train_stats", "ilg_probe_read_gbs", "ilg_set_lights", "ilg_radiance", "ilg_mlp_init_encoding"]

ILG_MLP_RAW = 16
ILG_MLP_WARP_MMA = 0x10
ILG_MLP_PARAMS = 23040
ILG_MLP_GRID_PARAMS = 1048576

# Largest batch ilg_intersect_noalloc accepts (include/ilg.h).
ILG_NOALLOC_MAX_RAYS = 262144

ILG_MAT_LAMBERT, ILG_MAT_GGX, ILG_MAT_MIRROR, ILG_MAT_GLASS = 0, 1, 2, 3


class IlgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class ilg_opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("build_flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 6)]


ILG_BUILD_FAST = 0x1


class ilg_stats(ctypes.Structure):
    _fields_ = [("n_tris", ctypes.c_uint32), ("n_nodes", ctypes.c_uint32), ("n_leaf_tris", ctypes.c_uint32),
                ("max_depth", ctypes.c_uint32), ("build_ms", ctypes.c_float), ("node_bytes", ctypes.c_uint64),
                ("tri_bytes", ctypes.c_uint64)]


class ilg_material(ctypes.Structure):
    _fields_ = [("albedo", ctypes.c_float * 3), ("kind", ctypes.c_uint32), ("f0", ctypes.c_float * 3),
                ("alpha", ctypes.c_float)]


class ilg_quad_light(ctypes.Structure):
    _fields_ = [("v", (ctypes.c_float * 3) * 4), ("emit", ctypes.c_float * 3), ("first_tri", ctypes.c_uint32)]


ILG_LIGHT_QUAD, ILG_LIGHT_MESH, ILG_LIGHT_INFINITE = 0, 1, 2


class ilg_light(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("emit", ctypes.c_float * 3), ("v", (ctypes.c_float * 3) * 4),
                ("first_tri", ctypes.c_uint32), ("tri_count", ctypes.c_uint32)]


class ilg_camera(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("target", ctypes.c_float * 3), ("up", ctypes.c_float * 3),
                ("fov_deg", ctypes.c_float), ("aspect", ctypes.c_float)]


class ilg_camera_frame(ctypes.Structure):
    _fields_ = [("centre", ctypes.c_float * 3), ("corner", ctypes.c_float * 3), ("across", ctypes.c_float * 3),
                ("up", ctypes.c_float * 3)]


class ilg_region(ctypes.Structure):
    _fields_ = [("x", ctypes.c_uint32), ("y", ctypes.c_uint32), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32)]


class ilg_batch_item(ctypes.Structure):
    pass


class ilg_render_opts(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("spp", ctypes.c_uint32),
                ("max_depth", ctypes.c_uint32), ("epsilon", ctypes.c_float), ("seed", ctypes.c_uint32),
                ("paths_per_wave", ctypes.c_uint32), ("sky", ctypes.c_float * 3), ("cache_depth", ctypes.c_uint32),
                ("train_every", ctypes.c_uint32), ("train_steps", ctypes.c_uint32), ("train_batch", ctypes.c_uint32),
                ("train_tail", ctypes.c_uint32), ("train_epochs", ctypes.c_uint32)]


ilg_batch_item._fields_ = [("scene", ctypes.c_void_p), ("camera", ilg_camera), ("width", ctypes.c_uint32),
                           ("height", ctypes.c_uint32), ("spp", ctypes.c_uint32), ("max_depth", ctypes.c_uint32),
                           ("epsilon", ctypes.c_float), ("seed", ctypes.c_uint32), ("sky", ctypes.c_float * 3),
                           ("out_rgb", ctypes.c_void_p)]

_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True) -> ctypes.CDLL:
    """Load libilg.so (building it first when it is absent or stale)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing:
        _build.build()
    if not os.path.exists(_build.LIB):
        raise IlgError(ILG_ESTATE, f"CUDA library not built: {_build.LIB}")
    L = ctypes.CDLL(_build.LIB)
    vp, u32, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32
    L.ilg_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(ilg_opts)]
    L.ilg_destroy.argtypes = [vp]
    L.ilg_last_error.argtypes = [vp]
    L.ilg_last_error.restype = ctypes.c_char_p
    L.ilg_set_mesh.argtypes = [vp, vp, u32, vp, u32, vp]
    L.ilg_build.argtypes = [vp]
    L.ilg_get_stats.argtypes = [vp, ctypes.POINTER(ilg_stats)]
    L.ilg_intersect.argtypes = [vp, vp, vp, u32, vp, vp, vp, vp, u32]
    L.ilg_intersect_counted.argtypes = [vp, vp, vp, u32, vp, vp, vp, vp, vp, u32]
    L.ilg_occluded.argtypes = [vp, vp, vp, u32, vp, u32]
    L.ilg_set_materials.argtypes = [vp, vp, u32]
    L.ilg_set_quad_lights.argtypes = [vp, vp, u32]
    L.ilg_set_lights.argtypes = [vp, vp, u32]
    L.ilg_radiance.argtypes = [vp, vp, vp, u32, ctypes.POINTER(ilg_render_opts), vp, vp, vp, u32]
    L.ilg_render.argtypes = [vp, ctypes.POINTER(ilg_camera), ctypes.POINTER(ilg_render_opts), vp, u32]
    L.ilg_intersect_noalloc.argtypes = [vp, vp, vp, u32, vp, vp, vp, vp]
    L.ilg_render_counts.argtypes = [vp, vp]
    L.ilg_hash_cache_reset.argtypes = [vp]
    L.ilg_last_train_stats.argtypes = [vp, vp, vp]
    L.ilg_probe_read_gbs.argtypes = [vp, ctypes.c_uint64, u32, vp]
    L.ilg_save.argtypes = [vp, ctypes.c_char_p]
    L.ilg_load.argtypes = [vp, ctypes.c_char_p]
    L.ilg_accumulate.argtypes = [vp, vp, u32, vp, u32]
    L.ilg_accumulate_reset.argtypes = [vp]
    L.ilg_tonemap.argtypes = [vp, vp, u32, vp, u32, u32]
    L.ilg_camera_frame_of.argtypes = [ctypes.POINTER(ilg_camera), ctypes.POINTER(ilg_camera_frame)]
    L.ilg_render_region.argtypes = [vp, ctypes.POINTER(ilg_camera_frame), ctypes.POINTER(ilg_render_opts),
                                    ctypes.POINTER(ilg_region), vp, vp, vp, u32]
    L.ilg_intersect_excluding.argtypes = [vp, vp, vp, u32, u32, u32, vp, vp, vp, vp, u32]
    L.ilg_occluded_excluding.argtypes = [vp, vp, vp, u32, u32, u32, vp, u32]
    L.ilg_intersect_noalloc.restype = i32
    L.ilg_mlp_init.argtypes = [vp, u32, ctypes.c_float]
    L.ilg_mlp_init_encoding.argtypes = [vp, u32, ctypes.c_float, u32]
    L.ilg_mlp_get_params.argtypes = [vp, vp]
    L.ilg_mlp_set_params.argtypes = [vp, vp]
    L.ilg_mlp_get_grid.argtypes = [vp, vp]
    L.ilg_mlp_set_grid.argtypes = [vp, vp]
    L.ilg_mlp_get_grid_grads.argtypes = [vp, vp]
    L.ilg_mlp_infer.argtypes = [vp, vp, u32, vp, u32]
    L.ilg_mlp_grads.argtypes = [vp, vp, vp, u32, vp, vp, u32]
    L.ilg_mlp_train_step.argtypes = [vp, vp, vp, u32, vp, u32]
    for f in ("ilg_mlp_init", "ilg_mlp_get_params", "ilg_mlp_set_params", "ilg_mlp_infer", "ilg_mlp_grads",
              "ilg_mlp_train_step"):
        getattr(L, f).restype = i32
    L.ilg_render_batch.argtypes = [vp, vp, u32, u32, u32, u32]
    L.ilg_render_batch.restype = i32
    L.ilg_sync.argtypes = [vp]
    L.ilg_stream.argtypes = [vp]
    L.ilg_stream.restype = vp
    for f in ("ilg_create", "ilg_destroy", "ilg_set_mesh", "ilg_build", "ilg_get_stats", "ilg_intersect",
              "ilg_intersect_counted", "ilg_occluded", "ilg_sync", "ilg_set_materials", "ilg_set_quad_lights",
              "ilg_render"):
        getattr(L, f).restype = i32
    _lib = L
    return L


def _ptr(a) -> int:
    """Address of a numpy array or a torch tensor."""
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


class GpuSpace:
    """A triangle scene on one GPU with batched closest-hit / any-hit queries."""

    def __init__(self, device: int = 0, fast_build: bool = False):
        """fast_build: ILG_BUILD_FAST (the Morton tree without treelet restructuring)."""
        self.L = load()
        self.h = ctypes.c_void_p()
        opts = ilg_opts(device=device, build_flags=ILG_BUILD_FAST if fast_build else 0)
        rc = self.L.ilg_create(ctypes.byref(self.h), ctypes.byref(opts))
        if rc != ILG_OK:
            raise IlgError(rc, f"ilg_create(device={device}) failed")
        self.device = device
        self.n_tris = 0

    def _check(self, rc: int):
        if rc != ILG_OK:
            raise IlgError(rc, self.L.ilg_last_error(self.h).decode(errors="replace"))

    # ISpace::Initialise + PrimitiveList fill
    def initialise(self, positions, indices, material_ids=None):
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        idx = np.ascontiguousarray(indices, np.uint32).reshape(-1, 3)
        mat = None if material_ids is None else np.ascontiguousarray(material_ids, np.uint32)
        self._check(self.L.ilg_set_mesh(self.h, pos.ctypes.data, pos.shape[0], idx.ctypes.data, idx.shape[0],
                                        None if mat is None else mat.ctypes.data))
        self.n_tris = idx.shape[0]

    # ISpace::Build
    def build(self):
        self._check(self.L.ilg_build(self.h))

    def stats(self) -> dict:
        s = ilg_stats()
        self._check(self.L.ilg_get_stats(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    @property
    def stream(self) -> int:
        return self.L.ilg_stream(self.h) or 0

    # ISpace::Intersects(ray, isect), batched; host arrays
    def intersects(self, o4: np.ndarray, d4: np.ndarray, watertight: bool = False):
        o4 = np.ascontiguousarray(o4, np.float32)
        d4 = np.ascontiguousarray(d4, np.float32)
        n = o4.shape[0]
        prim = np.empty(n, np.int32)
        t, u, v = (np.empty(n, np.float32) for _ in range(3))
        self._check(self.L.ilg_intersect(self.h, o4.ctypes.data, d4.ctypes.data, n, prim.ctypes.data,
                                         t.ctypes.data, u.ctypes.data, v.ctypes.data,
                                         ILG_WATERTIGHT if watertight else 0))
        return prim, t, u, v

    def intersects_into(self, o4, d4, prim, t, u, v, device_ptrs: bool, watertight: bool = False):
        """Same query on caller-owned buffers (numpy, pinned or device torch tensors)."""
        n = o4.shape[0]
        flags = (ILG_DEVICE_PTRS if device_ptrs else 0) | (ILG_WATERTIGHT if watertight else 0)
        self._check(self.L.ilg_intersect(self.h, _ptr(o4), _ptr(d4), n, _ptr(prim), _ptr(t), _ptr(u), _ptr(v),
                                         flags))

    def traversal_counts(self, o4, d4):
        """(node records read, triangle records tested) for one closest-hit pass
        over device-resident rays (torch tensors)."""
        import torch
        n = o4.shape[0]
        prim = torch.empty(n, dtype=torch.int32, device=o4.device)
        t, u, v = (torch.empty(n, dtype=torch.float32, device=o4.device) for _ in range(3))
        counts = np.zeros(2, np.uint64)
        self._check(self.L.ilg_intersect_counted(self.h, _ptr(o4), _ptr(d4), n, _ptr(prim), _ptr(t), _ptr(u),
                                                 _ptr(v), counts.ctypes.data, ILG_DEVICE_PTRS))
        return int(counts[0]), int(counts[1])

    # ISpace::Intersects(ray), batched
    def occluded(self, o4: np.ndarray, d4: np.ndarray, watertight: bool = False) -> np.ndarray:
        o4 = np.ascontiguousarray(o4, np.float32)
        d4 = np.ascontiguousarray(d4, np.float32)
        occ = np.empty(o4.shape[0], np.uint8)
        self._check(self.L.ilg_occluded(self.h, o4.ctypes.data, d4.ctypes.data, o4.shape[0], occ.ctypes.data,
                                        ILG_WATERTIGHT if watertight else 0))
        return occ

    # ISpace::Intersects(ray, isect, p_pExclude) / Intersects(ray, p_pExclude),
    # batched: input triangles [first, first + count) are ignored
    def intersects_excluding(self, o4: np.ndarray, d4: np.ndarray, first: int, count: int):
        o4 = np.ascontiguousarray(o4, np.float32)
        d4 = np.ascontiguousarray(d4, np.float32)
        n = o4.shape[0]
        prim = np.empty(n, np.int32)
        t, u, v = (np.empty(n, np.float32) for _ in range(3))
        self._check(self.L.ilg_intersect_excluding(self.h, o4.ctypes.data, d4.ctypes.data, n, first, count,
                                                   prim.ctypes.data, t.ctypes.data, u.ctypes.data, v.ctypes.data, 0))
        return prim, t, u, v

    def occluded_excluding(self, o4: np.ndarray, d4: np.ndarray, first: int, count: int) -> np.ndarray:
        o4 = np.ascontiguousarray(o4, np.float32)
        d4 = np.ascontiguousarray(d4, np.float32)
        occ = np.empty(o4.shape[0], np.uint8)
        self._check(self.L.ilg_occluded_excluding(self.h, o4.ctypes.data, d4.ctypes.data, o4.shape[0], first, count,
                                                  occ.ctypes.data, 0))
        return occ

    def occluded_into(self, o4, d4, occ, device_ptrs: bool):
        self._check(self.L.ilg_occluded(self.h, _ptr(o4), _ptr(d4), o4.shape[0], _ptr(occ),
                                        ILG_DEVICE_PTRS if device_ptrs else 0))

    # --- path tracing: PathIntegrator + RenderRegion over the whole image ----
    def set_materials(self, mats):
        """mats: sequence of dicts {albedo, kind=0, f0=(0,0,0), alpha=0}; kind 0 Lambertian,
        1 GGX (f0, alpha), 2 mirror (albedo = reflectivity), 3 glass (albedo = reflectivity,
        f0 = transmittance, alpha = eta_i / eta_t)."""
        arr = (ilg_material * len(mats))()
        for i, m in enumerate(mats):
            arr[i].albedo[:] = list(m.get("albedo", (0.0, 0.0, 0.0)))
            arr[i].kind = int(m.get("kind", ILG_MAT_LAMBERT))
            arr[i].f0[:] = list(m.get("f0", (0.0, 0.0, 0.0)))
            arr[i].alpha = float(m.get("alpha", 0.0))
        self._check(self.L.ilg_set_materials(self.h, ctypes.addressof(arr), len(mats)))

    def set_quad_lights(self, lights):
        """lights: sequence of dicts {v: 4x3 (reference Quad order), emit: 3, first_tri}."""
        arr = (ilg_quad_light * max(1, len(lights)))()
        for i, l in enumerate(lights):
            for k in range(4):
                arr[i].v[k][:] = [float(x) for x in l["v"][k]]
            arr[i].emit[:] = [float(x) for x in l["emit"]]
            arr[i].first_tri = int(l["first_tri"])
        self._check(self.L.ilg_set_quad_lights(self.h, ctypes.addressof(arr), len(lights)))

    def set_lights(self, lights):
        """lights: sequence of dicts with "kind" ("quad", "mesh" or "infinite")
        and "emit"; quads add "v" (4x3, reference Quad order) and "first_tri",
        meshes "first_tri" and "tri_count"."""
        kinds = {"quad": ILG_LIGHT_QUAD, "mesh": ILG_LIGHT_MESH, "infinite": ILG_LIGHT_INFINITE}
        arr = (ilg_light * max(1, len(lights)))()
        for i, l in enumerate(lights):
            arr[i].kind = kinds[l["kind"]]
            arr[i].emit[:] = [float(x) for x in l["emit"]]
            if "v" in l:
                for k in range(4):
                    arr[i].v[k][:] = [float(x) for x in l["v"][k]]
            arr[i].first_tri = int(l.get("first_tri", 0))
            arr[i].tri_count = int(l.get("tri_count", 2 if l["kind"] == "quad" else 0))
        self._check(self.L.ilg_set_lights(self.h, ctypes.addressof(arr), len(lights)))

    @staticmethod
    def _camera(camera: dict, width: int, height: int) -> ilg_camera:
        cam = ilg_camera()
        cam.eye[:] = list(camera["eye"])
        cam.target[:] = list(camera["target"])
        cam.up[:] = list(camera["up"])
        cam.fov_deg = float(camera["fov"])
        cam.aspect = float(camera.get("aspect", width / height))
        return cam

    def camera_frame(self, camera: dict, width: int, height: int) -> ilg_camera_frame:
        """The (centre, corner, across, up) frame the reference's PerspectiveCamera builds."""
        f = ilg_camera_frame()
        self._check(self.L.ilg_camera_frame_of(ctypes.byref(self._camera(camera, width, height)), ctypes.byref(f)))
        return f

    def render_region(self, frame: ilg_camera_frame, width: int, height: int, spp: int, region, max_depth: int = 6,
                      epsilon: float = 1e-4, seed: int = 1, sky=(0.0, 0.0, 0.0), aux: bool = True,
                      cache_depth: int = 0, train_every: int = 16, train_steps: int = 4, train_batch: int = 16384,
                      train_tail: int = 0, train_epochs: int = 1):
        """IRenderer::RenderRegion: region = (x, y, w, h) of the width x height image.
        Returns (final, direct, albedo), each (h, w, 3) float32 (direct/albedo None without aux).
        cache_depth > 0 renders with the radiance cache as render() does."""
        x, y, w, h = (int(v) for v in region)
        o = ilg_render_opts(width=width, height=height, spp=spp, max_depth=max_depth, epsilon=epsilon, seed=seed,
                            cache_depth=cache_depth, train_every=train_every, train_steps=train_steps,
                            train_batch=train_batch, train_tail=train_tail, train_epochs=train_epochs)
        o.sky[:] = list(sky)
        r = ilg_region(x=x, y=y, width=w, height=h)
        final = np.empty((h, w, 3), np.float32)
        direct = np.empty((h, w, 3), np.float32) if aux else None
        albedo = np.empty((h, w, 3), np.float32) if aux else None
        self._check(self.L.ilg_render_region(self.h, ctypes.byref(frame), ctypes.byref(o), ctypes.byref(r),
                                             final.ctypes.data, direct.ctypes.data if aux else None,
                                             albedo.ctypes.data if aux else None, 0))
        return final, direct, albedo

    def save(self, path: str):
        """Writes the mesh and its built BVH (ilg_save)."""
        self._check(self.L.ilg_save(self.h, str(path).encode()))

    def load(self, path: str):
        """Reads a scene written by save: the context is built, no rebuild (ilg_load)."""
        self._check(self.L.ilg_load(self.h, str(path).encode()))

    def render_counts(self):
        """Traversal work of the last render made with count=True:
        (closest rays, their node reads, their triangle tests, shadow rays, node reads, triangle tests)."""
        c = np.zeros(6, np.uint64)
        self._check(self.L.ilg_render_counts(self.h, c.ctypes.data))
        return tuple(int(x) for x in c)

    def render(self, camera: dict, width: int, height: int, spp: int, max_depth: int = 6, epsilon: float = 1e-4,
               seed: int = 1, sky=(0.0, 0.0, 0.0), paths_per_wave: int = 0, out=None, cache_depth: int = 0,
               train_every: int = 16, train_steps: int = 4, train_batch: int = 16384, count: bool = False,
               train_tail: int = 0, train_epochs: int = 1, hash_cache: bool = False, one_launch: bool = False):
        """Returns (height, width, 3) float32 (or fills `out`, a CUDA tensor, in place).
        one_launch renders with the persistent one-launch kernel (ILG_RENDER_PERSISTENT).
        cache_depth > 0 renders with the radiance cache (mlp_init first) and trains it afterwards;
        with hash_cache the non-learned hash-grid cache stands in for the network
        (hash_cache_reset first)."""
        cam = self._camera(camera, width, height)
        o = ilg_render_opts(width=width, height=height, spp=spp, max_depth=max_depth, epsilon=epsilon, seed=seed,
                            paths_per_wave=paths_per_wave, cache_depth=cache_depth, train_every=train_every,
                            train_steps=train_steps, train_batch=train_batch, train_tail=train_tail,
                            train_epochs=train_epochs)
        o.sky[:] = list(sky)
        flags = ((ILG_RENDER_COUNT if count else 0) | (ILG_RENDER_HASH_CACHE if hash_cache else 0)
                 | (ILG_RENDER_PERSISTENT if one_launch else 0))
        if out is not None:
            self._check(self.L.ilg_render(self.h, ctypes.byref(cam), ctypes.byref(o), _ptr(out),
                                          ILG_DEVICE_PTRS | flags))
            return out
        img = np.empty((height, width, 3), np.float32)
        self._check(self.L.ilg_render(self.h, ctypes.byref(cam), ctypes.byref(o), img.ctypes.data, flags))
        return img

    def radiance(self, o4, d4, spp: int = 1, max_depth: int = 6, epsilon: float = 1e-4, seed: int = 1,
                 sky=(0.0, 0.0, 0.0), aux: bool = False):
        """IIntegrator::Radiance over the rays (float32 (n, 4) origin/Min and
        direction/Max): per ray the average of spp device paths started with
        it; returns final (n, 3), or (final, direct, albedo) with aux."""
        o4 = np.ascontiguousarray(o4, np.float32)
        d4 = np.ascontiguousarray(d4, np.float32)
        n = o4.shape[0]
        o = ilg_render_opts(width=n, height=1, spp=spp, max_depth=max_depth, epsilon=epsilon, seed=seed)
        o.sky[:] = list(sky)
        outs = [np.empty((n, 3), np.float32) for _ in range(3 if aux else 1)]
        ptrs = [x.ctypes.data for x in outs] + [None] * (3 - len(outs))
        self._check(self.L.ilg_radiance(self.h, o4.ctypes.data, d4.ctypes.data, n, ctypes.byref(o), *ptrs, 0))
        return tuple(outs) if aux else outs[0]

    def hash_cache_reset(self):
        """Empties the hash-grid radiance cache (allocated on first use)."""
        self._check(self.L.ilg_hash_cache_reset(self.h))

    def probe_read_gbs(self, nbytes: int, reps: int = 64) -> float:
        """Streaming read bandwidth (GB/s) over a device buffer of nbytes."""
        g = ctypes.c_float(0.0)
        self._check(self.L.ilg_probe_read_gbs(self.h, int(nbytes), int(reps), ctypes.byref(g)))
        return float(g.value)

    def last_train_stats(self):
        """(training records of the last cached render, of those dropped by
        the hash-grid cache for want of a free cell)."""
        rec, drop = ctypes.c_uint32(0), ctypes.c_uint32(0)
        self._check(self.L.ilg_last_train_stats(self.h, ctypes.byref(rec), ctypes.byref(drop)))
        return int(rec.value), int(drop.value)

    # --- post-processing (AccumulationBuffer, tone operators) ---------------
    TONE = {"global": 0, "auto": 1, "drago": 2}

    def accumulate(self, frame, out=None):
        """AccumulationBuffer::Apply: running average of the frames given since
        the last reset (numpy in/out, or CUDA tensors with out given)."""
        if out is not None:
            self._check(self.L.ilg_accumulate(self.h, _ptr(frame), frame.numel() // 3, _ptr(out), ILG_DEVICE_PTRS))
            return out
        f = np.ascontiguousarray(frame, np.float32)
        o = np.empty_like(f)
        self._check(self.L.ilg_accumulate(self.h, f.ctypes.data, f.size // 3, o.ctypes.data, 0))
        return o

    def accumulate_reset(self):
        self._check(self.L.ilg_accumulate_reset(self.h))

    def tonemap(self, img, op: str = "global", out=None):
        if out is not None:
            self._check(self.L.ilg_tonemap(self.h, _ptr(img), img.numel() // 3, _ptr(out), self.TONE[op],
                                           ILG_DEVICE_PTRS))
            return out
        f = np.ascontiguousarray(img, np.float32)
        o = np.empty_like(f)
        self._check(self.L.ilg_tonemap(self.h, f.ctypes.data, f.size // 3, o.ctypes.data, self.TONE[op], 0))
        return o

    # --- radiance-cache network -------------------------------------------
    MLP_ENCODINGS = {"hashgrid": 0, "freq12": 1}

    def mlp_init(self, seed: int = 1, lr: float = 1e-2, encoding: str = "hashgrid"):
        """A fresh cache network; encoding "hashgrid" (hash grid + bands +
        spherical harmonics) or "freq12" (12 frequency bands of position and
        the raw direction, normal, roughness and albedo)."""
        self._check(self.L.ilg_mlp_init_encoding(self.h, seed, lr, self.MLP_ENCODINGS[encoding]))

    def mlp_params(self) -> np.ndarray:
        p = np.empty(ILG_MLP_PARAMS, np.float32)
        self._check(self.L.ilg_mlp_get_params(self.h, p.ctypes.data))
        return p

    def mlp_set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == ILG_MLP_PARAMS
        self._check(self.L.ilg_mlp_set_params(self.h, p.ctypes.data))

    def mlp_grid(self) -> np.ndarray:
        g = np.empty(ILG_MLP_GRID_PARAMS, np.float32)
        self._check(self.L.ilg_mlp_get_grid(self.h, g.ctypes.data))
        return g

    def mlp_set_grid(self, g):
        g = np.ascontiguousarray(g, np.float32)
        assert g.size == ILG_MLP_GRID_PARAMS
        self._check(self.L.ilg_mlp_set_grid(self.h, g.ctypes.data))

    def mlp_grid_grads(self) -> np.ndarray:
        """The grid part of the gradient of the last mlp_grads call."""
        g = np.empty(ILG_MLP_GRID_PARAMS, np.float32)
        self._check(self.L.ilg_mlp_get_grid_grads(self.h, g.ctypes.data))
        return g

    def mlp_infer(self, raw, warp_mma: bool = False) -> np.ndarray:
        """Cache network outputs (tcgen05 tensor cores; warp_mma selects the mma.sync kernel)."""
        raw = np.ascontiguousarray(raw, np.float32).reshape(-1, ILG_MLP_RAW)
        out = np.empty((raw.shape[0], 3), np.float32)
        self._check(self.L.ilg_mlp_infer(self.h, raw.ctypes.data, raw.shape[0], out.ctypes.data,
                                         ILG_MLP_WARP_MMA if warp_mma else 0))
        return out

    def mlp_grads(self, raw, target, warp_mma: bool = False):
        """(loss, gradient) of the batch; on the tcgen05 kernels, or with
        warp_mma on the warp-level mma.sync ones."""
        raw = np.ascontiguousarray(raw, np.float32).reshape(-1, ILG_MLP_RAW)
        target = np.ascontiguousarray(target, np.float32).reshape(-1, 3)
        g = np.empty(ILG_MLP_PARAMS, np.float32)
        loss = ctypes.c_float()
        self._check(self.L.ilg_mlp_grads(self.h, raw.ctypes.data, target.ctypes.data, raw.shape[0], g.ctypes.data,
                                         ctypes.byref(loss), ILG_MLP_WARP_MMA if warp_mma else 0))
        return loss.value, g

    def mlp_train_step(self, raw, target) -> float:
        raw = np.ascontiguousarray(raw, np.float32).reshape(-1, ILG_MLP_RAW)
        target = np.ascontiguousarray(target, np.float32).reshape(-1, 3)
        loss = ctypes.c_float()
        self._check(self.L.ilg_mlp_train_step(self.h, raw.ctypes.data, target.ctypes.data, raw.shape[0],
                                              ctypes.byref(loss), 0))
        return loss.value

    def render_batch(self, items, paths_per_wave: int = 0, block: int = 0, device_ptrs: bool = False,
                     count: bool = False, one_launch: bool = False):
        """items: list of dicts {space: GpuSpace, camera, width, height, spp, max_depth=6, epsilon=1e-4,
        seed=1, sky=(0,0,0), out=None}. Renders all in one wavefront on this context; returns the images
        (numpy arrays, or the given CUDA tensors when device_ptrs)."""
        arr = (ilg_batch_item * len(items))()
        outs = []
        for i, it in enumerate(items):
            cam = it["camera"]
            a = arr[i]
            a.scene = it["space"].h.value
            a.camera.eye[:] = list(cam["eye"])
            a.camera.target[:] = list(cam["target"])
            a.camera.up[:] = list(cam["up"])
            a.camera.fov_deg = float(cam["fov"])
            a.camera.aspect = float(cam.get("aspect", it["width"] / it["height"]))
            a.width, a.height, a.spp = it["width"], it["height"], it["spp"]
            a.max_depth = it.get("max_depth", 6)
            a.epsilon = it.get("epsilon", 1e-4)
            a.seed = it.get("seed", 1)
            a.sky[:] = list(it.get("sky", (0.0, 0.0, 0.0)))
            if device_ptrs:
                out = it["out"]
                a.out_rgb = out.data_ptr()
            else:
                out = np.empty((it["height"], it["width"], 3), np.float32)
                a.out_rgb = out.ctypes.data
            outs.append(out)
        flags = ((ILG_DEVICE_PTRS if device_ptrs else 0) | (ILG_RENDER_COUNT if count else 0)
                 | (ILG_RENDER_PERSISTENT if one_launch else 0))
        self._check(self.L.ilg_render_batch(self.h, ctypes.addressof(arr), len(items), paths_per_wave, block,
                                            flags))
        return outs

    def sync(self):
        self._check(self.L.ilg_sync(self.h))

    def close(self):
        if self.h:
            self.L.ilg_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
