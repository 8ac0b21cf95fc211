"""ctypes bindings for the two CPU checkers - TEST INFRASTRUCTURE ONLY.

* ``Oracle``: our C restatement of the reference's query (oracle/ilg_oracle.c).
* ``RefLib``: the reference's own sources compiled by oracle/Makefile into
  oracle/_ref/libilref.so (present only where the reference tree was
  available at build time, or where the built library was carried along).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libilref.so")
# the reference's Core tree: $ILLUMINA_CORE, else a checkout named "reference"
# beside this repository
REF_TREE = os.environ.get("ILLUMINA_CORE",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference", "Core"))

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


def build(ref: bool = True) -> None:
    """Compile the oracle (always) and the reference library (when its tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref and os.path.isdir(REF_TREE):
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={REF_TREE}"], check=True)


def _ensure_oracle():
    srcs = [os.path.join(HERE, f) for f in ("ilg_oracle.c", "ilg_oracle.h", "pt_oracle.c")]
    if not os.path.exists(ORACLE_SO) or any(os.path.getmtime(s) > os.path.getmtime(ORACLE_SO) for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


class Oracle:
    def __init__(self):
        _ensure_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_shirley.argtypes = [_f32p, _u32p, ctypes.c_uint32, _f32p, _f32p, ctypes.c_float,
                                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                  ctypes.POINTER(ctypes.c_float)]
        L.orc_shirley.restype = ctypes.c_int
        L.orc_intersect_brute.argtypes = [_f32p, _u32p, ctypes.c_uint32, _f32p, _f32p, ctypes.c_int64,
                                          _i32p, _f32p, _f32p, _f32p]
        L.orc_watertight_brute.argtypes = [_f32p, _u32p, ctypes.c_uint32, _f32p, _f32p, ctypes.c_int64,
                                           _i32p, _f32p, _f32p, _f32p, _u8p]
        L.orc_bvh_create.argtypes = [_f32p, ctypes.c_uint32, _u32p, ctypes.c_uint32]
        L.orc_bvh_create.restype = ctypes.c_void_p
        L.orc_bvh_destroy.argtypes = [ctypes.c_void_p]
        L.orc_bvh_intersect.argtypes = [ctypes.c_void_p, _f32p, _f32p, ctypes.c_int64, _i32p, _f32p, _f32p,
                                        _f32p, ctypes.c_int, ctypes.c_void_p]
        L.orc_bvh_occluded.argtypes = [ctypes.c_void_p, _f32p, _f32p, ctypes.c_int64, _u8p, ctypes.c_int]
        L.orc_render.argtypes = [_f32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, _u32p, ctypes.c_void_p,
                                 ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32, _f32p, ctypes.c_uint32,
                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32,
                                 _f32p, ctypes.c_int, _f32p]
        L.orc_last_render_seconds.restype = ctypes.c_double
        self.L = L

    def last_render_seconds(self) -> float:
        """Wall seconds of the last render's paths, its tree build excluded."""
        return float(self.L.orc_last_render_seconds())

    def render(self, pos, idx, mat_ids, mats, lights, camera, width, height, spp, max_depth=6, epsilon=1e-4,
               seed=1, sky=(0.0, 0.0, 0.0), nthreads=None):
        """CPU restatement of the path tracer with the device's random numbers.
        mats: list of dicts {albedo, kind, f0, alpha}; lights: list of dicts {v, emit, first_tri}."""
        M = np.zeros((len(mats), 8), np.float32)
        for i, m in enumerate(mats):
            M[i, 0:3] = m.get("albedo", (0, 0, 0))
            M[i, 3] = np.array([m.get("kind", 0)], np.uint32).view(np.float32)[0]
            M[i, 4:7] = m.get("f0", (0, 0, 0))
            M[i, 7] = m.get("alpha", 0.0)
        Lt = np.zeros((max(1, len(lights)), 16), np.float32)
        for i, l in enumerate(lights):
            Lt[i, 0:12] = np.asarray(l["v"], np.float32).reshape(-1)
            Lt[i, 12:15] = l["emit"]
            Lt[i, 15] = np.array([l["first_tri"]], np.uint32).view(np.float32)[0]
        cam = np.array([*camera["eye"], *camera["target"], *camera["up"], camera["fov"],
                        camera.get("aspect", width / height)], np.float32)
        out = np.zeros((height, width, 3), np.float32)
        pos = np.ascontiguousarray(pos, np.float32)
        idx = np.ascontiguousarray(idx, np.uint32)
        self.L.orc_render(pos.reshape(-1), pos.shape[0], idx.reshape(-1), idx.shape[0],
                          np.ascontiguousarray(mat_ids, np.uint32), M.ctypes.data, len(mats), Lt.ctypes.data,
                          len(lights), cam, width, height, spp, max_depth, epsilon, seed,
                          np.asarray(sky, np.float32), nthreads or os.cpu_count() or 1, out.reshape(-1))
        return out

    def shirley(self, pos, idx, tri, o, d, tmax=np.finfo(np.float32).max):
        t, b, g = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        ok = self.L.orc_shirley(pos, idx, int(tri), np.ascontiguousarray(o[:3], np.float32),
                                np.ascontiguousarray(d[:3], np.float32), float(tmax),
                                ctypes.byref(t), ctypes.byref(b), ctypes.byref(g))
        return bool(ok), t.value, b.value, g.value

    def intersect_brute(self, pos, idx, o4, d4):
        n = o4.shape[0]
        out = (np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.float32))
        self.L.orc_intersect_brute(pos, idx.reshape(-1), idx.shape[0], o4, d4, n, *out)
        return out

    def watertight_brute(self, pos, idx, o4, d4):
        """Closest hit and any hit with the watertight test: (prim, t, u, v, occ)."""
        n = o4.shape[0]
        out = (np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.float32),
               np.empty(n, np.uint8))
        self.L.orc_watertight_brute(np.ascontiguousarray(pos, np.float32), np.ascontiguousarray(idx, np.uint32).reshape(-1),
                                    idx.shape[0], np.ascontiguousarray(o4, np.float32),
                                    np.ascontiguousarray(d4, np.float32), n, *out)
        return out

    def bvh(self, pos, idx):
        return OracleBVH(self, pos, idx)


class OracleBVH:
    def __init__(self, orc: Oracle, pos, idx):
        self.o = orc
        self.pos = np.ascontiguousarray(pos, np.float32)
        self.idx = np.ascontiguousarray(idx, np.uint32)
        self.h = orc.L.orc_bvh_create(self.pos.reshape(-1), self.pos.shape[0], self.idx.reshape(-1), self.idx.shape[0])

    def intersect(self, o4, d4, nthreads=None, stats=False):
        n = o4.shape[0]
        nthreads = nthreads or os.cpu_count() or 1
        out = (np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.float32))
        st = np.zeros(2, np.uint64)
        self.o.L.orc_bvh_intersect(self.h, o4, d4, n, *out, nthreads, st.ctypes.data)
        return (out, st) if stats else out

    def occluded(self, o4, d4, nthreads=None):
        n = o4.shape[0]
        occ = np.empty(n, np.uint8)
        self.o.L.orc_bvh_occluded(self.h, o4, d4, n, occ, nthreads or os.cpu_count() or 1)
        return occ

    def __del__(self):
        try:
            self.o.L.orc_bvh_destroy(self.h)
        except Exception:
            pass


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class RefLib:
    """The reference's BasicSpace -> KDTreeMesh / BVHMesh path (compiled)."""

    def __init__(self):
        if not ref_available():
            raise FileNotFoundError(REF_SO)
        L = ctypes.CDLL(REF_SO)
        L.ilref_mesh_create.argtypes = [ctypes.c_int, _f32p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.ilref_mesh_create.restype = ctypes.c_void_p
        L.ilref_mesh_destroy.argtypes = [ctypes.c_void_p]
        L.ilref_mesh_build_seconds.argtypes = [ctypes.c_void_p]
        L.ilref_mesh_build_seconds.restype = ctypes.c_double
        L.ilref_intersect.argtypes = [ctypes.c_void_p, _f32p, _f32p, ctypes.c_long, _i32p, _f32p, _f32p, _f32p,
                                      ctypes.c_int]
        L.ilref_occluded.argtypes = [ctypes.c_void_p, _f32p, _f32p, ctypes.c_long, _u8p, ctypes.c_int]
        L.ilref_render_box.argtypes = [_f32p, _i32p, ctypes.c_int, ctypes.c_int, _f32p, ctypes.c_int, _f32p, _f32p,
                                       _f32p, _f32p, _f32p, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint32,
                                       ctypes.c_int, _f32p]
        c = ctypes
        L.ilref_render_box_plugin.argtypes = [c.c_char_p, c.c_char_p] + list(L.ilref_render_box.argtypes) + [
            c.c_char_p, c.c_int]
        L.ilref_render_box_aov.argtypes = list(L.ilref_render_box.argtypes) + [_f32p, _f32p]
        L.ilref_render_box_renderer.argtypes = ([c.c_char_p, c.c_char_p] + list(L.ilref_render_box.argtypes[:17])
                                                + [c.c_float, c.c_int, _f32p, _f32p, _f32p, c.c_void_p, c.c_void_p,
                                                   c.c_char_p, c.c_int])
        L.ilref_render_box_materials.argtypes = (list(L.ilref_render_box.argtypes[:8]) + [c.c_void_p, c.c_void_p]
                                                 + list(L.ilref_render_box.argtypes[8:]))
        L.ilref_render_box_lights.argtypes = (list(L.ilref_render_box.argtypes[:8]) + [c.c_void_p, c.c_void_p, c.c_int,
                                                                                      c.c_void_p]
                                              + list(L.ilref_render_box.argtypes[8:]) + [_f32p, _f32p])
        L.ilref_render_box_engine.argtypes = ([c.c_char_p] * 5 + list(L.ilref_render_box.argtypes[:8])
                                              + [c.c_void_p, c.c_void_p, c.c_int, c.c_void_p]
                                              + list(L.ilref_render_box.argtypes[8:17])
                                              + [c.c_float, c.c_int, _f32p, _f32p, _f32p, c.c_char_p, c.c_int])
        L.ilref_postprocess.argtypes = [c.c_int, _f32p, c.c_int, c.c_int, c.c_int, _f32p]
        L.ilref_render_script.argtypes = [c.c_char_p, c.c_char_p, c.c_int, c.c_int, c.c_int, _f32p, _f32p, _f32p,
                                          c.c_char_p, c.c_int, c.c_char_p, c.c_int]
        L.ilref_compare_spaces.argtypes = [c.c_char_p, c.c_char_p, _f32p, _i32p, c.c_int, c.c_int, _f32p, c.c_int,
                                           _f32p, _f32p, _f32p, _f32p, c.c_long, c.c_void_p, _u8p, _f32p,
                                           c.c_void_p, _u8p, _u8p, _f32p, _u8p, c.c_char_p, c.c_int]
        self.L = L

    @staticmethod
    def _material_args(scene):
        """(kinds, spec) pointers of a scene with per-primitive material kinds
        (scenes.box_scene(specular=True)) and the arrays that back them, or
        (None, None, ())."""
        if "kinds" not in scene:
            return None, None, ()
        kinds = np.ascontiguousarray(scene["kinds"], np.int32)
        spec = np.ascontiguousarray(scene["spec"], np.float32)
        return kinds.ctypes.data, spec.ctypes.data, (kinds, spec)

    def render_box(self, scene: dict, width: int, height: int, spp: int, seed: int = 1, nthreads=None):
        """The reference's PathIntegrator on the box scene; returns (H, W, 3) float32."""
        f = lambda a: np.ascontiguousarray(a, np.float32)
        cam = scene["camera"]
        out = np.zeros((height, width, 3), np.float32)
        if "kinds" in scene:
            kp, sp, keep = self._material_args(scene)
            self.L.ilref_render_box_materials(*self._scene_args(scene), kp, sp, f(cam["eye"]), f(cam["target"]),
                                              f(cam["up"]), float(cam["fov"]), float(cam["aspect"]), width, height,
                                              spp, int(scene["max_depth"]), float(scene["epsilon"]), seed,
                                              nthreads or os.cpu_count() or 1, out.reshape(-1))
            return out
        self.L.ilref_render_box(f(scene["pos"]).reshape(-1), np.ascontiguousarray(scene["prim_of_tri"], np.int32),
                                scene["pos"].shape[0] // 3, scene["albedo"].shape[0], f(scene["albedo"]).reshape(-1),
                                int(scene["light_prim"]), f(scene["light_quad"]).reshape(-1), f(scene["light_emit"]),
                                f(cam["eye"]), f(cam["target"]), f(cam["up"]), float(cam["fov"]),
                                float(cam["aspect"]), width, height, spp, int(scene["max_depth"]),
                                float(scene["epsilon"]), seed, nthreads or os.cpu_count() or 1, out.reshape(-1))
        return out

    @staticmethod
    def _scene_args(scene):
        f = lambda a: np.ascontiguousarray(a, np.float32)
        return (f(scene["pos"]).reshape(-1), np.ascontiguousarray(scene["prim_of_tri"], np.int32),
                scene["pos"].shape[0] // 3, scene["albedo"].shape[0], f(scene["albedo"]).reshape(-1),
                int(scene["light_prim"]), f(scene["light_quad"]).reshape(-1), f(scene["light_emit"]))

    def render_box_plugin(self, plugin: str, scene: dict, width: int, height: int, spp: int, seed: int = 1,
                          nthreads: int = 1, factory: str = "GPU"):
        """The reference's PathIntegrator on the box scene over the space that
        plug-in library `plugin` registers under `factory`. Raises RuntimeError
        with the loader's message on failure."""
        f = lambda a: np.ascontiguousarray(a, np.float32)
        cam = scene["camera"]
        out = np.zeros((height, width, 3), np.float32)
        err = ctypes.create_string_buffer(512)
        rc = self.L.ilref_render_box_plugin(plugin.encode(), factory.encode(), *self._scene_args(scene),
                                            f(cam["eye"]), f(cam["target"]), f(cam["up"]), float(cam["fov"]),
                                            float(cam["aspect"]), width, height, spp, int(scene["max_depth"]),
                                            float(scene["epsilon"]), seed, nthreads, out.reshape(-1), err, 512)
        if rc:
            raise RuntimeError(f"ilref_render_box_plugin: {rc}: {err.value.decode(errors='replace')}")
        return out

    @staticmethod
    def _light_args(scene):
        """(light_kind, inf pointer, backing arrays) of a box scene's lights."""
        inf = scene.get("inf")
        if inf is None:
            return int(scene.get("light_kind", 0)), None, ()
        inf = np.ascontiguousarray(inf, np.float32)
        return int(scene.get("light_kind", 0)), inf.ctypes.data, (inf,)

    def render_box_lights(self, scene: dict, width: int, height: int, spp: int, seed: int = 1, nthreads=None):
        """The reference's PathIntegrator on a box scene with any of its light
        choices (mesh light, infinite light) and materials: (final, direct, albedo)."""
        f = lambda a: np.ascontiguousarray(a, np.float32)
        cam = scene["camera"]
        outs = [np.zeros((height, width, 3), np.float32) for _ in range(3)]
        kp, sp, keep = self._material_args(scene)
        kind, ip, keep2 = self._light_args(scene)
        self.L.ilref_render_box_lights(*self._scene_args(scene), kp, sp, kind, ip, f(cam["eye"]), f(cam["target"]),
                                       f(cam["up"]), float(cam["fov"]), float(cam["aspect"]), width, height, spp,
                                       int(scene["max_depth"]), float(scene["epsilon"]), seed,
                                       nthreads or os.cpu_count() or 1, *(o.reshape(-1) for o in outs))
        return tuple(outs)

    def render_box_engine(self, plugin: str, scene: dict, width: int, height: int, spp: int, tile: int = 0,
                          space: str = "GPU", renderer: str = "GPU", integrator: str = "",
                          integrator_args: dict | None = None):
        """The box scene driven by the engine's objects over the plug-in's
        space, with the renderer made by factory `renderer` ("" = the
        reference's BasicRenderer) and the integrator made by factory
        `integrator` ("" = the reference's PathIntegrator) with
        `integrator_args`. Returns (final, direct, albedo) from the
        RadianceBuffer; raises RuntimeError with the engine's message."""
        f = lambda a: np.ascontiguousarray(a, np.float32)
        cam = scene["camera"]
        outs = [np.zeros((height, width, 3), np.float32) for _ in range(3)]
        err = ctypes.create_string_buffer(1024)
        kp, sp, keep = self._material_args(scene)
        kind, ip, keep2 = self._light_args(scene)
        extra = ";".join(f"{k}={v}" for k, v in (integrator_args or {}).items())
        rc = self.L.ilref_render_box_engine(plugin.encode(), space.encode(), renderer.encode(), integrator.encode(),
                                            extra.encode(), *self._scene_args(scene), kp, sp, kind, ip,
                                            f(cam["eye"]), f(cam["target"]), f(cam["up"]), float(cam["fov"]),
                                            float(cam["aspect"]), width, height, spp, int(scene["max_depth"]),
                                            float(scene["epsilon"]), tile, *(o.reshape(-1) for o in outs), err,
                                            1024)
        if rc:
            raise RuntimeError(f"ilref_render_box_engine: {rc}: {err.value.decode(errors='replace')}")
        return tuple(outs)

    def render_box_aov(self, scene: dict, width: int, height: int, spp: int, seed: int = 1, nthreads=None):
        """render_box plus the RadianceContext Direct and Albedo: (final, direct, albedo)."""
        f = lambda a: np.ascontiguousarray(a, np.float32)
        cam = scene["camera"]
        outs = [np.zeros((height, width, 3), np.float32) for _ in range(3)]
        self.L.ilref_render_box_aov(*self._scene_args(scene), f(cam["eye"]), f(cam["target"]), f(cam["up"]),
                                    float(cam["fov"]), float(cam["aspect"]), width, height, spp,
                                    int(scene["max_depth"]), float(scene["epsilon"]), seed,
                                    nthreads or os.cpu_count() or 1, *(o.reshape(-1) for o in outs))
        return tuple(outs)

    def render_box_renderer(self, plugin: str, scene: dict, width: int, height: int, spp: int, tile: int = 0,
                            factory: str = "GPU"):
        """The box scene through the plug-in's renderer over its space, driven by
        the engine's objects; tile > 0 renders tile x tile RenderRegion calls.
        Returns (final, direct, albedo) from the RadianceBuffer."""
        f = lambda a: np.ascontiguousarray(a, np.float32)
        cam = scene["camera"]
        outs = [np.zeros((height, width, 3), np.float32) for _ in range(3)]
        err = ctypes.create_string_buffer(512)
        kp, sp, keep = self._material_args(scene)
        rc = self.L.ilref_render_box_renderer(plugin.encode(), factory.encode(), *self._scene_args(scene),
                                              f(cam["eye"]), f(cam["target"]), f(cam["up"]), float(cam["fov"]),
                                              float(cam["aspect"]), width, height, spp, int(scene["max_depth"]),
                                              float(scene["epsilon"]), tile, *(o.reshape(-1) for o in outs),
                                              kp, sp, err, 512)
        if rc:
            raise RuntimeError(f"ilref_render_box_renderer: {rc}: {err.value.decode(errors='replace')}")
        return tuple(outs)

    def render_script(self, script: str, width: int, height: int, plugin: str | None = None, tile: int = 0):
        """A scene script loaded by the reference's Environment::Load and
        rendered by the renderer it names (see ilref_render_script); with
        `plugin`, the plug-in's factories are registered first. Returns
        (final, direct, albedo, info); raises RuntimeError with the loader's
        or renderer's reason."""
        outs = [np.zeros((height, width, 3), np.float32) for _ in range(3)]
        info = ctypes.create_string_buffer(256)
        err = ctypes.create_string_buffer(1024)
        rc = self.L.ilref_render_script((plugin or "").encode(), str(script).encode(), width, height, tile,
                                        *(o.reshape(-1) for o in outs), info, 256, err, 1024)
        if rc:
            raise RuntimeError(f"ilref_render_script: {rc}: {err.value.decode(errors='replace')}")
        return (*outs, info.value.decode())

    def postprocess(self, op: str, frames):
        """The reference's post-process on float32 images: op 'accumulate'
        (frames: (F, H, W, 3), returns the F-th accumulated output), 'global',
        'auto' or 'drago' (frames: (H, W, 3))."""
        codes = {"accumulate": 0, "global": 1, "auto": 2, "drago": 3}
        f = np.ascontiguousarray(frames, np.float32)
        if op != "accumulate":
            f = f[None]
        n, h, w = f.shape[0], f.shape[1], f.shape[2]
        out = np.zeros((h, w, 3), np.float32)
        self.L.ilref_postprocess(codes[op], f.reshape(-1), n, w, h, out.reshape(-1))
        return out

    def compare_spaces(self, plugin: str, scene: dict, o4, d4, exclude=None, factory: str = "GPU"):
        """BasicSpace vs the plug-in's space on the same primitives, ray by ray
        (see ilref_compare_spaces). Returns a dict of arrays."""
        o4 = np.ascontiguousarray(o4, np.float32)
        d4 = np.ascontiguousarray(d4, np.float32)
        n = o4.shape[0]
        hit, occ, xhit, xocc = (np.zeros((n, 2), np.uint8) for _ in range(4))
        t, xt = np.zeros((n, 2), np.float32), np.zeros((n, 2), np.float32)
        diff = np.zeros(n, np.uint32)
        ex = None if exclude is None else np.ascontiguousarray(exclude, np.int32)
        err = ctypes.create_string_buffer(512)
        rc = self.L.ilref_compare_spaces(plugin.encode(), factory.encode(), *self._scene_args(scene),
                                         o4.reshape(-1), d4.reshape(-1), n, None if ex is None else ex.ctypes.data,
                                         hit.reshape(-1), t.reshape(-1), diff.ctypes.data, occ.reshape(-1),
                                         xhit.reshape(-1), xt.reshape(-1), xocc.reshape(-1), err, 512)
        if rc:
            raise RuntimeError(f"ilref_compare_spaces: {rc}: {err.value.decode(errors='replace')}")
        return dict(hit=hit, t=t, diff=diff, occ=occ, xhit=xhit, xt=xt, xocc=xocc)

    def mesh(self, pos, idx, kind: str = "bvh"):
        return RefMesh(self, pos, idx, 0 if kind == "kd" else 1)


class RefMesh:
    def __init__(self, lib: RefLib, pos, idx, kind: int):
        self.lib = lib
        pos = np.ascontiguousarray(pos, np.float32)
        idx32 = np.ascontiguousarray(idx, np.int32)
        self.h = lib.L.ilref_mesh_create(kind, pos.reshape(-1), pos.shape[0], idx32.ctypes.data, idx32.shape[0])
        self.build_seconds = lib.L.ilref_mesh_build_seconds(self.h)

    def intersect(self, o4, d4, nthreads=None):
        n = o4.shape[0]
        out = (np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.float32))
        self.lib.L.ilref_intersect(self.h, o4, d4, n, *out, nthreads or os.cpu_count() or 1)
        return out

    def occluded(self, o4, d4, nthreads=None):
        n = o4.shape[0]
        occ = np.empty(n, np.uint8)
        self.lib.L.ilref_occluded(self.h, o4, d4, n, occ, nthreads or os.cpu_count() or 1)
        return occ

    def __del__(self):
        try:
            self.lib.L.ilref_mesh_destroy(self.h)
        except Exception:
            pass
