"""Seeded procedural workloads for the intersection and path-tracing paths.

Nothing here is a reference dataset: the reference ships no scenes, so every
workload is generated from a seed with the shapes and sizes it is quoted on.

* ``heightfield`` - a W x H grid of cells over [0,1]^2, two triangles per cell,
  height = amplitude * value-noise fBm. The noise is defined here: a PCG
  lattice hash of (ix, iy, octave, seed) mapped to [0,1), smoothstep
  interpolation, base frequency 8, lacunarity 2, gain 0.5, normalised to [0,1).
* ``coherent_rays`` - one pinhole ray per pixel centre.
* ``incoherent_rays`` - origins uniform on random triangles (uniform triangle
  index, point by the reference's UniformSampleTriangle warp,
  Core/Maths/Montecarlo.h:59-64), lifted 1e-4 along the +z-facing geometric
  normal, directions cosine-distributed about that normal
  (Montecarlo.h:31-37 in the frame of Core/Geometry/Basis.cpp:85-99).

Rays are two float32 (N, 4) arrays: (ox, oy, oz, tmin) and (dx, dy, dz, tmax).
"""
from __future__ import annotations

import numpy as np

FLT_MAX = np.float32(np.finfo(np.float32).max)

_M32 = np.uint64(0xFFFFFFFF)


def _pcg_hash(x: np.ndarray) -> np.ndarray:
    """32-bit PCG output permutation of a linear step (Jarzynski & Olano 2020)."""
    x = x.astype(np.uint64) & _M32
    state = (x * np.uint64(747796405) + np.uint64(2891336453)) & _M32
    shift = (state >> np.uint64(28)) + np.uint64(4)
    word = (((state >> shift) ^ state) * np.uint64(277803737)) & _M32
    return ((word >> np.uint64(22)) ^ word) & _M32


def _lattice(ix, iy, octave: int, seed: int) -> np.ndarray:
    h = _pcg_hash(np.full(np.shape(ix), seed, dtype=np.uint64))
    h = _pcg_hash(h + np.uint64(octave))
    h = _pcg_hash(h + (np.asarray(iy).astype(np.int64).astype(np.uint64) & _M32))
    h = _pcg_hash(h + (np.asarray(ix).astype(np.int64).astype(np.uint64) & _M32))
    return h.astype(np.float64) * (1.0 / 4294967296.0)


def value_noise_fbm(x, y, seed: int = 1, octaves: int = 6, base_freq: float = 8.0,
                    lacunarity: float = 2.0, gain: float = 0.5) -> np.ndarray:
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    total = np.zeros(np.broadcast(x, y).shape)
    norm = 0.0
    freq, amp = base_freq, 1.0
    for o in range(octaves):
        X, Y = x * freq, y * freq
        ix, iy = np.floor(X), np.floor(Y)
        fx, fy = X - ix, Y - iy
        sx, sy = fx * fx * (3 - 2 * fx), fy * fy * (3 - 2 * fy)
        v00 = _lattice(ix, iy, o, seed)
        v10 = _lattice(ix + 1, iy, o, seed)
        v01 = _lattice(ix, iy + 1, o, seed)
        v11 = _lattice(ix + 1, iy + 1, o, seed)
        a = v00 + (v10 - v00) * sx
        b = v01 + (v11 - v01) * sx
        total += amp * (a + (b - a) * sy)
        norm += amp
        freq *= lacunarity
        amp *= gain
    return total / norm


def heightfield(nx: int = 1024, ny: int = 512, amplitude: float = 0.2, seed: int = 1):
    """Return (positions float32 (V,3), indices uint32 (T,3)) with T = 2*nx*ny."""
    gx = np.arange(nx + 1, dtype=np.float64) / nx
    gy = np.arange(ny + 1, dtype=np.float64) / ny
    X, Y = np.meshgrid(gx, gy)                      # (ny+1, nx+1)
    Z = amplitude * value_noise_fbm(X, Y, seed=seed)
    pos = np.stack([X, Y, Z], axis=-1).reshape(-1, 3).astype(np.float32)
    i = np.arange(nx)[None, :]
    j = np.arange(ny)[:, None]
    a = j * (nx + 1) + i
    b = a + 1
    c = a + (nx + 1) + 1
    d = a + (nx + 1)
    t0 = np.stack([a, b, c], axis=-1)
    t1 = np.stack([a, c, d], axis=-1)
    idx = np.stack([t0, t1], axis=2).reshape(-1, 3).astype(np.uint32)
    return pos, idx


def _normalize(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def pinhole_rays(width: int, height: int, eye, look_at, up, vfov_deg: float):
    """One ray per pixel centre, row-major, rows top to bottom."""
    eye = np.asarray(eye, np.float64)
    fwd = _normalize(np.asarray(look_at, np.float64) - eye)
    right = _normalize(np.cross(fwd, np.asarray(up, np.float64)))
    upv = np.cross(right, fwd)
    th = np.tan(np.radians(vfov_deg) * 0.5)
    aspect = width / height
    px = (np.arange(width) + 0.5) / width * 2 - 1
    py = 1 - (np.arange(height) + 0.5) / height * 2
    PX, PY = np.meshgrid(px * th * aspect, py * th)
    d = fwd[None, None, :] + PX[..., None] * right + PY[..., None] * upv
    d = _normalize(d).reshape(-1, 3)
    n = d.shape[0]
    o4 = np.empty((n, 4), np.float32)
    d4 = np.empty((n, 4), np.float32)
    o4[:, :3] = eye
    o4[:, 3] = 0.0
    d4[:, :3] = d
    d4[:, 3] = FLT_MAX
    return o4, d4


def coherent_rays(side: int = 2048):
    return pinhole_rays(side, side, (0.5, -0.6, 0.8), (0.5, 0.5, 0.0), (0, 0, 1), 60.0)


def onb_from_w(w):
    """Frame of Core/Geometry/Basis.cpp:85-99 (InitFromW), vectorised."""
    w = _normalize(w)
    use_x = np.abs(w[:, 0]) > np.abs(w[:, 1])
    v = np.empty_like(w)
    inv_a = 1.0 / np.sqrt(w[:, 0] ** 2 + w[:, 2] ** 2)
    inv_b = 1.0 / np.sqrt(w[:, 1] ** 2 + w[:, 2] ** 2)
    v[:, 0] = np.where(use_x, -w[:, 2] * inv_a, 0.0)
    v[:, 1] = np.where(use_x, 0.0, w[:, 2] * inv_b)
    v[:, 2] = np.where(use_x, w[:, 0] * inv_a, -w[:, 1] * inv_b)
    u = np.cross(w, v)
    return u, v, w


def incoherent_rays(pos, idx, n: int = 4194304, seed: int = 2, offset: float = 1e-4):
    rng = np.random.Generator(np.random.PCG64(seed))
    tri = rng.integers(0, idx.shape[0], size=n)
    u1, u2, u3, u4 = (rng.random(n) for _ in range(4))
    p0 = pos[idx[tri, 0]].astype(np.float64)
    p1 = pos[idx[tri, 1]].astype(np.float64)
    p2 = pos[idx[tri, 2]].astype(np.float64)
    su = np.sqrt(u1)
    b0 = 1.0 - su
    b1 = u2 * su
    p = b0[:, None] * p0 + b1[:, None] * p1 + (1.0 - b0 - b1)[:, None] * p2
    nrm = _normalize(np.cross(p1 - p0, p2 - p0))
    nrm = np.where(nrm[:, 2:3] < 0, -nrm, nrm)
    U, V, W = onb_from_w(nrm)
    a = 2 * np.pi * u4
    r = np.sqrt(u3)
    lx, ly, lz = r * np.cos(a), r * np.sin(a), np.sqrt(np.maximum(0.0, 1 - u3))
    d = _normalize(lx[:, None] * U + ly[:, None] * V + lz[:, None] * W)
    o4 = np.empty((n, 4), np.float32)
    d4 = np.empty((n, 4), np.float32)
    o4[:, :3] = p + offset * nrm
    o4[:, 3] = 0.0
    d4[:, :3] = d
    d4[:, 3] = FLT_MAX
    return o4, d4


def ray_batch_workload(nx=1024, ny=512, side=2048, n_incoherent=4194304, seed=1):
    """The 1,048,576-triangle heightfield with coherent + incoherent ray sets."""
    pos, idx = heightfield(nx, ny, 0.2, seed)
    co, cd = coherent_rays(side)
    io, idr = incoherent_rays(pos, idx, n_incoherent, seed + 1)
    return pos, idx, (co, cd), (io, idr)


# ---------------------------------------------------------------------------
# Procedural box scene (the reference's CPU-runnable path-tracing case)
# ---------------------------------------------------------------------------
GREY = (0.73, 0.73, 0.73)
RED = (0.63, 0.065, 0.05)
GREEN = (0.14, 0.45, 0.09)


def _rot_y(deg):
    a = np.radians(deg)
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])


def _box_tris(center, half, rot_deg):
    """12 triangles of an axis-aligned box rotated about y, normals outward
    (n = (v1 - v0) x (v2 - v0), the reference's edge convention)."""
    hx, hy, hz = half
    c = np.array([[-hx, -hy, -hz], [hx, -hy, -hz], [hx, hy, -hz], [-hx, hy, -hz],
                  [-hx, -hy, hz], [hx, -hy, hz], [hx, hy, hz], [-hx, hy, hz]], np.float64)
    faces = [(1, 0, 3, 2), (4, 5, 6, 7), (0, 4, 7, 3), (5, 1, 2, 6), (3, 7, 6, 2), (0, 1, 5, 4)]
    R = _rot_y(rot_deg)
    p = c @ R.T + np.asarray(center)
    tris = []
    for a, b, cc, d in faces:
        tris.append((p[a], p[b], p[cc]))
        tris.append((p[a], p[cc], p[d]))
    return tris


def _quad_tris(v0, v1, v2, v3):
    return [(v0, v1, v2), (v0, v2, v3)]


def _fan_light_tris(yl: float):
    """A flat 6-triangle fan under the ceiling, emitting downward (every
    triangle's (v1 - v0) x (v2 - v0) points to -y), with triangles of unequal
    area, so the reference's index-uniform choice of a triangle to sample
    (ITriangleMesh::SamplePoint) is not the area-uniform one."""
    c = np.array((0.02, yl, -0.01))
    ang = np.radians([0.0, 50.0, 110.0, 170.0, 235.0, 300.0])
    rad = [0.28, 0.22, 0.30, 0.20, 0.26, 0.24]
    pts = [c + np.array((r * np.cos(a), 0.0, r * np.sin(a))) for r, a in zip(rad, ang)]
    tris = []
    for k in range(6):
        a, b = pts[k], pts[(k + 1) % 6]
        if np.cross(a - c, b - c)[1] > 0:
            a, b = b, a
        tris.append((c, a, b))
    return tris


def box_scene(specular: bool = False, light: str = "quad", infinite=None, fov: float = 40.0):
    """Closed box [-1,1]^3 with the front (z = +1) open, walls two triangles
    each (normals inward), left wall red, right green, others grey; two inner
    boxes rotated +-17 deg about y; a 0.5 x 0.4 ceiling quad light with
    radiance (17, 12, 4) facing -y; pinhole camera at z = 3.5, 40 deg.

    With specular=True the short box is a mirror (MirrorMaterial, reflectivity
    0.9) and the tall one glass (GlassMaterial, reflectivity 0.45,
    transmittance 0.45, eta 1 / 1.52): "kinds" (0 matte, 2 mirror, 3 glass)
    and "spec" (per primitive: transmittance rgb, eta_i, eta_t) are added.

    With light="mesh" the ceiling light is a 6-triangle mesh of unequal
    triangles (a DiffuseAreaLight on a triangle mesh, "light_kind" 1) with the
    same radiance; with infinite = (r, g, b) an InfiniteAreaLight of that
    intensity (no texture) joins the lights ("inf"). fov: the camera's field
    of view (at 60 deg the border pixels see past the box, where an infinite
    light is seen directly).

    Returns a dict with flattened world-space triangles (unshared vertices),
    a per-triangle primitive index, per-primitive albedo, the light quad in
    the reference's Quad vertex order, and the camera.
    """
    prims = []  # (triangles, albedo)
    L, H = -1.0, 1.0
    walls = [
        ("floor", _quad_tris((L, L, L), (L, L, H), (H, L, H), (H, L, L)), GREY),      # +y
        ("ceiling", _quad_tris((L, H, L), (H, H, L), (H, H, H), (L, H, H)), GREY),    # -y
        ("back", _quad_tris((L, L, L), (H, L, L), (H, H, L), (L, H, L)), GREY),       # +z
        ("left", _quad_tris((L, L, L), (L, H, L), (L, H, H), (L, L, H)), RED),        # +x
        ("right", _quad_tris((H, L, L), (H, L, H), (H, H, H), (H, H, L)), GREEN),     # -x
    ]
    for _, tris, alb in walls:
        prims.append((tris, alb))
    prims.append((_box_tris((0.35, -0.7, 0.35), (0.3, 0.3, 0.3), -17.0), GREY))
    prims.append((_box_tris((-0.35, -0.4, -0.3), (0.3, 0.6, 0.3), 17.0), GREY))
    # light quad, reference Quad vertex order: its triangles are (v1, v3, v2)
    # and (v1, v4, v3) (Core/Shape/Quad.cpp), normal (v3-v1) x (v2-v1) = -y
    yl = 0.999
    q = np.array([(-0.25, yl, -0.2), (-0.25, yl, 0.2), (0.25, yl, 0.2), (0.25, yl, -0.2)], np.float64)
    # the mesh light hangs 0.2 below the ceiling: the reference samples mesh
    # lights from both sides (the normal turned toward the shaded point), so
    # ceiling points right above a light flush with it would see it at ~0
    # distance (fireflies); at 0.2 the ceiling gets a smooth glow instead
    light_tris = [(q[0], q[2], q[1]), (q[0], q[3], q[2])] if light == "quad" else _fan_light_tris(0.8)
    prims.append((light_tris, GREY))
    pos, prim_of_tri = [], []
    for pi, (tris, _) in enumerate(prims):
        for t in tris:
            pos.extend(t)
            prim_of_tri.append(pi)
    pos = np.asarray(pos, np.float32).reshape(-1, 3)
    n_tris = pos.shape[0] // 3
    out = {
        "pos": pos,
        "idx": np.arange(3 * n_tris, dtype=np.uint32).reshape(-1, 3),
        "prim_of_tri": np.asarray(prim_of_tri, np.uint32),
        "albedo": np.asarray([p[1] for p in prims], np.float32),
        "light_prim": len(prims) - 1,
        "light_quad": q.astype(np.float32),
        "light_emit": np.array([17.0, 12.0, 4.0], np.float32),
        "camera": {"eye": (0.0, 0.0, 3.5), "target": (0.0, 0.0, 0.0), "up": (0.0, 1.0, 0.0),
                   "fov": float(fov), "aspect": 1.0},
        "max_depth": 6, "epsilon": 1e-4,
        "light_kind": 0 if light == "quad" else 1,
    }
    if infinite is not None:
        out["inf"] = np.asarray(infinite, np.float32)
    if specular:
        n = len(prims)
        kinds = np.zeros(n, np.int32)
        spec = np.zeros((n, 5), np.float32)
        spec[:, 3], spec[:, 4] = 1.0, 1.52
        albedo = out["albedo"]
        kinds[5], albedo[5] = 2, (0.9, 0.9, 0.9)                        # short box: mirror
        kinds[6], albedo[6], spec[6, :3] = 3, (0.45, 0.45, 0.45), 0.45  # tall box: glass
        out["kinds"], out["spec"] = kinds, spec
    return out


def box_materials(scene):
    """One material dict per primitive of a box scene (GpuSpace.set_materials
    form): matte by default; with the scene's "kinds", mirror (reflectivity =
    albedo) and glass (transmittance and eta_i / eta_t from "spec")."""
    kinds = scene.get("kinds")
    spec = scene.get("spec")
    mats = []
    for p, a in enumerate(scene["albedo"]):
        k = 0 if kinds is None else int(kinds[p])
        m = {"albedo": tuple(float(x) for x in a), "kind": k}
        if k == 3:
            m["f0"] = tuple(float(x) for x in spec[p, :3])
            m["alpha"] = float(spec[p, 3] / spec[p, 4])
        mats.append(m)
    return mats


def load_box_scene(space, scene=None):
    """Upload the box scene to a GpuSpace: mesh with per-triangle material
    ids (one material per primitive, as MatteMaterial per primitive), the
    light quad, then build."""
    scene = scene or box_scene()
    space.initialise(scene["pos"], scene["idx"], scene["prim_of_tri"])
    space.build()
    space.set_materials(box_materials(scene))
    space.set_lights(box_lights(scene))
    return scene


def box_lights(scene):
    """The box scene's lights (GpuSpace.set_lights form), in the order of the
    reference scene's LightList: the area light, then the infinite light."""
    sel = np.nonzero(scene["prim_of_tri"] == scene["light_prim"])[0]
    first = int(sel[0])
    if scene.get("light_kind", 0) == 1:
        lights = [{"kind": "mesh", "emit": scene["light_emit"], "first_tri": first, "tri_count": int(sel.size)}]
    else:
        lights = [{"kind": "quad", "v": scene["light_quad"], "emit": scene["light_emit"], "first_tri": first}]
    if "inf" in scene:
        lights.append({"kind": "infinite", "emit": scene["inf"]})
    return lights


def _g(x) -> str:
    """A float32 in the shortest text that reads back to the same value."""
    return np.format_float_positional(np.float32(x), trim="-")


def write_box_script(directory, scene=None, width: int = 64, height: int = 64, spp: int = 16,
                     space: str = "GPU", renderer: str = "GPU", seed: int = 1, container: str = "BVHMesh",
                     integrator: str = "PathTracing", integrator_args: dict | None = None) -> str:
    """Write the box scene as files the reference's own scene loader reads and
    return the script's path: ``box.obj`` + ``box.mtl`` (every non-light
    triangle, one MTL material per primitive with Kd = its albedo, a flat
    per-face normal), and ``box.ilm``, an environment script
    (Core/Scene/EnvironmentLoader.cpp:150-921 syntax: ``Name = value`` lines
    and ``Name {`` ... ``}`` blocks) that loads the OBJ as a WavefrontModel
    into one mesh with a MaterialGroup, adds the light as a Quad shape with a
    DiffuseArea light and an Emissive primitive, and names the space and
    renderer factories (``"GPU"`` for the plug-in's, ``"Basic"`` for the
    reference's), an integrator of type `integrator` (``"PathTracing"``, or
    the plug-in's ``"GPU"``) with the scene's depth and epsilon plus
    `integrator_args` (e.g. ``{"Cache": "MLP"}``), a Random sampler, a Box
    filter and a ``Memory`` device of width x height.

    For a scene with material kinds (box_scene(specular=True)) a mirror
    primitive's MTL material gets ``illum 5`` and Ks = its reflectivity (the
    loader's Mirror, WavefrontSceneLoader.cpp:212-232), and a glass primitive
    goes to ``glass.obj``, its own Geometry primitive with a Glass material
    declared in the script (Reflectivity = {reflectivity, transmittance},
    Absorption, Eta = {eta_i, eta_t}; MaterialFactories.h:105-135): the MTL
    route has no indices for glass."""
    import os
    scene = scene or box_scene()
    directory = os.path.abspath(str(directory))
    os.makedirs(directory, exist_ok=True)
    obj, mtl, ilm = (os.path.join(directory, n) for n in ("box.obj", "box.mtl", "box.ilm"))
    light = scene["light_prim"]
    kinds = scene.get("kinds")
    kind_of = (lambda p: 0) if kinds is None else (lambda p: int(kinds[p]))
    glass = [p for p in range(len(scene["albedo"])) if kind_of(p) == 3]
    with open(mtl, "w") as f:
        for p, a in enumerate(scene["albedo"]):
            if p == light or p in glass:
                continue
            f.write(f"newmtl prim{p}\nKd {_g(a[0])} {_g(a[1])} {_g(a[2])}\n")
            if kind_of(p) == 2:
                f.write(f"Ks {_g(a[0])} {_g(a[1])} {_g(a[2])}\nillum 5\n")
            f.write("\n")
    pos = scene["pos"].reshape(-1, 3, 3).astype(np.float32)
    if glass:
        with open(os.path.join(directory, "glass.obj"), "w") as f:
            nv = 0
            for t, p in enumerate(scene["prim_of_tri"]):
                if p not in glass:
                    continue
                v = pos[t].astype(np.float64)
                n = np.cross(v[1] - v[0], v[2] - v[0])
                n /= np.linalg.norm(n)
                for c in range(3):
                    f.write(f"v {_g(v[c, 0])} {_g(v[c, 1])} {_g(v[c, 2])}\n")
                f.write(f"vn {_g(n[0])} {_g(n[1])} {_g(n[2])}\n")
                k = nv // 3 + 1
                f.write(f"f {nv + 1}//{k} {nv + 2}//{k} {nv + 3}//{k}\n")
                nv += 3
    with open(obj, "w") as f:
        f.write("mtllib box.mtl\n")
        current, nv = None, 0
        for t, p in enumerate(scene["prim_of_tri"]):
            if p == light or p in glass:
                continue
            v = pos[t].astype(np.float64)
            n = np.cross(v[1] - v[0], v[2] - v[0])
            n /= np.linalg.norm(n)
            for c in range(3):
                f.write(f"v {_g(v[c, 0])} {_g(v[c, 1])} {_g(v[c, 2])}\n")
            f.write(f"vn {_g(n[0])} {_g(n[1])} {_g(n[2])}\n")
            if p != current:
                f.write(f"usemtl prim{p}\n")
                current = p
            k = nv // 3 + 1  # this triangle's vn
            f.write(f"f {nv + 1}//{k} {nv + 2}//{k} {nv + 3}//{k}\n")
            nv += 3
    q, e, cam = scene["light_quad"], scene["light_emit"], scene["camera"]
    alb = scene["albedo"][light]
    vec = lambda v: "{" + ",".join(_g(x) for x in v) + "}"
    extra = "".join(f"\t\t{k} = {v}\n" for k, v in (integrator_args or {}).items())
    glass_shape = glass_material = glass_prim = ""
    if glass:
        g = glass[0]
        r, t, eta = scene["albedo"][g], scene["spec"][g, :3], scene["spec"][g, 3:5]
        gobj = os.path.join(directory, "glass.obj")
        glass_shape = (f"\tShape {{\n\t\tId = glass_mesh\n\t\tType = WavefrontModel\n\t\tFilename = {gobj}\n"
                       f"\t\tContainer = {container}\n\t}}\n")
        glass_material = (f"\tMaterial {{\n\t\tId = glass_material\n\t\tType = Glass\n"
                          f"\t\tReflectivity = {{{vec(r)},{vec(t)}}}\n\t\tAbsorption = 1\n"
                          f"\t\tEta = {vec(eta)}\n\t}}\n")
        glass_prim = ("\t\t\t\tPrimitive {\n\t\t\t\t\tId = glass\n\t\t\t\t\tType = Geometry\n"
                      "\t\t\t\t\tMaterial = glass_material\n\t\t\t\t\tShape = glass_mesh\n\t\t\t\t}\n")
    script = f"""# box scene: walls, two boxes and a ceiling quad light
Shapes {{
\tShape {{
\t\tId = box_mesh
\t\tType = WavefrontModel
\t\tFilename = {obj}
\t\tContainer = {container}
\t\tMaterialGroupId = box_materials
\t}}
\tShape {{
\t\tId = light_quad
\t\tType = Quad
\t\tVertices = {{{",".join(vec(v) for v in q)}}}
\t}}
{glass_shape}}}
Materials {{
\tMaterial {{
\t\tId = light_material
\t\tType = Matte
\t\tReflectivity = {vec(alb)}
\t}}
{glass_material}}}
Lights {{
\tLight {{
\t\tId = ceiling_light
\t\tType = DiffuseArea
\t\tPower = {vec(e)}
\t\tShape = light_quad
\t}}
}}
Cameras {{
\tCamera {{
\t\tId = camera
\t\tType = Perspective
\t\tPosition = {vec(cam["eye"])}
\t\tTarget = {vec(cam["target"])}
\t\tUp = {vec(cam["up"])}
\t\tFov = {_g(cam["fov"])}
\t\tAspect = {_g(cam["aspect"])}
\t}}
}}
Filters {{
\tFilter {{
\t\tId = filter
\t\tType = Box
\t}}
}}
Samplers {{
\tSampler {{
\t\tId = sampler
\t\tType = Random
\t}}
}}
Devices {{
\tDevice {{
\t\tId = device
\t\tType = Memory
\t\tWidth = {int(width)}
\t\tHeight = {int(height)}
\t}}
}}
Integrators {{
\tIntegrator {{
\t\tId = integrator
\t\tType = {integrator}
\t\tRayDepth = {int(scene["max_depth"])}
\t\tShadowRays = 1
\t\tEpsilon = {_g(scene["epsilon"])}
{extra}\t}}
}}
Renderers {{
\tRenderer {{
\t\tId = renderer
\t\tType = {renderer}
\t\tSamples = {int(spp)}
\t\tSeed = {int(seed)}
\t\tIntegrator = integrator
\t\tFilter = filter
\t\tDevice = device
\t}}
}}
Environment {{
\tRenderer = renderer
\tScene {{
\t\tSampler = sampler
\t\tCamera = camera
\t\tLights = {{ceiling_light}}
\t\tSpace {{
\t\t\tId = space
\t\t\tType = {space}
\t\t\tPrimitives {{
\t\t\t\tPrimitive {{
\t\t\t\t\tId = box
\t\t\t\t\tType = Geometry
\t\t\t\t\tMaterial = box_materials
\t\t\t\t\tShape = box_mesh
\t\t\t\t}}
\t\t\t\tPrimitive {{
\t\t\t\t\tId = light
\t\t\t\t\tType = Emissive
\t\t\t\t\tMaterial = light_material
\t\t\t\t\tShape = light_quad
\t\t\t\t\tLight = ceiling_light
\t\t\t\t}}
{glass_prim}\t\t\t}}
\t\t}}
\t}}
}}
"""
    with open(ilm, "w") as f:
        f.write(script)
    return ilm


# ---------------------------------------------------------------------------
# Icosphere field (the at-scale path-tracing scene)
# ---------------------------------------------------------------------------
def icosphere(subdiv: int):
    """Unit icosphere: (verts float64 (V,3), faces int64 (F,3)), F = 20 * 4^subdiv,
    outward winding ((v1 - v0) x (v2 - v0) points out)."""
    t = (1.0 + 5 ** 0.5) / 2
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t],
                  [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(subdiv):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (v.shape[0] + 1) + e[:, 1]
        uk, inv = np.unique(key, return_inverse=True)
        a, b = uk // (v.shape[0] + 1), uk % (v.shape[0] + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1).T + v.shape[0]  # midpoints of edges (01, 12, 20)
        v = np.concatenate([v, mid])
        f0, f1, f2 = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([f0, m01, m20], 1), np.stack([f1, m12, m01], 1),
                            np.stack([f2, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    # make the winding outward
    p = v[f]
    n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    flip = (n * p.mean(1)).sum(1) < 0
    f[flip] = f[flip][:, [0, 2, 1]]
    return v, f


def sphere_field(n_side: int = 8, subdiv: int = 7, seed: int = 3, width: int = 1920, height: int = 1080):
    """n_side^2 icospheres on a jittered grid (radius U[0.3, 0.6], resting on a
    ground plane), 50% Lambertian (albedo U[0.1, 0.9]^3) and 50% GGX conductors
    (alpha U[0.05, 0.5], F0 U[0.5, 1]^3), four 2 x 2 quad lights at height 6
    with radiance U[10, 30], a constant sky of 0.1. Material 0 is the ground
    (Lambertian 0.5); materials 1.. belong to the spheres in order; the lights
    use material 0."""
    rng = np.random.Generator(np.random.PCG64(seed))
    uv, uf = icosphere(subdiv)
    ns = n_side * n_side
    coords = (np.arange(n_side) - (n_side - 1) / 2.0)
    gx, gz = np.meshgrid(coords, coords)
    cx = gx.reshape(-1) + rng.uniform(-0.15, 0.15, ns)
    cz = gz.reshape(-1) + rng.uniform(-0.15, 0.15, ns)
    r = rng.uniform(0.3, 0.6, ns)
    nv, nf = uv.shape[0], uf.shape[0]
    pos = np.empty((ns * nv + 4 + 16, 3), np.float32)
    idx = np.empty((ns * nf + 2 + 8, 3), np.uint32)
    mat = np.empty(ns * nf + 2 + 8, np.uint32)
    mats = [{"albedo": (0.5, 0.5, 0.5), "kind": 0}]
    is_ggx = rng.permutation(np.arange(ns) < ns // 2)  # exactly half the spheres are conductors
    for i in range(ns):
        pos[i * nv:(i + 1) * nv] = uv * r[i] + np.array([cx[i], r[i], cz[i]])
        idx[i * nf:(i + 1) * nf] = uf + i * nv
        mat[i * nf:(i + 1) * nf] = i + 1
        if not is_ggx[i]:
            mats.append({"albedo": tuple(rng.uniform(0.1, 0.9, 3)), "kind": 0})
        else:
            mats.append({"albedo": (0.0, 0.0, 0.0), "kind": 1, "f0": tuple(rng.uniform(0.5, 1.0, 3)),
                         "alpha": float(rng.uniform(0.05, 0.5))})
    base_v, base_f = ns * nv, ns * nf
    G = 50.0
    pos[base_v:base_v + 4] = [(-G, 0, -G), (-G, 0, G), (G, 0, G), (G, 0, -G)]
    idx[base_f:base_f + 2] = [(base_v, base_v + 1, base_v + 2), (base_v, base_v + 2, base_v + 3)]  # +y
    mat[base_f:base_f + 2] = 0
    lights = []
    vi, fi = base_v + 4, base_f + 2
    for k, (lx, lz) in enumerate([(-3, -3), (3, -3), (-3, 3), (3, 3)]):
        y = 6.0
        q = np.array([(lx - 1, y, lz - 1), (lx - 1, y, lz + 1), (lx + 1, y, lz + 1), (lx + 1, y, lz - 1)], np.float32)
        pos[vi:vi + 4] = q
        # reference Quad tessellation (v1, v3, v2), (v1, v4, v3): normal -y
        idx[fi:fi + 2] = [(vi, vi + 2, vi + 1), (vi, vi + 3, vi + 2)]
        mat[fi:fi + 2] = 0
        e = float(rng.uniform(10.0, 30.0))
        lights.append({"v": q, "emit": (e, e, e), "first_tri": fi})
        vi += 4
        fi += 2
    return {
        "pos": pos, "idx": idx, "mat_ids": mat, "materials": mats, "lights": lights,
        "camera": {"eye": (0.0, 3.5, 9.5), "target": (0.0, 0.3, 0.0), "up": (0.0, 1.0, 0.0), "fov": 40.0,
                   "aspect": width / height},
        "width": width, "height": height, "sky": (0.1, 0.1, 0.1), "max_depth": 12, "spp": 64,
        "epsilon": 1e-4,
    }


def matte_field(n_side: int = 8, subdiv: int = 3, seed: int = 3, width: int = 480, height: int = 270):
    """The icosphere field in the box-scene form (write_box_script,
    load_box_scene), with what the reference's own integrators can render:
    every sphere Lambertian (a conductor of sphere_field gets its F0 as
    albedo), the 100 x 100 ground (albedo 0.5), and one 4 x 4 quad light at
    height 6 over the field's centre with radiance 20 (the power of
    sphere_field's four 2 x 2 lights at their mean radiance); no sky. The
    camera looks down on the field so that every camera ray hits the ground
    (the reference's ICIntegrator answers a camera ray that escapes with a
    fixed colour, ICIntegrator.cpp:432). The scene on which the reference's
    irradiance cache and this project's learned cache are compared."""
    f = sphere_field(n_side, subdiv, seed, width, height)
    n_geo = f["idx"].shape[0] - 8  # the spheres and the ground (the four lights' triangles dropped)
    tris = f["pos"][f["idx"][:n_geo].astype(np.int64)]  # (n_geo, 3, 3)
    prim_of_tri = f["mat_ids"][:n_geo].astype(np.uint32)
    albedo = [m["albedo"] if m["kind"] == 0 else m["f0"] for m in f["materials"]]
    y, h = 6.0, 2.0
    q = np.array([(-h, y, -h), (-h, y, h), (h, y, h), (h, y, -h)], np.float32)
    light_tris = np.array([(q[0], q[2], q[1]), (q[0], q[3], q[2])], np.float32)  # normal -y
    light_prim = len(albedo)
    albedo.append((0.0, 0.0, 0.0))
    pos = np.concatenate([tris, light_tris]).reshape(-1, 3).astype(np.float32)
    n_tris = pos.shape[0] // 3
    return {
        "pos": pos,
        "idx": np.arange(3 * n_tris, dtype=np.uint32).reshape(-1, 3),
        "prim_of_tri": np.concatenate([prim_of_tri, np.full(2, light_prim, np.uint32)]),
        "albedo": np.asarray(albedo, np.float32),
        "light_prim": light_prim,
        "light_quad": q,
        "light_emit": np.array([20.0, 20.0, 20.0], np.float32),
        "camera": {"eye": (0.0, 4.5, 8.0), "target": (0.0, 0.0, 0.0), "up": (0.0, 1.0, 0.0), "fov": 40.0,
                   "aspect": width / height},
        "max_depth": 12, "epsilon": 1e-4, "light_kind": 0,
    }


def load_sphere_field(space, scene):
    space.initialise(scene["pos"], scene["idx"], scene["mat_ids"])
    space.build()
    space.set_materials(scene["materials"])
    space.set_quad_lights(scene["lights"])
    return scene


def batch_workload(n_scenes: int = 32, seed: int = 9, tri_range=(10_000, 2_000_000), side_range=(256, 1024)):
    """Independent icosphere-field scenes with uneven sizes: triangle counts
    log-uniform in tri_range (grid side and subdivision picked to match),
    square images with side log-uniform in side_range, spp from
    {4, 8, 16, 32, 64}, max depth uniform in [4, 16]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    items = []
    for i in range(n_scenes):
        target = float(np.exp(rng.uniform(np.log(tri_range[0]), np.log(tri_range[1]))))
        best = None
        for s in range(2, 8):
            for n_side in range(1, 9):
                t = n_side * n_side * 20 * 4 ** s
                err = abs(np.log(t / target))
                if best is None or err < best[0]:
                    best = (err, n_side, s)
        _, n_side, subdiv = best
        side = int(round(np.exp(rng.uniform(np.log(side_range[0]), np.log(side_range[1])))))
        scene = sphere_field(n_side, subdiv, seed=1000 + i, width=side, height=side)
        scene["spp"] = int(rng.choice([4, 8, 16, 32, 64]))
        scene["max_depth"] = int(rng.integers(4, 17))
        scene["target_tris"] = int(target)
        items.append(scene)
    return items
