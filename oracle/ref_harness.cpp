// Test-infrastructure harness around the reference's own compiled sources.
//
// This file is ours; everything it calls is the reference's code, compiled
// unmodified from the reference tree by oracle/Makefile (with the two
// replacement headers under illuminaprt_b200/plugin/compat). It exposes a small C ABI so the
// tests and the CPU baseline of bench.py can drive the reference path:
//
//   closest hit  BasicSpace::Intersects(ray, isect)      Core/Space/BasicSpace.cpp:58-73
//                -> GeometricPrimitive::Intersects       Core/Scene/GeometricPrimitive.cpp:68-185
//                -> KDTreeMesh::Intersect_New            Core/Shape/KDTreeMesh.cpp:467-577
//                   or BVHMesh::Intersect                Core/Shape/BVHMesh.cpp:169-198
//                -> IndexedTriangle::Intersects          Core/Shape/IndexedTriangle.cpp:92-253
//   any hit      BasicSpace::Intersects(ray)             Core/Space/BasicSpace.cpp:94-103
//   path tracing PathIntegrator::Radiance                Core/Integrator/PathIntegrator.cpp:357-367
//                driven per pixel as BaseRenderer::RenderRegion does
//                (Core/Renderer/BaseRenderer.cpp:62-169) over a 16x16 tile
//                queue with an atomic counter (Utility/Sandbox/Multithreaded.h:207-259)
//
// Barycentrics: DifferentialSurface stores none, so every triangle gets its
// own three vertices with UVs (0,0), (1,0), (0,1); the interpolated UV
// (IndexedTriangle.cpp:231-233) is then exactly (beta, gamma). The primitive
// id is the triangle's index in the mesh's TriangleList.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// the library this file builds.
#include <thread>
#include <vector>
#include <atomic>
#include <cstring>
#include <cstdint>
#include <chrono>

#include "Shape/KDTreeMesh.h"
#include "Shape/BVHMesh.h"
#include "Shape/Quad.h"
#include "Space/BasicSpace.h"
#include "Scene/GeometricPrimitive.h"
#include "Scene/EmissivePrimitive.h"
#include "Scene/Scene.h"
#include "Geometry/Intersection.h"
#include "Camera/PerspectiveCamera.h"
#include "Integrator/PathIntegrator.h"
#include "Light/DiffuseAreaLight.h"
#include "Light/InfiniteAreaLight.h"
#include "Renderer/BasicRenderer.h"
#include "Material/Glass.h"
#include "Material/Matte.h"
#include "Material/Mirror.h"
#include "Sampler/RandomSampler.h"
#include "Filter/BoxFilter.h"
#include "System/EngineKernel.h"
#include "Postproc/AccumulationBuffer.h"
#include "Postproc/GlobalTone.h"
#include "Postproc/AutoTone.h"
#include "Postproc/DragoTone.h"
#include "System/ArgumentMap.h"
#include "Device/Device.h"
#include "Renderer/Renderer.h"
#include "Exception/Exception.h"
#include "System/PlugIn.h"
#include "System/PlugInManager.h"

#include <dlfcn.h>
#include <map>
#include <string>

using namespace Illumina::Core;

namespace {

struct RefMesh
{
	ITriangleMesh *mesh;
	GeometricPrimitive *prim;
	BasicSpace *space;
	int ntris;
	double build_seconds;
};

template <class F>
void parallel_chunks(long n, int nthreads, F f)
{
	if (nthreads <= 1 || n < 1024) { f(0L, n); return; }
	std::vector<std::thread> pool;
	long chunk = (n + nthreads - 1) / nthreads;
	for (int i = 0; i < nthreads; i++) {
		long b = i * chunk, e = std::min(n, b + chunk);
		if (b >= e) break;
		pool.emplace_back([=]() { f(b, e); });
	}
	for (auto &th : pool) th.join();
}

void report(char *err, int err_len, const std::string &msg)
{
	if (err && err_len > 0) {
		std::strncpy(err, msg.c_str(), (size_t)err_len - 1);
		err[err_len - 1] = 0;
	}
}

bool same(float a, float b) { return std::memcmp(&a, &b, sizeof(float)) == 0; }
bool same(const Vector3 &a, const Vector3 &b) { return same(a.X, b.X) && same(a.Y, b.Y) && same(a.Z, b.Z); }

uint32_t intersection_diff(const Intersection &a, const Intersection &b)
{
	const DifferentialSurface &p = a.Surface, &q = b.Surface;
	uint32_t m = 0;
	if (!same(p.Distance, q.Distance)) m |= 1u;
	if (!same(p.Point, q.Point)) m |= 2u;
	if (!same(p.PointUV.U, q.PointUV.U) || !same(p.PointUV.V, q.PointUV.V)) m |= 4u;
	if (!same(p.GeometryNormal, q.GeometryNormal)) m |= 8u;
	if (!same(p.ShadingNormal, q.ShadingNormal)) m |= 16u;
	if (!same(p.PointWS, q.PointWS)) m |= 32u;
	if (!same(p.GeometryBasisWS.U, q.GeometryBasisWS.U) || !same(p.GeometryBasisWS.V, q.GeometryBasisWS.V) ||
	    !same(p.GeometryBasisWS.W, q.GeometryBasisWS.W) || !same(p.ShadingBasisWS.U, q.ShadingBasisWS.U) ||
	    !same(p.ShadingBasisWS.V, q.ShadingBasisWS.V) || !same(p.ShadingBasisWS.W, q.ShadingBasisWS.W))
		m |= 64u;
	if (!same(p.RayOrigin, q.RayOrigin) || !same(p.RayDirection, q.RayDirection) ||
	    !same(p.RayOriginWS, q.RayOriginWS) || !same(p.RayDirectionWS, q.RayDirectionWS))
		m |= 128u;
	if (a.GetPrimitive() != b.GetPrimitive()) m |= 256u;
	if (a.GetMaterial() != b.GetMaterial()) m |= 512u;
	if (a.GetLight() != b.GetLight()) m |= 1024u;
	if (p.GetShape() != q.GetShape()) m |= 2048u;
	return m;
}

// The box scene in reference objects (see ilref_render_box). Owns them.
struct BoxScene
{
	std::vector<ITriangleMesh *> meshes;
	std::vector<IPrimitive *> prims;
	std::vector<IMaterial *> mats;
	ILight *light = nullptr;
	ILight *infinite = nullptr;
	IShape *quadShape = nullptr;

	// The scene's LightList: the area light, then the infinite light.
	std::vector<ILight *> lights() const
	{
		std::vector<ILight *> l;
		if (light) l.push_back(light);
		if (infinite) l.push_back(infinite);
		return l;
	}

	// kinds (optional, one per primitive): 0 MatteMaterial(albedo), 2
	// MirrorMaterial(albedo), 3 GlassMaterial(albedo, transmittance, 1,
	// eta_i, eta_t) with spec[5 * p ..] = transmittance rgb, eta_i, eta_t.
	// light_kind 0: primitive light_prim is the Quad(quad) light; 1: it is
	// the BVHMesh of its own triangles, emitting as a DiffuseAreaLight on
	// that mesh; -1: no area light. inf (optional): an InfiniteAreaLight
	// of that intensity, without a texture, joins the lights.
	void create(const float *pos, const int32_t *prim_of_tri, int ntris, int nprims, const float *albedo,
	            int light_prim, const float *quad, const float *emit, const int32_t *kinds = nullptr,
	            const float *spec = nullptr, int light_kind = 0, const float *inf = nullptr)
	{
		if (inf) infinite = new InfiniteAreaLight(Spectrum(inf[0], inf[1], inf[2]));
		for (int p = 0; p < nprims; p++) {
			const Spectrum a(albedo[3 * p], albedo[3 * p + 1], albedo[3 * p + 2]);
			const int kind = kinds ? kinds[p] : 0;
			IMaterial *m;
			if (kind == 2)
				m = new MirrorMaterial(a);
			else if (kind == 3)
				m = new GlassMaterial(a, Spectrum(spec[5 * p], spec[5 * p + 1], spec[5 * p + 2]), 1.f, spec[5 * p + 3],
				                      spec[5 * p + 4]);
			else
				m = new MatteMaterial(a);
			mats.push_back(m);
			if (p == light_prim && light_kind == 0) {
				Quad *qs = new Quad(Vector3(quad[0], quad[1], quad[2]), Vector3(quad[3], quad[4], quad[5]),
				                    Vector3(quad[6], quad[7], quad[8]), Vector3(quad[9], quad[10], quad[11]));
				qs->ComputeBoundingVolume();
				quadShape = qs;
				EmissivePrimitive *ep = new EmissivePrimitive();
				ep->SetShape(qs);
				ep->SetMaterial(m);
				DiffuseAreaLight *dl = new DiffuseAreaLight(nullptr, qs, Spectrum(emit[0], emit[1], emit[2]));
				ep->SetLight(dl);
				light = dl;
				prims.push_back(ep);
				continue;
			}
			BVHMesh *mesh = new BVHMesh(10, 35);
			int nv = 0;
			for (int t = 0; t < ntris; t++) {
				if (prim_of_tri[t] != p) continue;
				const float *a = pos + 9 * t;
				Vector3 v0(a[0], a[1], a[2]), v1(a[3], a[4], a[5]), v2(a[6], a[7], a[8]);
				Vector3 n = Vector3::Normalize(Vector3::Cross(v1 - v0, v2 - v0));
				for (int c = 0; c < 3; c++) {
					Vertex v;
					v.Position.Set(a[3 * c], a[3 * c + 1], a[3 * c + 2]);
					v.Normal = n;
					v.UV.Set(c == 1 ? 1.f : 0.f, c == 2 ? 1.f : 0.f);
					mesh->AddVertex(v);
				}
				mesh->AddIndexedTriangle(nv, nv + 1, nv + 2);
				nv += 3;
			}
			mesh->ComputeBoundingVolume();
			mesh->Compile();
			meshes.push_back(mesh);
			if (p == light_prim && light_kind == 1) {
				EmissivePrimitive *ep = new EmissivePrimitive();
				ep->SetShape(mesh);
				ep->SetMaterial(m);
				DiffuseAreaLight *dl = new DiffuseAreaLight(nullptr, mesh, Spectrum(emit[0], emit[1], emit[2]));
				ep->SetLight(dl);
				light = dl;
				prims.push_back(ep);
				continue;
			}
			GeometricPrimitive *gp = new GeometricPrimitive();
			gp->SetShape(mesh);
			gp->SetMaterial(m);
			prims.push_back(gp);
		}
	}

	void fill(ISpace &space)
	{
		for (auto *p : prims) space.PrimitiveList.PushBack(p);
		space.Initialise();
		space.Build();
	}

	~BoxScene()
	{
		for (auto *pr : prims) delete pr;
		for (auto *m : meshes) delete m;
		for (auto *m : mats) delete m;
		delete light;
		delete infinite;
		delete quadShape;
	}
};

// Reference renderer loop over any space (see ilref_render_box).
void render_over(ISpace &space, const std::vector<ILight *> &lights, const float *eye, const float *target,
                 const float *up, float fov, float aspect, int width, int height, int spp, int max_depth, float eps,
                 uint32_t seed, int nthreads, float *out, float *out_direct = nullptr, float *out_albedo = nullptr)
{
	PerspectiveCamera camera(Vector3(eye[0], eye[1], eye[2]),
	                         Vector3::Normalize(Vector3(target[0], target[1], target[2]) - Vector3(eye[0], eye[1], eye[2])),
	                         Vector3(up[0], up[1], up[2]), -1.f, 1.f, -1.f, 1.f, 1.f);
	camera.SetFieldOfView(fov, aspect);

	const int tile = 16;
	const int tiles_x = (width + tile - 1) / tile, tiles_y = (height + tile - 1) / tile;
	const int ntiles = tiles_x * tiles_y;
	std::atomic<int> next(0);
	if (nthreads < 1) nthreads = 1;

	auto worker = [&]() {
		RandomSampler sampler;
		Scene scene(&space, &camera, &sampler);
		for (ILight *l : lights) scene.LightList.PushBack(l);
		PathIntegrator integrator(max_depth, 1, eps);
		integrator.Initialise(&scene, &camera);
		BoxFilter filter;
		IntegratorContext ctx;
		ctx.SampleCount = spp;
		Intersection isect;
		RadianceContext rc;
		std::vector<Vector2> samples(spp);
		const float rcpW = 1.f / width, rcpH = 1.f / height, rcpS = 1.f / spp;
		int tid;
		while ((tid = next.fetch_add(1)) < ntiles) {
			sampler.Reset(seed * 7919u + (uint32_t)tid);
			int x0 = (tid % tiles_x) * tile, y0 = (tid / tiles_x) * tile;
			for (int y = y0; y < std::min(height, y0 + tile); y++)
				for (int x = x0; x < std::min(width, x0 + tile); x++) {
					sampler.Get2DSamples(samples.data(), spp);
					filter(samples.data(), spp);
					ctx.SurfacePosition.Set((float)x, (float)y);
					ctx.NormalisedPosition.Set(x * rcpW, y * rcpH);
					Spectrum acc(0.f), direct(0.f), albedo(0.f);
					for (ctx.SampleIndex = 0; ctx.SampleIndex < spp; ctx.SampleIndex++) {
						Ray ray;
						camera.GetRay(ctx.NormalisedPosition.X, ctx.NormalisedPosition.Y,
						              samples[ctx.SampleIndex].U * rcpW, samples[ctx.SampleIndex].V * rcpH, ray);
						acc += integrator.Radiance(&ctx, &scene, ray, isect, &rc);
						direct += rc.Direct;
						albedo += rc.Albedo;
					}
					acc *= rcpS;
					const size_t px = 3 * ((size_t)y * width + x);
					float *o = out + px;
					o[0] = acc[0]; o[1] = acc[1]; o[2] = acc[2];
					if (out_direct) {
						direct *= rcpS;
						for (int c = 0; c < 3; c++) out_direct[px + c] = direct[c];
					}
					if (out_albedo) {
						albedo *= rcpS;
						for (int c = 0; c < 3; c++) out_albedo[px + c] = albedo[c];
					}
				}
		}
	};
	std::vector<std::thread> pool;
	for (int i = 0; i < nthreads; i++) pool.emplace_back(worker);
	for (auto &th : pool) th.join();
}

// An IDevice that only has a size: what BaseRenderer asks of its device
// (GetWidth / GetHeight for normalisation) plus no-op frame calls.
class MemoryDevice : public IDevice
{
	int m_w, m_h;

public:
	MemoryDevice(int w, int h) : m_w(w), m_h(h) {}
	int GetWidth(void) const { return m_w; }
	int GetHeight(void) const { return m_h; }
	AccessType GetAccessType(void) const { return Write; }
	bool Open(void) { return true; }
	void Close(void) {}
	void BeginFrame(void) {}
	void EndFrame(void) {}
	void Set(int, int, const Spectrum &) {}
	void Set(float, float, const Spectrum &) {}
	void Get(int, int, Spectrum &s) const { s = Spectrum(0.f); }
	void Get(float, float, Spectrum &s) const { s = Spectrum(0.f); }
	Spectrum Get(int, int) const { return Spectrum(0.f); }
	Spectrum Get(float, float) const { return Spectrum(0.f); }
	void WriteRadianceBufferToDevice(int, int, int, int, RadianceBuffer *, int, int) {}
};

// A space made by a plug-in's factory (see ilref_render_box_plugin).
struct PluginSpace
{
	void *lib = nullptr;
	EngineKernel *kernel = nullptr;
	IPlugIn *plugin = nullptr;
	ISpace *space = nullptr;

	int open(const char *path, const char *factory, char *err, int err_len)
	{
		// The plug-in resolves the engine's symbols against this library, so
		// make this library's symbols global before loading it.
		Dl_info self;
		if (dladdr((void *)&report, &self) && self.dli_fname)
			dlopen(self.dli_fname, RTLD_NOW | RTLD_NOLOAD | RTLD_GLOBAL);
		lib = dlopen(path, RTLD_NOW | RTLD_LOCAL);
		if (!lib) {
			const char *e = dlerror();
			report(err, err_len, e ? e : "dlopen failed");
			return -1;
		}
		typedef IPlugIn *(*GetSingleton)(void);
		GetSingleton get = (GetSingleton)dlsym(lib, "GetPlugInSingleton");
		if (!get) {
			report(err, err_len, "no GetPlugInSingleton in plug-in");
			return -2;
		}
		kernel = new EngineKernel();
		plugin = get();
		kernel->GetPlugInManager()->Register(plugin);
		Factory<ISpace> *f = kernel->GetSpaceManager()->RequestFactory(factory);
		if (!f) {
			report(err, err_len, std::string("no space factory named ") + factory);
			return -3;
		}
		space = f->CreateInstance();
		return space ? 0 : -3;
	}

	// ISpace::Build returns only a bool; a plug-in may say why.
	void report_build_failure(char *err, int err_len)
	{
		typedef const char *(*LastError)(const ISpace *);
		LastError why = lib ? (LastError)dlsym(lib, "GpuSpaceLastError") : nullptr;
		report(err, err_len, std::string("space Initialise/Build returned false: ") + (why ? why(space) : ""));
	}

	~PluginSpace()
	{
		delete space;
		if (plugin) kernel->GetPlugInManager()->Unregister(plugin);
		delete kernel;
		if (lib) {
			typedef void (*Dispose)(void);
			Dispose d = (Dispose)dlsym(lib, "DisposePlugInSingleton");
			if (d) d();
			dlclose(lib);
		}
	}
};

} // namespace

extern "C" {

// kind 0 = KDTreeMesh (factory defaults: 10 tris / leaf, depth 35,
// Core/Shape/ShapeFactories.h:231-235); kind 1 = BVHMesh (10 tris / leaf,
// depth 35, ShapeFactories.h:311-315).
void *ilref_mesh_create(int kind, const float *pos, int nverts, const int *idx, int ntris)
{
	RefMesh *rm = new RefMesh();
	if (kind == 0) rm->mesh = new KDTreeMesh(10, 35);
	else rm->mesh = new BVHMesh(10, 35);
	rm->ntris = ntris;

	for (int t = 0; t < ntris; t++) {
		for (int c = 0; c < 3; c++) {
			Vertex v;
			int vi = idx[3 * t + c];
			v.Position.Set(pos[3 * vi + 0], pos[3 * vi + 1], pos[3 * vi + 2]);
			v.Normal.Set(0.f, 0.f, 1.f);
			v.UV.Set(c == 1 ? 1.f : 0.f, c == 2 ? 1.f : 0.f);
			rm->mesh->AddVertex(v);
		}
	}
	for (int t = 0; t < ntris; t++)
		rm->mesh->AddIndexedTriangle(3 * t, 3 * t + 1, 3 * t + 2);

	auto t0 = std::chrono::steady_clock::now();
	rm->mesh->ComputeBoundingVolume();
	rm->mesh->Compile();
	rm->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

	rm->prim = new GeometricPrimitive();
	rm->prim->SetShape(rm->mesh);
	rm->space = new BasicSpace();
	rm->space->PrimitiveList.PushBack(rm->prim);
	rm->space->Initialise();
	rm->space->Build();
	return rm;
}

double ilref_mesh_build_seconds(void *h) { return ((RefMesh *)h)->build_seconds; }

void ilref_mesh_destroy(void *h)
{
	RefMesh *rm = (RefMesh *)h;
	delete rm->space;
	delete rm->prim;
	delete rm->mesh;
	delete rm;
}

// Rays are two float4 streams: (ox, oy, oz, tmin) and (dx, dy, dz, tmax).
// Misses write prim = -1, t = +inf, u = v = 0.
int ilref_intersect(void *h, const float *o4, const float *d4, long n,
                    int32_t *prim, float *t, float *u, float *v, int nthreads)
{
	RefMesh *rm = (RefMesh *)h;
	const IndexedTriangle *base = &rm->mesh->TriangleList[0];
	parallel_chunks(n, nthreads, [&](long b, long e) {
		Intersection isect;
		for (long i = b; i < e; i++) {
			Ray ray(Vector3(o4[4 * i], o4[4 * i + 1], o4[4 * i + 2]),
			        Vector3(d4[4 * i], d4[4 * i + 1], d4[4 * i + 2]),
			        o4[4 * i + 3], d4[4 * i + 3]);
			isect.Prepare();
			if (rm->space->Intersects(ray, isect)) {
				prim[i] = (int32_t)((const IndexedTriangle *)isect.Surface.GetShape() - base);
				t[i] = isect.Surface.Distance;
				u[i] = isect.Surface.PointUV.U;
				v[i] = isect.Surface.PointUV.V;
			} else {
				prim[i] = -1; t[i] = __builtin_inff(); u[i] = 0.f; v[i] = 0.f;
			}
		}
	});
	return 0;
}

int ilref_occluded(void *h, const float *o4, const float *d4, long n, uint8_t *occ, int nthreads)
{
	RefMesh *rm = (RefMesh *)h;
	parallel_chunks(n, nthreads, [&](long b, long e) {
		for (long i = b; i < e; i++) {
			Ray ray(Vector3(o4[4 * i], o4[4 * i + 1], o4[4 * i + 2]),
			        Vector3(d4[4 * i], d4[4 * i + 1], d4[4 * i + 2]),
			        o4[4 * i + 3], d4[4 * i + 3]);
			occ[i] = rm->space->Intersects(ray) ? 1 : 0;
		}
	});
	return 0;
}

// Box-scene render through the reference's own path integrator.
//
// Scene input (flattened, world space): nprims primitives; triangles of
// primitive p are those with prim_of_tri == p, each given its own vertices
// with the face normal as vertex normal. Primitive light_prim is not a mesh:
// it is a Quad(q0..q3) in an EmissivePrimitive with a DiffuseAreaLight of
// radiance emit (Core/Shape/Quad.cpp, Core/Scene/EmissivePrimitive.cpp,
// Core/Light/DiffuseAreaLight.cpp). Every primitive gets a MatteMaterial of
// its albedo. Camera: PerspectiveCamera(eye, normalize(target-eye), up,
// -1,1,-1,1, 1) + SetFieldOfView(fov, aspect) as the camera factory builds it
// (Core/Camera/CameraFactories.h:40-80). PathIntegrator(max_depth, 1, eps).
//
// Each thread owns a Scene over the shared space and camera with its own
// RandomSampler reseeded per tile (seed * 7919 + tile): the reference shares
// one sampler across threads (a data race); per-tile seeding keeps the image
// independent of the thread count. out: height*width*3 floats, row y = the
// renderer's y (camera 'up' grows with y).
int ilref_render_box(const float *pos, const int32_t *prim_of_tri, int ntris, int nprims,
                     const float *albedo, int light_prim, const float *quad, const float *emit,
                     const float *eye, const float *target, const float *up, float fov, float aspect,
                     int width, int height, int spp, int max_depth, float eps, uint32_t seed,
                     int nthreads, float *out)
{
	BoxScene scene;
	scene.create(pos, prim_of_tri, ntris, nprims, albedo, light_prim, quad, emit);
	BasicSpace space;
	scene.fill(space);
	render_over(space, scene.lights(), eye, target, up, fov, aspect, width, height, spp, max_depth, eps, seed,
	            nthreads, out);
	return 0;
}

// ilref_render_box with a material kind per primitive (BoxScene::create):
// mirrors and glass next to the matte walls.
int ilref_render_box_materials(const float *pos, const int32_t *prim_of_tri, int ntris, int nprims,
                               const float *albedo, int light_prim, const float *quad, const float *emit,
                               const int32_t *kinds, const float *spec,
                               const float *eye, const float *target, const float *up, float fov, float aspect,
                               int width, int height, int spp, int max_depth, float eps, uint32_t seed,
                               int nthreads, float *out)
{
	BoxScene scene;
	scene.create(pos, prim_of_tri, ntris, nprims, albedo, light_prim, quad, emit, kinds, spec);
	BasicSpace space;
	scene.fill(space);
	render_over(space, scene.lights(), eye, target, up, fov, aspect, width, height, spp, max_depth, eps, seed,
	            nthreads, out);
	return 0;
}

// ilref_render_box plus the RadianceContext's Direct and Albedo per pixel,
// averaged over the samples as BaseRenderer::RenderRegion averages them
// (Core/Renderer/BaseRenderer.cpp:95-130).
int ilref_render_box_aov(const float *pos, const int32_t *prim_of_tri, int ntris, int nprims,
                         const float *albedo, int light_prim, const float *quad, const float *emit,
                         const float *eye, const float *target, const float *up, float fov, float aspect,
                         int width, int height, int spp, int max_depth, float eps, uint32_t seed,
                         int nthreads, float *out, float *out_direct, float *out_albedo)
{
	BoxScene scene;
	scene.create(pos, prim_of_tri, ntris, nprims, albedo, light_prim, quad, emit);
	BasicSpace space;
	scene.fill(space);
	render_over(space, scene.lights(), eye, target, up, fov, aspect, width, height, spp, max_depth, eps, seed,
	            nthreads, out, out_direct, out_albedo);
	return 0;
}

// The box scene rendered by the engine's own objects (Scene,
// PerspectiveCamera, BoxFilter, RadianceBuffer) over a plug-in's space (made
// by the factory `space_factory`), wired to a renderer as the Sandbox wires
// one: the renderer made by `renderer_factory` (or the reference's
// BasicRenderer when it is empty) and the integrator made by
// `integrator_factory` with the arguments RayDepth = max_depth, ShadowRays =
// 1, Epsilon = eps plus `integrator_args` ("Key=Value;..."; or the
// reference's PathIntegrator(max_depth, 1, eps) when the factory name is
// empty). Rendered with IRenderer::Render(buffer) (tile <= 0) or with
// RenderRegion(buffer, x, y, w, h, x, y) over tile x tile regions. Outputs the
// buffer's Final, Direct and Albedo (height x width x 3 each). light_kind and
// inf choose the lights as BoxScene::create does.
int ilref_render_box_engine(const char *plugin_path, const char *space_factory, const char *renderer_factory,
                            const char *integrator_factory, const char *integrator_args,
                            const float *pos, const int32_t *prim_of_tri, int ntris, int nprims,
                            const float *albedo, int light_prim, const float *quad, const float *emit,
                            const int32_t *kinds, const float *spec, int light_kind, const float *inf,
                            const float *eye, const float *target, const float *up, float fov, float aspect,
                            int width, int height, int spp, int max_depth, float eps, int tile,
                            float *out, float *out_direct, float *out_albedo, char *err, int err_len)
{
	PluginSpace ps;
	int rc = ps.open(plugin_path, space_factory, err, err_len);
	if (rc) return rc;
	Factory<IRenderer> *rf = nullptr;
	if (renderer_factory && *renderer_factory) {
		rf = ps.kernel->GetRendererManager()->RequestFactory(renderer_factory);
		if (!rf) {
			report(err, err_len, std::string("no renderer factory named ") + renderer_factory);
			return -3;
		}
	}
	Factory<IIntegrator> *inf_factory = nullptr;
	if (integrator_factory && *integrator_factory) {
		inf_factory = ps.kernel->GetIntegratorManager()->RequestFactory(integrator_factory);
		if (!inf_factory) {
			report(err, err_len, std::string("no integrator factory named ") + integrator_factory);
			return -3;
		}
	}
	BoxScene boxes;
	boxes.create(pos, prim_of_tri, ntris, nprims, albedo, light_prim, quad, emit, kinds, spec, light_kind, inf);
	boxes.fill(*ps.space);
	if (!ps.space->Initialise() || !ps.space->Build()) {
		ps.report_build_failure(err, err_len);
		return -4;
	}
	PerspectiveCamera camera(Vector3(eye[0], eye[1], eye[2]),
	                         Vector3::Normalize(Vector3(target[0], target[1], target[2]) - Vector3(eye[0], eye[1], eye[2])),
	                         Vector3(up[0], up[1], up[2]), -1.f, 1.f, -1.f, 1.f, 1.f);
	camera.SetFieldOfView(fov, aspect);
	RandomSampler sampler;
	Scene scene(ps.space, &camera, &sampler);
	for (ILight *l : boxes.lights()) scene.LightList.PushBack(l);
	BoxFilter filter;
	MemoryDevice device(width, height);
	RadianceBuffer buffer(width, height);
	IRenderer *renderer = nullptr;
	IIntegrator *integrator = nullptr;
	try {
		if (inf_factory) {
			std::map<std::string, std::string> args;
			args["RayDepth"] = std::to_string(max_depth);
			args["ShadowRays"] = "1";
			char e[32];
			snprintf(e, sizeof(e), "%.9g", eps);
			args["Epsilon"] = e;
			std::string extra = integrator_args ? integrator_args : "";
			size_t at = 0;
			while (at < extra.size()) {
				size_t semi = extra.find(';', at);
				if (semi == std::string::npos) semi = extra.size();
				const std::string kv = extra.substr(at, semi - at);
				const size_t eq = kv.find('=');
				if (eq != std::string::npos) args[kv.substr(0, eq)] = kv.substr(eq + 1);
				at = semi + 1;
			}
			ArgumentMap am(args);
			integrator = inf_factory->CreateInstance(am);
		} else {
			integrator = new PathIntegrator(max_depth, 1, eps);
		}
		integrator->Initialise(&scene, &camera);
		if (rf) {
			std::map<std::string, std::string> args;
			args["Samples"] = std::to_string(spp);
			ArgumentMap am(args);
			renderer = rf->CreateInstance(am);
			renderer->SetScene(&scene);
			renderer->SetIntegrator(integrator);
			renderer->SetDevice(&device);
			renderer->SetFilter(&filter);
		} else {
			renderer = new BasicRenderer(&scene, integrator, &device, &filter, &buffer, spp);
		}
		// (IRenderer::SetRadianceBuffer is declared but never defined in the
		// engine, so the buffer goes to the calls that take one)
		renderer->Initialise();
		if (tile <= 0) {
			renderer->Render(&buffer);
		} else {
			for (int y = 0; y < height; y += tile)
				for (int x = 0; x < width; x += tile)
					renderer->RenderRegion(&buffer, x, y, std::min(tile, width - x), std::min(tile, height - y), x, y);
		}
		renderer->Commit(&buffer);
	} catch (const Exception &e) {
		report(err, err_len, e.GetMessage());
		delete renderer;
		delete integrator;
		return -5;
	} catch (const Exception *e) {
		report(err, err_len, e->GetMessage());
		delete renderer;
		delete integrator;
		return -5;
	}
	for (int y = 0; y < height; y++)
		for (int x = 0; x < width; x++) {
			const RadianceContext *c = buffer.GetP(x, y);
			const size_t px = 3 * ((size_t)y * width + x);
			for (int k = 0; k < 3; k++) {
				out[px + k] = c->Final[k];
				out_direct[px + k] = c->Direct[k];
				out_albedo[px + k] = c->Albedo[k];
			}
		}
	delete renderer;
	delete integrator;
	return 0;
}

// ilref_render_box_engine with the plug-in's renderer (factory `factory`), its
// space (the same factory name) and the reference's PathIntegrator.
int ilref_render_box_renderer(const char *plugin_path, const char *factory,
                              const float *pos, const int32_t *prim_of_tri, int ntris, int nprims,
                              const float *albedo, int light_prim, const float *quad, const float *emit,
                              const float *eye, const float *target, const float *up, float fov, float aspect,
                              int width, int height, int spp, int max_depth, float eps, int tile,
                              float *out, float *out_direct, float *out_albedo, const int32_t *kinds,
                              const float *spec, char *err, int err_len)
{
	return ilref_render_box_engine(plugin_path, factory, factory, "", "", pos, prim_of_tri, ntris, nprims, albedo,
	                               light_prim, quad, emit, kinds, spec, 0, nullptr, eye, target, up, fov, aspect,
	                               width, height, spp, max_depth, eps, tile, out, out_direct, out_albedo, err,
	                               err_len);
}

// The box scene through the reference's PathIntegrator (render_over) with a
// choice of lights (BoxScene::create: light_kind, inf) and materials, plus
// the RadianceContext's Direct and Albedo (either may be null).
int ilref_render_box_lights(const float *pos, const int32_t *prim_of_tri, int ntris, int nprims,
                            const float *albedo, int light_prim, const float *quad, const float *emit,
                            const int32_t *kinds, const float *spec, int light_kind, const float *inf,
                            const float *eye, const float *target, const float *up, float fov, float aspect,
                            int width, int height, int spp, int max_depth, float eps, uint32_t seed,
                            int nthreads, float *out, float *out_direct, float *out_albedo)
{
	BoxScene scene;
	scene.create(pos, prim_of_tri, ntris, nprims, albedo, light_prim, quad, emit, kinds, spec, light_kind, inf);
	BasicSpace space;
	scene.fill(space);
	render_over(space, scene.lights(), eye, target, up, fov, aspect, width, height, spp, max_depth, eps, seed,
	            nthreads, out, out_direct, out_albedo);
	return 0;
}

// The same render with the space a plug-in registers: the plug-in library is
// loaded, its GetPlugInSingleton() handed to the engine's PlugInManager
// (which calls IPlugIn::Register(EngineKernel*)), and the space is made by
// the factory registered under `factory` in the kernel's SpaceManager. The
// reference's own library loader has no Linux implementation
// (System/LibraryManager.cpp:16-23 throws), so the load is a dlopen here.
// Returns 0, or a negative code: -1 load, -2 symbol, -3 factory, -4 Build().
int ilref_render_box_plugin(const char *plugin_path, const char *factory,
                            const float *pos, const int32_t *prim_of_tri, int ntris, int nprims,
                            const float *albedo, int light_prim, const float *quad, const float *emit,
                            const float *eye, const float *target, const float *up, float fov, float aspect,
                            int width, int height, int spp, int max_depth, float eps, uint32_t seed,
                            int nthreads, float *out, char *err, int err_len)
{
	PluginSpace ps;
	int rc = ps.open(plugin_path, factory, err, err_len);
	if (rc) return rc;
	BoxScene scene;
	scene.create(pos, prim_of_tri, ntris, nprims, albedo, light_prim, quad, emit);
	scene.fill(*ps.space);
	if (!ps.space->Initialise() || !ps.space->Build()) {
		ps.report_build_failure(err, err_len);
		return -4;
	}
	render_over(*ps.space, scene.lights(), eye, target, up, fov, aspect, width, height, spp, max_depth, eps, seed,
	            nthreads, out);
	return 0;
}

// Field-by-field comparison of the plug-in space with BasicSpace over the
// same primitives (the box scene), for n rays (float4 streams as above).
// Per ray: hit[2*i + s] (s = 0 BasicSpace, 1 plug-in) for the closest-hit
// overload, t[2*i + s] its Distance (+inf on a miss), diff[i] a bit mask of
// the Intersection fields that differ when both hit (1 Distance, 2 Point,
// 4 PointUV, 8 GeometryNormal, 16 ShadingNormal, 32 PointWS, 64 bases,
// 128 ray fields, 256 primitive, 512 material, 1024 light, 2048 shape),
// occ[2*i + s] the any-hit overload, and with exclude[i] >= 0 also
// xhit/xt/xocc[2*i + s] for the p_pExclude overloads excluding primitive
// exclude[i]. batch_diff counts rays whose IntersectsBatch-style answer
// (every ray in one call, when the plug-in is a GpuSpace) differs from its
// scalar answer; the comparison uses the space only through ISpace, so
// batching is exercised by the caller's choice of ray count.
int ilref_compare_spaces(const char *plugin_path, const char *factory,
                         const float *pos, const int32_t *prim_of_tri, int ntris, int nprims,
                         const float *albedo, int light_prim, const float *quad, const float *emit,
                         const float *o4, const float *d4, long n, const int32_t *exclude,
                         uint8_t *hit, float *t, uint32_t *diff, uint8_t *occ,
                         uint8_t *xhit, float *xt, uint8_t *xocc, char *err, int err_len)
{
	PluginSpace ps;
	int rc = ps.open(plugin_path, factory, err, err_len);
	if (rc) return rc;
	BoxScene scene;
	scene.create(pos, prim_of_tri, ntris, nprims, albedo, light_prim, quad, emit);
	BasicSpace basic;
	scene.fill(basic);
	scene.fill(*ps.space);
	basic.Initialise();
	basic.Build();
	if (!ps.space->Initialise() || !ps.space->Build()) {
		ps.report_build_failure(err, err_len);
		return -4;
	}
	ISpace *spaces[2] = {&basic, ps.space};
	const float inf = __builtin_inff();
	for (long i = 0; i < n; i++) {
		Ray ray(Vector3(o4[4 * i], o4[4 * i + 1], o4[4 * i + 2]), Vector3(d4[4 * i], d4[4 * i + 1], d4[4 * i + 2]),
		        o4[4 * i + 3], d4[4 * i + 3]);
		Intersection is[2];
		for (int s = 0; s < 2; s++) {
			is[s].Prepare();
			hit[2 * i + s] = spaces[s]->Intersects(ray, is[s]) ? 1 : 0;
			t[2 * i + s] = hit[2 * i + s] ? is[s].Surface.Distance : inf;
			occ[2 * i + s] = spaces[s]->Intersects(ray) ? 1 : 0;
		}
		diff[i] = (hit[2 * i] && hit[2 * i + 1]) ? intersection_diff(is[0], is[1]) : 0u;
		if (exclude && exclude[i] >= 0 && exclude[i] < (int)scene.prims.size()) {
			IPrimitive *ex = scene.prims[exclude[i]];
			for (int s = 0; s < 2; s++) {
				Intersection x;
				x.Prepare();
				xhit[2 * i + s] = spaces[s]->Intersects(ray, x, ex) ? 1 : 0;
				xt[2 * i + s] = xhit[2 * i + s] ? x.Surface.Distance : inf;
				xocc[2 * i + s] = spaces[s]->Intersects(ray, ex) ? 1 : 0;
			}
		}
	}
	return 0;
}

// The reference's post-processes on w x h rgb images (Core/Postproc/*.h).
// op 0: AccumulationBuffer fed n_frames frames in turn, out = the last
// Apply's output; op 1 GlobalTone, 2 AutoTone, 3 DragoTone on frames[0].
int ilref_postprocess(int op, const float *frames, int n_frames, int w, int h, float *out)
{
	RadianceBuffer in(w, h), res(w, h), acc(w, h);
	auto load = [&](const float *img) {
		for (int y = 0; y < h; y++)
			for (int x = 0; x < w; x++) {
				const float *p = img + 3 * ((size_t)y * w + x);
				RadianceContext *c = in.GetP(x, y);
				c->Final = Spectrum(p[0], p[1], p[2]);
				c->Flags = 0;
			}
	};
	if (op == 0) {
		AccumulationBuffer ab;
		ab.SetAccumulationBuffer(&acc);
		ab.Reset();
		for (int f = 0; f < n_frames; f++) {
			load(frames + 3 * (size_t)w * h * f);
			ab.Apply(&in, &res);
		}
	} else {
		load(frames);
		GlobalTone g;
		AutoTone a;
		DragoTone d;
		IPostProcess *pp = op == 1 ? (IPostProcess *)&g : (op == 2 ? (IPostProcess *)&a : (IPostProcess *)&d);
		pp->Apply(&in, &res);
	}
	for (int y = 0; y < h; y++)
		for (int x = 0; x < w; x++)
			for (int k = 0; k < 3; k++) out[3 * ((size_t)y * w + x) + k] = res.GetP(x, y)->Final[k];
	return 0;
}

} // extern "C"
