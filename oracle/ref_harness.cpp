// Test-infrastructure harness around the reference's own compiled sources.
//
// This file is ours; everything it calls is the reference's code, compiled
// unmodified from the reference tree by oracle/Makefile (with the two
// replacement headers under oracle/refshim). It exposes a small C ABI so the
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
#include "Material/Matte.h"
#include "Sampler/RandomSampler.h"
#include "Filter/BoxFilter.h"

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
	std::vector<ITriangleMesh *> meshes;
	std::vector<IPrimitive *> prims;
	std::vector<IMaterial *> mats;
	BasicSpace space;
	ILight *light = nullptr;
	IShape *quadShape = nullptr;

	for (int p = 0; p < nprims; p++) {
		IMaterial *m = new MatteMaterial(Spectrum(albedo[3 * p], albedo[3 * p + 1], albedo[3 * p + 2]));
		mats.push_back(m);
		if (p == light_prim) {
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
			space.PrimitiveList.PushBack(ep);
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
		GeometricPrimitive *gp = new GeometricPrimitive();
		gp->SetShape(mesh);
		gp->SetMaterial(m);
		prims.push_back(gp);
		space.PrimitiveList.PushBack(gp);
	}
	space.Initialise();
	space.Build();

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
		if (light) scene.LightList.PushBack(light);
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
					Spectrum acc(0.f);
					for (ctx.SampleIndex = 0; ctx.SampleIndex < spp; ctx.SampleIndex++) {
						Ray ray;
						camera.GetRay(ctx.NormalisedPosition.X, ctx.NormalisedPosition.Y,
						              samples[ctx.SampleIndex].U * rcpW, samples[ctx.SampleIndex].V * rcpH, ray);
						acc += integrator.Radiance(&ctx, &scene, ray, isect, &rc);
					}
					acc *= rcpS;
					float *o = out + 3 * ((size_t)y * width + x);
					o[0] = acc[0]; o[1] = acc[1]; o[2] = acc[2];
				}
		}
	};
	std::vector<std::thread> pool;
	for (int i = 0; i < nthreads; i++) pool.emplace_back(worker);
	for (auto &th : pool) th.join();

	for (auto *pr : prims) delete pr;
	for (auto *m : meshes) delete m;
	for (auto *m : mats) delete m;
	delete light;
	delete quadShape;
	return 0;
}

} // extern "C"
