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
#include "Space/BasicSpace.h"
#include "Scene/GeometricPrimitive.h"
#include "Geometry/Intersection.h"

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

} // extern "C"
