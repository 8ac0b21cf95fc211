// GpuSpace: ISpace over the device BVH. See GpuSpace.h for the contract.
#include "GpuSpace.h"
#include "EngineAccess.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>

#include "Exception/Exception.h"
#include "Geometry/Intersection.h"
#include "Geometry/Ray.h"
#include "Light/AreaLight.h"
#include "Material/MaterialGroup.h"
#include "Scene/EmissivePrimitive.h"
#include "Scene/GeometricPrimitive.h"
#include "Shape/IndexedTriangle.h"
#include "Shape/Quad.h"
#include "Shape/Triangle.h"
#include "Shape/TriangleMesh.h"

using namespace Illumina::Core;

namespace Illumina {
namespace PlugIn {

namespace {

// te1 x te2 in the component order of the reference's CROSS macro
// (Shape/IndexedTriangle.cpp:16-19); the plug-in is compiled without FMA
// contraction, so each component rounds as there.
inline Vector3 EdgeCross(const Vector3 &a, const Vector3 &b)
{
    return Vector3(a.Y * b.Z - a.Z * b.Y, a.Z * b.X - a.X * b.Z, a.X * b.Y - a.Y * b.X);
}

}  // namespace

GpuSpace::GpuSpace(const std::string &p_strName, int p_nDevice)
    : ISpace(p_strName), m_nDevice(p_nDevice), m_pContext(NULL), m_bBuilt(false), m_nBuildCount(0),
      m_pPreparedScene(NULL), m_nPreparedBuild(0), m_pOrigin4(NULL), m_pDirection4(NULL)
{
}

GpuSpace::GpuSpace(void)
    : ISpace(), m_nDevice(0), m_pContext(NULL), m_bBuilt(false), m_nBuildCount(0), m_pPreparedScene(NULL),
      m_nPreparedBuild(0), m_pOrigin4(NULL), m_pDirection4(NULL)
{
}

GpuSpace::~GpuSpace(void) { Shutdown(); }

IBoundingVolume *GpuSpace::GetBoundingVolume(void) { return &m_aabb; }

bool GpuSpace::Fail(const std::string &p_strReason)
{
    m_strLastError = p_strReason;
    m_bBuilt = false;
    return false;
}

void GpuSpace::Check(int p_nStatus, const char *p_szWhere) const
{
    if (p_nStatus == ILG_OK) return;
    std::ostringstream s;
    s << "GpuSpace: " << p_szWhere << " failed (status " << p_nStatus << "): "
      << (m_pContext ? ilg_last_error(m_pContext) : "no context");
    throw Exception(s.str(), __FILE__, __LINE__);
}

bool GpuSpace::Initialise(void)
{
    std::lock_guard<std::mutex> lock(m_mutex);
    if (m_pContext) return true;
    ilg_opts opts;
    std::memset(&opts, 0, sizeof(opts));
    opts.device = m_nDevice;
    const int status = ilg_create(&m_pContext, &opts);
    if (status != ILG_OK) {
        m_pContext = NULL;
        std::ostringstream s;
        s << "GpuSpace: ilg_create on device " << m_nDevice << " failed (status " << status << ")";
        return Fail(s.str());
    }
    return true;
}

void GpuSpace::Shutdown(void)
{
    std::lock_guard<std::mutex> lock(m_mutex);
    if (m_pContext) ilg_destroy(m_pContext);
    m_pContext = NULL;
    m_bBuilt = false;
}

// The reference's spaces rebuild on Update only when primitives moved; the
// device BVH is rebuilt from scratch, which is what Build does.
bool GpuSpace::Update(void) { return Build(); }

bool GpuSpace::Build(void)
{
    if (!m_pContext && !Initialise()) return false;
    std::lock_guard<std::mutex> lock(m_mutex);
    m_triangles.clear();
    m_ranges.clear();
    m_materials.clear();
    m_aabb.Invalidate();
    std::vector<float> positions;
    std::vector<uint32_t> indices, slots;

    // material slot of one triangle, resolved as FillIntersection resolves it
    auto slot_of = [&](IMaterial *material, const IShape *triangle) -> uint32_t {
        if (material != NULL && material->IsComposite()) {
            MaterialGroup *group = (MaterialGroup *)material;
            material = triangle->HasGroup() ? group->GetByGroupId(triangle->GetGroupId()) : group->GetByIndex(0);
        }
        for (size_t k = 0; k < m_materials.size(); k++)
            if (m_materials[k] == material) return (uint32_t)k;
        m_materials.push_back(material);
        return (uint32_t)(m_materials.size() - 1);
    };

    // One world-space triangle: three fresh vertices (no sharing), so each
    // device triangle's edges are p1 - p0 and p2 - p0 of exactly these floats.
    auto push = [&](const Vector3 &p0, const Vector3 &p1, const Vector3 &p2, const Transformation &xf) {
        const Vector3 *corner[3] = {&p0, &p1, &p2};
        for (int c = 0; c < 3; c++) {
            const Vector3 p = xf.IsIdentity() ? *corner[c] : xf.Apply(*corner[c]);
            indices.push_back((uint32_t)(positions.size() / 3));
            positions.push_back(p.X);
            positions.push_back(p.Y);
            positions.push_back(p.Z);
        }
    };

    for (int index = 0, count = (int)PrimitiveList.Size(); index < count; index++) {
        IPrimitive *primitive = PrimitiveList[index];
        GeometricPrimitive *geometric = dynamic_cast<GeometricPrimitive *>(primitive);
        if (!geometric || !geometric->GetShape()) {
            std::ostringstream s;
            s << "GpuSpace: primitive " << index << " is not a GeometricPrimitive with a shape";
            return Fail(s.str());
        }
        PrimitiveRange range;
        range.primitive = primitive;
        range.geometric = geometric;
        EmissivePrimitive *emissive = dynamic_cast<EmissivePrimitive *>(primitive);
        range.light = emissive ? emissive->GetLight() : NULL;
        range.first = (uint32_t)m_triangles.size();
        const Transformation &xf = geometric->WorldTransform;
        IShape *shape = geometric->GetShape();

        if (ITriangleMesh *mesh = dynamic_cast<ITriangleMesh *>(shape)) {
            for (int k = 0, n = (int)mesh->TriangleList.Size(); k < n; k++) {
                IndexedTriangle &tri = mesh->TriangleList[k];
                push(mesh->VertexList[tri.GetVertexIndex(0)].Position, mesh->VertexList[tri.GetVertexIndex(1)].Position,
                     mesh->VertexList[tri.GetVertexIndex(2)].Position, xf);
                TriangleSource src = {(uint32_t)index, kMesh, &tri, mesh};
                m_triangles.push_back(src);
                slots.push_back(slot_of(geometric->GetMaterial(), &tri));
            }
        } else if (Quad *quad = dynamic_cast<Quad *>(shape)) {
            const Triangle *half = Access::QuadTriangles::Of(quad);
            for (int k = 0; k < 2; k++) {
                push(half[k].Vertex[0], half[k].Vertex[1], half[k].Vertex[2], xf);
                TriangleSource src = {(uint32_t)index, kTriangle, &half[k], NULL};
                m_triangles.push_back(src);
                slots.push_back(slot_of(geometric->GetMaterial(), &half[k]));
            }
        } else if (Triangle *tri = dynamic_cast<Triangle *>(shape)) {
            push(tri->Vertex[0], tri->Vertex[1], tri->Vertex[2], xf);
            TriangleSource src = {(uint32_t)index, kTriangle, tri, NULL};
            m_triangles.push_back(src);
            slots.push_back(slot_of(geometric->GetMaterial(), tri));
        } else {
            std::ostringstream s;
            s << "GpuSpace: primitive " << index << " has a shape the device space does not trace ("
              << shape->ToString() << "); only triangle meshes, quads and triangles are supported";
            return Fail(s.str());
        }
        range.count = (uint32_t)m_triangles.size() - range.first;
        m_ranges.push_back(range);
        if (primitive->IsBounded()) m_aabb.Union(*(primitive->GetWorldBounds()));
    }
    if (m_triangles.empty()) return Fail("GpuSpace: no triangles to build");
    if (m_triangles.size() > 0x7fffffffu) return Fail("GpuSpace: too many triangles");

    int status = ilg_set_mesh(m_pContext, positions.data(), (uint32_t)(positions.size() / 3), indices.data(),
                              (uint32_t)m_triangles.size(), slots.data());
    if (status == ILG_OK) status = ilg_build(m_pContext);
    if (status != ILG_OK) {
        std::ostringstream s;
        s << "GpuSpace: device build failed (status " << status << "): " << ilg_last_error(m_pContext);
        return Fail(s.str());
    }
    m_bBuilt = true;
    m_nBuildCount++;
    m_strLastError.clear();
    return true;
}

bool GpuSpace::GetTriangleRange(const IPrimitive *p_pPrimitive, uint32_t &p_nFirst, uint32_t &p_nCount) const
{
    const PrimitiveRange *range = FindRange(p_pPrimitive);
    if (!range) return false;
    p_nFirst = range->first;
    p_nCount = range->count;
    return true;
}

const GpuSpace::PrimitiveRange *GpuSpace::FindRange(const IPrimitive *p_pPrimitive) const
{
    for (size_t i = 0; i < m_ranges.size(); i++)
        if (m_ranges[i].primitive == p_pPrimitive) return &m_ranges[i];
    return NULL;
}

void GpuSpace::StageRays(const Ray *p_pRays, size_t p_nCount) const
{
    if (!m_bBuilt) throw Exception("GpuSpace: query before a successful Build()", __FILE__, __LINE__);
    m_origin.resize(4 * p_nCount + 4);
    m_direction.resize(4 * p_nCount + 4);
    // 16-byte aligned views into the staging vectors (ilg wants float4 rays)
    float *o = m_origin.data(), *d = m_direction.data();
    o += ((16 - ((uintptr_t)o & 15u)) & 15u) / sizeof(float);
    d += ((16 - ((uintptr_t)d & 15u)) & 15u) / sizeof(float);
    m_pOrigin4 = o;
    m_pDirection4 = d;
    for (size_t i = 0; i < p_nCount; i++) {
        const Ray &r = p_pRays[i];
        // The reference's triangle window ignores Ray::Min (only t >= 1e-5
        // and t <= Max - 1e-5 count), so the device ray starts at 0.
        o[4 * i + 0] = r.Origin.X;
        o[4 * i + 1] = r.Origin.Y;
        o[4 * i + 2] = r.Origin.Z;
        o[4 * i + 3] = 0.f;
        d[4 * i + 0] = r.Direction.X;
        d[4 * i + 1] = r.Direction.Y;
        d[4 * i + 2] = r.Direction.Z;
        d[4 * i + 3] = r.Max;
    }
    m_prim.resize(p_nCount);
    m_t.resize(p_nCount);
    m_u.resize(p_nCount);
    m_v.resize(p_nCount);
    m_occluded.resize(p_nCount);
}

void GpuSpace::FillIntersection(const Ray &p_ray, int32_t p_nTriangle, float p_fDistance, float p_fBeta,
                                float p_fGamma, Intersection &p_intersection) const
{
    const TriangleSource &src = m_triangles[(size_t)p_nTriangle];
    const PrimitiveRange &range = m_ranges[src.primitive];  // one range per primitive, in list order
    GeometricPrimitive *geometric = range.geometric;
    const Transformation &xf = geometric->WorldTransform;
    const bool identity = xf.IsIdentity();
    DifferentialSurface &surface = p_intersection.Surface;

    // the shape's part (object space)
    const Ray objectRay = identity ? p_ray : p_ray.ApplyInverse(xf);
    const float beta = p_fBeta, gamma = p_fGamma, alpha = 1.f - beta - gamma;
    if (src.kind == kMesh) {
        IndexedTriangle *tri = (IndexedTriangle *)src.shape;
        const Vertex &v0 = src.mesh->VertexList[tri->GetVertexIndex(0)];
        const Vertex &v1 = src.mesh->VertexList[tri->GetVertexIndex(1)];
        const Vertex &v2 = src.mesh->VertexList[tri->GetVertexIndex(2)];
        surface.SetShape(tri);
        surface.Distance = p_fDistance;
        surface.Point = objectRay.PointAlongRay(p_fDistance);
        surface.PointUV.Set(v0.UV.U * alpha + v1.UV.U * beta + v2.UV.U * gamma,
                            v0.UV.V * alpha + v1.UV.V * beta + v2.UV.V * gamma);
        surface.ShadingNormal.Set(v0.Normal.X * alpha + v1.Normal.X * beta + v2.Normal.X * gamma,
                                  v0.Normal.Y * alpha + v1.Normal.Y * beta + v2.Normal.Y * gamma,
                                  v0.Normal.Z * alpha + v1.Normal.Z * beta + v2.Normal.Z * gamma);
        surface.ShadingNormal.Normalize();
        surface.GeometryNormal = EdgeCross(tri->GetEdge(0), tri->GetEdge(1));
        surface.GeometryNormal.Normalize();
    } else {
        const Triangle *tri = (const Triangle *)src.shape;
        surface.SetShape(tri);
        surface.Distance = p_fDistance;
        surface.Point = objectRay.PointAlongRay(p_fDistance);
        surface.PointUV.Set(tri->UV[0].U * alpha + tri->UV[1].U * beta + tri->UV[2].U * gamma,
                            tri->UV[0].V * alpha + tri->UV[1].V * beta + tri->UV[2].V * gamma);
        Vector3::Cross(tri->Vertex[1] - tri->Vertex[0], tri->Vertex[2] - tri->Vertex[0], surface.GeometryNormal);
        surface.GeometryNormal.Normalize();
        surface.ShadingNormal = surface.GeometryNormal;
    }

    // the primitive's part (world space)
    if (identity) {
        surface.GeometryBasisWS.InitFromW(surface.GeometryNormal);
        surface.ShadingBasisWS.InitFromW(surface.ShadingNormal);
        surface.PointWS = p_ray.PointAlongRay(p_fDistance);
        surface.RayOrigin = surface.RayOriginWS = p_ray.Origin;
        surface.RayDirection = surface.RayDirectionWS = p_ray.Direction;
        p_intersection.WorldTransform.Reset();
    } else {
        Vector3 geometryNormalWS, shadingNormalWS;
        xf.Rotate(surface.GeometryNormal, geometryNormalWS);
        surface.GeometryBasisWS.InitFromW(geometryNormalWS);
        xf.Rotate(surface.ShadingNormal, shadingNormalWS);
        surface.ShadingBasisWS.InitFromW(shadingNormalWS);
        surface.PointWS = p_ray.PointAlongRay(p_fDistance);
        surface.RayOriginWS = p_ray.Origin;
        surface.RayDirectionWS = p_ray.Direction;
        surface.RayOrigin = objectRay.Origin;
        surface.RayDirection = objectRay.Direction;
        p_intersection.WorldTransform = xf;
    }
    p_intersection.SetPrimitive(range.primitive);
    p_intersection.SetLight(NULL);
    IMaterial *material = geometric->GetMaterial();
    if (material != NULL && material->IsComposite()) {
        MaterialGroup *group = (MaterialGroup *)material;
        if (surface.GeometryFragment.HasGroup())
            p_intersection.SetMaterial(group->GetByGroupId(surface.GeometryFragment.GetGroupId()));
        else if (surface.GetShape()->HasGroup())
            p_intersection.SetMaterial(group->GetByGroupId(surface.GetShape()->GetGroupId()));
        else
            p_intersection.SetMaterial(group->GetByIndex(0));
    } else {
        p_intersection.SetMaterial(material);
    }
    if (range.light) p_intersection.SetLight(range.light);
}

bool GpuSpace::Intersects(const Ray &p_ray, Intersection &p_intersection) const
{
    bool hit = false;
    IntersectsBatch(&p_ray, 1, &p_intersection, &hit);
    return hit;
}

bool GpuSpace::Intersects(const Ray &p_ray, Intersection &p_intersection, IPrimitive *p_pExclude) const
{
    const PrimitiveRange *skip = p_pExclude ? FindRange(p_pExclude) : NULL;
    if (!skip) return Intersects(p_ray, p_intersection);
    std::lock_guard<std::mutex> lock(m_mutex);
    StageRays(&p_ray, 1);
    Check(ilg_intersect_excluding(m_pContext, m_pOrigin4, m_pDirection4, 1, skip->first, skip->count, m_prim.data(),
                                  m_t.data(), m_u.data(), m_v.data(), 0),
          "ilg_intersect_excluding");
    if (m_prim[0] < 0) return false;
    FillIntersection(p_ray, m_prim[0], m_t[0], m_u[0], m_v[0], p_intersection);
    return true;
}

bool GpuSpace::Intersects(const Ray &p_ray) const
{
    bool occluded = false;
    OccludedBatch(&p_ray, 1, &occluded);
    return occluded;
}

bool GpuSpace::Intersects(const Ray &p_ray, IPrimitive *p_pExclude) const
{
    const PrimitiveRange *skip = p_pExclude ? FindRange(p_pExclude) : NULL;
    if (!skip) return Intersects(p_ray);
    std::lock_guard<std::mutex> lock(m_mutex);
    StageRays(&p_ray, 1);
    Check(ilg_occluded_excluding(m_pContext, m_pOrigin4, m_pDirection4, 1, skip->first, skip->count, m_occluded.data(), 0),
          "ilg_occluded_excluding");
    return m_occluded[0] != 0;
}

void GpuSpace::IntersectsBatch(const Ray *p_pRays, size_t p_nCount, Intersection *p_pIntersection,
                               bool *p_pHit) const
{
    if (p_nCount == 0) return;
    if (p_nCount > 0xffffffffu) throw Exception("GpuSpace: batch too large", __FILE__, __LINE__);
    std::lock_guard<std::mutex> lock(m_mutex);
    StageRays(p_pRays, p_nCount);
    Check(ilg_intersect(m_pContext, m_pOrigin4, m_pDirection4, (uint32_t)p_nCount, m_prim.data(), m_t.data(), m_u.data(),
                        m_v.data(), 0),
          "ilg_intersect");
    for (size_t i = 0; i < p_nCount; i++) {
        p_pHit[i] = m_prim[i] >= 0;
        if (p_pHit[i]) FillIntersection(p_pRays[i], m_prim[i], m_t[i], m_u[i], m_v[i], p_pIntersection[i]);
    }
}

void GpuSpace::OccludedBatch(const Ray *p_pRays, size_t p_nCount, bool *p_pOccluded) const
{
    if (p_nCount == 0) return;
    if (p_nCount > 0xffffffffu) throw Exception("GpuSpace: batch too large", __FILE__, __LINE__);
    std::lock_guard<std::mutex> lock(m_mutex);
    StageRays(p_pRays, p_nCount);
    Check(ilg_occluded(m_pContext, m_pOrigin4, m_pDirection4, (uint32_t)p_nCount, m_occluded.data(), 0), "ilg_occluded");
    for (size_t i = 0; i < p_nCount; i++) p_pOccluded[i] = m_occluded[i] != 0;
}

}  // namespace PlugIn
}  // namespace Illumina
