// GpuSpace: an ISpace (Core/Space/Space.h:20-43) whose ray queries run on
// the B200 through the C ABI of libilg.so (include/ilg.h). It is a drop-in
// for BasicSpace (Core/Space/BasicSpace.cpp) under the reference's Scene,
// integrators and renderers: the same four Intersects overloads, the same
// Intersection record on a hit, the same untouched record on a miss.
//
// Build() flattens every primitive's triangles, in PrimitiveList order, into
// one world-space triangle array and builds the device BVH over it. Shapes:
// ITriangleMesh (every mesh kind: BasicMesh, KDTreeMesh, BVHMesh, ...),
// Quad (its two tessellated triangles) and Triangle. Any other shape (Sphere,
// PersistentMesh) makes Build() return false, with the reason in
// GetLastError(); there is no CPU fallback.
//
// Hit records are filled the way GeometricPrimitive::Intersects
// (Scene/GeometricPrimitive.cpp:60-180) fills them after
// IndexedTriangle::Intersects (Shape/IndexedTriangle.cpp:92-243) or
// Triangle::Intersects (Shape/Triangle.cpp:107-163), and
// EmissivePrimitive::Intersects (Scene/EmissivePrimitive.cpp:27-33) adds its
// light. Distance, beta and gamma come from the device in the reference's
// own arithmetic, so for untransformed primitives every field equals the
// reference's bit for bit. Primitives with a WorldTransform are traced in
// world space (their vertices transformed once at Build), where the
// reference intersects the inverse-transformed ray in object space: the hit
// is the same surface up to float rounding of the transform.
//
// The reference's scalar calls each cost one device round trip (tens of
// microseconds); IntersectsBatch / OccludedBatch answer a whole array of rays
// in one launch and are what a wavefront caller should use.
#pragma once

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "Geometry/BoundingBox.h"
#include "Space/Space.h"
#include "ilg.h"

namespace Illumina {
namespace Core {
class GeometricPrimitive;
class ITriangleMesh;
class IndexedTriangle;
class Triangle;
class IAreaLight;
class IMaterial;
}  // namespace Core

namespace PlugIn {

class GpuSpace : public Illumina::Core::ISpace {
public:
    explicit GpuSpace(const std::string &p_strName, int p_nDevice = 0);
    GpuSpace(void);
    ~GpuSpace(void);

    Illumina::Core::IBoundingVolume *GetBoundingVolume(void);

    bool Initialise(void);
    void Shutdown(void);
    bool Update(void);
    bool Build(void);

    bool Intersects(const Illumina::Core::Ray &p_ray, Illumina::Core::Intersection &p_intersection,
                    Illumina::Core::IPrimitive *p_pExclude) const;
    bool Intersects(const Illumina::Core::Ray &p_ray, Illumina::Core::Intersection &p_intersection) const;
    bool Intersects(const Illumina::Core::Ray &p_ray, Illumina::Core::IPrimitive *p_pExclude) const;
    bool Intersects(const Illumina::Core::Ray &p_ray) const;

    // Batched forms of the two hot overloads. p_pHit[i] says whether ray i
    // hit; p_pIntersection[i] is written only for hits, as above.
    void IntersectsBatch(const Illumina::Core::Ray *p_pRays, size_t p_nCount,
                         Illumina::Core::Intersection *p_pIntersection, bool *p_pHit) const;
    void OccludedBatch(const Illumina::Core::Ray *p_pRays, size_t p_nCount, bool *p_pOccluded) const;

    // Triangles handed to the device (valid after Build).
    size_t GetTriangleCount(void) const { return m_triangles.size(); }

    // For a device renderer over this space (GpuRenderer): the device
    // context, the material of every device triangle as a slot into
    // GetMaterialSlots() (one slot per distinct IMaterial*, MaterialGroups
    // resolved per triangle as the hit record resolves them; a primitive
    // without material gets a NULL slot), a primitive's triangle range, and
    // a counter that changes with every successful Build.
    ilg_ctx *GetContext(void) const { return m_pContext; }
    const std::vector<Illumina::Core::IMaterial *> &GetMaterialSlots(void) const { return m_materials; }
    bool GetTriangleRange(const Illumina::Core::IPrimitive *p_pPrimitive, uint32_t &p_nFirst,
                          uint32_t &p_nCount) const;
    uint64_t GetBuildCount(void) const { return m_nBuildCount; }
    const std::string &GetLastError(void) const { return m_strLastError; }

    // Whether the device's materials and lights were last uploaded for this
    // scene and this build (PrepareDeviceScene, DeviceScene.h).
    bool IsPreparedFor(const void *p_pScene) const
    {
        return m_pPreparedScene == p_pScene && m_nPreparedBuild == m_nBuildCount;
    }
    void SetPreparedFor(const void *p_pScene)
    {
        m_pPreparedScene = p_pScene;
        m_nPreparedBuild = m_nBuildCount;
    }
    std::string ToString(void) const { return "GpuSpace"; }

private:
    // What produced one device triangle.
    struct TriangleSource {
        uint32_t primitive;      // index into PrimitiveList at Build time
        uint32_t kind;           // kMesh or kTriangle
        const void *shape;       // the IndexedTriangle or the Triangle
        const Illumina::Core::ITriangleMesh *mesh;
    };
    struct PrimitiveRange {
        Illumina::Core::IPrimitive *primitive;
        Illumina::Core::GeometricPrimitive *geometric;
        Illumina::Core::IAreaLight *light;  // EmissivePrimitive's light, else null
        uint32_t first, count;              // its triangles in the device array
    };
    static const uint32_t kMesh = 0, kTriangle = 1;

    bool Fail(const std::string &p_strReason);
    void Check(int p_nStatus, const char *p_szWhere) const;
    const PrimitiveRange *FindRange(const Illumina::Core::IPrimitive *p_pPrimitive) const;
    void StageRays(const Illumina::Core::Ray *p_pRays, size_t p_nCount) const;
    void FillIntersection(const Illumina::Core::Ray &p_ray, int32_t p_nTriangle, float p_fDistance, float p_fBeta,
                          float p_fGamma, Illumina::Core::Intersection &p_intersection) const;

    int m_nDevice;
    ilg_ctx *m_pContext;
    bool m_bBuilt;
    Illumina::Core::AxisAlignedBoundingBox m_aabb;
    std::vector<TriangleSource> m_triangles;
    std::vector<PrimitiveRange> m_ranges;
    std::vector<Illumina::Core::IMaterial *> m_materials;
    uint64_t m_nBuildCount;
    const void *m_pPreparedScene;
    uint64_t m_nPreparedBuild;
    std::string m_strLastError;

    // staging for the device calls (guarded by m_mutex)
    mutable std::mutex m_mutex;
    mutable std::vector<float> m_origin, m_direction, m_t, m_u, m_v;
    mutable float *m_pOrigin4, *m_pDirection4;  // 16-byte aligned views of m_origin, m_direction
    mutable std::vector<int32_t> m_prim;
    mutable std::vector<uint8_t> m_occluded;
};

}  // namespace PlugIn
}  // namespace Illumina
