// Materials and lights of a scene on the device. See DeviceScene.h.
#include "DeviceScene.h"

#include <cstring>
#include <sstream>
#include <vector>

#include "EngineAccess.h"
#include "Exception/Exception.h"
#include "GpuSpace.h"
#include "Light/DiffuseAreaLight.h"
#include "Light/InfiniteAreaLight.h"
#include "Material/Glass.h"
#include "Material/Matte.h"
#include "Material/Mirror.h"
#include "Scene/EmissivePrimitive.h"
#include "Scene/Scene.h"
#include "Shape/Quad.h"
#include "Shape/TriangleMesh.h"

using namespace Illumina::Core;

namespace Illumina {
namespace PlugIn {

namespace {

void Put(float *p_pDst, const Vector3 &p_v)
{
    p_pDst[0] = p_v.X;
    p_pDst[1] = p_v.Y;
    p_pDst[2] = p_v.Z;
}

void PutSpectrum(float *p_pDst, const Spectrum &p_s)
{
    p_pDst[0] = p_s[0];
    p_pDst[1] = p_s[1];
    p_pDst[2] = p_s[2];
}

}  // namespace

GpuSpace *PrepareDeviceScene(Scene *p_pScene, const std::string &p_strWho)
{
    auto Refuse = [&](const std::string &p_strWhat) {
        throw Exception(p_strWho + ": " + p_strWhat, __FILE__, __LINE__);
    };
    auto Check = [&](ilg_ctx *p_pContext, int p_nStatus, const char *p_szWhere) {
        if (p_nStatus == ILG_OK) return;
        std::ostringstream s;
        s << p_szWhere << " failed (status " << p_nStatus << "): " << ilg_last_error(p_pContext);
        Refuse(s.str());
    };
    if (!p_pScene) Refuse("no scene");
    GpuSpace *space = dynamic_cast<GpuSpace *>(p_pScene->GetSpace());
    if (!space) Refuse("the scene's space is not a GpuSpace (the device path tracer has no CPU path)");
    ilg_ctx *ctx = space->GetContext();
    if (!ctx || space->GetBuildCount() == 0) Refuse("the GpuSpace has not been built");
    if (space->IsPreparedFor(p_pScene)) return space;

    // materials, one per slot of the space
    const std::vector<IMaterial *> &slots = space->GetMaterialSlots();
    std::vector<ilg_material> materials(slots.size());
    for (size_t k = 0; k < slots.size(); k++) {
        ilg_material &m = materials[k];
        std::memset(&m, 0, sizeof(m));
        m.kind = ILG_MAT_LAMBERT;
        if (slots[k] == NULL) continue;  // no material: black
        const std::string name = slots[k]->GetName();
        if (const MatteMaterial *matte = dynamic_cast<const MatteMaterial *>(slots[k])) {
            if (Access::Matte::Texture(matte)) Refuse("textured material '" + name + "'");
            PutSpectrum(m.albedo, Access::Matte::Reflectivity(matte));
        } else if (const MirrorMaterial *mirror = dynamic_cast<const MirrorMaterial *>(slots[k])) {
            if (Access::Mirror::Texture(mirror)) Refuse("textured material '" + name + "'");
            m.kind = ILG_MAT_MIRROR;
            PutSpectrum(m.albedo, Access::Mirror::Reflectivity(mirror));
        } else if (const GlassMaterial *glass = dynamic_cast<const GlassMaterial *>(slots[k])) {
            if (Access::Glass::Texture(glass)) Refuse("textured material '" + name + "'");
            const float ei = Access::Glass::EtaI(glass), et = Access::Glass::EtaT(glass);
            if (!(ei > 0.f && et > 0.f)) Refuse("glass material '" + name + "' needs positive indices");
            m.kind = ILG_MAT_GLASS;
            PutSpectrum(m.albedo, Access::Glass::Reflectivity(glass));
            PutSpectrum(m.f0, Access::Glass::Transmittance(glass));
            m.alpha = ei / et;
        } else {
            Refuse("material '" + name + "' is not a MatteMaterial, MirrorMaterial or GlassMaterial");
        }
    }
    Check(ctx, ilg_set_materials(ctx, materials.data(), (uint32_t)materials.size()), "ilg_set_materials");

    // lights, in LightList order
    std::vector<ilg_light> lights;
    for (int l = 0, n = (int)p_pScene->LightList.Size(); l < n; l++) {
        ILight *light = p_pScene->LightList[l];
        ilg_light d;
        std::memset(&d, 0, sizeof(d));
        if (const InfiniteAreaLight *sky = dynamic_cast<const InfiniteAreaLight *>(light)) {
            if (sky->GetTexture()) Refuse("infinite light " + light->GetName() + " has a texture");
            d.kind = ILG_LIGHT_INFINITE;
            PutSpectrum(d.emit, sky->GetIntensity());
            lights.push_back(d);
            continue;
        }
        const DiffuseAreaLight *area = dynamic_cast<const DiffuseAreaLight *>(light);
        if (!area) Refuse("light " + light->GetName() + " is not a DiffuseAreaLight or an InfiniteAreaLight");
        const IShape *shape = area->GetShape();
        const Quad *quad = dynamic_cast<const Quad *>(shape);
        const ITriangleMesh *mesh = dynamic_cast<const ITriangleMesh *>(shape);
        if (!quad && !mesh) Refuse("area light " + light->GetName() + " is not on a Quad or a triangle mesh");
        uint32_t first = 0, count = 0;
        bool found = false;
        for (int p = 0, np = (int)space->PrimitiveList.Size(); p < np && !found; p++) {
            const EmissivePrimitive *ep = dynamic_cast<const EmissivePrimitive *>(space->PrimitiveList[p]);
            if (ep && ep->GetLight() == area && ep->GetShape() == shape)
                found = space->GetTriangleRange(ep, first, count);
        }
        if (!found || count == 0 || (quad && count != 2))
            Refuse("area light " + light->GetName() + " has no emissive primitive in the space");
        const Transformation *xf = area->GetWorldTransform();
        PutSpectrum(d.emit, Access::AreaLight::Emit(area));
        d.first_tri = first;
        if (quad) {
            // the reference's vertex order from its tessellation: (v1, v3, v2), (v1, v4, v3)
            const Triangle *half = Access::QuadTriangles::Of(quad);
            Vector3 v[4] = {half[0].Vertex[0], half[0].Vertex[2], half[0].Vertex[1], half[1].Vertex[1]};
            d.kind = ILG_LIGHT_QUAD;
            for (int c = 0; c < 4; c++) Put(d.v[c], (xf && !xf->IsIdentity()) ? xf->Apply(v[c]) : v[c]);
            d.tri_count = 2;
        } else {
            // the device samples the mesh's world-space triangles; a light
            // with a transform of its own would sample other points
            if (xf && !xf->IsIdentity()) Refuse("mesh light " + light->GetName() + " has a world transform");
            d.kind = ILG_LIGHT_MESH;
            d.tri_count = count;
        }
        lights.push_back(d);
    }
    Check(ctx, ilg_set_lights(ctx, lights.empty() ? NULL : lights.data(), (uint32_t)lights.size()),
          "ilg_set_lights");
    space->SetPreparedFor(p_pScene);
    return space;
}

}  // namespace PlugIn
}  // namespace Illumina
