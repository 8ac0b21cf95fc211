// GpuRenderer: IRenderer over the device path tracer. See GpuRenderer.h.
#include "GpuRenderer.h"

#include <cstring>
#include <sstream>
#include <vector>

#include "Camera/Camera.h"
#include "Device/Device.h"
#include "EngineAccess.h"
#include "Exception/Exception.h"
#include "Geometry/Intersection.h"
#include "GpuPathIntegrator.h"
#include "GpuSpace.h"
#include "Integrator/PathIntegrator.h"
#include "Light/DiffuseAreaLight.h"
#include "Material/Glass.h"
#include "Material/Matte.h"
#include "Material/Mirror.h"
#include "Scene/EmissivePrimitive.h"
#include "Scene/Scene.h"
#include "Shape/Quad.h"

using namespace Illumina::Core;

namespace Illumina {
namespace PlugIn {

namespace {

void Refuse(const std::string &p_strWhat) { throw Exception("GpuRenderer: " + p_strWhat, __FILE__, __LINE__); }

void Check(ilg_ctx *p_pContext, int p_nStatus, const char *p_szWhere)
{
    if (p_nStatus == ILG_OK) return;
    std::ostringstream s;
    s << p_szWhere << " failed (status " << p_nStatus << "): " << ilg_last_error(p_pContext);
    Refuse(s.str());
}

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

GpuRenderer::GpuRenderer(const std::string &p_strName, Scene *p_pScene, IIntegrator *p_pIntegrator,
                         IDevice *p_pDevice, IFilter *p_pFilter, RadianceBuffer *p_pRadianceBuffer,
                         int p_nSampleCount, uint32_t p_nSeed)
    : BaseRenderer(p_strName, p_pScene, p_pIntegrator, p_pDevice, p_pFilter, p_pRadianceBuffer, p_nSampleCount),
      m_nSeed(p_nSeed), m_pPreparedScene(NULL), m_nPreparedBuild(0), m_pCacheContext(NULL), m_nCacheBuild(0)
{
}

GpuRenderer::GpuRenderer(Scene *p_pScene, IIntegrator *p_pIntegrator, IDevice *p_pDevice, IFilter *p_pFilter,
                         RadianceBuffer *p_pRadianceBuffer, int p_nSampleCount, uint32_t p_nSeed)
    : BaseRenderer(p_pScene, p_pIntegrator, p_pDevice, p_pFilter, p_pRadianceBuffer, p_nSampleCount),
      m_nSeed(p_nSeed), m_pPreparedScene(NULL), m_nPreparedBuild(0), m_pCacheContext(NULL), m_nCacheBuild(0)
{
}

GpuSpace *GpuRenderer::PrepareScene(void)
{
    if (!m_pScene) Refuse("no scene");
    GpuSpace *space = dynamic_cast<GpuSpace *>(m_pScene->GetSpace());
    if (!space) Refuse("the scene's space is not a GpuSpace");
    ilg_ctx *ctx = space->GetContext();
    if (!ctx || space->GetBuildCount() == 0) Refuse("the GpuSpace has not been built");
    if (m_pPreparedScene == m_pScene && m_nPreparedBuild == space->GetBuildCount()) return space;

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

    // lights: each a DiffuseAreaLight on a Quad whose primitive is in the space
    std::vector<ilg_quad_light> lights;
    for (int l = 0, n = (int)m_pScene->LightList.Size(); l < n; l++) {
        ILight *light = m_pScene->LightList[l];
        const DiffuseAreaLight *area = dynamic_cast<const DiffuseAreaLight *>(light);
        if (!area) Refuse("light " + light->GetName() + " is not a DiffuseAreaLight");
        const Quad *quad = dynamic_cast<const Quad *>(area->GetShape());
        if (!quad) Refuse("area light " + light->GetName() + " is not on a Quad");
        uint32_t first = 0, count = 0;
        bool found = false;
        for (int p = 0, np = (int)space->PrimitiveList.Size(); p < np && !found; p++) {
            const EmissivePrimitive *ep = dynamic_cast<const EmissivePrimitive *>(space->PrimitiveList[p]);
            if (ep && ep->GetLight() == area && ep->GetShape() == quad)
                found = space->GetTriangleRange(ep, first, count);
        }
        if (!found || count != 2) Refuse("area light " + light->GetName() + " has no emissive primitive in the space");
        // the reference's vertex order from its tessellation: (v1, v3, v2), (v1, v4, v3)
        const Triangle *half = Access::QuadTriangles::Of(quad);
        Vector3 v[4] = {half[0].Vertex[0], half[0].Vertex[2], half[0].Vertex[1], half[1].Vertex[1]};
        const Transformation *xf = area->GetWorldTransform();
        ilg_quad_light q;
        std::memset(&q, 0, sizeof(q));
        for (int c = 0; c < 4; c++) Put(q.v[c], (xf && !xf->IsIdentity()) ? xf->Apply(v[c]) : v[c]);
        const Spectrum &e = Access::AreaLight::Emit(area);
        q.emit[0] = e[0];
        q.emit[1] = e[1];
        q.emit[2] = e[2];
        q.first_tri = first;
        lights.push_back(q);
    }
    Check(ctx, ilg_set_quad_lights(ctx, lights.empty() ? NULL : lights.data(), (uint32_t)lights.size()),
          "ilg_set_quad_lights");
    m_pPreparedScene = m_pScene;
    m_nPreparedBuild = space->GetBuildCount();
    return space;
}

void GpuRenderer::RenderRegion(RadianceBuffer *p_pRadianceBuffer, int p_nRegionX, int p_nRegionY,
                               int p_nRegionWidth, int p_nRegionHeight, int p_nBufferX, int p_nBufferY)
{
    if (!p_pRadianceBuffer || !m_pDevice || !m_pIntegrator) Refuse("buffer, device and integrator must be set");
    if (!m_pScene || !m_pScene->GetCamera()) Refuse("no scene camera");
    if (p_nRegionWidth <= 0 || p_nRegionHeight <= 0) return;
    if (p_nRegionX < 0 || p_nRegionY < 0 || p_nBufferX < 0 || p_nBufferY < 0 ||
        p_nBufferX + p_nRegionWidth > (int)p_pRadianceBuffer->GetWidth() ||
        p_nBufferY + p_nRegionHeight > (int)p_pRadianceBuffer->GetHeight())
        Refuse("region outside the radiance buffer");
    const PathIntegrator *path = dynamic_cast<const PathIntegrator *>(m_pIntegrator);
    if (!path) Refuse("the integrator is not a PathIntegrator");
    if (Access::PathTracer::ShadowSampleCount(path) != 1) Refuse("more than one shadow ray per light");
    if (m_nSampleCount < 1) Refuse("sample count below 1");
    GpuSpace *space = PrepareScene();
    ilg_ctx *ctx = space->GetContext();

    ilg_camera_frame frame;
    Vector3 centre, corner, across, up;
    Access::Camera::Frame(m_pScene->GetCamera(), centre, corner, across, up);
    Put(frame.centre, centre);
    Put(frame.corner, corner);
    Put(frame.across, across);
    Put(frame.up, up);

    ilg_render_opts opts;
    std::memset(&opts, 0, sizeof(opts));
    opts.width = (uint32_t)m_pDevice->GetWidth();
    opts.height = (uint32_t)m_pDevice->GetHeight();
    opts.spp = (uint32_t)m_nSampleCount;
    opts.max_depth = (uint32_t)Access::PathTracer::MaxRayDepth(path);
    opts.epsilon = Access::PathTracer::ReflectEpsilon(path);
    opts.seed = m_nSeed;
    const GpuPathIntegrator *gpu = dynamic_cast<const GpuPathIntegrator *>(path);
    if (gpu && gpu->GetCacheSettings().enabled) {
        const RadianceCacheSettings &c = gpu->GetCacheSettings();
        if (c.depth < 1 || c.depth >= opts.max_depth) Refuse("the radiance cache depth must be in [1, RayDepth)");
        // a fresh network for every built scene; it then learns across regions and frames
        if (m_pCacheContext != ctx || m_nCacheBuild != space->GetBuildCount()) {
            Check(ctx, ilg_mlp_init(ctx, c.seed, c.learning_rate), "ilg_mlp_init");
            m_pCacheContext = ctx;
            m_nCacheBuild = space->GetBuildCount();
        }
        opts.cache_depth = c.depth;
        opts.train_every = c.train_every;
        opts.train_steps = c.train_steps;
        opts.train_batch = c.train_batch;
        opts.train_tail = c.train_tail;
        opts.train_epochs = c.train_epochs;
    }
    ilg_region region = {(uint32_t)p_nRegionX, (uint32_t)p_nRegionY, (uint32_t)p_nRegionWidth,
                         (uint32_t)p_nRegionHeight};
    const size_t n = (size_t)p_nRegionWidth * p_nRegionHeight;
    std::vector<float> final_rgb(3 * n), direct_rgb(3 * n), albedo_rgb(3 * n);
    Check(ctx, ilg_render_region(ctx, &frame, &opts, &region, final_rgb.data(), direct_rgb.data(),
                                 albedo_rgb.data(), 0),
          "ilg_render_region");

    const float rcpWidth = 1.f / opts.width, rcpHeight = 1.f / opts.height;
    for (int j = 0; j < p_nRegionHeight; j++) {
        for (int i = 0; i < p_nRegionWidth; i++) {
            const size_t k = 3 * ((size_t)j * p_nRegionWidth + i);
            RadianceContext *rc = p_pRadianceBuffer->GetP(p_nBufferX + i, p_nBufferY + j);
            rc->Final = Spectrum(final_rgb[k], final_rgb[k + 1], final_rgb[k + 2]);
            rc->Direct = Spectrum(direct_rgb[k], direct_rgb[k + 1], direct_rgb[k + 2]);
            rc->Indirect = rc->Final - rc->Direct;
            rc->Albedo = Spectrum(albedo_rgb[k], albedo_rgb[k + 1], albedo_rgb[k + 2]);
            // the ray through the pixel's corner sample, as RenderRegion's last GetRay would
            m_pScene->GetCamera()->GetRay((p_nRegionX + i) * rcpWidth, (p_nRegionY + j) * rcpHeight, 0.f, 0.f,
                                          rc->ViewRay);
            rc->Flags |= RadianceContext::DF_Computed;
        }
    }
}

void GpuRenderer::Commit(RadianceBuffer *p_pRadianceBuffer)
{
    BaseRenderer::Commit(p_pRadianceBuffer);
    m_nSeed++;  // the next frame draws new samples
}

}  // namespace PlugIn
}  // namespace Illumina
