// GpuRenderer: IRenderer over the device path tracer. See GpuRenderer.h.
#include "GpuRenderer.h"

#include <cstring>
#include <memory>
#include <sstream>
#include <vector>

#include "Camera/Camera.h"
#include "Device/Device.h"
#include "DeviceScene.h"
#include "EngineAccess.h"
#include "Exception/Exception.h"
#include "Geometry/Intersection.h"
#include "GpuPathIntegrator.h"
#include "GpuSpace.h"
#include "Integrator/PathIntegrator.h"
#include "Scene/Scene.h"

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

}  // namespace

GpuRenderer::GpuRenderer(const std::string &p_strName, Scene *p_pScene, IIntegrator *p_pIntegrator,
                         IDevice *p_pDevice, IFilter *p_pFilter, RadianceBuffer *p_pRadianceBuffer,
                         int p_nSampleCount, uint32_t p_nSeed)
    : BaseRenderer(p_strName, p_pScene, p_pIntegrator, p_pDevice, p_pFilter, p_pRadianceBuffer, p_nSampleCount),
      m_nSeed(p_nSeed), m_pCacheContext(NULL), m_nCacheBuild(0)
{
}

GpuRenderer::GpuRenderer(Scene *p_pScene, IIntegrator *p_pIntegrator, IDevice *p_pDevice, IFilter *p_pFilter,
                         RadianceBuffer *p_pRadianceBuffer, int p_nSampleCount, uint32_t p_nSeed)
    : BaseRenderer(p_pScene, p_pIntegrator, p_pDevice, p_pFilter, p_pRadianceBuffer, p_nSampleCount),
      m_nSeed(p_nSeed), m_pCacheContext(NULL), m_nCacheBuild(0)
{
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
    GpuSpace *space = PrepareDeviceScene(m_pScene, "GpuRenderer");
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
    // the view ray of every pixel (its corner sample, as RenderRegion's last
    // GetRay would make it) and its first hit, in one batched device query:
    // the spatial fields PathIntegrator::Radiance sets from that hit
    // (RadianceContext::SetSpatialContext, Core/Geometry/Intersection.h:92-103)
    std::vector<Ray> rays(n);
    std::vector<Intersection> hits(n);
    std::unique_ptr<bool[]> hit(new bool[n]);
    for (int j = 0; j < p_nRegionHeight; j++)
        for (int i = 0; i < p_nRegionWidth; i++)
            m_pScene->GetCamera()->GetRay((p_nRegionX + i) * rcpWidth, (p_nRegionY + j) * rcpHeight, 0.f, 0.f,
                                          rays[(size_t)j * p_nRegionWidth + i]);
    space->IntersectsBatch(rays.data(), n, hits.data(), hit.get());
    for (int j = 0; j < p_nRegionHeight; j++) {
        for (int i = 0; i < p_nRegionWidth; i++) {
            const size_t p = (size_t)j * p_nRegionWidth + i, k = 3 * p;
            RadianceContext *rc = p_pRadianceBuffer->GetP(p_nBufferX + i, p_nBufferY + j);
            rc->Final = Spectrum(final_rgb[k], final_rgb[k + 1], final_rgb[k + 2]);
            rc->Direct = Spectrum(direct_rgb[k], direct_rgb[k + 1], direct_rgb[k + 2]);
            rc->Indirect = rc->Final - rc->Direct;
            rc->Albedo = Spectrum(albedo_rgb[k], albedo_rgb[k + 1], albedo_rgb[k + 2]);
            rc->ViewRay = rays[p];
            if (hit[p]) rc->SetSpatialContext(&hits[p]);
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
