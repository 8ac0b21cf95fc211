// GpuPathIntegrator: PathIntegrator whose Radiance runs on the device, plus
// radiance-cache settings. See GpuPathIntegrator.h.
#include "GpuPathIntegrator.h"

#include <cstring>
#include <sstream>

#include "DeviceScene.h"
#include "Exception/Exception.h"
#include "Geometry/Intersection.h"
#include "GpuSpace.h"
#include "Scene/Scene.h"
#include "ilg.h"

using namespace Illumina::Core;

namespace Illumina {
namespace PlugIn {

GpuPathIntegrator::GpuPathIntegrator(const std::string &p_strName, int p_nMaxRayDepth, int p_nShadowSampleCount,
                                     float p_fReflectEpsilon, const RadianceCacheSettings &p_cache)
    : PathIntegrator(p_strName, p_nMaxRayDepth, p_nShadowSampleCount, p_fReflectEpsilon), m_cache(p_cache),
      m_nPaths(0)
{
}

GpuPathIntegrator::GpuPathIntegrator(int p_nMaxRayDepth, int p_nShadowSampleCount, float p_fReflectEpsilon,
                                     const RadianceCacheSettings &p_cache)
    : PathIntegrator(p_nMaxRayDepth, p_nShadowSampleCount, p_fReflectEpsilon), m_cache(p_cache), m_nPaths(0)
{
}

// PathIntegrator::Radiance(context, scene, ray, intersection, rc)
// (Core/Integrator/PathIntegrator.cpp:357-367): the scene finds the first
// intersection (a miss keeps the ray in the record), then the path.
Spectrum GpuPathIntegrator::Radiance(IntegratorContext *p_pContext, Scene *p_pScene, const Ray &p_ray,
                                     Intersection &p_intersection, RadianceContext *p_pRadianceContext)
{
    (void)p_pContext;
    if (!p_pScene) throw Exception("GpuPathIntegrator: no scene", __FILE__, __LINE__);
    if (!p_pScene->Intersects(Ray(p_ray), p_intersection)) {
        p_intersection.Surface.RayOriginWS = p_ray.Origin;
        p_intersection.Surface.RayDirectionWS = p_ray.Direction;
    }
    return DeviceRadiance(p_pScene, p_ray, p_intersection, p_pRadianceContext);
}

// PathIntegrator::Radiance(context, scene, intersection, rc)
// (PathIntegrator.cpp:44-355): the path continues the ray stored in the
// intersection record, which the device intersects again with the
// reference's Ray(origin, direction) window [0, FLT_MAX].
Spectrum GpuPathIntegrator::Radiance(IntegratorContext *p_pContext, Scene *p_pScene, Intersection &p_intersection,
                                     RadianceContext *p_pRadianceContext)
{
    (void)p_pContext;
    if (!p_pScene) throw Exception("GpuPathIntegrator: no scene", __FILE__, __LINE__);
    const Ray ray(p_intersection.Surface.RayOriginWS, p_intersection.Surface.RayDirectionWS);
    return DeviceRadiance(p_pScene, ray, p_intersection, p_pRadianceContext);
}

Spectrum GpuPathIntegrator::DeviceRadiance(Scene *p_pScene, const Ray &p_ray, Intersection &p_intersection,
                                           RadianceContext *p_pRadianceContext)
{
    if (m_cache.enabled)
        throw Exception("GpuPathIntegrator: Cache = MLP trains on whole regions and needs GpuRenderer; the "
                        "renderer calling Radiance per sample would leave it untrained",
                        __FILE__, __LINE__);
    if (m_nShadowSampleCount != 1)
        throw Exception("GpuPathIntegrator: the device takes one shadow ray per light", __FILE__, __LINE__);
    std::lock_guard<std::mutex> lock(m_mutex);
    GpuSpace *space = PrepareDeviceScene(p_pScene, "GpuPathIntegrator");
    ilg_ctx *ctx = space->GetContext();

    alignas(16) float o4[4] = {p_ray.Origin.X, p_ray.Origin.Y, p_ray.Origin.Z, p_ray.Min};
    alignas(16) float d4[4] = {p_ray.Direction.X, p_ray.Direction.Y, p_ray.Direction.Z, p_ray.Max};
    ilg_render_opts opts;
    std::memset(&opts, 0, sizeof(opts));
    opts.spp = 1;
    opts.max_depth = (uint32_t)m_nMaxRayDepth;
    opts.epsilon = m_fReflectEpsilon;
    // every call draws a fresh sample sequence (the reference's shared
    // sampler advances with every path)
    opts.seed = (uint32_t)(m_nPaths * 0x9E3779B1ull + 1u);
    m_nPaths++;
    float final_rgb[3], direct_rgb[3], albedo_rgb[3];
    const int status = ilg_radiance(ctx, o4, d4, 1, &opts, final_rgb, direct_rgb, albedo_rgb, 0);
    if (status != ILG_OK) {
        std::ostringstream s;
        s << "GpuPathIntegrator: ilg_radiance failed (status " << status << "): " << ilg_last_error(ctx);
        throw Exception(s.str(), __FILE__, __LINE__);
    }

    RadianceContext local;
    RadianceContext *rc = p_pRadianceContext ? p_pRadianceContext : &local;
    rc->Flags = 0;
    rc->Direct = Spectrum(direct_rgb[0], direct_rgb[1], direct_rgb[2]);
    rc->Albedo = Spectrum(albedo_rgb[0], albedo_rgb[1], albedo_rgb[2]);
    if (!p_intersection.IsValid()) {
        // a missed ray: Direct only (PathIntegrator.cpp:84-92)
        rc->Indirect = 0.f;
        rc->Flags |= RadianceContext::DF_Computed | RadianceContext::DF_Direct;
        return rc->Direct;
    }
    rc->SetSpatialContext(&p_intersection);
    const Spectrum final_s(final_rgb[0], final_rgb[1], final_rgb[2]);
    rc->Indirect = final_s - rc->Direct;
    rc->Flags |= RadianceContext::DF_Albedo | RadianceContext::DF_Direct | RadianceContext::DF_Indirect;
    return rc->Direct + rc->Indirect;
}

}  // namespace PlugIn
}  // namespace Illumina
