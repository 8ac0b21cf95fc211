// GpuPathIntegrator: PathIntegrator plus radiance-cache settings. See GpuPathIntegrator.h.
#include "GpuPathIntegrator.h"

namespace Illumina {
namespace PlugIn {

GpuPathIntegrator::GpuPathIntegrator(const std::string &p_strName, int p_nMaxRayDepth, int p_nShadowSampleCount,
                                     float p_fReflectEpsilon, const RadianceCacheSettings &p_cache)
    : PathIntegrator(p_strName, p_nMaxRayDepth, p_nShadowSampleCount, p_fReflectEpsilon), m_cache(p_cache)
{
}

GpuPathIntegrator::GpuPathIntegrator(int p_nMaxRayDepth, int p_nShadowSampleCount, float p_fReflectEpsilon,
                                     const RadianceCacheSettings &p_cache)
    : PathIntegrator(p_nMaxRayDepth, p_nShadowSampleCount, p_fReflectEpsilon), m_cache(p_cache)
{
}

}  // namespace PlugIn
}  // namespace Illumina
