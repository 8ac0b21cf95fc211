// GpuPathIntegrator: the reference's PathIntegrator
// (Core/Integrator/PathIntegrator.h:19-50) whose bounce loop runs on the
// device, with the settings of the device renderer's learned radiance cache
// attached. It is what a scene script's Integrator { Type = GPU ... } makes
// (factory "GPU" in the IntegratorManager, registered by the plug-in).
//
// Under the reference's own renderers (BasicRenderer and the others, which
// call Radiance once per pixel sample) both Radiance overloads run the path
// on the device: the first intersection is found by the scene (so
// p_intersection and the RadianceContext's spatial fields are filled as
// PathIntegrator::Radiance fills them), and the path itself, started with the
// same ray, is one ilg_radiance call (Direct, Indirect and Albedo come back).
// There is no CPU path: the scene's space must be a GpuSpace, the
// materials and lights ones the device renders (DeviceScene.h), one shadow
// ray per light, and Cache = MLP is refused there (the cache trains on
// whole regions; use GpuRenderer). Calls are serialised on one device
// context. Under GpuRenderer its RayDepth and
// Epsilon drive the device path tracer as a PathIntegrator's do, and with
// Cache = MLP rendering paths stop into the radiance cache at their
// CacheDepth-th bounce vertex while one path in 1 / TrainFraction trains it
// (TrainSteps Adam steps of TrainBatch records, at LearningRate, after every
// rendered region); a training path stops into the cache TrainTail vertices
// later and the cache's answer completes its targets (0: it is traced to
// RayDepth). The reference has no such
// cache; its nearest relative is the irradiance cache of
// Core/Integrator/ICIntegrator.*.
#pragma once

#include <cstdint>
#include <mutex>
#include <string>

#include "Integrator/PathIntegrator.h"

namespace Illumina {
namespace PlugIn {

struct RadianceCacheSettings {
    bool enabled;
    uint32_t depth;         // bounce vertex where rendering paths stop into the cache (>= 1)
    uint32_t train_every;   // one training path in this many
    uint32_t train_steps;   // Adam steps after each rendered region (0 = frozen)
    uint32_t train_batch;   // records per step
    uint32_t train_tail;    // training paths stop into the cache this many vertices after
                            // the query vertex (self-training); 0 = traced to RayDepth
    uint32_t train_epochs;  // passes over each region's training records
    float learning_rate;
    uint32_t seed;          // network initialisation

    RadianceCacheSettings(void)
        : enabled(false), depth(1), train_every(16), train_steps(4), train_batch(16384), train_tail(2),
          train_epochs(2), learning_rate(1e-2f), seed(1)
    {
    }
};

class GpuPathIntegrator : public Illumina::Core::PathIntegrator {
public:
    GpuPathIntegrator(const std::string &p_strName, int p_nMaxRayDepth, int p_nShadowSampleCount,
                      float p_fReflectEpsilon, const RadianceCacheSettings &p_cache);
    GpuPathIntegrator(int p_nMaxRayDepth, int p_nShadowSampleCount, float p_fReflectEpsilon,
                      const RadianceCacheSettings &p_cache);

    const RadianceCacheSettings &GetCacheSettings(void) const { return m_cache; }
    std::string ToString(void) const { return "GpuPathIntegrator"; }

    // IIntegrator::Radiance on the device (see above).
    Illumina::Core::Spectrum Radiance(Illumina::Core::IntegratorContext *p_pContext,
                                      Illumina::Core::Scene *p_pScene, const Illumina::Core::Ray &p_ray,
                                      Illumina::Core::Intersection &p_intersection,
                                      Illumina::Core::RadianceContext *p_pRadianceContext = NULL);
    Illumina::Core::Spectrum Radiance(Illumina::Core::IntegratorContext *p_pContext,
                                      Illumina::Core::Scene *p_pScene, Illumina::Core::Intersection &p_intersection,
                                      Illumina::Core::RadianceContext *p_pRadianceContext = NULL);

    // Paths started so far; the next call's sample sequence starts after them.
    uint64_t GetPathCount(void) const { return m_nPaths; }

private:
    // The path of p_ray (its first hit p_intersection, found by the scene)
    // traced on the device.
    Illumina::Core::Spectrum DeviceRadiance(Illumina::Core::Scene *p_pScene, const Illumina::Core::Ray &p_ray,
                                            Illumina::Core::Intersection &p_intersection,
                                            Illumina::Core::RadianceContext *p_pRadianceContext);

    RadianceCacheSettings m_cache;
    std::mutex m_mutex;
    uint64_t m_nPaths;
};

}  // namespace PlugIn
}  // namespace Illumina
