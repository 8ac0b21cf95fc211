// The plug-in that registers the device space and renderer with the engine:
// factory "GPU" in the EngineKernel's SpaceManager (System/EngineKernel.h:54,
// FactoryManager<ISpace>, Space/Space.h:42) makes a GpuSpace, and factory
// "GPU" in its RendererManager (FactoryManager<IRenderer>,
// Renderer/Renderer.h:80) makes a GpuRenderer, so a scene description naming
// space or renderer type "GPU" gets the device path. It exports the
// symbol set that the reference's LibraryManager looks up in a plug-in
// library (System/LibrarySymbols.h, System/LibraryManager.cpp:62-170):
// GetPlugInSingleton, DisposePlugInSingleton, CreatePlugInInstance,
// GetPlugInInstance, DisposePlugInInstance, DisposePlugInInstances.
//
// Factory "GPU" in its IntegratorManager makes a GpuPathIntegrator, a
// PathIntegrator that also carries the settings of the device renderer's
// radiance cache.
//
// Factory arguments (ArgumentMap). Space: Id (instance name), Device (CUDA
// ordinal, default 0). Renderer: Id, Samples (per pixel, default 1, as
// BasicRendererFactory, Renderer/RendererFactories.h:34-44), Seed (default 1).
// Integrator: Id, RayDepth (6), ShadowRays (1), Epsilon (1e-4), as the
// reference's PathIntegratorFactory (Integrator/IntegratorFactories.h:41-58);
// Cache (None or MLP, default None), CacheDepth (1), TrainFraction (1/16),
// TrainSteps (4), TrainBatch (16384), TrainTail (2), TrainEpochs (2),
// LearningRate (0.01), CacheSeed (1).
// Bad values throw the engine's Exception, as its factories do.
#include <cmath>
#include <string>

#include "Exception/Exception.h"
#include "GpuPathIntegrator.h"
#include "GpuRenderer.h"
#include "GpuSpace.h"
#include "System/ArgumentMap.h"
#include "System/EngineKernel.h"
#include "System/Factory.h"
#include "System/LibrarySymbols.h"
#include "System/PlugIn.h"
#include "System/Version.h"

using namespace Illumina::Core;

namespace Illumina {
namespace PlugIn {

class GpuSpaceFactory : public Factory<ISpace> {
public:
    ISpace *CreateInstance(void) { return new GpuSpace(); }

    ISpace *CreateInstance(ArgumentMap &p_argumentMap)
    {
        std::string id = "GpuSpace";
        int device = 0;
        p_argumentMap.GetArgument("Id", id);
        p_argumentMap.GetArgument("Device", device);
        return new GpuSpace(id, device);
    }
};

class GpuRendererFactory : public Factory<IRenderer> {
public:
    IRenderer *CreateInstance(void) { return new GpuRenderer(); }

    IRenderer *CreateInstance(ArgumentMap &p_argumentMap)
    {
        int samples = 1, seed = 1;
        std::string id = "GpuRenderer";
        p_argumentMap.GetArgument("Samples", samples);
        p_argumentMap.GetArgument("Seed", seed);
        p_argumentMap.GetArgument("Id", id);
        return new GpuRenderer(id, NULL, NULL, NULL, NULL, NULL, samples, (uint32_t)seed);
    }
};

class GpuPathIntegratorFactory : public Factory<IIntegrator> {
public:
    IIntegrator *CreateInstance(void) { return new GpuPathIntegrator(6, 1, 1e-4f, RadianceCacheSettings()); }

    IIntegrator *CreateInstance(ArgumentMap &p_argumentMap)
    {
        int depth = 6, shadow = 1, cache_depth = 1, steps = 4, batch = 16384, tail = 2, epochs = 2, seed = 1;
        float epsilon = 1e-4f, fraction = 1.f / 16.f, lr = 1e-2f;
        std::string id, cache = "None";
        p_argumentMap.GetArgument("RayDepth", depth);
        p_argumentMap.GetArgument("ShadowRays", shadow);
        p_argumentMap.GetArgument("Epsilon", epsilon);
        p_argumentMap.GetArgument("Cache", cache);
        p_argumentMap.GetArgument("CacheDepth", cache_depth);
        p_argumentMap.GetArgument("TrainFraction", fraction);
        p_argumentMap.GetArgument("TrainSteps", steps);
        p_argumentMap.GetArgument("TrainBatch", batch);
        p_argumentMap.GetArgument("TrainTail", tail);
        p_argumentMap.GetArgument("TrainEpochs", epochs);
        p_argumentMap.GetArgument("LearningRate", lr);
        p_argumentMap.GetArgument("CacheSeed", seed);

        RadianceCacheSettings c;
        if (cache == "MLP")
            c.enabled = true;
        else if (cache != "None")
            throw new Exception("GpuPathIntegratorFactory: Cache must be None or MLP, not '" + cache + "'");
        if (c.enabled && (cache_depth < 1 || cache_depth >= depth))
            throw new Exception("GpuPathIntegratorFactory: CacheDepth must be at least 1 and below RayDepth");
        if (!(fraction > 0.f && fraction <= 1.f))
            throw new Exception("GpuPathIntegratorFactory: TrainFraction must be in (0, 1]");
        if (steps < 0 || batch < 1 || !(lr > 0.f) || tail < 0 || tail > 64 || epochs < 1 || epochs > 64)
            throw new Exception(
                "GpuPathIntegratorFactory: TrainSteps >= 0, TrainBatch >= 1, TrainTail 0..64, TrainEpochs 1..64, "
                "LearningRate > 0");
        c.depth = (uint32_t)cache_depth;
        c.train_every = (uint32_t)std::max(1.f, std::floor(1.f / fraction + 0.5f));
        c.train_steps = (uint32_t)steps;
        c.train_batch = (uint32_t)batch;
        c.train_tail = (uint32_t)tail;
        c.train_epochs = (uint32_t)epochs;
        c.learning_rate = lr;
        c.seed = (uint32_t)seed;
        if (p_argumentMap.GetArgument("Id", id)) return new GpuPathIntegrator(id, depth, shadow, epsilon, c);
        return new GpuPathIntegrator(depth, shadow, epsilon, c);
    }
};

class GpuPlugIn : public IPlugIn {
public:
    GpuPlugIn(void)
        : m_strName("GPU Space"), m_version(1, 0, 0), m_pFactory(NULL), m_pRendererFactory(NULL),
          m_pIntegratorFactory(NULL)
    {
    }
    ~GpuPlugIn(void)
    {
        delete m_pFactory;
        delete m_pRendererFactory;
        delete m_pIntegratorFactory;
    }

    const std::string &GetName(void) const { return m_strName; }
    const Version &GetVersion(void) const { return m_version; }

    void Register(EngineKernel *p_pEngineKernel)
    {
        if (!m_pFactory) m_pFactory = new GpuSpaceFactory();
        if (!m_pRendererFactory) m_pRendererFactory = new GpuRendererFactory();
        if (!m_pIntegratorFactory) m_pIntegratorFactory = new GpuPathIntegratorFactory();
        p_pEngineKernel->GetSpaceManager()->RegisterFactory("GPU", m_pFactory);
        p_pEngineKernel->GetRendererManager()->RegisterFactory("GPU", m_pRendererFactory);
        p_pEngineKernel->GetIntegratorManager()->RegisterFactory("GPU", m_pIntegratorFactory);
    }

    void Unregister(EngineKernel *p_pEngineKernel)
    {
        p_pEngineKernel->GetSpaceManager()->UnregisterFactory("GPU");
        p_pEngineKernel->GetRendererManager()->UnregisterFactory("GPU");
        p_pEngineKernel->GetIntegratorManager()->UnregisterFactory("GPU");
    }

    void Initialise(void) {}
    void Shutdown(void) {}

private:
    std::string m_strName;
    Version m_version;
    GpuSpaceFactory *m_pFactory;
    GpuRendererFactory *m_pRendererFactory;
    GpuPathIntegratorFactory *m_pIntegratorFactory;
};

}  // namespace PlugIn
}  // namespace Illumina

namespace {
Illumina::PlugIn::GpuPlugIn *g_pGpuPlugIn = NULL;
}

// One plug-in object serves every handle: the space factory holds no state.
extern "C" {

__attribute__((visibility("default"))) IPlugIn *GetPlugInSingleton(void)
{
    if (!g_pGpuPlugIn) g_pGpuPlugIn = new Illumina::PlugIn::GpuPlugIn();
    return g_pGpuPlugIn;
}

__attribute__((visibility("default"))) void DisposePlugInSingleton(void)
{
    delete g_pGpuPlugIn;
    g_pGpuPlugIn = NULL;
}

__attribute__((visibility("default"))) PlugInHandle CreatePlugInInstance(void)
{
    GetPlugInSingleton();
    return (PlugInHandle)1;
}

__attribute__((visibility("default"))) IPlugIn *GetPlugInInstance(PlugInHandle p_hInstance)
{
    return p_hInstance ? GetPlugInSingleton() : NULL;
}

__attribute__((visibility("default"))) void DisposePlugInInstance(PlugInHandle p_hInstance) { (void)p_hInstance; }

__attribute__((visibility("default"))) void DisposePlugInInstances(void) { DisposePlugInSingleton(); }

// Why the last Initialise/Build of a GpuSpace failed ("" when it did not, or
// when the space is not a GpuSpace): ISpace::Build reports only a bool.
__attribute__((visibility("default"))) const char *GpuSpaceLastError(const ISpace *p_pSpace)
{
    const Illumina::PlugIn::GpuSpace *space = dynamic_cast<const Illumina::PlugIn::GpuSpace *>(p_pSpace);
    return space ? space->GetLastError().c_str() : "";
}

}  // extern "C"
