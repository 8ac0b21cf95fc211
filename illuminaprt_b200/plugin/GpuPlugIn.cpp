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
// Factory arguments (ArgumentMap). Space: Id (instance name), Device (CUDA
// ordinal, default 0). Renderer: Id, Samples (per pixel, default 1, as
// BasicRendererFactory, Renderer/RendererFactories.h:34-44), Seed (default 1).
#include <string>

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

class GpuPlugIn : public IPlugIn {
public:
    GpuPlugIn(void) : m_strName("GPU Space"), m_version(1, 0, 0), m_pFactory(NULL), m_pRendererFactory(NULL) {}
    ~GpuPlugIn(void)
    {
        delete m_pFactory;
        delete m_pRendererFactory;
    }

    const std::string &GetName(void) const { return m_strName; }
    const Version &GetVersion(void) const { return m_version; }

    void Register(EngineKernel *p_pEngineKernel)
    {
        if (!m_pFactory) m_pFactory = new GpuSpaceFactory();
        if (!m_pRendererFactory) m_pRendererFactory = new GpuRendererFactory();
        p_pEngineKernel->GetSpaceManager()->RegisterFactory("GPU", m_pFactory);
        p_pEngineKernel->GetRendererManager()->RegisterFactory("GPU", m_pRendererFactory);
    }

    void Unregister(EngineKernel *p_pEngineKernel)
    {
        p_pEngineKernel->GetSpaceManager()->UnregisterFactory("GPU");
        p_pEngineKernel->GetRendererManager()->UnregisterFactory("GPU");
    }

    void Initialise(void) {}
    void Shutdown(void) {}

private:
    std::string m_strName;
    Version m_version;
    GpuSpaceFactory *m_pFactory;
    GpuRendererFactory *m_pRendererFactory;
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
