// GpuRenderer: an IRenderer (Core/Renderer/Renderer.h:21-81) that renders a
// region of the image on the B200 in one call: the device wavefront path
// tracer of libilg.so (ilg_render_region) instead of one
// IIntegrator::Radiance call per pixel sample. It is a drop-in for
// BasicRenderer (Core/Renderer/BasicRenderer.cpp, BaseRenderer.cpp:62-169)
// under the reference's own driver loops: Render(), RenderRegion(...) and
// Commit() keep their meaning, and the RadianceBuffer receives Final,
// Direct, Indirect (= Final - Direct) and Albedo per pixel with
// DF_Computed set, each averaged over the renderer's samples per pixel, and
// the view ray through the pixel's corner with its first hit's Position,
// Normal and Distance (one batched device query per region).
//
// What it takes from the engine's objects, and what it refuses (with an
// Exception, never a CPU fallback):
//   space       must be a GpuSpace (its device BVH and material slots)
//   integrator  a PathIntegrator: its RayDepth and Epsilon are used; more
//               than one shadow ray per light is refused. A
//               GpuPathIntegrator with Cache = MLP also turns on the
//               device's learned radiance cache (a fresh network for each
//               built scene, trained after every region)
//   materials   MatteMaterial, MirrorMaterial or GlassMaterial without a
//               texture (reflectivity; for glass also transmittance and
//               the two indices); a primitive without material renders black
//   lights      DiffuseAreaLight on a Quad or on a triangle mesh whose
//               EmissivePrimitive is in the space, and InfiniteAreaLight
//               without a texture (PrepareDeviceScene, DeviceScene.h)
//   camera      any ICamera: its centre / corner / across / up frame, the
//               same numbers its GetRay uses
//   device      GetWidth() / GetHeight() give the image size, as in
//               BaseRenderer
//
// Samples come from a counter-based sequence keyed by (seed, pixel,
// sample), not from the scene's ISampler: images agree with the reference's
// statistically, not bit for bit. A region renders exactly the samples the
// whole image gives those pixels, so tiles meet seamlessly. The seed
// advances at every Commit(), so successive frames differ, as the
// reference's advancing sampler makes them.
#pragma once

#include <cstdint>
#include <string>

#include "Renderer/BaseRenderer.h"
#include "ilg.h"

namespace Illumina {
namespace PlugIn {

class GpuSpace;

class GpuRenderer : public Illumina::Core::BaseRenderer {
public:
    GpuRenderer(const std::string &p_strName, Illumina::Core::Scene *p_pScene = NULL,
                Illumina::Core::IIntegrator *p_pIntegrator = NULL, Illumina::Core::IDevice *p_pDevice = NULL,
                Illumina::Core::IFilter *p_pFilter = NULL, Illumina::Core::RadianceBuffer *p_pRadianceBuffer = NULL,
                int p_nSampleCount = 1, uint32_t p_nSeed = 1);
    GpuRenderer(Illumina::Core::Scene *p_pScene = NULL, Illumina::Core::IIntegrator *p_pIntegrator = NULL,
                Illumina::Core::IDevice *p_pDevice = NULL, Illumina::Core::IFilter *p_pFilter = NULL,
                Illumina::Core::RadianceBuffer *p_pRadianceBuffer = NULL, int p_nSampleCount = 1,
                uint32_t p_nSeed = 1);

    using Illumina::Core::BaseRenderer::RenderRegion;
    void RenderRegion(Illumina::Core::RadianceBuffer *p_pRadianceBuffer, int p_nRegionX, int p_nRegionY,
                      int p_nRegionWidth, int p_nRegionHeight, int p_nBufferX = 0, int p_nBufferY = 0);

    using Illumina::Core::BaseRenderer::Commit;
    void Commit(Illumina::Core::RadianceBuffer *p_pRadianceBuffer);

    void SetSeed(uint32_t p_nSeed) { m_nSeed = p_nSeed; }
    uint32_t GetSeed(void) const { return m_nSeed; }
    int GetSampleCount(void) const { return m_nSampleCount; }
    void SetSampleCount(int p_nSampleCount) { m_nSampleCount = p_nSampleCount; }

    std::string ToString(void) const { return "GpuRenderer"; }

private:
    uint32_t m_nSeed;
    const ilg_ctx *m_pCacheContext;  // context whose radiance cache this renderer initialised
    uint64_t m_nCacheBuild;
};

}  // namespace PlugIn
}  // namespace Illumina
