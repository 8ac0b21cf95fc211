// The shading data a device path tracer needs besides the GpuSpace's BVH:
// the scene's materials (one per material slot of the space) and its lights,
// uploaded to the space's device context. Shared by GpuRenderer (whole
// regions) and GpuPathIntegrator (IIntegrator::Radiance per ray); refuses
// what the device cannot render with an Exception, never a CPU fallback.
//
//   materials  MatteMaterial, MirrorMaterial or GlassMaterial without a
//              texture; a primitive without material renders black
//   lights     DiffuseAreaLight on a Quad or on a triangle mesh whose
//              EmissivePrimitive is in the space (a mesh light without a
//              world transform of its own), and InfiniteAreaLight without a
//              texture, in the scene's LightList order (at most 8)
#pragma once

#include <string>

namespace Illumina {
namespace Core {
class Scene;
}
namespace PlugIn {

class GpuSpace;

// The scene's GpuSpace, with its materials and lights on the device (uploaded
// again only when the space was rebuilt or the scene changed). p_strWho
// prefixes the refusals.
GpuSpace *PrepareDeviceScene(Illumina::Core::Scene *p_pScene, const std::string &p_strWho);

}  // namespace PlugIn
}  // namespace Illumina
