// Test-infrastructure harness: a scene script loaded by the reference's own
// loader and rendered by the renderer the script names.
//
// This file is ours; the loader it drives is the reference's, compiled
// unmodified by oracle/Makefile:
//   Environment::Load                     Core/Scene/Environment.cpp:102-106
//   EnvironmentLoader::Parse              Core/Scene/EnvironmentLoader.cpp:150-210
//     ParseShapes (WavefrontModel -> WavefrontSceneLoader::Import, else the
//     ShapeManager factory)               Core/Scene/EnvironmentLoader.cpp:567-647
//     ParseRenderers (binds Integrator, Filter, Device by Id)  :649-713
//     ParseEnvironment (Renderer, Scene{Sampler, Camera, Lights}, Space{Type,
//     Primitives}, then ISpace::Initialise / Build)            :715-921
//   WavefrontSceneLoader::LoadGeometry / LoadMaterials (OBJ + MTL into one
//   triangle mesh and a MaterialGroup)    Core/Scene/WavefrontSceneLoader.cpp:126-570
// and then the Sandbox's start-up and frame (Utility/Sandbox/Environment.h:
// 436-446): IIntegrator::Initialise(scene, camera), IRenderer::Initialise(),
// Render(buffer) or RenderRegion over tiles, Commit(buffer).
//
// The factories are the reference's own (Camera/CameraFactories.h,
// Light/LightFactories.h, Space/SpaceFactories.h, Shape/ShapeFactories.h,
// Filter/FilterFactories.h, Sampler/SamplerFactories.h,
// Material/MaterialFactories.h, Renderer/RendererFactories.h), registered
// under the names the Sandbox gives them (Utility/Sandbox/Environment.h:
// 77-189), with three exceptions written here:
//   "PathTracing"  Integrator/IntegratorFactories.h does not compile with a
//                  current compiler (Integrator/IntegratorHelper.h:285, :444),
//                  so this file has a factory with the same arguments and
//                  defaults (RayDepth 6, ShadowRays 1, Epsilon 1e-4) making
//                  the same PathIntegrator (IntegratorFactories.h:26-69).
//   "IC"           likewise for the irradiance-cache integrator: the same
//                  arguments and defaults (IntegratorFactories.h:160-205)
//                  making the reference's ICIntegrator.
//   "Memory"       an IDevice that only has a size (Width, Height): the
//                  reference's devices write image files or displays.
// A plug-in library, when given, is loaded and registered with the kernel's
// PlugInManager (its "GPU" space and renderer factories).
//
// Only tests/ load the library this file builds.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>

#include <dlfcn.h>

#include "Camera/CameraFactories.h"
#include "Device/Device.h"
#include "Exception/Exception.h"
#include "Filter/FilterFactories.h"
#include "Integrator/ICIntegrator.h"
#include "Integrator/PathIntegrator.h"
#include "Light/LightFactories.h"
#include "Material/MaterialFactories.h"
#include "Renderer/Renderer.h"
#include "Renderer/RendererFactories.h"
#include "Sampler/SamplerFactories.h"
#include "Scene/Environment.h"
#include "Scene/Scene.h"
#include "Shape/ShapeFactories.h"
#include "Space/SpaceFactories.h"
#include "System/EngineKernel.h"
#include "System/PlugIn.h"
#include "System/PlugInManager.h"

using namespace Illumina::Core;

namespace {

void report(char *err, int err_len, const std::string &msg)
{
	if (!err || err_len <= 0) return;
	std::strncpy(err, msg.c_str(), err_len - 1);
	err[err_len - 1] = 0;
}

class ScriptPathIntegratorFactory : public Factory<IIntegrator>
{
public:
	IIntegrator *CreateInstance(void) { throw new Exception("Method not supported!"); }

	IIntegrator *CreateInstance(ArgumentMap &p_argumentMap)
	{
		int depth = 6, shadow = 1;
		float epsilon = 1e-4f;
		std::string id;
		p_argumentMap.GetArgument("RayDepth", depth);
		p_argumentMap.GetArgument("ShadowRays", shadow);
		p_argumentMap.GetArgument("Epsilon", epsilon);
		if (p_argumentMap.GetArgument("Id", id)) return new PathIntegrator(id, depth, shadow, epsilon);
		return new PathIntegrator(depth, shadow, epsilon);
	}
};

class ScriptICIntegratorFactory : public Factory<IIntegrator>
{
public:
	IIntegrator *CreateInstance(void) { throw new Exception("Method not supported!"); }

	IIntegrator *CreateInstance(ArgumentMap &p_argumentMap)
	{
		int depth = 6, cache_depth = 16, azimuth = 12, altitude = 4, shadow = 1;
		float error = 1.f, resolution = 1e-3f, multiplier = 1e+3f, epsilon = 1e-4f;
		std::string id;
		p_argumentMap.GetArgument("CacheDepth", cache_depth);
		p_argumentMap.GetArgument("ErrorThreshold", error);
		p_argumentMap.GetArgument("AzimuthStrata", azimuth);
		p_argumentMap.GetArgument("AltitudeStrata", altitude);
		p_argumentMap.GetArgument("AmbientResolution", resolution);
		p_argumentMap.GetArgument("AmbientMultiplier", multiplier);
		p_argumentMap.GetArgument("RayDepth", depth);
		p_argumentMap.GetArgument("ShadowRays", shadow);
		p_argumentMap.GetArgument("Epsilon", epsilon);
		if (p_argumentMap.GetArgument("Id", id))
			return new ICIntegrator(id, cache_depth, error, resolution, multiplier, azimuth, altitude, depth, shadow,
			                        epsilon);
		return new ICIntegrator(cache_depth, error, resolution, multiplier, azimuth, altitude, depth, shadow, epsilon);
	}
};

class ScriptDevice : public IDevice
{
	int m_w, m_h;

public:
	ScriptDevice(const std::string &id, int w, int h) : IDevice(id), m_w(w), m_h(h) {}
	int GetWidth(void) const { return m_w; }
	int GetHeight(void) const { return m_h; }
	AccessType GetAccessType(void) const { return Write; }
	bool Open(void) { return true; }
	void Close(void) {}
	void BeginFrame(void) {}
	void EndFrame(void) {}
	void Set(int, int, const Spectrum &) {}
	void Set(float, float, const Spectrum &) {}
	void Get(int, int, Spectrum &s) const { s = Spectrum(0.f); }
	void Get(float, float, Spectrum &s) const { s = Spectrum(0.f); }
	Spectrum Get(int, int) const { return Spectrum(0.f); }
	Spectrum Get(float, float) const { return Spectrum(0.f); }
	void WriteRadianceBufferToDevice(int, int, int, int, RadianceBuffer *, int, int) {}
};

class ScriptDeviceFactory : public Factory<IDevice>
{
public:
	IDevice *CreateInstance(void) { return new ScriptDevice("Memory", 64, 64); }

	IDevice *CreateInstance(ArgumentMap &p_argumentMap)
	{
		int w = 64, h = 64;
		std::string id = "Memory";
		p_argumentMap.GetArgument("Width", w);
		p_argumentMap.GetArgument("Height", h);
		p_argumentMap.GetArgument("Id", id);
		if (w <= 0 || h <= 0) throw new Exception("Memory device: Width and Height must be positive");
		return new ScriptDevice(id, w, h);
	}
};

void register_factories(EngineKernel *k)
{
	k->GetSamplerManager()->RegisterFactory("Random", new RandomSamplerFactory());
	k->GetFilterManager()->RegisterFactory("Box", new BoxFilterFactory());
	k->GetSpaceManager()->RegisterFactory("Basic", new BasicSpaceFactory());
	k->GetIntegratorManager()->RegisterFactory("PathTracing", new ScriptPathIntegratorFactory());
	k->GetIntegratorManager()->RegisterFactory("IC", new ScriptICIntegratorFactory());
	k->GetRendererManager()->RegisterFactory("Basic", new BasicRendererFactory());
	k->GetDeviceManager()->RegisterFactory("Memory", new ScriptDeviceFactory());
	k->GetCameraManager()->RegisterFactory("Perspective", new PerspectiveCameraFactory());
	k->GetLightManager()->RegisterFactory("DiffuseArea", new DiffuseAreaLightFactory());
	k->GetShapeManager()->RegisterFactory("BasicMesh", new BasicMeshShapeFactory());
	k->GetShapeManager()->RegisterFactory("KDTreeMesh", new KDTreeMeshShapeFactory());
	k->GetShapeManager()->RegisterFactory("BVHMesh", new BVHMeshShapeFactory());
	k->GetShapeManager()->RegisterFactory("Quad", new QuadMeshShapeFactory());
	k->GetShapeManager()->RegisterFactory("Triangle", new TriangleShapeFactory());
	k->GetMaterialManager()->RegisterFactory("Matte", new MatteMaterialFactory());
	k->GetMaterialManager()->RegisterFactory("Mirror", new MirrorMaterialFactory());
	k->GetMaterialManager()->RegisterFactory("Glass", new GlassMaterialFactory());
	k->GetMaterialManager()->RegisterFactory("Group", new MaterialGroupFactory());
}

// The OBJ loader ends the process when a file it is given cannot be opened
// (WavefrontSceneLoader.cpp:418-422), so every "Filename = ..." of the script
// is checked here first.
bool files_exist(const std::string &script, std::string &missing)
{
	std::ifstream in(script.c_str());
	std::string line;
	while (std::getline(in, line)) {
		const size_t k = line.find("Filename");
		const size_t eq = line.find('=');
		if (k == std::string::npos || eq == std::string::npos || eq < k) continue;
		std::string name = line.substr(eq + 1);
		const size_t b = name.find_first_not_of(" \t\r");
		const size_t e = name.find_last_not_of(" \t\r");
		if (b == std::string::npos) continue;
		name = name.substr(b, e - b + 1);
		struct stat st;
		if (stat(name.c_str(), &st) != 0) {
			missing = name;
			return false;
		}
	}
	return true;
}

} // namespace

extern "C" {

// Loads `script` with the reference's Environment::Load into a fresh engine
// kernel (with the plug-in at plugin_path registered when it is not NULL or
// empty), initialises the integrator and renderer as the Sandbox does, and
// renders one frame of the device's size (width x height, which must match
// the script's device) with Render (tile <= 0) or RenderRegion over tile x
// tile regions, then Commit. Outputs Final, Direct and Albedo (height x width
// x 3 each) and, in info, "space=<name> renderer=<name> primitives=<n>
// lights=<n> render_s=<seconds from the integrator's Initialise to Commit>".
// Returns 0, or a negative code with the reason in err: -1
// script or a file it names missing, -2 plug-in load, -3 load or parse
// exception, -4 the script left no renderer, scene, camera, integrator or
// device, -5 device size differs, -6 render exception.
//
// The kernel, environment and everything the script made are left allocated:
// FactoryManager's destructor erases from its map while iterating it
// (System/FactoryManager.inl:15-26), so the kernel is never deleted; the
// space is shut down (a GpuSpace frees its device context there). A loaded
// plug-in stays loaded.
int ilref_render_script(const char *plugin_path, const char *script, int width, int height, int tile,
                        float *out, float *out_direct, float *out_albedo, char *info, int info_len, char *err,
                        int err_len)
{
	struct stat st;
	if (!script || stat(script, &st) != 0) {
		report(err, err_len, std::string("no script file ") + (script ? script : "(null)"));
		return -1;
	}
	std::string missing;
	if (!files_exist(script, missing)) {
		report(err, err_len, "the script names a file that does not exist: " + missing);
		return -1;
	}

	EngineKernel *kernel = new EngineKernel();
	register_factories(kernel);
	if (plugin_path && plugin_path[0]) {
		// the plug-in resolves the engine's symbols against this library
		Dl_info self;
		if (dladdr((void *)&report, &self) && self.dli_fname)
			dlopen(self.dli_fname, RTLD_NOW | RTLD_NOLOAD | RTLD_GLOBAL);
		void *lib = dlopen(plugin_path, RTLD_NOW | RTLD_LOCAL);
		typedef IPlugIn *(*GetSingleton)(void);
		GetSingleton get = lib ? (GetSingleton)dlsym(lib, "GetPlugInSingleton") : NULL;
		if (!get) {
			const char *e = dlerror();
			report(err, err_len, std::string("plug-in: ") + (e ? e : "no GetPlugInSingleton"));
			return -2;
		}
		kernel->GetPlugInManager()->Register(get());
	}

	Environment *env = new Environment(kernel);
	try {
		if (!env->Load(script)) {
			report(err, err_len, "Environment::Load returned false");
			return -3;
		}
	} catch (Exception *e) {
		report(err, err_len, "load: " + e->GetMessage());
		return -3;
	} catch (Exception &e) {
		report(err, err_len, "load: " + e.GetMessage());
		return -3;
	}

	IRenderer *renderer = env->GetRenderer();
	Scene *scene = renderer ? renderer->GetScene() : NULL;
	if (!renderer || !scene || !scene->GetCamera() || !scene->GetSpace() || !renderer->GetIntegrator() ||
	    !renderer->GetDevice()) {
		report(err, err_len, "the script left no renderer, scene, camera, space, integrator or device");
		return -4;
	}
	IDevice *device = renderer->GetDevice();
	if (device->GetWidth() != width || device->GetHeight() != height) {
		std::ostringstream s;
		s << "device is " << device->GetWidth() << " x " << device->GetHeight() << ", asked " << width << " x "
		  << height;
		report(err, err_len, s.str());
		return -5;
	}
	{
		std::ostringstream s;
		s << "space=" << scene->GetSpace()->ToString() << " renderer=" << renderer->ToString()
		  << " primitives=" << scene->GetSpace()->PrimitiveList.Size() << " lights=" << scene->LightList.Size();
		report(info, info_len, s.str());
	}

	RadianceBuffer buffer(width, height);
	int rc = 0;
	const auto t0 = std::chrono::steady_clock::now();
	try {
		renderer->GetIntegrator()->Initialise(scene, scene->GetCamera());
		renderer->Initialise();
		if (tile <= 0) {
			renderer->Render(&buffer);
		} else {
			for (int y = 0; y < height; y += tile)
				for (int x = 0; x < width; x += tile)
					renderer->RenderRegion(&buffer, x, y, std::min(tile, width - x), std::min(tile, height - y), x, y);
		}
		renderer->Commit(&buffer);
	} catch (Exception *e) {
		report(err, err_len, "render: " + e->GetMessage());
		rc = -6;
	} catch (Exception &e) {
		report(err, err_len, "render: " + e.GetMessage());
		rc = -6;
	}
	if (rc == 0) {
		const double render_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
		if (info && info_len > 0) {
			std::ostringstream s;
			s << info << " render_s=" << render_s;
			report(info, info_len, s.str());
		}
		for (int y = 0; y < height; y++)
			for (int x = 0; x < width; x++) {
				const RadianceContext *c = buffer.GetP(x, y);
				const size_t px = 3 * ((size_t)y * width + x);
				for (int k = 0; k < 3; k++) {
					out[px + k] = c->Final[k];
					out_direct[px + k] = c->Direct[k];
					out_albedo[px + k] = c->Albedo[k];
				}
			}
	}
	scene->GetSpace()->Shutdown();
	return rc;
}

} // extern "C"
