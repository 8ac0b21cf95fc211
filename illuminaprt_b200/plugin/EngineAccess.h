// Read access to engine state that the engine keeps protected but a device
// renderer must copy to the GPU: a member pointer formed in a derived
// class's scope reads a protected member of any object of the base class
// without changing the class or the object.
#pragma once

#include "Camera/Camera.h"
#include "Integrator/PathIntegrator.h"
#include "Light/DiffuseAreaLight.h"
#include "Material/Glass.h"
#include "Material/Matte.h"
#include "Material/Mirror.h"
#include "Shape/Quad.h"
#include "Shape/Triangle.h"

namespace Illumina {
namespace PlugIn {
namespace Access {

// Quad's two triangles (Shape/Quad.h:23): (v1, v3, v2) and (v1, v4, v3).
struct QuadTriangles : public Illumina::Core::Quad {
    static const Illumina::Core::Triangle *Of(const Illumina::Core::Quad *p)
    {
        Illumina::Core::Triangle(Illumina::Core::Quad::*m)[2] = &QuadTriangles::m_tesselatedQuad;
        return p->*m;
    }
};

// MatteMaterial's reflectivity and texture (Material/Matte.h).
struct Matte : public Illumina::Core::MatteMaterial {
    static const Illumina::Core::Spectrum &Reflectivity(const Illumina::Core::MatteMaterial *p)
    {
        Illumina::Core::Spectrum Illumina::Core::MatteMaterial::*m = &Matte::m_reflectivity;
        return p->*m;
    }
    static const Illumina::Core::ITexture *Texture(const Illumina::Core::MatteMaterial *p)
    {
        Illumina::Core::ITexture *Illumina::Core::MatteMaterial::*m = &Matte::m_pTexture;
        return p->*m;
    }
};

// MirrorMaterial's reflectivity and texture (Material/Mirror.h).
struct Mirror : public Illumina::Core::MirrorMaterial {
    static const Illumina::Core::Spectrum &Reflectivity(const Illumina::Core::MirrorMaterial *p)
    {
        Illumina::Core::Spectrum Illumina::Core::MirrorMaterial::*m = &Mirror::m_reflectivity;
        return p->*m;
    }
    static const Illumina::Core::ITexture *Texture(const Illumina::Core::MirrorMaterial *p)
    {
        Illumina::Core::ITexture *Illumina::Core::MirrorMaterial::*m = &Mirror::m_pTexture;
        return p->*m;
    }
};

// GlassMaterial's reflectivity, transmittance, indices and texture
// (Material/Glass.h).
struct Glass : public Illumina::Core::GlassMaterial {
    static const Illumina::Core::Spectrum &Reflectivity(const Illumina::Core::GlassMaterial *p)
    {
        Illumina::Core::Spectrum Illumina::Core::GlassMaterial::*m = &Glass::m_reflectivity;
        return p->*m;
    }
    static const Illumina::Core::Spectrum &Transmittance(const Illumina::Core::GlassMaterial *p)
    {
        Illumina::Core::Spectrum Illumina::Core::GlassMaterial::*m = &Glass::m_transmittance;
        return p->*m;
    }
    static float EtaI(const Illumina::Core::GlassMaterial *p)
    {
        float Illumina::Core::GlassMaterial::*m = &Glass::m_fEtaI;
        return p->*m;
    }
    static float EtaT(const Illumina::Core::GlassMaterial *p)
    {
        float Illumina::Core::GlassMaterial::*m = &Glass::m_fEtaT;
        return p->*m;
    }
    static const Illumina::Core::ITexture *Texture(const Illumina::Core::GlassMaterial *p)
    {
        Illumina::Core::ITexture *Illumina::Core::GlassMaterial::*m = &Glass::m_pTexture;
        return p->*m;
    }
};

// DiffuseAreaLight's emitted radiance (Light/DiffuseAreaLight.h).
struct AreaLight : public Illumina::Core::DiffuseAreaLight {
    static const Illumina::Core::Spectrum &Emit(const Illumina::Core::DiffuseAreaLight *p)
    {
        Illumina::Core::Spectrum Illumina::Core::DiffuseAreaLight::*m = &AreaLight::m_emit;
        return p->*m;
    }
};

// PathIntegrator's parameters (Integrator/PathIntegrator.h:20-23).
struct PathTracer : public Illumina::Core::PathIntegrator {
    static int MaxRayDepth(const Illumina::Core::PathIntegrator *p)
    {
        int Illumina::Core::PathIntegrator::*m = &PathTracer::m_nMaxRayDepth;
        return p->*m;
    }
    static int ShadowSampleCount(const Illumina::Core::PathIntegrator *p)
    {
        int Illumina::Core::PathIntegrator::*m = &PathTracer::m_nShadowSampleCount;
        return p->*m;
    }
    static float ReflectEpsilon(const Illumina::Core::PathIntegrator *p)
    {
        float Illumina::Core::PathIntegrator::*m = &PathTracer::m_fReflectEpsilon;
        return p->*m;
    }
};

// ICamera's frame (Camera/Camera.h:23-28), what GetRay combines.
struct Camera : public Illumina::Core::ICamera {
    static void Frame(const Illumina::Core::ICamera *p, Illumina::Core::Vector3 &centre,
                      Illumina::Core::Vector3 &corner, Illumina::Core::Vector3 &across, Illumina::Core::Vector3 &up)
    {
        Illumina::Core::Vector3 Illumina::Core::ICamera::*c = &Camera::m_centre;
        Illumina::Core::Vector3 Illumina::Core::ICamera::*k = &Camera::m_corner;
        Illumina::Core::Vector3 Illumina::Core::ICamera::*a = &Camera::m_across;
        Illumina::Core::Vector3 Illumina::Core::ICamera::*u = &Camera::m_up;
        centre = p->*c;
        corner = p->*k;
        across = p->*a;
        up = p->*u;
    }
};

}  // namespace Access
}  // namespace PlugIn
}  // namespace Illumina
