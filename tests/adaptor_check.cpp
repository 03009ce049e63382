// Compile check of include/bunnykiller_gpu.hpp against the reference's own headers: the
// adaptor must derive from TransientRenderer and override render() with the reference's
// signature.  Built by tests/test_abi.py::test_reference_adaptor_compiles (reference sources
// needed; the reference's headers are included in the order its main program uses).
#include "Utils/RandomNumbers.h"
#include "Camera/PinholeCamera.h"
#include "RayTracing/World.h"
#include "Renderer/TransientRenderer.h"
#include "Film/StreakCameraFilm.h"
#include "Geometry/Primitives/3D/Triangle.h"
#include "Geometry/Aggregate/BVH.h"
#include "Geometry/ObjectPointer.h"
#include "Material/UberMaterial.h"
#include "Material/Reflectance/Lambertian.h"
#include "LightSource/PointLightSource.h"
#include "LightSource/RectangularAreaLightSource.h"
#include "Sampling/StratifiedSampler.h"
#include "Integrator/BidirectionalPathTracing.h"
#include "bunnykiller_gpu.hpp"

template class tr::GpuTransientRenderer<3, Spectrum, Spectrum>;

int main() {
    tr::SceneCapture scene;
    float p[3] = {0.5f, 0.5f, -1.37f}, f[3] = {0.5f, 0.5f, 0.5f}, u[3] = {0.f, 1.f, 0.f};
    tr_camera cam = tr::pinhole(p, f, u, 2.7474775f);
    RenderEngine<3, Spectrum, Spectrum>* engine =
        new tr::GpuTransientRenderer<3, Spectrum, Spectrum>(nullptr, scene, cam, 6, 8, 1, 1);
    delete engine;
    return 0;
}
