// Runs include/bunnykiller_gpu.hpp for real: the reference's own objects (World with its Embree
// scene, PinholeCamera, StreakCameraFilm, StratifiedSampler, BidirectionalPathTracing) are set
// up the way the reference's main() sets them up (src/bunnykiller.cpp:1504-1824), the meshes
// are captured with tr::SceneCapture from the same OBJ files, and
// tr::GpuTransientRenderer::render is called through a RenderEngine pointer as main() calls it
// (bunnykiller.cpp:1824).  The GPU path then writes the reference's files: <name>_%04d.hdr per
// scanline and <name>.hdr.
//
// Built by `make -C oracle adaptor` (the reference's headers and Embree are needed to compile
// it, so the binary is built where the reference sources are and run wherever the library is).
//
// Usage: adaptor_render DIR NAME [W H T EXPOSURE SQRT_SPP [SAMPLER_SQRT_SPP]]
//   writes DIR/room.obj and DIR/box.obj, renders, writes DIR/NAME*.hdr.  SAMPLER_SQRT_SPP
//   (default SQRT_SPP) sets the reference sampler's strata; a value that disagrees with the
//   captured configuration must make render() throw.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "Utils/RandomNumbers.h"
#include "Camera/PinholeCamera.h"
#include "RayTracing/World.h"
#include "Renderer/TransientRenderer.h"
#include "Film/StreakCameraFilm.h"
#include "Material/UberMaterial.h"
#include "Material/Reflectance/Lambertian.h"
#include "LightSource/PointLightSource.h"
#include "Sampling/StratifiedSampler.h"
#include "Integrator/BidirectionalPathTracing.h"
#include "bunnykiller_gpu.hpp"

static void write_file(const std::string& path, const char* text) {
    FILE* f = fopen(path.c_str(), "w");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
    fputs(text, f);
    fclose(f);
}

int main(int argc, char** argv) {
    if (argc < 3) { fprintf(stderr, "usage: adaptor_render DIR NAME [W H T EXPOSURE SQRT_SPP [SAMPLER_SQRT_SPP]]\n"); return 2; }
    const std::string dir = argv[1], name = dir + "/" + argv[2];
    const unsigned W = argc > 3 ? atoi(argv[3]) : 24, H = argc > 4 ? atoi(argv[4]) : 16;
    const unsigned T = argc > 5 ? atoi(argv[5]) : 64;
    const float exposure = argc > 6 ? (float)atof(argv[6]) : 0.05f;
    const unsigned sqrt_spp = argc > 7 ? atoi(argv[7]) : 4;
    const unsigned sampler_sqrt_spp = argc > 8 ? atoi(argv[8]) : sqrt_spp;

    // a room with floor, ceiling and back wall (inward normals under cross(p2 - p0, p1 - p0)),
    // and a box standing on the floor
    write_file(dir + "/room.obj",
               "v 0 0 0\nv 1 0 0\nv 1 0 1\nv 0 0 1\nv 0 1 0\nv 1 1 0\nv 1 1 1\nv 0 1 1\n"
               "f 1 3 2\nf 1 4 3\nf 5 6 7\nf 5 7 8\nf 4 7 3\nf 4 8 7\n");
    write_file(dir + "/box.obj",
               "v 0.3 0 0.3\nv 0.6 0 0.3\nv 0.6 0 0.6\nv 0.3 0 0.6\n"
               "v 0.3 0.4 0.3\nv 0.6 0.4 0.3\nv 0.6 0.4 0.6\nv 0.3 0.4 0.6\n"
               "f 5 6 7\nf 5 7 8\nf 1 2 6\nf 1 6 5\nf 2 3 7\nf 2 7 6\nf 3 4 8\nf 3 8 7\nf 4 1 5\nf 4 5 8\n");

    // -name-mesh FILE -lambertian r g b (bunnykiller.cpp:995-1002, :328-337), into World and capture
    World<3, Spectrum> world;
    tr::SceneCapture capture;
    const struct { const char* file; float kd[3]; } meshes[] = {{"room.obj", {0.75f, 0.75f, 0.75f}},
                                                               {"box.obj", {0.25f, 0.75f, 0.25f}}};
    for (const auto& m : meshes) {
        UberMaterial3D* mat = new UberMaterial3D();
        mat->add_bsdf(new Lambertian3D(Spectrum(m.kd[0], m.kd[1], m.kd[2])));
        world.add_triangle_mesh(dir + "/" + m.file, mat);
        capture.add_triangle_mesh(dir + "/" + m.file, m.kd[0], m.kd[1], m.kd[2]);
    }
    // -point-light-source 0.5 0.9 0.5 1 1 1 (bunnykiller.cpp:1194-1207)
    const float lp[3] = {0.5f, 0.9f, 0.5f}, li[3] = {1.f, 1.f, 1.f};
    world.add_light(new PointLightSource<3, Spectrum>(&world, Vector3(lp[0], lp[1], lp[2]), Spectrum(1.f)));
    capture.add_point_light(lp, li);
    world.set_background(Spectrum(0.));
    world.freeze();

    // -camera-position / -camera-focus / -camera-up / -camera-fov 40 (bunnykiller.cpp:1156-1161)
    const float cp[3] = {0.5f, 0.5f, -1.37f}, cf[3] = {0.5f, 0.5f, 0.5f}, cu[3] = {0.f, 1.f, 0.f};
    const Real fd = 1. / tan(M_PI / 180. * 40. / 2);
    PinholeCamera camera(Vector3(cp[0], cp[1], cp[2]), Vector3(cf[0], cf[1], cf[2]), Vector3(cu[0], cu[1], cu[2]), fd);
    const tr_camera gcam = tr::pinhole(cp, cf, cu, (float)fd);

    StreakCameraFilm<3, Spectrum> film(W, H, T, exposure, false, nullptr);   // bunnykiller.cpp:1700-1716
    StratifiedSampler sampler(W, H, sampler_sqrt_spp, true);                  // bunnykiller.cpp:1675
    BidirectionalPathTracing<3, Spectrum, Spectrum> integrator(world, 1, nullptr, &film);
    integrator.set_max_path_size(6);

    RenderEngine<3, Spectrum, Spectrum>* engine =
        new tr::GpuTransientRenderer<3, Spectrum, Spectrum>(nullptr, capture, gcam, 6, sqrt_spp, 1, 7);
    int rc = 0;
    try {
        engine->render(name.c_str(), world, &integrator, camera, &film, &sampler);   // bunnykiller.cpp:1824
        printf("{\"rendered\": true, \"width\": %u, \"height\": %u, \"bins\": %u}\n", W, H, T);
    } catch (const std::exception& e) {
        printf("{\"rendered\": false, \"error\": \"%s\"}\n", e.what());
        rc = 3;
    }
    delete engine;
    return rc;
}
