// bunnykiller_gpu.hpp - reference-side adaptor: renders BunnyKiller's transient scenes on a B200.
//
// Included by the reference's src/bunnykiller.cpp after its own headers.  It provides
//   * tr::SceneCapture   - records what parse_args feeds to World (meshes with their Lambertian
//                          albedo, point / rectangular lights, the homogeneous medium), reading
//                          OBJ files with the rules of World::add_triangle_mesh (World.h:209-420);
//   * tr::GpuTransientRenderer<D, Radiance, RadianceAttenuation>
//                        - a TransientRenderer whose render() (TransientRenderer.h:76-201) runs
//                          the GPU path through include/transient_b200.h and then writes the
//                          same files as StreakCameraFilm::write (StreakCameraFilm.h:233-242).
// World's geometry is private to its Embree scene (World.h:107-108), so the meshes are captured
// at parse time instead of being read back from World.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "transient_b200.h"

namespace tr {

class SceneCapture {
public:
    std::vector<float> vertices;
    std::vector<uint32_t> triangles;
    std::vector<uint32_t> triangle_material;
    std::vector<tr_material> materials;
    std::vector<tr_light> lights;
    tr_medium medium{};

    // -name-mesh FILE -lambertian r g b   (bunnykiller.cpp:995-1002, :328-337)
    void add_triangle_mesh(const std::string& path, float kd_r, float kd_g, float kd_b) {
        std::ifstream in(path);
        if (!in) throw std::runtime_error("Error: failed to open model file: \"" + path + "\"");
        tr_material m{};
        m.kind = TR_MAT_LAMBERTIAN;
        m.kd[0] = kd_r; m.kd[1] = kd_g; m.kd[2] = kd_b;
        materials.push_back(m);
        const uint32_t mat = (uint32_t)materials.size() - 1;
        const uint32_t base = (uint32_t)(vertices.size() / 3);
        std::vector<float> v;
        size_t nvt = 0, nvn = 0;
        std::string line;
        unsigned line_num = 0;
        auto index = [&](long i, size_t n) -> uint32_t {
            long j = i > 0 ? i - 1 : (long)n + i;
            if (j < 0 || j > (long)n - 1)
                throw std::out_of_range("Error: reading open model file \"" + path + "\": out of range index " +
                                        std::to_string(i) + " at line " + std::to_string(line_num));
            return (uint32_t)j;
        };
        while (std::getline(in, line)) {
            ++line_num;
            std::istringstream ls(line);
            std::string tag;
            if (!(ls >> tag) || tag[0] == '#') continue;
            if (tag == "v") {
                float x, y, z;
                if (!(ls >> x >> y >> z)) throw std::runtime_error("Error: reading open model file \"" + path + "\"");
                v.push_back(x); v.push_back(y); v.push_back(z);
            } else if (tag == "vt") {
                ++nvt;
            } else if (tag == "vn") {
                ++nvn;
            } else if (tag == "f") {
                std::string c[4];
                int k = 0;
                while (k < 4 && (ls >> c[k])) ++k;
                if (k != 3) throw std::runtime_error("Error: reading open model file \"" + path + "\": invalid face");
                for (int j = 0; j < 3; ++j) {
                    long vi = std::stol(c[j].substr(0, c[j].find('/')));
                    triangles.push_back(base + index(vi, v.size() / 3));
                }
                triangle_material.push_back(mat);
            }
        }
        vertices.insert(vertices.end(), v.begin(), v.end());
    }

    // -point-light-source x y z r g b   (bunnykiller.cpp:1194-1207)
    void add_point_light(const float pos[3], const float intensity[3]) {
        tr_light L{};
        L.kind = TR_LIGHT_POINT;
        for (int k = 0; k < 3; ++k) { L.position[k] = pos[k]; L.intensity[k] = intensity[k]; }
        lights.push_back(L);
    }

    // -rectangular-area-light-source p t size I   (bunnykiller.cpp:1242-1262); frame as
    // RectangularAreaLightSource::setup (RectangularAreaLightSource.h:66-80)
    void add_rect_light(const float pos[3], const float target[3], const float size[2], float intensity) {
        tr_light L{};
        L.kind = TR_LIGHT_RECT;
        float n[3] = {target[0] - pos[0], target[1] - pos[1], target[2] - pos[2]};
        float l = std::sqrt((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2]);
        for (float& c : n) c /= l;
        float up[3] = {0.f, 1.f, 0.f};
        if (!(std::fabs(n[1]) < 0.9999f)) { up[1] = 0.f; up[2] = 1.f; }
        float left[3] = {n[1] * up[2] - n[2] * up[1], n[2] * up[0] - n[0] * up[2], n[0] * up[1] - n[1] * up[0]};
        float u2[3] = {n[1] * left[2] - n[2] * left[1], n[2] * left[0] - n[0] * left[2], n[0] * left[1] - n[1] * left[0]};
        for (int k = 0; k < 3; ++k) {
            L.position[k] = pos[k];
            L.intensity[k] = intensity;
            L.left[k] = left[k] * size[0];
            L.up[k] = u2[k] * size[1];
            L.normal[k] = n[k];
        }
        L.area = size[0] * size[1];
        lights.push_back(L);
    }

    // -homogeneous-medium sa(3) ss(3) -pf-hg g   (bunnykiller.cpp:184-227)
    void set_medium(const float sa[3], const float ss[3], float g) {
        medium.enabled = 1;
        for (int k = 0; k < 3; ++k) { medium.sigma_a[k] = sa[k]; medium.sigma_s[k] = ss[k]; }
        medium.g = g;
    }

    tr_scene view() const {
        tr_scene s{};
        s.vertices = vertices.data();
        s.num_vertices = (uint32_t)(vertices.size() / 3);
        s.triangles = triangles.data();
        s.num_triangles = (uint32_t)(triangles.size() / 3);
        s.triangle_material = triangle_material.data();
        s.materials = materials.data();
        s.num_materials = (uint32_t)materials.size();
        s.lights = lights.data();
        s.num_lights = (uint32_t)lights.size();
        s.medium = medium;
        return s;
    }
};

// Pinhole basis as PinholeCamera builds it (PinholeCamera.h:56-75).
inline tr_camera pinhole(const float pos[3], const float focus[3], const float up_in[3], float focal_distance) {
    auto norm = [](float* v) {
        float l = std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
        v[0] /= l; v[1] /= l; v[2] /= l;
    };
    auto cross = [](const float* a, const float* b, float* o) {
        o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; o[2] = a[0] * b[1] - a[1] * b[0];
    };
    tr_camera c{};
    float up[3] = {up_in[0], up_in[1], up_in[2]};
    norm(up);
    for (int k = 0; k < 3; ++k) { c.position[k] = pos[k]; c.nv[k] = focus[k] - pos[k]; }
    norm(c.nv);
    cross(c.nv, up, c.uv);
    norm(c.uv);
    cross(c.uv, c.nv, c.vv);
    norm(c.vv);
    c.focal_distance = focal_distance;
    return c;
}

inline void check(tr_status s) {
    if (s != TR_OK) throw std::runtime_error(std::string("GPU renderer: ") + tr_status_string(s) + ": " + tr_last_error());
}

#ifdef _TRANSIENT_RENDERER_H_
// The renderer the maintainer swaps in for TransientRenderer in main() (bunnykiller.cpp:1754).
template <unsigned D, class Radiance, class RadianceAttenuation>
class GpuTransientRenderer : public TransientRenderer<D, Radiance, RadianceAttenuation> {
    using Base = TransientRenderer<D, Radiance, RadianceAttenuation>;
    const SceneCapture& m_scene;
    tr_camera m_camera;
    tr_integrator m_integrator;
    int m_device;

public:
    // time_sampling: the reference's TransientRenderer(f_log, time_sampling) argument
    // (TransientRenderer.h:61-62, "-time-sampling"), i.e. TR_FLAG_TIME_SAMPLING.
    // path_tracing_only: what the caller passed to BidirectionalPathTracing::set_path_tracing_only
    // (BidirectionalPathTracing.h:214-217); false adds light subpaths and vertex connections
    // (TR_FLAG_BIDIRECTIONAL, defined with time sampling in scenes without a medium).
    GpuTransientRenderer(FILE* f_log, const SceneCapture& scene, const tr_camera& camera, unsigned max_bounces,
                         unsigned sqrt_spp, unsigned incoming_samples, uint64_t seed, int device = 0,
                         bool time_sampling = false, bool path_tracing_only = true)
        : Base(f_log, time_sampling), m_scene(scene), m_camera(camera), m_integrator{}, m_device(device) {
        m_integrator.max_bounces = max_bounces;
        m_integrator.sqrt_spp = sqrt_spp;
        m_integrator.incoming_samples = incoming_samples;
        m_integrator.seed = seed;
        if (time_sampling) m_integrator.flags |= TR_FLAG_TIME_SAMPLING;
        if (!path_tracing_only) m_integrator.flags |= TR_FLAG_BIDIRECTIONAL;
    }

    void render(const char* name, World<D, Radiance>& world, Integrator<D, Radiance, RadianceAttenuation>* integrator,
                const Camera<D>& camera, Film<D, Radiance>* film, Sampler* sampler) const override {
        if (!integrator) throw std::runtime_error("Error: Need to define an integrator for rendering\n");
        if (!film || !sampler) throw std::runtime_error("GPU renderer: film and sampler are required");
        tr_film f{};
        f.width = (uint32_t)film->get_width();
        f.height = (uint32_t)film->get_height();
        f.time_bins = film->get_time_resolution();
        f.exposure = film->get_exposure_time();
        f.offset = film->get_time_offset();
        // the GPU renders the captured configuration: the reference's film and sampler must
        // describe the same frame (StratifiedSampler::get_nb_samples = W x H x sqrt_spp^2)
        const size_t spp = (size_t)m_integrator.sqrt_spp * m_integrator.sqrt_spp;
        const size_t want = (size_t)f.width * f.height * spp;
        if (sampler->get_nb_samples() != want)
            throw std::runtime_error("GPU renderer: the sampler draws " + std::to_string(sampler->get_nb_samples()) +
                                     " samples but the film (" + std::to_string(f.width) + "x" +
                                     std::to_string(f.height) + ") at the captured " + std::to_string(spp) +
                                     " samples per pixel needs " + std::to_string(want));
        tr_scene s = m_scene.view();
        tr_ctx* ctx = nullptr;
        check(tr_create(&s, &m_camera, &f, &m_integrator, m_device, &ctx));
        tr_status st = tr_render(ctx, 0, m_integrator.sqrt_spp * m_integrator.sqrt_spp);
        if (st == TR_OK) st = tr_write_film(ctx, name);
        tr_destroy(ctx);
        check(st);
    }
};
#endif

}  // namespace tr
