/*
 * ref_harness.cpp - runs the reference renderer's own transient path tracer on a scene file.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/): built by `make -C oracle ref` into oracle/_ref/ from the
 * reference's header sources where they lie; it is the statistical pin of the CPU oracle and
 * the CPU baseline of bench.py.  Nothing in the product links it.
 *
 * Everything on the sampling path is the reference's code: World, PinholeCamera,
 * StratifiedSampler, BidirectionalPathTracing in path-tracing-only steady-state mode,
 * UberMaterial+Lambertian, PointLightSource, RectangularAreaLightSource, HomogeneousMedium with
 * Henyey-Greenstein / isotropic phase, TransientRenderer::render.  Set-up follows main()
 * (src/bunnykiller.cpp:1504-1827).  Two builds:
 *   - ref_render: the shipped configuration (src/bunnykiller.h defines _USE_EMBREE_).  Every
 *     mesh is written to an OBJ file and loaded by World::add_triangle_mesh
 *     (src/RayTracing/World.h:209-541), as `-name-mesh FILE -lambertian ...` does, and rays are
 *     cast by the vendored Embree 2.17.4 (compiled by oracle/embree.mk);
 *   - ref_render_bvh: the reference's own non-Embree backend (ref_globals.h pre-defines the
 *     src/bunnykiller.h include guard): triangles are the smooth Triangle
 *     (src/Geometry/Primitives/3D/Triangle.h) with all three shading normals = the Embree
 *     geometric normal normalize(cross(p2-p0, p1-p0)) (World.h:449,514-540), placed in the
 *     reference's BVH (src/Geometry/Aggregate/BVH.h).
 * The one piece that is the harness's own: the film is a StreakCameraFilm whose add_samples
 * (StreakCameraFilm.h:139-192) is overridden to accumulate the same (pixel, bin) sums in double
 * precision into one buffer instead of averaging and writing RGBE scanlines; with `filmopts U N`
 * it also applies the camera unwarp of StreakCameraFilm.h:167 (sample time minus the record's
 * camera distance) and, for N > 0, routes the samples to N per-bounce films with the weights of
 * MultibounceStreakFilm::add_samples (MultibounceStreakCameraFilm.h:151-171), the main steady
 * image then being the base Film's (all samples, Film.h:263-284); `mode transient` selects the
 * time-sampling mode (-time-sampling, bunnykiller.cpp:1337-1345, 1754, 1812-1817); `bidir 1`
 * turns off path-tracing-only (light subpaths and vertex connections;
 * BidirectionalPathTracing::set_path_tracing_only, reachable through the API).
 *
 * Usage: ref_render SCENE OUT [y0 y1 | --rows y,y,...] [--no-streak] [--timing]
 *   SCENE: text file written by oracle/refscene.py; y0 y1 / --rows: render only scanlines
 *   [y0, y1) / the listed ones (-film-scanline, one call of TransientRenderer::render per line;
 *   the film then holds only those rows, in that order, H below = their count; with --timing
 *   every scanline is added into one stored row - the same splat work in a film of one row, for
 *   timing many scanlines per process); OUT: raw doubles
 *   streak [H][W][T][3] (unless --no-streak), steady [H][W][3], weight [H][W], then with N
 *   bounce films bstreak [N][H][W][T][3], bsteady [N][H][W][3], bweight [N][H][W], then with
 *   components (`filmopts U N C`, C != 0) depth [H][W], positions [H][W][3], normals [H][W][3]
 *   summed from each camera sample's record (Film::add_components, Film.h:127-145).
 *   Prints one JSON line on stderr: paths, seconds and paths/s of the render loop, and with a
 *   scanline range the seconds of each scanline's render call.
 */
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <unistd.h>

#include "Utils/RandomNumbers.h"
#include "Camera/PinholeCamera.h"
#include "RayTracing/World.h"
#include "Renderer/TransientRenderer.h"
#include "Film/StreakCameraFilm.h"
#ifndef _USE_EMBREE_
#include "Geometry/Primitives/3D/Triangle.h"
#include "Geometry/Aggregate/BVH.h"
#include "Geometry/ObjectPointer.h"
#endif
#include "Material/UberMaterial.h"
#include "Material/Reflectance/Lambertian.h"
#include "LightSource/PointLightSource.h"
#include "LightSource/RectangularAreaLightSource.h"
#include "Sampling/StratifiedSampler.h"
#include "Integrator/BidirectionalPathTracing.h"
#include "Media/HomogeneousMedium.h"
#include "Media/PhaseFunction/IsotropicPhaseFunction.h"
#include "Media/PhaseFunction/HenyeyGreensteinPhaseFunction.h"

typedef Spectrum Radiance;
typedef Spectrum RadianceAttenuation;

class AccumStreakFilm : public StreakCameraFilm<3, Radiance> {
    using Base = StreakCameraFilm<3, Radiance>;
public:
    unsigned W, H, T;
    std::vector<int> row_of;           /* scanline -> stored row (the film holds only rendered rows) */
    Real exposure, offset;
    std::vector<double> streak, steady, weight;
    bool keep_streak;
    bool unwarp;
    unsigned NB;
    unsigned comps;
    std::vector<double> bstreak, bsteady, bweight;
    std::vector<double> cdepth, cpos, cnorm;
    AccumStreakFilm(unsigned w, unsigned full_h, const std::vector<int>& rows, unsigned t, Real exp_, Real off,
                    bool ks, bool uw, unsigned nb, unsigned cm)
        : Base(w, full_h, t, exp_, uw, nullptr), W(w), H((unsigned)rows.size()), T(t), exposure(exp_), offset(off),
          keep_streak(ks), unwarp(uw), NB(nb), comps(cm) {
        const unsigned h = H;
        row_of.assign(full_h, -1);
        for (size_t i = 0; i < rows.size(); ++i) row_of[rows[i]] = (int)i;
        if (cm) {
            cdepth.assign((size_t)h * w, 0.0);
            cpos.assign((size_t)h * w * 3, 0.0);
            cnorm.assign((size_t)h * w * 3, 0.0);
        }
        if (off > 0) this->set_offset(off);
        if (ks) streak.assign((size_t)h * w * t * 3, 0.0);
        steady.assign((size_t)h * w * 3, 0.0);
        weight.assign((size_t)h * w, 0.0);
        if (nb) {
            bstreak.assign((size_t)nb * h * w * t * 3, 0.0);
            bsteady.assign((size_t)nb * h * w * 3, 0.0);
            bweight.assign((size_t)nb * h * w, 0.0);
        }
    }
    /* StreakCameraFilm::add_samples with the box filter of size 1 (weight 1, one pixel): */
    void add_samples(const Sample& sample, const RadianceSampleRecordVector<3, Radiance>& rec) override {
        unsigned x = (unsigned)std::floor(sample.position[0]);
        unsigned y = (unsigned)row_of[(unsigned)std::floor(sample.position[1])];
        size_t pix = (size_t)y * W + x;
        const size_t npix = (size_t)W * H;
        weight[pix] += sample.weight;
        std::vector<char> present(NB, 0);
        for (const RadianceSample<3, Radiance>& r : rec.samples) {
            const unsigned b = NB ? (r.bounce < NB ? r.bounce : NB - 1) : 0;
            if (NB) present[b] = 1;
            Real cam_time = unwarp ? (r.time - rec.distance) : r.time;
            Real pos_sensor = (cam_time - offset) / exposure;
            const bool inside = pos_sensor < T && pos_sensor >= 0.0;
            for (int c = 0; c < 3; ++c)
                if (inside || NB) steady[pix * 3 + c] += (double)r.radiance[c];
            if (!inside) continue;
            size_t t = (size_t)std::floor(pos_sensor);
            for (int c = 0; c < 3; ++c) {
                if (keep_streak) streak[(pix * T + t) * 3 + c] += (double)r.radiance[c];
                if (NB) {
                    bstreak[(((size_t)b * npix + pix) * T + t) * 3 + c] += (double)r.radiance[c];
                    bsteady[((size_t)b * npix + pix) * 3 + c] += (double)r.radiance[c];
                }
            }
        }
        for (unsigned b = 0; b < NB; ++b)
            if (present[b]) bweight[(size_t)b * npix + pix] += sample.weight;
        if (comps) {                                     /* Film::add_components, Film.h:127-145 */
            cdepth[pix] += (double)(rec.distance * sample.weight);
            for (int c = 0; c < 3; ++c) {
                cpos[pix * 3 + c] += (double)(rec.pos[c] * sample.weight);
                cnorm[pix * 3 + c] += (double)(rec.normal[c] * sample.weight);
            }
        }
    }
    void write(const char*) override {}
};

static void fail(const char* m) { fprintf(stderr, "ref_render: %s\n", m); exit(2); }

int main(int argc, char** argv) {
    if (argc < 3) fail("usage: ref_render SCENE OUT [y0 y1 | --rows y,y,...] [--no-streak] [--timing]");
    bool keep_streak = true;
    bool one_row = false;                  /* --timing: every scanline splats into one stored row */
    std::vector<int> rows;                 /* scanlines to render; empty = the whole film */
    std::vector<std::string> pos;
    for (int i = 3; i < argc; ++i) {
        if (!strcmp(argv[i], "--no-streak")) keep_streak = false;
        else if (!strcmp(argv[i], "--timing")) one_row = true;
        else if (!strcmp(argv[i], "--rows") && i + 1 < argc) {
            std::stringstream ss(argv[++i]);
            std::string item;
            while (std::getline(ss, item, ',')) rows.push_back(atoi(item.c_str()));
        } else pos.push_back(argv[i]);
    }
    if (pos.size() >= 2)
        for (int y = atoi(pos[0].c_str()); y < atoi(pos[1].c_str()); ++y) rows.push_back(y);
    const bool region = !rows.empty() || pos.size() >= 2;
    std::ifstream in(argv[1]);
    if (!in) fail("cannot open scene");
    std::string tag;
    unsigned W = 0, H = 0, T = 0, maxb = 0, sqrt_spp = 0, ninc = 1, unwarp = 0, nbounce = 0, comps = 0;
    bool time_sampling = false;
    int bidir = 0;
    Real exposure = 0, offset = 0, fov = 40;
    unsigned long long seed = 1;
    Vector3 cpos, cfoc, cup;
    int med_on = 0; float sa[3] = {0, 0, 0}, ss[3] = {0, 0, 0}, g = 0;
    std::vector<UberMaterial3D*> mats;
    World<3, Radiance> w;
#ifdef _USE_EMBREE_
    char tmpl[] = "/tmp/tr_ref_render_XXXXXX";
    if (!mkdtemp(tmpl)) fail("cannot create a temporary directory");
    const std::string objdir(tmpl);
    std::vector<std::string> objs;
#else
    BVH<Object3DPointer, 3>* bvh = new BVH<Object3DPointer, 3>();
#endif
    std::vector<std::string> light_lines;
    while (in >> tag) {
        if (tag == "film") { in >> W >> H >> T >> exposure >> offset; }
        else if (tag == "filmopts") { in >> unwarp >> nbounce >> comps; }
        else if (tag == "mode") { std::string m; in >> m; time_sampling = (m == "transient"); }
        else if (tag == "bidir") { in >> bidir; }
        else if (tag == "camera") {
            float a[9]; for (float& v : a) in >> v; in >> fov;
            cpos = Vector3(a[0], a[1], a[2]); cfoc = Vector3(a[3], a[4], a[5]); cup = Vector3(a[6], a[7], a[8]);
        } else if (tag == "integrator") { in >> maxb >> sqrt_spp >> ninc >> seed; }
        else if (tag == "medium") { in >> med_on >> sa[0] >> sa[1] >> sa[2] >> ss[0] >> ss[1] >> ss[2] >> g; }
        else if (tag == "material") {
            unsigned kind; float kd[3], alpha; in >> kind >> kd[0] >> kd[1] >> kd[2] >> alpha;
            if (kind != 0) fail("the reference has no GGX material");
            UberMaterial3D* um = new UberMaterial3D();     /* bunnykiller.cpp:328-337 */
            um->add_bsdf(new Lambertian3D(Spectrum(kd[0], kd[1], kd[2])));
            mats.push_back(um);
        } else if (tag == "light") { std::string l; std::getline(in, l); light_lines.push_back(l); }
        else if (tag == "mesh") {
            size_t nv, nt; unsigned m; in >> nv >> nt >> m;
            if (m >= mats.size()) fail("bad material index");
#ifdef _USE_EMBREE_
            /* the CLI's `-name-mesh FILE -lambertian ...` (bunnykiller.cpp:328-337): an OBJ file
               loaded by World::add_triangle_mesh; %.9g round-trips every float */
            std::string path = objdir + "/mesh" + std::to_string(objs.size()) + ".obj";
            FILE* f = fopen(path.c_str(), "w");
            if (!f) fail("cannot write an OBJ file");
            for (size_t i = 0; i < nv; ++i) { float a, b, c; in >> a >> b >> c; fprintf(f, "v %.9g %.9g %.9g\n", a, b, c); }
            for (size_t i = 0; i < nt; ++i) { size_t a, b, c; in >> a >> b >> c; fprintf(f, "f %zu %zu %zu\n", a + 1, b + 1, c + 1); }
            fclose(f);
            w.add_triangle_mesh(path, mats[m]);
            unlink(path.c_str());
            objs.push_back(path);
#else
            std::vector<Vector3f> v(nv);
            for (size_t i = 0; i < nv; ++i) { float a, b, c; in >> a >> b >> c; v[i] = Vector3f(a, b, c); }
            for (size_t i = 0; i < nt; ++i) {
                size_t a, b, c; in >> a >> b >> c;
                Vector3f p0 = v[a], p1 = v[b], p2 = v[c];
                Vector3f ngf = cross(p2 - p0, p1 - p0).normalized();      /* World.h:449 */
                Vector3 ng(ngf[0], ngf[1], ngf[2]);
                Vector2 uv0(0., 0.);
                Triangle* tri = new Triangle(Vector3(p0[0], p0[1], p0[2]), ng, uv0,
                                             Vector3(p1[0], p1[1], p1[2]), ng, uv0,
                                             Vector3(p2[0], p2[1], p2[2]), ng, uv0, mats[m]);
                bvh->add_primitive(Object3DPointer(tri));
            }
#endif
        } else if (tag == "end") break;
        else fail("unknown tag");
    }
    for (const std::string& l : light_lines) {
        std::istringstream ls(l);
        std::string kind; ls >> kind;
        if (kind == "point") {
            float p[3], I[3]; ls >> p[0] >> p[1] >> p[2] >> I[0] >> I[1] >> I[2];
            w.add_light(new PointLightSource<3, Radiance>(&w, Vector3(p[0], p[1], p[2]), Radiance(I[0], I[1], I[2])));
        } else if (kind == "rect") {
            float p[3], t[3], sz[2], I; ls >> p[0] >> p[1] >> p[2] >> t[0] >> t[1] >> t[2] >> sz[0] >> sz[1] >> I;
            Vector3 pp(p[0], p[1], p[2]), tt(t[0], t[1], t[2]);          /* bunnykiller.cpp:1242-1262 */
            w.add_light(new RectangularAreaLightSource<Radiance>(&w, pp, (tt - pp).normalized(),
                                                                 Vector2(sz[0], sz[1]), Radiance(I), nullptr));
        } else fail("unknown light");
    }
    if (med_on) {                                                       /* bunnykiller.cpp:184-227 */
        Spectrum a(sa[0], sa[1], sa[2]), s(ss[0], ss[1], ss[2]);
        if (g == 0.f)
            w.set_medium(new HomogeneousMedium<3, PhaseFunction::Isotropic<3>>(a, s, PhaseFunction::Isotropic<3>(0.)));
        else
            w.set_medium(new HomogeneousMedium<3, PhaseFunction::HenyeyGreenstein<3>>(a, s,
                         PhaseFunction::HenyeyGreenstein<3>(g, 0.)));
    }
#ifdef _USE_EMBREE_
    rmdir(objdir.c_str());
#else
    bvh->freeze();
    w.add_object(Object3DPointer(bvh));
#endif
    w.set_background(Spectrum(0.));
    w.freeze();

    Real fovr = M_PI / 180. * fov / 2;                                   /* bunnykiller.cpp:1156-1161 */
    Real fd = 1. / tan(fovr);
    PinholeCamera camera(cpos, cfoc, cup, fd);
    /* a scanline set stores only its own rows, so a full-size streak film fits per process */
    std::vector<int> stored = rows;
    if (!region) for (unsigned y = 0; y < H; ++y) stored.push_back((int)y);
    if (one_row && region) stored.assign(1, rows[0]);
    if (region && rows.empty()) fail("empty scanline range");
    for (size_t i = 0; i < stored.size(); ++i) {
        if (stored[i] < 0 || (unsigned)stored[i] >= H) fail("scanline out of range");
        for (size_t j = 0; j < i; ++j) if (stored[j] == stored[i]) fail("repeated scanline");
    }
    AccumStreakFilm film(W, H, stored, T, exposure, offset, keep_streak, unwarp != 0, nbounce, comps);
    if (one_row && region) for (int y : rows) film.row_of[y] = 0;
    StratifiedSampler sampler(W, H, sqrt_spp, true);
    TransientRenderer<3, Radiance, RadianceAttenuation> engine(nullptr, time_sampling);   /* bunnykiller.cpp:1754 */
    Random::StdRNG.seed(seed);                                           /* bunnykiller.cpp:1794 */
    BidirectionalPathTracing<3, Radiance, RadianceAttenuation> bpt(w, ninc, nullptr, &film);
    bpt.set_max_path_size(maxb);
    bpt.set_path_tracing_only(bidir == 0);                              /* bunnykiller.cpp:1809 (API only) */
    bpt.set_scattering_components(Scattering::ALL);
    bpt.set_mode(time_sampling                                           /* bunnykiller.cpp:1812-1817 */
                     ? BidirectionalPathTracing<3, Radiance, RadianceAttenuation>::SamplingMode::Transient
                     : BidirectionalPathTracing<3, Radiance, RadianceAttenuation>::SamplingMode::SteadyState);

    FILE* devnull = freopen("/dev/null", "w", stdout);   /* the renderer prints progress */
    (void)devnull;
    auto t0 = std::chrono::steady_clock::now();
    unsigned long long paths = 0;
    std::vector<double> row_seconds;
    if (region) {
        for (int y : rows) {
            auto r0 = std::chrono::steady_clock::now();
            sampler.set_scanline(y);                                     /* -film-scanline, :1782-1791 */
            engine.render("ref", w, &bpt, camera, &film, &sampler);
            paths += (unsigned long long)W * sqrt_spp * sqrt_spp * ninc;
            row_seconds.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - r0).count());
        }
    } else {
        engine.render("ref", w, &bpt, camera, &film, &sampler);
        paths = (unsigned long long)W * H * sqrt_spp * sqrt_spp * ninc;
    }
    auto t1 = std::chrono::steady_clock::now();
    double secs = std::chrono::duration<double>(t1 - t0).count();
    FILE* out = fopen(argv[2], "wb");
    if (!out) fail("cannot write output");
    if (keep_streak) fwrite(film.streak.data(), sizeof(double), film.streak.size(), out);
    fwrite(film.steady.data(), sizeof(double), film.steady.size(), out);
    fwrite(film.weight.data(), sizeof(double), film.weight.size(), out);
    if (nbounce) {
        fwrite(film.bstreak.data(), sizeof(double), film.bstreak.size(), out);
        fwrite(film.bsteady.data(), sizeof(double), film.bsteady.size(), out);
        fwrite(film.bweight.data(), sizeof(double), film.bweight.size(), out);
    }
    if (comps) {
        fwrite(film.cdepth.data(), sizeof(double), film.cdepth.size(), out);
        fwrite(film.cpos.data(), sizeof(double), film.cpos.size(), out);
        fwrite(film.cnorm.data(), sizeof(double), film.cnorm.size(), out);
    }
    fclose(out);
    FILE* tty = fopen("/dev/stderr", "w");
    fprintf(tty, "{\"paths\": %llu, \"seconds\": %.6f, \"paths_per_s\": %.3f, \"row_seconds\": [",
            paths, secs, paths / secs);
    for (size_t i = 0; i < row_seconds.size(); ++i) fprintf(tty, "%s%.6f", i ? ", " : "", row_seconds[i]);
    fprintf(tty, "]}\n");
    fclose(tty);
    return 0;
}
