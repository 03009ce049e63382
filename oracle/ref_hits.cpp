/*
 * ref_hits.cpp - closest-hit records of the reference's own ray caster on a ray batch.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/): built by `make -C oracle ref` into oracle/_ref/ from the
 * reference's sources where they lie, linked with the vendored Embree 2.17.4 that
 * oracle/embree.mk compiles.  It is the hit-record pin of the GPU traversal; nothing in the
 * product links it.
 *
 * The scene goes through the reference's World exactly as its CLI builds it: every mesh is
 * written to an OBJ file and loaded with World::add_triangle_mesh (src/RayTracing/World.h:209-541:
 * vertex split, geometric normal, Embree buffers), in mesh order, so geomID = mesh index and
 * primID = face order; World::World creates the device and scene with the reference's flags
 * (World.h:141-157: RTC_SCENE_STATIC | RTC_SCENE_INCOHERENT, RTC_INTERSECT1 | RTC_INTERPOLATE,
 * FTZ/DAZ on) and World::freeze commits it (World.h:543-550).  Each ray is initialised as
 * World::first_intersection does (World.h:570-583) and cast with rtcIntersect (:585).
 * World keeps its Embree scene private; the harness reads it through the standard
 * explicit-instantiation access idiom instead of changing the reference.
 *
 * Usage: ref_hits SCENE RAYS OUT
 *   SCENE: text scene of oracle/refscene.py (only its meshes are used); RAYS: float32 [N][8]
 *   (ox, oy, oz, tnear, dx, dy, dz, tfar); OUT: per ray geomID u32, primID u32, tfar f32,
 *   u f32, v f32 (20 bytes; geomID = primID = 0xFFFFFFFF and tfar unchanged on a miss).
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>
#include <unistd.h>

#include "RayTracing/World.h"
#include "Material/UberMaterial.h"
#include "Material/Reflectance/Lambertian.h"

typedef World<3, Spectrum> World3;

/* Access to World::g_scene without modifying the reference: an explicit instantiation may
 * name a private member, and the friend function it defines hands the pointer out. */
struct SceneTag { typedef RTCScene World3::*type; friend type scene_member(SceneTag); };
template <typename Tag, typename Tag::type M> struct Expose { friend typename Tag::type scene_member(Tag) { return M; } };
template struct Expose<SceneTag, &World3::g_scene>;

static void fail(const char* m) { fprintf(stderr, "ref_hits: %s\n", m); exit(2); }

int main(int argc, char** argv) {
    if (argc != 4) fail("usage: ref_hits SCENE RAYS OUT");
    std::ifstream in(argv[1]);
    if (!in) fail("cannot open scene");
    char tmpl[] = "/tmp/tr_ref_hits_XXXXXX";
    if (!mkdtemp(tmpl)) fail("cannot create a temporary directory");
    const std::string dir(tmpl);

    World3 world;
    UberMaterial3D* mat = new UberMaterial3D();
    mat->add_bsdf(new Lambertian3D(Spectrum(0.5f)));
    std::vector<std::string> objs;
    std::string tag;
    while (in >> tag) {
        if (tag == "mesh") {
            size_t nv, nt; unsigned m; in >> nv >> nt >> m;
            std::vector<std::string> vl(nv), tl(nt);
            std::string path = dir + "/mesh" + std::to_string(objs.size()) + ".obj";
            FILE* f = fopen(path.c_str(), "w");
            if (!f) fail("cannot write an OBJ file");
            for (size_t i = 0; i < nv; ++i) {             /* %.9g round-trips every float */
                float a, b, c; in >> a >> b >> c;
                fprintf(f, "v %.9g %.9g %.9g\n", a, b, c);
            }
            for (size_t i = 0; i < nt; ++i) {
                size_t a, b, c; in >> a >> b >> c;
                fprintf(f, "f %zu %zu %zu\n", a + 1, b + 1, c + 1);
            }
            fclose(f);
            objs.push_back(path);
        } else if (tag == "end") {
            break;
        } else {
            std::string rest; std::getline(in, rest);     /* film, camera, lights, ...: unused */
        }
    }
    for (const std::string& p : objs) world.add_triangle_mesh(p, mat);
    world.freeze();
    for (const std::string& p : objs) unlink(p.c_str());
    rmdir(dir.c_str());

    FILE* fr = fopen(argv[2], "rb");
    if (!fr) fail("cannot open rays");
    fseek(fr, 0, SEEK_END);
    const long bytes = ftell(fr);
    fseek(fr, 0, SEEK_SET);
    const size_t n = (size_t)bytes / (8 * sizeof(float));
    std::vector<float> rays(n * 8);
    if (fread(rays.data(), sizeof(float), n * 8, fr) != n * 8) fail("short ray file");
    fclose(fr);

    RTCScene scene = world.*scene_member(SceneTag());
    struct Rec { unsigned geom, prim; float t, u, v; };
    static_assert(sizeof(Rec) == 20, "record layout");
    std::vector<Rec> out(n);
    for (size_t i = 0; i < n; ++i) {
        const float* r = &rays[i * 8];
        RTCRay rr;                                        /* World::first_intersection, :570-583 */
        rr.org[0] = r[0]; rr.org[1] = r[1]; rr.org[2] = r[2];
        rr.dir[0] = r[4]; rr.dir[1] = r[5]; rr.dir[2] = r[6];
        rr.tnear = r[3];
        rr.tfar = r[7];
        rr.time = 0.f;
        rr.mask = 0xFFFFFFFF;
        rr.geomID = RTC_INVALID_GEOMETRY_ID;
        rr.primID = RTC_INVALID_GEOMETRY_ID;
        rtcIntersect(scene, rr);
        out[i] = Rec{rr.geomID, rr.primID, rr.tfar, rr.u, rr.v};
    }
    FILE* fo = fopen(argv[3], "wb");
    if (!fo || fwrite(out.data(), sizeof(Rec), n, fo) != n) fail("cannot write output");
    fclose(fo);
    return 0;
}
