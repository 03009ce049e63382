"""Known answers the reference's sources imply but its repository never checks (it has no tests):
the arrival time of the first bounce and the normalisation of the learned proposal's lobes.

* First bounce (BidirectionalPathTracing.h:485-692,975-1045; StreakCameraFilm.h:139-192): in an
  empty room every wall point sees a point light inside it, so with one camera sample per pixel
  and a path depth of 1, each pixel's bounce-0 film holds exactly one radiance sample, in time
  bin floor((|camera - x| + |x - light| - offset) / exposure), x the camera ray's first hit
  (taken from the film's position component, Film.h:127-145).
* vMF lobes (Jakob 2012, oracle/guide_oracle.py): the density integrates to one over the sphere
  and the samples' mean cosine to the lobe axis is coth(kappa) - 1/kappa."""
import numpy as np

from jarabotransientrendering_b200 import scenes as S


def _room_scene():
    mats = [S.Material(S.MAT_LAMBERTIAN, S.WHITE)]
    meshes = [S.Mesh(name, v, t, 0) for name, v, t in S.room()]
    light = S.Light(S.LIGHT_POINT, (0.5, 0.99, 0.5), (1.0, 1.0, 1.0))
    cam = S.Camera((0.5, 0.5, -1.37), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0), 40.0)
    return S.Scene("room", meshes, mats, [light], cam, 16, 12, 2048, 0.002, 0.0, 1, 1, 1,
                   bounce_films=2, components=S.COMP_POSITIONS)


def test_first_bounce_arrives_at_the_geometric_path_length(oracle_lib):
    sc = _room_scene()
    o = oracle_lib.Oracle(sc)
    f = o.render(0, 1, bounces=True, components=True)
    b0 = f["bstreak"][0]                                   # [H][W][T][3]
    cam = np.array(sc.camera.position, np.float64)
    light = np.array(sc.lights[0].position, np.float64)
    checked = 0
    for y in range(sc.height):
        for x in range(sc.width):
            assert f["weight"][y, x] == 1.0
            hit = f["positions"][y, x]
            t = np.linalg.norm(hit - cam) + np.linalg.norm(light - hit)
            q = (t - sc.offset) / sc.exposure
            nz = np.nonzero(b0[y, x].sum(axis=-1))[0]
            assert len(nz) == 1, (y, x, nz)
            want = int(np.floor(q))
            if abs(q - round(q)) < 1e-3:                   # on a bin edge: float32 may round either way
                assert nz[0] in (want, want - 1, want + 1), (y, x, q, nz)
            else:
                assert nz[0] == want, (y, x, q, nz)
                checked += 1
    assert checked > sc.width * sc.height * 0.9


def test_vmf_lobes_are_normalised_and_sample_their_mean_cosine():
    from oracle import guide_oracle as G
    rng = np.random.default_rng(3)
    c = np.linspace(-1.0, 1.0, 4_000_001)
    for kappa in (0.05, 1.0, 10.0, 200.0):
        # over the sphere: integral of f(cos theta) d omega = 2 pi * integral over c in [-1, 1]
        total = 2.0 * np.pi * np.trapezoid(np.exp(G.log_vmf(kappa, c)), c)
        assert abs(total - 1.0) < 1e-6, (kappa, total)
        mu = rng.normal(size=3)
        mu /= np.linalg.norm(mu)
        n = 400_000
        d = G.sample_vmf(np.broadcast_to(mu, (n, 3)), kappa, rng.random(n), rng.random(n))
        assert np.allclose(np.linalg.norm(d, axis=-1), 1.0, atol=1e-9)
        w = d @ mu
        mean = 1.0 / np.tanh(kappa) - 1.0 / kappa
        assert abs(w.mean() - mean) < 5.0 * w.std() / np.sqrt(n), (kappa, w.mean(), mean)


def test_hg_phase_function_is_normalised_with_mean_cosine_g(oracle_lib):
    """The oracle's Henyey-Greenstein density (HenyeyGreensteinPhaseFunction.h:254-276; the GPU's
    is the same operation sequence, compared per path) integrates to one over the sphere with
    mean cosine g, and its inverse-CDF sampler (:218-240) draws cosines with that density."""
    L = oracle_lib.lib()
    c = np.linspace(-1.0, 1.0, 200_001)
    rng = np.random.default_rng(11)
    xs = rng.random(200_000).astype(np.float32)
    for g in (-0.9, -0.3, 0.0, 0.3, 0.9):
        f = np.array([L.orc_hg_eval(g, float(v)) for v in c[::20]], np.float64)
        cc = c[::20]
        total = 2.0 * np.pi * np.trapezoid(f, cc)
        mean = 2.0 * np.pi * np.trapezoid(f * cc, cc)
        assert abs(total - 1.0) < 2e-3 and abs(mean - g) < 2e-3, (g, total, mean)
        s = np.array([L.orc_hg_sample_cos(g, float(x)) for x in xs], np.float64)
        assert (np.abs(s) <= 1.0).all()
        assert abs(s.mean() - g) < 5.0 * s.std() / np.sqrt(len(s)) + 1e-4, (g, s.mean())
        # the sampled cosines follow the density: counts per interval against its integral
        edges = np.linspace(-1.0, 1.0, 21)
        counts, _ = np.histogram(s, edges)
        fine = np.linspace(-1.0, 1.0, 20 * 200 + 1)
        fv = np.array([L.orc_hg_eval(g, float(v)) for v in fine], np.float64)
        p = np.array([2.0 * np.pi * np.trapezoid(fv[i * 200:(i + 1) * 200 + 1], fine[i * 200:(i + 1) * 200 + 1])
                      for i in range(20)])
        expect = p / p.sum() * len(s)
        z = (counts - expect) / np.sqrt(np.maximum(expect, 1.0))
        assert np.abs(z).max() < 5.0, (g, z)
