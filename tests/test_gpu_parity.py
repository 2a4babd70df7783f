"""GPU parity: every kernel, called through the C ABI, against the CPU oracle
on the same seeded inputs.

Bar: bit-exact for hit ids, t, u, v, masks, heights, noise values, SDF
positions, normals and step counts (the kernels and the oracle share one
rounding policy).  Against the reference as shipped (brute force over one
leaf), hit ids must match except where the FP64 edge margin of either
triangle is below 1e-6 (counted), and t/u/v within 1e-5 relative.
"""
import numpy as np
import pytest
import torch

import rayengine_b200 as rb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

MARGIN = 1e-6
REL_TOL = 1e-5


def _kd(sc):
    st = sc.stats()
    nodes, leaves, tris = sc.export()
    return st, po.KdTree(nodes, leaves, tris, st["bmin"], st["bmax"])


def _hits(t):
    return t.cpu().numpy().reshape(-1, 4)


def _assert_vs_bruteforce(got, packed, st, cam, w, h, pixels, mode=0, label=None):
    """Reference-as-shipped comparison with the FP64 edge-margin exemption.

    Returns a report: rays compared, hits, id mismatches (every one of them
    must be edge-margin exempt), and the largest t/u/v relative difference on
    the rays whose ids agree (bound REL_TOL).  Printed when `label` is given."""
    bf = po.primary_bruteforce(packed, st["bmin"], st["bmax"], cam, w, h, mode=mode, pixels=pixels)
    g = got[pixels].view(np.int32).reshape(-1, 4)
    gid, bid = g[:, 0], bf["id"]
    diff = np.nonzero(gid != bid)[0]
    exempt = 0
    if diff.size:
        o, d = po.camera_rays(cam, w, h, pixels[diff])
        m = np.full(diff.size, np.inf)
        for ids in (gid[diff], bid[diff]):
            ok = ids >= 0
            m[ok] = np.minimum(m[ok], po.edge_margin(packed, ids[ok], o[ok], d[ok]))
        assert np.all(m < MARGIN), f"{int((m >= MARGIN).sum())} id mismatches outside the edge margin"
        exempt = diff.size
    same = (gid == bid) & (bid >= 0)
    gf = g[same, 1:].view(np.float32)
    bfv = np.stack([bf["t"], bf["u"], bf["v"]], 1)[same]
    rel = np.abs(gf - bfv) / np.maximum(np.abs(bfv), 1e-3)
    rel_max = float(rel.max(initial=0))
    assert rel_max <= REL_TOL
    report = {"rays": int(len(pixels)), "hits": int((bid >= 0).sum()),
              "id_mismatch_edge_exempt": int(exempt), "max_rel_tuv": rel_max}
    if label:
        print(f"parity vs reference brute force [{label}]: {report}")
    return exempt, int((bid >= 0).sum())


def test_soup_small_bitexact(cuda):
    cfg = rb.configs.SoupConfig(num_tris=4096, width=128, height=128)
    packed = cfg.packed()
    cam = cfg.camera()
    with rb.KDScene.from_packed(packed) as sc:
        st, kd = _kd(sc)
        for mode in (rb.TRACE_TWO_SIDED, rb.TRACE_ONE_SIDED):
            got = _hits(sc.trace_primary(cam, 128, 128, mode))
            ref = po.primary_kd(kd, cam, 128, 128, mode=mode)
            assert np.array_equal(got, ref.view(np.int32).reshape(-1, 4)), mode
            pix = np.arange(128 * 128, dtype=np.uint32)
            exempt, nhit = _assert_vs_bruteforce(got, packed, st, cam, 128, 128, pix, mode)
            assert nhit > (1000 if mode == 0 else 500)


def test_golden_reference_scenes(cuda):
    """The committed fixtures of the reference's own build + traversal."""
    import os

    for name in ("ref_soup.npz", "ref_grid.npz"):
        g = np.load(os.path.join(os.path.dirname(__file__), "golden", name))
        cam = rb.build_camera(g["campos"], (0, 0, 0), g["fov"])
        cam.view[:] = [float(x) for x in g["view"]]
        w, h = int(g["w"]), int(g["h"])
        with rb.KDScene.from_mesh(g["verts"], g["faces"]) as sc:
            got = _hits(sc.trace_primary(cam, w, h))
        gid, rid = got[:, 0], g["hits"][:, 0]
        diff = np.nonzero(gid != rid)[0]
        if diff.size:
            packed = rb.pack_triangles(g["verts"], g["faces"])
            o, d = po.camera_rays(cam, w, h, diff)
            m = np.full(diff.size, np.inf)
            for ids in (gid[diff], rid[diff]):
                ok = ids >= 0
                m[ok] = np.minimum(m[ok], po.edge_margin(packed, ids[ok], o[ok], d[ok]))
            assert np.all(m < MARGIN), name
        same = (gid == rid) & (rid >= 0)
        assert np.array_equal(got[same], g["hits"][same]), name


def test_soup_config0_full(cuda):
    """65,536 triangles, 512x512: bit-exact against the oracle's traversal of
    the same tree on every ray; against brute force on a ray sample."""
    cfg = rb.configs.SoupConfig()
    packed = cfg.packed()
    cam = cfg.camera()
    with rb.KDScene.from_packed(packed) as sc:
        st, kd = _kd(sc)
        got = _hits(sc.trace_primary(cam, 512, 512))
        cnt = sc.count_primary(cam, 512, 512).cpu().numpy()
    ref, rc = po.primary_kd(kd, cam, 512, 512, counts=True)
    assert np.array_equal(got, ref.view(np.int32).reshape(-1, 4))
    assert np.array_equal(cnt, rc.view(np.uint32).reshape(-1, 4).astype(np.int32))
    pix = np.random.default_rng(3).choice(512 * 512, 3000, replace=False).astype(np.uint32)
    _assert_vs_bruteforce(got, packed, st, cam, 512, 512, pix)


def test_caller_rays_closest_and_anyhit(cuda):
    cfg = rb.configs.SoupConfig(num_tris=20000)
    packed = cfg.packed()
    rng = np.random.default_rng(4)
    n = 50000
    o = rng.uniform(-1.5, 1.5, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d[: n // 10, 1:] = 0.0  # axis-parallel rays (zero direction components)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    tmax = rng.choice([np.inf, 0.5, 1e20], n).astype(np.float32)
    rays = np.concatenate([o, tmax[:, None], d, np.zeros((n, 1), np.float32)], 1)
    with rb.KDScene.from_packed(packed) as sc:
        st, kd = _kd(sc)
        dr = torch.from_numpy(rays).cuda()
        for flags in (0, 1, 2, 3):
            got = _hits(sc.trace_rays(dr, flags))
            ref = po.rays_kd(kd, rays, mode=flags & 1, anyhit=bool(flags & 2))
            if flags & 2:
                # any-hit: occlusion must agree; the reported triangle may differ
                assert np.array_equal(got[:, 0] >= 0, ref["id"] >= 0)
            else:
                assert np.array_equal(got, ref.view(np.int32).reshape(-1, 4))


def test_ray_refill_threshold_changes_only_speed(cuda):
    """Primary and caller-ray kernels refill idle lanes; every threshold gives
    the oracle's hits (and per-pixel work counts)."""
    cfg = rb.configs.SoupConfig(num_tris=8192, width=200, height=120)
    packed = cfg.packed()
    cam = cfg.camera()
    rng = np.random.default_rng(9)
    n = 20011  # not a multiple of 32
    o = rng.uniform(-1.5, 1.5, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    rays = np.concatenate([o, np.full((n, 1), np.inf, np.float32), d, np.zeros((n, 1), np.float32)], 1)
    with rb.KDScene.from_packed(packed) as sc:
        st, kd = _kd(sc)
        ref = po.primary_kd(kd, cam, 200, 120).view(np.int32).reshape(-1, 4)
        _, rc = po.primary_kd(kd, cam, 200, 120, counts=True)
        rref = po.rays_kd(kd, rays).view(np.int32).reshape(-1, 4)
        dr = torch.from_numpy(rays).cuda()
        t = sc.tuning()
        assert t["ray_refill_min"] == 32
        for refill in (1, 3, 8, 32):
            sc.set_tuning(t["stage_nodes"], t["queue_kind_major"], t["refill_min"], refill)
            assert np.array_equal(_hits(sc.trace_primary(cam, 200, 120)), ref), refill
            cnt = sc.count_primary(cam, 200, 120).cpu().numpy()
            assert np.array_equal(cnt, rc.view(np.uint32).reshape(-1, 4).astype(np.int32)), refill
            assert np.array_equal(_hits(sc.trace_rays(dr, 0)), rref), refill
        with pytest.raises(rb.RayEngineError):
            sc.set_tuning(t["stage_nodes"], t["queue_kind_major"], t["refill_min"], 0)
        best = sc.autotune_primary(cam, 200, 120)
        assert best["ray_refill_min"] in (4, 8, 16, 32) and best["frame_ms"] > 0
        assert sc.tuning()["ray_refill_min"] == best["ray_refill_min"]
        assert np.array_equal(_hits(sc.trace_primary(cam, 200, 120)), ref)


@pytest.mark.parametrize("leaf,mode", [(8, 0), (8, 1), (32, 0)])
def test_lanes_per_ray_same_hits(cuda, leaf, mode):
    """2, 4 or 8 lanes per primary ray split each leaf's triangle tests and
    keep the smallest (t, id), and with 32 the warp tests all its lanes'
    leaves together: every hit (id, t, u, v) equals the oracle's one-lane
    walk, on an image whose sides are no multiple of the tiles, with leaves
    holding more references than lanes."""
    cfg = rb.configs.SoupConfig(num_tris=16384, width=203, height=119)
    packed = cfg.packed()
    cam = cfg.camera()
    W, H = cfg.width, cfg.height
    with rb.KDScene.from_packed(packed, rb.kd_params(leaf_size=leaf, max_depth=24)) as sc:
        st, kd = _kd(sc)
        assert st["max_leaf_size"] > (8 if leaf > 8 else 1)
        ref = po.primary_kd(kd, cam, W, H, mode=mode).view(np.int32).reshape(-1, 4)
        assert (ref[:, 0] >= 0).mean() > 0.2
        t = sc.tuning()
        assert t["ray_lanes"] == 1
        for lanes in (2, 4, 8, 32, 1):
            for stage in (0, 1024):
                sc.set_tuning(stage, t["queue_kind_major"], t["refill_min"], 32, lanes)
                got = _hits(sc.trace_primary(cam, W, H, mode))
                assert np.array_equal(got, ref), (lanes, stage)
        # the counting pass is one lane per ray whatever the setting
        sc.set_tuning(t["stage_nodes"], t["queue_kind_major"], t["refill_min"], 32, 4)
        _, rc = po.primary_kd(kd, cam, W, H, mode=mode, counts=True)
        cnt = sc.count_primary(cam, W, H, mode).cpu().numpy()
        assert np.array_equal(cnt, rc.view(np.uint32).reshape(-1, 4).astype(np.int32))


@pytest.mark.parametrize("lanes", [2, 4, 32])
def test_lanes_per_ray_visit_cap(cuda, lanes):
    """With several lanes per ray a walk stopped at the leaf-visit cap is
    counted once and keeps the oracle's hit."""
    cfg = rb.configs.SoupConfig(num_tris=8192, width=160, height=120)
    cam = cfg.camera()
    W, H = cfg.width, cfg.height
    with rb.KDScene.from_packed(cfg.packed(), rb.kd_params(leaf_size=8, max_leaf_visits=2)) as sc:
        st, kd = _kd(sc)
        ref, rc = po.primary_kd(kd, cam, W, H, max_visits=2, counts=True)
        t = sc.tuning()
        sc.set_tuning(t["stage_nodes"], t["queue_kind_major"], t["refill_min"], 32, lanes)
        got = _hits(sc.trace_primary(cam, W, H))
        assert np.array_equal(got, ref.view(np.int32).reshape(-1, 4))
        n_cut = int((rc["status"] == 1).sum())
        assert n_cut > 100 and sc.truncated() == n_cut


def test_autotune_primary_considers_lanes(cuda):
    cfg = rb.configs.SoupConfig(num_tris=65536)
    with rb.KDScene.from_packed(cfg.packed(), cfg.kd_params()) as sc:
        st, kd = _kd(sc)
        cam = cfg.camera()
        best = sc.autotune_primary(cam, 128, 128)
        assert best["ray_lanes"] in (1, 2, 4, 8, 32)
        assert sc.tuning()["ray_lanes"] == best["ray_lanes"]
        ref = po.primary_kd(kd, cam, 128, 128).view(np.int32).reshape(-1, 4)
        assert np.array_equal(_hits(sc.trace_primary(cam, 128, 128)), ref)


def test_heightfield_kernel_bitexact(cuda):
    cfg = rb.configs.HeightfieldConfig()
    P = po.perm(cfg.seed)
    for cells in (7, 256, 1024):
        v = rb.heightfield(cfg.fbm(), cells, cfg.lo, cfg.hi).cpu().numpy()
        ov, of = po.heightfield(P, cells, cfg.lo, cfg.hi, cfg.octaves, cfg.amplitude)
        assert np.array_equal(v, ov), cells
        assert np.array_equal(rb.grid_faces(cells), of)


def test_fbm_kernel_bitexact(cuda):
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "noise.npz"))
    pts = torch.from_numpy(g["pts"]).cuda()
    for o in (1, 6, 8):
        got = rb.generate_noise(rb.fbm_params(seed=2016, octaves=o), pts).cpu().numpy()
        assert np.array_equal(got, g[f"fbm{o}"]), o
    rng = np.random.default_rng(5)
    big = rng.uniform(-1000, 1000, (1 << 20, 3)).astype(np.float32)
    got = rb.generate_noise(rb.fbm_params(seed=7, octaves=8, scale=0.25, amplitude=3.0),
                            torch.from_numpy(big).cuda()).cpu().numpy()
    assert np.array_equal(got, po.fbm_batch(po.perm(7), big, 8, scale=0.25, amp=3.0))


def test_fbm_lattice_edges_bitexact(cuda):
    """Points on and next to lattice planes (fractional parts 0 and just
    below 1), at the 255/256 wrap of the table, negative, and with
    coordinates of large magnitude: every corner case of the lattice
    indexing and of the gradient selection, bit-exact against the oracle."""
    rng = np.random.default_rng(11)
    ints = rng.integers(-600, 600, (40000, 3)).astype(np.float32)
    wrap = np.array([255.0, 256.0, -1.0, -256.0, 511.0, 512.0], np.float32)
    ints[:6000] = rng.choice(wrap, (6000, 3))
    below = np.nextafter(ints, np.float32(-np.inf))
    above = np.nextafter(ints, np.float32(np.inf))
    half = ints + np.float32(0.5)
    large = rng.uniform(-1e6, 1e6, (20000, 3)).astype(np.float32)
    pts = np.concatenate([ints, below, above, half, large, -ints]).astype(np.float32)
    for seed, octaves in ((2016, 1), (3, 8)):
        params = rb.fbm_params(seed=seed, octaves=octaves)
        got = rb.generate_noise(params, torch.from_numpy(pts).cuda()).cpu().numpy()
        assert np.array_equal(got.view(np.uint32),
                              po.fbm_batch(po.perm(seed), pts, octaves).view(np.uint32)), seed


def test_render_ao_small_bitexact(cuda):
    cfg = rb.configs.HeightfieldConfig(cells=128, width=320, height=180)
    P = po.perm(cfg.seed)
    verts, faces = po.heightfield(P, cfg.cells, cfg.lo, cfg.hi, cfg.octaves, cfg.amplitude)
    packed = rb.pack_triangles(verts, faces)
    cam = cfg.camera()
    light = rb.unit(cfg.light_dir)
    with rb.KDScene.from_mesh(verts, faces) as sc:
        st, kd = _kd(sc)
        hits, mask, nsec = sc.render_ao(cam, cfg.width, cfg.height, light, cfg.ao_length,
                                        cfg.bias, cfg.ao_seed)
        hits, mask, nsec = _hits(hits), mask.cpu().numpy(), int(nsec.item())
    rh, rm, rn = po.frame_ao(kd, packed, cam, cfg.width, cfg.height, light, cfg.ao_length,
                             cfg.bias, cfg.ao_seed)
    assert np.array_equal(hits, rh.view(np.int32).reshape(-1, 4))
    assert np.array_equal(mask.view(np.uint32), rm)
    assert nsec == rn == 5 * int((rh["id"] >= 0).sum())
    # the AO and shadow bits are not trivially all-set or all-clear
    hit = (rm & 1) == 1
    assert 0.05 < ((rm[hit] >> 1) & 1).mean() < 0.98
    assert 0.05 < ((rm[hit] >> 2) & 15).astype(bool).mean() <= 1.0


def test_render_ao_config1_sampled(cuda):
    """Full 2.1M-triangle heightfield at 1920x1080: heights from the GPU,
    bit-exact hits/masks on a pixel sample, size-independent checks on all."""
    cfg = rb.configs.HeightfieldConfig()
    verts, faces = cfg.mesh_on_device()
    packed = rb.pack_triangles(verts, faces)
    cam = cfg.camera()
    light = rb.unit(cfg.light_dir)
    W, H = cfg.width, cfg.height
    with rb.KDScene.from_mesh(verts, faces) as sc:
        st, kd = _kd(sc)
        hits, mask, nsec = sc.render_ao(cam, W, H, light, cfg.ao_length, cfg.bias, cfg.ao_seed)
        hits2, mask2, _ = sc.render_ao(cam, W, H, light, cfg.ao_length, cfg.bias, cfg.ao_seed)
        hits, mask, nsec = _hits(hits), mask.cpu().numpy().view(np.uint32), int(nsec.item())
        prim = _hits(sc.trace_primary(cam, W, H))
    # deterministic frame to frame, and the AO frame's primary pass equals the plain one
    assert np.array_equal(hits, _hits(hits2)) and np.array_equal(mask, mask2.cpu().numpy().view(np.uint32))
    assert np.array_equal(hits, prim)
    assert nsec == 5 * int((hits[:, 0] >= 0).sum())
    assert np.array_equal(mask & 1, (hits[:, 0] >= 0).astype(np.uint32))
    pix = np.random.default_rng(6).choice(W * H, 4000, replace=False).astype(np.uint32)
    rh, rm, _ = po.frame_ao(kd, packed, cam, W, H, light, cfg.ao_length, cfg.bias, cfg.ao_seed,
                            pixels=pix)
    assert np.array_equal(hits[pix], rh.view(np.int32).reshape(-1, 4))
    assert np.array_equal(mask[pix], rm)
    _assert_vs_bruteforce(hits, packed, st, cam, W, H, pix[:300])


def test_sdf_small_bitexact(cuda):
    tc = rb.configs.TerrainConfig(width=96, height=54)
    out = rb.sphere_trace(tc.params(), tc.camera(), tc.width, tc.height).cpu().numpy()
    ref = po.sdf_image(po.perm(tc.seed), tc.camera(), tc.width, tc.height)
    f = out.view(np.float32)
    assert np.array_equal(out[:, 7].view(np.uint32), ref["status"])
    assert np.array_equal(out[:, 6].view(np.uint32), ref["steps"])
    hit = ref["status"] == 1
    assert hit.sum() > 1000
    assert np.array_equal(f[hit, 0:3], ref["pos"][hit])
    assert np.array_equal(f[hit, 3:6], ref["normal"][hit])


def test_sdf_config2_sampled(cuda):
    tc = rb.configs.TerrainConfig()
    W, H = tc.width, tc.height
    out = rb.sphere_trace(tc.params(), tc.camera(), W, H).cpu().numpy()
    pix = np.random.default_rng(8).choice(W * H, 3000, replace=False).astype(np.uint32)
    ref = po.sdf_image(po.perm(tc.seed), tc.camera(), W, H, pixels=pix)
    assert np.array_equal(out[pix, 7].view(np.uint32), ref["status"])
    assert np.array_equal(out[pix, 6].view(np.uint32), ref["steps"])
    f = out.view(np.float32)
    hit = ref["status"] == 1
    assert np.array_equal(f[pix][hit, 0:6], np.concatenate([ref["pos"], ref["normal"]], 1)[hit])
    # whole image: hits lie on the surface and normals are unit length
    st = out[:, 7].view(np.uint32)
    allhit = st == 1
    P = po.perm(tc.seed)
    pos = f[allhit, 0:3]
    # the kernel's density is fma(-3, fbm, y); 3*fbm is exact in float64
    dens = pos[:, 1].astype(np.float64) - 3.0 * po.fbm_batch(P, pos, 8, scale=0.25).astype(np.float64)
    assert np.all(dens < 1e-4 + 1e-9)
    nrm = np.linalg.norm(f[allhit, 3:6], axis=1)
    assert np.all(np.abs(nrm - 1) < 1e-5)
    assert allhit.mean() > 0.3


def test_tunings_give_identical_frames(cuda):
    """Staging depth, queue layout and refill threshold change only speed."""
    cfg = rb.configs.HeightfieldConfig(cells=128, width=320, height=180)
    P = po.perm(cfg.seed)
    verts, faces = po.heightfield(P, cfg.cells, cfg.lo, cfg.hi, cfg.octaves, cfg.amplitude)
    cam = cfg.camera()
    light = rb.unit(cfg.light_dir)
    with rb.KDScene.from_mesh(verts, faces) as sc:
        ref = None
        for stage, km, refill in ((0, 0, 32), (64, 1, 4), (4096, 0, 8), (4096, 1, 1), (1, 1, 32),
                                  (0, 2, 8), (4096, 2, 1), (64, 2, 32)):
            sc.set_tuning(stage, km, refill)
            got = [x.cpu().numpy() for x in sc.render_ao(cam, cfg.width, cfg.height, light,
                                                         cfg.ao_length, cfg.bias, cfg.ao_seed)]
            if ref is None:
                ref = got
            else:
                for a, b in zip(got, ref):
                    assert np.array_equal(a, b), (stage, km, refill)
        params = rb.ao_params(cfg.light_dir, cfg.ao_length, cfg.bias, cfg.ao_seed)
        best = sc.autotune_ao(cam, cfg.width, cfg.height, params)
        assert best["frame_ms"] > 0 and 1 <= best["refill_min"] <= 32
        assert sc.tuning()["refill_min"] == best["refill_min"]
        got = [x.cpu().numpy() for x in sc.render_ao(cam, cfg.width, cfg.height, light,
                                                     cfg.ao_length, cfg.bias, cfg.ao_seed)]
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("cap", [1, 2])
def test_visit_cap_is_reported(cuda, cap):
    """The reference stops a walk after 50 leaves without saying so
    (ray_functions.cuh:284).  Here a walk that reaches max_leaf_visits stops
    too, with the closest hit among the leaves it reached, and is reported:
    the per-ray status of re_count_primary, the scene's truncated-ray count
    and bit 6 of the AO mask, each equal to the oracle's."""
    cfg = rb.configs.SoupConfig(num_tris=8192, width=160, height=120)
    packed = cfg.packed()
    cam = cfg.camera()
    W, H = cfg.width, cfg.height
    with rb.KDScene.from_packed(packed, rb.kd_params(leaf_size=8, max_leaf_visits=cap)) as sc:
        st, kd = _kd(sc)
        ref, rc = po.primary_kd(kd, cam, W, H, max_visits=cap, counts=True)
        got = _hits(sc.trace_primary(cam, W, H))
        assert np.array_equal(got, ref.view(np.int32).reshape(-1, 4))
        n_cut = int((rc["status"] == 1).sum())
        assert n_cut > 100
        assert sc.truncated() == n_cut
        cnt = sc.count_primary(cam, W, H).cpu().numpy()
        assert np.array_equal(cnt[:, 3], rc["status"].astype(np.int32))
        assert sc.truncated() == n_cut
    hcfg = rb.configs.HeightfieldConfig(cells=96, width=200, height=120)
    verts, faces = po.heightfield(po.perm(hcfg.seed), hcfg.cells, hcfg.lo, hcfg.hi,
                                  hcfg.octaves, hcfg.amplitude)
    packed = rb.pack_triangles(verts, faces)
    hcam = hcfg.camera()
    light = rb.unit(hcfg.light_dir)
    hcap = 4 * cap  # 4: 1.7k of 24k pixels hit; 8: 9.8k (both with truncated shadow/AO rays)
    with rb.KDScene.from_mesh(verts, faces, rb.kd_params(max_leaf_visits=hcap)) as sc:
        st, kd = _kd(sc)
        hits, mask, nsec = sc.render_ao(hcam, hcfg.width, hcfg.height, light, hcfg.ao_length,
                                        hcfg.bias, hcfg.ao_seed)
        cut = sc.truncated()
        rh, rm, rn, tot = po.frame_ao(kd, packed, hcam, hcfg.width, hcfg.height, light,
                                      hcfg.ao_length, hcfg.bias, hcfg.ao_seed, max_visits=hcap,
                                      totals=True)
        assert np.array_equal(_hits(hits), rh.view(np.int32).reshape(-1, 4))
        assert np.array_equal(mask.cpu().numpy().view(np.uint32), rm)
        assert int(nsec.item()) == rn
        assert cut == int(tot[8] + tot[9]) and tot[8] > 0 and tot[9] > 0
        assert ((rm >> 6) & 1).sum() > 0
    # without a cap in reach nothing is reported
    with rb.KDScene.from_mesh(verts, faces) as sc:
        _, mask, _ = sc.render_ao(hcam, hcfg.width, hcfg.height, light, hcfg.ao_length,
                                  hcfg.bias, hcfg.ao_seed)
        assert sc.truncated() == 0
        assert not ((mask.cpu().numpy().view(np.uint32) >> 6) & 1).any()
