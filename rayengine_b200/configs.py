"""The seeded synthetic workloads (no dataset is involved; every input is
generated from a seed with the shapes and distributions below).

soup:        N triangles, centroid ~ U[-1,1]^3, vertex offsets ~ N(0, 0.02)
             per axis (mt19937_64 seed 0); camera at (0,0,3) looking at the
             origin, 60x60 degree field of view, 512x512 primary rays.  The
             "1M-triangle scene" is the same generator with N = 2^20.
heightfield: 1024x1024 cells over [-10,10]^2 (2,097,152 triangles), height =
             2 * fBm(x, 0, z) with RPerlinNoise(2016), 6 octaves, lacunarity 2,
             gain 0.5; camera at (0,8,-14) looking at the origin, 60 degree
             horizontal field of view, 1920x1080, plus one shadow ray toward
             normalize(0.3,1,0.2) and four cosine-weighted AO rays of length 1
             per primary hit.
terrain SDF: d(p) = p.y - 3 * fBm(0.25 p), RPerlinNoise(2016), 8 octaves;
             camera at (0,6,-20) looking at the origin, 60 degree horizontal
             field of view, 1920x1080, step 0.6 d, eps 1e-4, tmax 200, at most
             512 steps.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import api

PERLIN_SEED = 2016  # RPerlinNoise's default seed (PerlinNoise.h:16)


@dataclass
class SoupConfig:
    num_tris: int = 65536
    seed: int = 0
    width: int = 512
    height: int = 512
    campos: tuple = (0.0, 0.0, 3.0)
    lookat: tuple = (0.0, 0.0, 0.0)
    fov: tuple = (60.0, 60.0)

    def camera(self):
        return api.build_camera(self.campos, self.lookat, self.fov)

    def kd_params(self):
        """Tree parameters for random soups: the configured SAH tree (depth
        <= 24, leaves of up to 8 references: their large overlapping
        triangles duplicate heavily when split finer) with an empty-side
        bonus of 0.15.  Measured on B200: the 2^16 soup's primary pass is
        3.6 % faster than at depth 40 (the 2^20 soup is level)."""
        return api.kd_params(max_depth=24, leaf_size=8, empty_bonus=0.15)

    def packed(self) -> np.ndarray:
        v = api.triangle_soup(self.num_tris, self.seed)
        p = np.zeros((self.num_tris, 12), np.float32)
        p[:, 0:3] = v[:, 0]
        p[:, 4:7] = v[:, 1] - v[:, 0]
        p[:, 8:11] = v[:, 2] - v[:, 0]
        return p


@dataclass
class HeightfieldConfig:
    cells: int = 1024
    lo: float = -10.0
    hi: float = 10.0
    octaves: int = 6
    amplitude: float = 2.0
    seed: int = PERLIN_SEED
    width: int = 1920
    height: int = 1080
    campos: tuple = (0.0, 8.0, -14.0)
    lookat: tuple = (0.0, 0.0, 0.0)
    fov_x: float = 60.0
    light_dir: tuple = (0.3, 1.0, 0.2)
    ao_length: float = 1.0
    bias: float = 1e-4
    ao_seed: int = 7

    def camera(self):
        fy = api.vertical_fov(self.fov_x, self.width, self.height)
        return api.build_camera(self.campos, self.lookat, (self.fov_x, fy))

    def fbm(self):
        return api.fbm_params(seed=self.seed, octaves=self.octaves, amplitude=self.amplitude)

    def mesh_on_device(self, stream=None):
        """(vertices as a host array, faces) with heights computed on the GPU."""
        verts = api.heightfield(self.fbm(), self.cells, self.lo, self.hi, stream=stream)
        return verts.cpu().numpy(), api.grid_faces(self.cells)


@dataclass
class TerrainConfig:
    seed: int = PERLIN_SEED
    octaves: int = 8
    scale: float = 0.25
    amplitude: float = 3.0
    step_factor: float = 0.6
    eps: float = 1e-4
    tmax: float = 200.0
    max_steps: int = 512
    width: int = 1920
    height: int = 1080
    campos: tuple = (0.0, 6.0, -20.0)
    lookat: tuple = (0.0, 0.0, 0.0)
    fov_x: float = 60.0

    def camera(self):
        fy = api.vertical_fov(self.fov_x, self.width, self.height)
        return api.build_camera(self.campos, self.lookat, (self.fov_x, fy))

    def params(self):
        return api.sdf_params(self.seed, self.octaves, self.scale, self.amplitude,
                              self.step_factor, self.eps, self.tmax, self.max_steps)


@dataclass
class SdfFrameConfig:
    """The shaded terrain frame: TerrainConfig's field and camera with the
    shading settings of re_sdf_shade_params_default (the light at (20, 40,
    20) with intensity 30000, the reference's soft-shadow factor 32, shadow
    rays from 0.05 to 40 in at most 128 steps, the sun at 0.18 pi from the
    zenith, terrain top 2, soft shadows and light on)."""
    terrain: TerrainConfig = None
    light_pos: tuple = (20.0, 40.0)
    light_intensity: float = 30000.0
    soft_shadow_k: float = 32.0
    shadow_tmin: float = 0.05
    shadow_tmax: float = 40.0
    shadow_max_steps: int = 128
    sun_dir: tuple = (0.0, 0.844327926, 0.535826795)  # (0, cos a, sin a), a = 0.18 pi
    max_y: float = 2.0
    fog_density: float = 0.02
    vignetting_k: float = 0.25
    flags: int = 1  # RE_SDF_SHADE

    def __post_init__(self):
        if self.terrain is None:
            self.terrain = TerrainConfig()

    def shade(self):
        """re_sdf_shade_params built in Python (no library call)."""
        from ._lib import re_sdf_shade_params

        p = re_sdf_shade_params()
        p.light_pos[:] = [float(x) for x in self.light_pos]
        p.light_intensity, p.soft_shadow_k = self.light_intensity, self.soft_shadow_k
        p.shadow_tmin, p.shadow_tmax = self.shadow_tmin, self.shadow_tmax
        p.shadow_max_steps = self.shadow_max_steps
        p.sun_dir[:] = [float(x) for x in self.sun_dir]
        p.max_y, p.fog_density, p.vignetting_k = self.max_y, self.fog_density, self.vignetting_k
        p.flags = self.flags
        return p


@dataclass
class NeuralTerrainConfig:
    """Neural SDF surrogate of the terrain field above: training set, network
    and tracer settings."""
    terrain: TerrainConfig = None
    box_tmax: float = 200.0      # network box: the view frustum up to this t ...
    box_y: tuple = (-6.0, 12.0)  # ... with y clamped to this range
    f0: float = 2.0              # lowest feature frequency (cycles per box half-width)
    init_seed: int = 5
    num_points: int = 8 << 20    # 50% uniform in the box, 50% near the surface
    data_seed: int = 11
    train_steps: int = 20000
    batch: int = 65536
    lr: float = 1e-3
    lipschitz_samples: int = 200000
    lipschitz_h: float = 1e-2
    lipschitz_quantile: float = 0.5
    # Network phase: one cone per 16x16 pixel tile, 16 lanes per cone
    # evaluating guessed successive steps in one pass, each step safety
    # `cone_safety` / L (measured on B200, 1080p, 20k-step network: cone +
    # exact phase 3.21 ms against 7.62 ms for the per-ray network march
    # below, the exact tracer then 4.17 ms; on the faster field 2.12 ms
    # with 16 lanes and safety 1.5 against 2.19 ms with 8 lanes and 1.2,
    # same median error, p95 and silhouettes).
    # Exact phase from the cone's stop: the exact tracer's steps allowed to
    # grow 1.5x along the secant of the last two samples (median hit error
    # 8e-5, ~850 of 2.07M pixels whose hit/miss differs from the exact
    # tracer; relax 1.0: 27 pixels, 3.98 ms with 8x8 cones of one lane;
    # relax 2.0: 2.94 ms, 2,100 pixels, median error 4e-4); the root search
    # ends when its secant point moves less than 1e-4 (3.23 -> 3.17 ms, same
    # median error).
    safety: float = 1.2          # the per-ray network march's step safety
    cone_safety: float = 1.5
    switch_dist: float = 0.3
    min_step: float = 0.05
    max_network_steps: int = 64  # per-ray march steps
    # passes of a cone (16 steps guessed per pass): the cone phase lasts as
    # long as its longest chains of passes; capped at 12 the far tiles hand
    # over earlier (measured on B200: 2.10 -> 2.01 ms per frame, cone phase
    # 0.27 -> 0.20 ms, exact evaluations 14.41 -> 14.59 per ray, the same
    # median error and p95; 8 passes: 2.05 ms)
    cone_max_passes: int = 12
    root_steps: int = 4
    cone_tile: int = 16
    cone_lanes: int = 16
    relax: float = 1.5
    root_tol: float = 1e-4
    # the normal: the exact field's analytic gradient at the hit, in a
    # second pass over the hits (about 1.8 field evaluations of arithmetic
    # per hit, against 4 for the reference's tetrahedral normal
    # compute_sdf_normal_tet or 6 for central differences, taken inside the
    # march).  Measured on B200: 2.93 -> 2.66-2.70 ms per frame, hits
    # unchanged, and the normal within 1e-5 deg (median) of the FP64
    # gradient, where the finite-difference stencils at the exact tracer's
    # radius 0.002 t are 18 deg (median) from it
    normal_taps: int = 1
    # the per-ray network march (cone_tile 0), measured on B200: safety 1.2
    # with the hand-over at 0.6 gives 7.49 ms against 8.97 ms at (0.9,
    # 0.3), with the same median error (8e-6) and ~45 of 2.07M pixels whose
    # hit/miss differs from the exact tracer; larger steps (1.5-2.5) or the
    # 0.25 gradient quantile run faster but let rays through thin ridges
    # (550-3500 pixels)
    per_ray_switch_dist: float = 0.6

    def __post_init__(self):
        if self.terrain is None:
            self.terrain = TerrainConfig()

    def box(self):
        t = self.terrain
        return api.NeuralSDF.box_for_camera(t.camera(), t.width, t.height, self.box_tmax,
                                            self.box_y[0], self.box_y[1])

    def build(self, train_steps=None):
        """Generate the training set, train, and return (model, trace params, losses)."""
        t = self.terrain
        lo, hi = self.box()
        m = api.NeuralSDF(lo, hi, self.f0, self.init_seed)
        m.generate(t.params(), t.camera(), t.width, t.height, self.num_points, self.data_seed)
        losses = m.train(self.train_steps if train_steps is None else train_steps, self.batch,
                         self.lr)
        lip = m.lipschitz(self.lipschitz_samples, self.lipschitz_h, self.lipschitz_quantile)
        tp = self.trace_params(lip)
        return m, tp, losses

    def trace_params(self, lipschitz):
        """The cone tracer's settings (the default method)."""
        return api.nsdf_trace_params(lipschitz, self.cone_safety, self.switch_dist, self.min_step,
                                     self.cone_max_passes, 0, self.root_steps, self.relax,
                                     cone_tile=self.cone_tile, cone_lanes=self.cone_lanes,
                                     normal_taps=self.normal_taps, root_tol=self.root_tol)

    def per_ray_params(self, lipschitz):
        """The per-ray network march with its hand-over queue, the exact
        tracer's plain steps and central-difference normal."""
        return api.nsdf_trace_params(lipschitz, self.safety, self.per_ray_switch_dist,
                                     self.min_step, self.max_network_steps, 0, self.root_steps)


@dataclass
class BatchConfig:
    """Batched wavefront workload: seeded scenes of uneven size, soups
    (triangle counts log-uniform in tri_range, cameras as SoupConfig) and
    volumetric terrains (TerrainConfig with a per-scene seed and
    amplitude), each at a resolution drawn from `resolutions`."""
    num_scenes: int = 32
    seed: int = 4
    terrain_fraction: float = 0.25
    tri_range: tuple = (10_000, 2_000_000)
    resolutions: tuple = ((640, 360), (1280, 720), (1920, 1080))
    max_depth: int = 4
    path_seed: int = 11
    mesh_bias: float = 1e-4

    def specs(self):
        """Scene descriptions (no device work): dicts with kind, size and seeds."""
        rng = np.random.default_rng(self.seed)
        out = []
        for i in range(self.num_scenes):
            w, h = self.resolutions[int(rng.integers(len(self.resolutions)))]
            albedo = float(rng.uniform(0.5, 0.8))
            if rng.random() < self.terrain_fraction:
                out.append(dict(kind="terrain", seed=PERLIN_SEED + i,
                                amplitude=float(rng.uniform(2.0, 3.5)), width=w, height=h,
                                albedo=albedo))
            else:
                lo, hi = np.log(self.tri_range[0]), np.log(self.tri_range[1])
                n = int(round(float(np.exp(rng.uniform(lo, hi)))))
                out.append(dict(kind="soup", num_tris=n, seed=1000 + i, width=w, height=h,
                                albedo=albedo))
        return out

    @staticmethod
    def shard(specs, rank: int, world: int):
        """This rank's scenes when a batch is split across `world` GPUs:
        largest scenes first, each to the rank with the fewest pixels so
        far (ties to the lower rank); deterministic on every rank."""
        load = [0] * world
        owner = {}
        order = sorted(range(len(specs)),
                       key=lambda i: (-specs[i]["width"] * specs[i]["height"], i))
        for i in order:
            r = min(range(world), key=lambda k: (load[k], k))
            owner[i] = r
            load[r] += specs[i]["width"] * specs[i]["height"]
        return [specs[i] for i in range(len(specs)) if owner[i] == rank]

    def build(self, rank: int = 0, world: int = 1):
        """(Batch, [KDScene]) on the current device: all scenes, or this
        rank's shard when world > 1."""
        scenes, meshes = [], []
        specs = self.specs() if world <= 1 else self.shard(self.specs(), rank, world)
        for s in specs:
            w, h = s["width"], s["height"]
            if s["kind"] == "soup":
                sc = SoupConfig(num_tris=s["num_tris"], seed=s["seed"], width=w, height=h)
                m = api.KDScene.from_packed(sc.packed(), sc.kd_params())
                meshes.append(m)
                cam = api.build_camera(sc.campos, sc.lookat,
                                       (60.0, api.vertical_fov(60.0, w, h)))
                scenes.append(dict(mesh=m, camera=cam, width=w, height=h, albedo=s["albedo"]))
            else:
                tc = TerrainConfig(seed=s["seed"], amplitude=s["amplitude"], width=w, height=h)
                scenes.append(dict(terrain=tc.params(), camera=tc.camera(), width=w, height=h,
                                   albedo=s["albedo"]))
        b = api.Batch(scenes, self.max_depth, self.path_seed, self.mesh_bias)
        return b, meshes
