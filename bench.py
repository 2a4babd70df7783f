#!/usr/bin/env python
"""Throughput benchmark of the rope kd-tree ray-query path on B200.

Default workload (one "step" = one frame): the 1024x1024-cell fBm heightfield
(2,097,152 triangles, SAH kd-tree with ropes built once on the host and
resident in HBM), 1920x1080 primary rays + one shadow ray and four
cosine-weighted AO rays (length 1) per primary hit.  Metric: Mrays/s over all
rays traced in the frame.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config heightfield_ao|soup|soup1m|soup1m_2k|terrain_sdf|sdf_frame|nsdf_terrain|batch32]
                    [--tree tuned|configured]

The mesh workloads run over the library's B200-tuned kd-tree; the same
frame over the tree the configuration names (SAH, depth <= 24, leaf <= 8)
is timed after the headline and reported under "configured_tree" (hits do
not depend on the tree).  On one GPU the line also carries the CPU baseline
(the oracle's traversal of the same tree on all host cores) and "parity",
the checker's comparison of the last frame with the oracle and with the
reference as shipped.

Under torchrun (N > 1) every rank holds a replica of the scene and renders
its own frame (rays are independent, nothing is exchanged): weak scaling,
value = rays of all ranks / the slowest rank's time.  Rank 0 prints one JSON
line.  `--impl reference` times the reference's own CPU path on all host
cores over a bounded pixel sample of the same frame: for meshes its
RKDTreeCPU and CPU ray query compiled from its sources (the tree ships as a
single leaf, so every query is brute-force Moller-Trumbore); for the SDF
and batch workloads the oracle's restatement of its march.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


# ------------------------------------------------------------- plumbing
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world: int, backend: str = "nccl"):
    import datetime

    import torch.distributed as dist

    if world > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return dist


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Slowest rank's time (the only cross-rank exchange of the benchmark)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: int, world: int, device=None) -> int:
    """Total of a per-rank count (set-up only, outside the timed region)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


# FP32 issue peak of the SIMT pipes, nominal: 148 SMs x 128 FP32 lanes x
# 1965 MHz, one operation (an FMA counts once) per lane per clock.  The
# roofline's denominator is the FMA rate measured in the run
# (re_measure_fp32_fma); the nominal figure is printed beside it.
FP32_TOPS_NOMINAL = 148 * 128 * 1.965e9 / 1e12
# FP32 operations of one evaluation of d(p) = p.y - 3 fBm(0.25 p), 8
# octaves, counted from the formula (FMA = 1): Perlin 70 (3 floor, 3 frac,
# 15 quintic, 3 offsets, 16 gradient dots, 19 for k1..k7, 11 interpolation)
# + 5 fBm bookkeeping per octave, + 4 for the scale and the final FMA
SDF_OPS_PER_EVAL = 8 * 75 + 4
# one analytic gradient of the field (the neural tracer's normal): per
# octave 3 floor, 3 frac, 15 quintic, 3 offsets, 12 fade derivatives, 16
# gradient dots, 19 for k1..k7, 23 corner weights, 36 for the three
# components, 3 accumulations, 3 coordinate doublings; + 6 for the scale
# and the final FMA, + 8 to normalise
SDF_GRAD_OPS_PER_EVAL = 8 * 136 + 14
# BF16 tensor FLOPs of one network evaluation: 2 (128*64 + 3*64*64 + 64)
NSDF_FLOPS_PER_EVAL = 41088


def measure_l2_gbs(torch) -> float:
    """L2 read bandwidth measured in this run by the library's probe
    (re_measure_l2_read: 16-byte L2-only loads over a 32 MB L2-resident
    buffer, 100 passes in one launch).  The traversal kernels' reads mostly
    hit L2; no measured L2 figure comes with the hardware peaks."""
    import rayengine_b200 as rb

    return round(rb.measure_l2_read_gbs(32 << 20, 100), 1)


def measure_fp32_tops(torch) -> float:
    """FP32 FMA rate measured in this run by the library's probe
    (re_measure_fp32_fma: 8 independent FMA chains per thread, 8 blocks of
    256 threads per SM), in 10^12 FMAs/s."""
    import rayengine_b200 as rb

    return round(rb.measure_fp32_fma_tops(1 << 16), 3)


def fp32_roofline(kernel, ops, ms, peaks, name, **extra):
    """Roofline of a SIMT field kernel: `ops` algorithmic FP32 operations
    (FMA = 1) in `ms`, against the FMA rate measured in the run."""
    achieved = ops / (ms / 1e3) / 1e12
    peak = peaks.get("fp32_tops") or FP32_TOPS_NOMINAL
    src = ("measured in this run (re_measure_fp32_fma)" if peaks.get("fp32_tops")
           else "nominal 148 SMs x 128 FP32 lanes x 1965 MHz")
    out = {"bound": "fp32-simt", "kernel": kernel, "achieved": round(achieved, 3),
           "peak": round(peak, 2), "unit": "Tops/s", "frac": round(achieved / peak, 4),
           "peak_source": src, "nominal_peak": round(FP32_TOPS_NOMINAL, 2),
           "alg_ops_per_launch": ops}
    out.update(extra)
    out["traffic"] = ncu_traffic(f"{name}:{kernel}")
    return out


def hbm_roofline(wl, phase_ms, peaks):
    ab = wl.alg_bytes()
    lb = wl.layout_bytes() if hasattr(wl, "layout_bytes") else {}
    dom = max(phase_ms, key=phase_ms.get)
    achieved = ab[dom] / (phase_ms[dom] / 1e3) / 1e9
    out = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1),
           "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4),
           "peak_source": peaks["source"], "alg_bytes_per_launch": ab[dom],
           "alg_bytes_model": "per ray 16 (hit) + 16/inner node + 48/leaf + 4/reference + "
                              "48/triangle test (+32 per stored ray)",
           "traffic": ncu_traffic(f"{wl.name}:{dom}")}
    if dom in lb:
        out["layout_bytes_per_launch"] = lb[dom]
    if peaks.get("l2_gbs"):
        out["l2"] = {"peak": peaks["l2_gbs"], "frac": round(achieved / peaks["l2_gbs"], 4),
                     "peak_source": "measured in this run (re_measure_l2_read)"}
    return out


def traversal_bytes(rays, inner, leaf, tests, stored=0):
    """Algorithmic bytes of a traversal launch: 16 (hit out) per ray, 16 per
    inner-node visit, 48 per leaf visit (24-byte box + 24-byte ropes), 4 per
    triangle reference read and 48 per triangle test, plus 32 per stored ray
    read or written.  The visit and test counts are the traversal's own
    (equal to the oracle's walk of the same tree on the same rays)."""
    return 16 * rays + 16 * inner + 48 * leaf + 52 * tests + 32 * stored


def layout_bytes(rays, inner, leaf, tests, stored=0, hit_bytes=16):
    """Bytes the kernels' own records move: 8 per inner node, 36 per leaf
    (32-byte box and range, 4-byte rope), 48 per triangle reference (with
    its vertex data), plus the hit records and stored rays."""
    return hit_bytes * rays + 8 * inner + 36 * leaf + 48 * tests + 32 * stored


def kd_description(params, choice):
    return {"max_depth": params.max_depth, "leaf_size": params.leaf_size,
            "empty_bonus": round(params.empty_bonus, 4),
            "cost_traversal": params.cost_traversal, "cost_intersect": params.cost_intersect,
            "choice": choice}


CONFIGURED_TREE = dict(max_depth=24, leaf_size=8)  # configs 0/1: SAH, depth <= 24, leaf <= 8


def hit_parity(got, packed, st, kd, cam, W, H, pix_kd, pix_ref, ref_mesh=None):
    """Checker (oracle) comparison of a primary pass's hits `got` (W*H, 4 int32):
    bit-exact against the oracle's walk of the same tree on pix_kd; against the
    reference as shipped (brute force in index order, strict <) on pix_ref with
    the FP64 edge-margin rule; and, when ref_mesh = (verts, faces) is given,
    hit/miss and t against the reference's own compiled CPU query."""
    from oracle import pyoracle as po

    out = {}
    ref = po.primary_kd(kd, cam, W, H, pixels=pix_kd)
    g = got[pix_kd]
    out["vs_oracle_same_tree"] = {"rays": int(pix_kd.size),
                                  "bitexact": int((g == ref.view(np.int32).reshape(-1, 4)).all(1).sum())}
    bf = po.primary_bruteforce(packed, st["bmin"], st["bmax"], cam, W, H, pixels=pix_ref)
    g = got[pix_ref]
    gid, bid = g[:, 0], bf["id"]
    diff = np.nonzero(gid != bid)[0]
    exempt = 0
    if diff.size:
        o, d = po.camera_rays(cam, W, H, pix_ref[diff])
        m = np.full(diff.size, np.inf)
        for ids in (gid[diff], bid[diff]):
            ok = ids >= 0
            m[ok] = np.minimum(m[ok], po.edge_margin(packed, ids[ok], o[ok], d[ok]))
        exempt = int((m < 1e-6).sum())
    same = (gid == bid) & (bid >= 0)
    gf = g[same, 1:].view(np.float32)
    bv = np.stack([bf["t"], bf["u"], bf["v"]], 1)[same]
    rel = np.abs(gf - bv) / np.maximum(np.abs(bv), 1e-3)
    out["vs_reference_as_shipped"] = {
        "rays": int(pix_ref.size), "hits": int((bid >= 0).sum()), "id_mismatch": int(diff.size),
        "id_mismatch_edge_exempt": exempt, "max_rel_tuv": float(rel.max(initial=0.0)),
        "rule": "ids equal except rays whose FP64 edge margin < 1e-6; t, u, v within 1e-5 relative"}
    if ref_mesh is not None and po.ref_lib() is not None:
        tree = po.RefTree(*ref_mesh)
        o, d = po.camera_rays(cam, W, H, pix_ref)
        t, _, _ = tree.trace(o, d)
        tree.close()
        rh = t < 1e19
        gh = g[:, 0] >= 0
        both = rh & gh
        gt = g[both, 1].view(np.float32)
        out["vs_reference_compiled_query"] = {
            "rays": int(pix_ref.size), "hit_miss_disagree": int((rh != gh).sum()),
            "max_rel_t": float((np.abs(gt - t[both]) / np.abs(t[both])).max(initial=0.0)),
            "what": "RKDTreeCPU::singleRayStacklessIntersect compiled from the reference's sources"}
    return out


def ncu_traffic(key: str):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f).get(key)


# ------------------------------------------------------------ workloads
class HeightfieldAO:
    """Primary + shadow + 4 AO rays over the 2.1M-triangle heightfield."""

    name = "heightfield_ao"

    def __init__(self, torch, tree="tuned", mesh=None):
        import rayengine_b200 as rb

        self.rb = rb
        self.tree = tree
        self.cfg = cfg = rb.configs.HeightfieldConfig()
        self.verts, self.faces = mesh if mesh is not None else cfg.mesh_on_device()
        if tree == "configured":
            self.kd = rb.kd_params(**CONFIGURED_TREE)
            choice = "as configured: SAH, depth <= 24, leaf <= 8 (library defaults for the rest)"
        else:
            self.kd = rb.kd_params()
            choice = ("tuned on B200 (library default); hits do not depend on the tree, "
                      "see configured_tree for the configured one")
        self.kd_desc = kd_description(self.kd, choice)
        t0 = time.time()
        self.scene = rb.KDScene.from_mesh(self.verts, self.faces, self.kd)
        self.build_s = time.time() - t0
        self.cam = cfg.camera()
        self.params = rb.ao_params(cfg.light_dir, cfg.ao_length, cfg.bias, cfg.ao_seed)
        W, H = cfg.width, cfg.height
        self.primary = torch.empty((H * W, 4), dtype=torch.int32, device="cuda")
        self.mask = torch.empty(H * W, dtype=torch.int32, device="cuda")
        self.nsec = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.counts = self.scene.render_ao_counts(self.cam, W, H, self.params)
        self.rays_per_step = self.counts["primary"]["rays"] + self.counts["secondary"]["rays"]
        self.kernels_per_step = 2
        # set-up: the autotuner picks staging depth, queue layout and refill threshold
        self.tuning = self.scene.autotune_ao(self.cam, W, H, self.params)

    def config(self):
        st = self.scene.stats()
        c = self.cfg
        return {"workload": "heightfield 1024x1024 cells (2,097,152 tris) rope kd-tree; 1920x1080 "
                            "primary + 1 shadow + 4 AO rays per hit",
                "triangles": st["num_tris"], "kd_nodes": st["num_nodes"],
                "kd_leaves": st["num_leaves"], "kd_refs": st["num_refs"],
                "kd_build_s": round(self.build_s, 3), "kd_tree": self.kd_desc,
                "image": [c.width, c.height],
                "rays_per_step": self.rays_per_step,
                "secondary_rays_per_step": self.counts["secondary"]["rays"],
                "work_per_ray": {
                    k: {f: round(v[f] / max(1, v["rays"]), 2) for f in ("inner", "leaf", "tests")}
                    for k, v in self.counts.items()},
                "tuning": self.tuning,
                "l2": "flushed between steps (256 MB write)"}

    def phases(self, stream):
        W, H = self.cfg.width, self.cfg.height
        return [
            ("ao_primary", lambda: self.scene.render_ao_primary(self.cam, W, H, self.params,
                                                                self.primary, self.mask, stream)),
            ("ao_secondary", lambda: self.scene.render_ao_secondary(self.mask, self.nsec, stream)),
        ]

    def alg_bytes(self):
        """Algorithmic bytes per launch (traversal_bytes): the primary pass also
        stores the five secondary rays of every hit, the secondary pass reads
        them."""
        p, s = self.counts["primary"], self.counts["secondary"]
        return {"ao_primary": traversal_bytes(p["rays"], p["inner"], p["leaf"], p["tests"], s["rays"]),
                "ao_secondary": traversal_bytes(s["rays"], s["inner"], s["leaf"], s["tests"], s["rays"])}

    def layout_bytes(self):
        p, s = self.counts["primary"], self.counts["secondary"]
        return {"ao_primary": layout_bytes(p["rays"], p["inner"], p["leaf"], p["tests"], s["rays"], 20),
                "ao_secondary": layout_bytes(0, s["inner"], s["leaf"], s["tests"], s["rays"])}

    def configured_variant(self, torch):
        """The same frame over the configured tree (depth 24, leaf 8)."""
        if self.tree == "configured":
            return None
        return HeightfieldAO(torch, tree="configured", mesh=(self.verts, self.faces))

    def parity(self):
        """Checker comparison of the bench's last frame (see hit_parity)."""
        from oracle import pyoracle as po

        st = self.scene.stats()
        nodes, leaves, tris = self.scene.export()
        kd = po.KdTree(nodes, leaves, tris, st["bmin"], st["bmax"])
        packed = self.rb.pack_triangles(self.verts, self.faces)
        W, H = self.cfg.width, self.cfg.height
        got = self.primary.cpu().numpy().reshape(-1, 4)
        mask = self.mask.cpu().numpy().view(np.uint32)
        rng = np.random.default_rng(12)
        pix = rng.choice(W * H, 4000, replace=False).astype(np.uint32)
        light = self.rb.unit(self.cfg.light_dir)
        rh, rm, _ = po.frame_ao(kd, packed, self.cam, W, H, light, self.cfg.ao_length,
                                self.cfg.bias, self.cfg.ao_seed, pixels=pix)
        out = {"ao_frame_vs_oracle_same_tree": {
            "pixels": int(pix.size),
            "hits_bitexact": int((got[pix] == rh.view(np.int32).reshape(-1, 4)).all(1).sum()),
            "masks_equal": int((mask[pix] == rm).sum()),
            "truncated_pixels": int(((mask >> 6) & 1).sum())}}
        out.update(hit_parity(got, packed, st, kd, self.cam, W, H, pix[:2000], pix[:150],
                              (self.verts, self.faces)))
        return out

    def e2e_compute(self, torch, stream):
        W, H = self.cfg.width, self.cfg.height
        self.scene.render_ao(self.cam, W, H, self.cfg.light_dir, self.cfg.ao_length,
                             self.cfg.bias, self.cfg.ao_seed, self.primary, self.mask, self.nsec,
                             stream)

    def e2e_outputs(self):
        return [self.primary, self.mask]

    def e2e_bytes(self):
        W, H = self.cfg.width, self.cfg.height
        import ctypes

        h2d = ctypes.sizeof(self.rb.RCamera) + ctypes.sizeof(self.params)
        return h2d, W * H * 16 + W * H * 4

    def cpu_baseline(self, budget_s=12.0):
        """The oracle's rope traversal of the same tree on the host cores."""
        from oracle import pyoracle as po

        st = self.scene.stats()
        nodes, leaves, tris = self.scene.export()
        kd = po.KdTree(nodes, leaves, tris, st["bmin"], st["bmax"])
        packed = self.rb.pack_triangles(self.verts, self.faces)
        W, H = self.cfg.width, self.cfg.height
        rng = np.random.default_rng(0)
        light = self.rb.unit(self.cfg.light_dir)
        n = 20000
        while True:
            pix = rng.choice(W * H, n, replace=False).astype(np.uint32)
            t0 = time.perf_counter()
            _, _, nsec = po.frame_ao(kd, packed, self.cam, W, H, light, self.cfg.ao_length,
                                     self.cfg.bias, self.cfg.ao_seed, pixels=pix)
            dt = time.perf_counter() - t0
            if dt > budget_s / 4 or n >= W * H:
                break
            n = min(W * H, int(n * min(8.0, budget_s / max(dt, 1e-3))))
        return {"value": round((n + nsec) / dt / 1e6, 4), "unit": "Mrays/s", "cores": po.threads(),
                "kind": "port",
                "sample": f"{n} seeded-random pixels of the 1920x1080 frame with their shadow+AO "
                          f"rays ({n + nsec} rays); oracle rope traversal over the same SAH tree, "
                          "OpenMP schedule(dynamic) over pixels"}



class SoupPrimary:
    name = "soup"

    def __init__(self, torch, num_tris=65536, tree="tuned", packed=None, size=512):
        import rayengine_b200 as rb

        self.rb = rb
        self.tree = tree
        self.num_tris = num_tris
        self.size = size
        if num_tris == 1 << 20:
            self.name = "soup1m" if size == 512 else f"soup1m_{size // 1024}k"
        self.cfg = cfg = rb.configs.SoupConfig(num_tris=num_tris, width=size, height=size)
        self.packed = cfg.packed() if packed is None else packed
        if tree == "configured":
            self.kd = cfg.kd_params()
            for k, v in CONFIGURED_TREE.items():
                setattr(self.kd, k, v)
            choice = "as configured: SAH, depth <= 24, leaf <= 8 (soup empty bonus 0.15)"
        else:
            self.kd = cfg.kd_params()
            choice = ("the configured SAH tree (depth <= 24, leaf <= 8) with the soups' empty "
                      "bonus 0.15, measured on B200 as fast as or faster than deeper trees")
        self.kd_desc = kd_description(self.kd, choice)
        t0 = time.time()
        self.scene = rb.KDScene.from_packed(self.packed, self.kd)
        self.build_s = time.time() - t0
        self.cam = cfg.camera()
        W, H = cfg.width, cfg.height
        self.out = torch.empty((H * W, 4), dtype=torch.int32, device="cuda")
        # set-up: the autotuner picks staging depth and ray refill threshold
        self.tuning = self.scene.autotune_primary(self.cam, W, H)
        c = self.scene.count_primary(self.cam, W, H).cpu().numpy().astype(np.int64)
        self.tot = {"inner": int(c[:, 0].sum()), "leaf": int(c[:, 1].sum()),
                    "tests": int(c[:, 2].sum()), "rays": W * H}
        self.rays_per_step = W * H
        self.kernels_per_step = 1

    def config(self):
        st = self.scene.stats()
        return {"workload": f"triangle soup {st['num_tris']} tris rope kd-tree; "
                            f"{self.cfg.width}x{self.cfg.height} primary rays",
                "triangles": st["num_tris"], "kd_nodes": st["num_nodes"],
                "kd_refs": st["num_refs"], "kd_build_s": round(self.build_s, 3),
                "kd_tree": self.kd_desc,
                "work_per_ray": {f: round(self.tot[f] / self.tot["rays"], 2)
                                 for f in ("inner", "leaf", "tests")},
                "rays_per_step": self.rays_per_step, "tuning": self.tuning,
                "l2": "flushed between steps (256 MB write)"}

    def phases(self, stream):
        W, H = self.cfg.width, self.cfg.height
        return [("primary", lambda: self.scene.trace_primary(self.cam, W, H, 0, self.out, stream))]

    def alg_bytes(self):
        t = self.tot
        return {"primary": traversal_bytes(t["rays"], t["inner"], t["leaf"], t["tests"])}

    def layout_bytes(self):
        t = self.tot
        return {"primary": layout_bytes(t["rays"], t["inner"], t["leaf"], t["tests"])}

    def configured_variant(self, torch):
        if self.tree == "configured" or (self.kd.max_depth, self.kd.leaf_size) == (
                CONFIGURED_TREE["max_depth"], CONFIGURED_TREE["leaf_size"]):
            return None  # the headline already runs the configured tree
        return SoupPrimary(torch, self.num_tris, tree="configured", packed=self.packed,
                           size=self.size)

    def parity(self):
        from oracle import pyoracle as po

        st = self.scene.stats()
        nodes, leaves, tris = self.scene.export()
        kd = po.KdTree(nodes, leaves, tris, st["bmin"], st["bmax"])
        W, H = self.cfg.width, self.cfg.height
        got = self.out.cpu().numpy().reshape(-1, 4)
        full = np.arange(W * H, dtype=np.uint32)
        pix = np.random.default_rng(12).choice(W * H, 600, replace=False).astype(np.uint32)
        v = self.packed[:, 0:3]
        verts = np.stack([v, v + self.packed[:, 4:7], v + self.packed[:, 8:11]], 1).reshape(-1, 3)
        faces = np.arange(verts.shape[0], dtype=np.uint32).reshape(-1, 3)
        return hit_parity(got, self.packed, st, kd, self.cam, W, H, full, pix, (verts, faces))

    def e2e_compute(self, torch, stream):
        W, H = self.cfg.width, self.cfg.height
        self.scene.trace_primary(self.cam, W, H, 0, self.out, stream)

    def e2e_outputs(self):
        return [self.out]

    def e2e_bytes(self):
        import ctypes

        return ctypes.sizeof(self.rb.RCamera), self.cfg.width * self.cfg.height * 16

    def cpu_baseline(self, budget_s=12.0):
        from oracle import pyoracle as po

        st = self.scene.stats()
        nodes, leaves, tris = self.scene.export()
        kd = po.KdTree(nodes, leaves, tris, st["bmin"], st["bmax"])
        W, H = self.cfg.width, self.cfg.height
        t0 = time.perf_counter()
        reps = 0
        while time.perf_counter() - t0 < budget_s / 2:
            po.primary_kd(kd, self.cam, W, H)
            reps += 1
        dt = time.perf_counter() - t0
        return {"value": round(reps * W * H / dt / 1e6, 4), "unit": "Mrays/s", "cores": po.threads(),
                "kind": "port", "sample": f"{reps} full {W}x{H} frames; oracle rope traversal over "
                                          "the same SAH tree, OpenMP"}



class TerrainSDF:
    name = "terrain_sdf"

    def __init__(self, torch):
        import rayengine_b200 as rb

        self.rb = rb
        self.cfg = cfg = rb.configs.TerrainConfig()
        self.cam = cfg.camera()
        self.params = cfg.params()
        W, H = cfg.width, cfg.height
        self.out = torch.empty((H * W, 8), dtype=torch.int32, device="cuda")
        rb.sphere_trace(self.params, self.cam, W, H, self.out)
        o = self.out.cpu().numpy()
        self.steps = int(o[:, 6].astype(np.int64).sum())
        self.hits = int((o[:, 7] == 1).sum())
        self.rays_per_step = W * H
        self.kernels_per_step = 1

    def config(self):
        return {"workload": "exact-SDF sphere tracing of d(p)=p.y-3fBm(0.25p), 8 octaves, "
                            "1920x1080, step 0.6d, eps 1e-4, tmax 200, <=512 steps",
                "field_evals_per_step": self.steps + 6 * self.hits,
                "rays_per_step": self.rays_per_step, "l2": "flushed between steps (256 MB write)"}

    def phases(self, stream):
        W, H = self.cfg.width, self.cfg.height
        return [("sdf", lambda: self.rb.sphere_trace(self.params, self.cam, W, H, self.out, stream))]

    def alg_bytes(self):
        return {"sdf": 32 * self.rays_per_step}

    def roofline(self, phase_ms, peaks):
        evals = self.steps + 6 * self.hits
        return fp32_roofline("sdf", evals * SDF_OPS_PER_EVAL, phase_ms["sdf"], peaks, self.name)

    def parity(self):
        """Bit-exact agreement with the oracle's march on a pixel sample, and
        the hit error against the FP64 arbiter (the float march's rule in
        double precision, its first crossing bisected to the root)."""
        from oracle import pyoracle as po

        W, H = self.cfg.width, self.cfg.height
        out = self.out.cpu().numpy()
        pix = np.random.default_rng(12).choice(W * H, 3000, replace=False).astype(np.uint32)
        P = po.perm(self.cfg.seed)
        ref = po.sdf_image(P, self.cam, W, H, pixels=pix)
        f = out.view(np.float32)[pix]
        u = out.view(np.uint32)[pix]
        same = ((u[:, 7] == ref["status"]) & (u[:, 6] == ref["steps"]) &
                (f[:, 0:3].view(np.uint32) == ref["pos"].view(np.uint32)).all(1) &
                (f[:, 3:6].view(np.uint32) == ref["normal"].view(np.uint32)).all(1))
        jp, jh = po.sdf_arbiter(P, self.cam, W, H, pix[:1000])
        err, disagree, both = po.hit_errors(out, jp, jh, pix[:1000])
        return {"vs_oracle": {"pixels": int(pix.size), "bitexact": int(same.sum())},
                "vs_fp64_arbiter": {"pixels": 1000, "hit_miss_disagree": disagree,
                                    "median_hit_error": float(np.median(err)) if both else None,
                                    "p95_hit_error": float(np.quantile(err, 0.95)) if both else None}}

    def e2e_compute(self, torch, stream):
        W, H = self.cfg.width, self.cfg.height
        self.rb.sphere_trace(self.params, self.cam, W, H, self.out, stream)

    def e2e_outputs(self):
        return [self.out]

    def e2e_bytes(self):
        import ctypes

        return (ctypes.sizeof(self.rb.RCamera) + ctypes.sizeof(self.params),
                self.cfg.width * self.cfg.height * 32)

    def cpu_baseline(self, budget_s=12.0):
        from oracle import pyoracle as po

        W, H = self.cfg.width, self.cfg.height
        rng = np.random.default_rng(0)
        n = 4000
        P = po.perm(self.cfg.seed)
        while True:
            pix = rng.choice(W * H, n, replace=False).astype(np.uint32)
            t0 = time.perf_counter()
            po.sdf_image(P, self.cam, W, H, pixels=pix)
            dt = time.perf_counter() - t0
            if dt > budget_s / 4 or n >= W * H:
                break
            n = min(W * H, int(n * min(8.0, budget_s / max(dt, 1e-3))))
        return {"value": round(n / dt / 1e6, 4), "unit": "Mrays/s", "cores": po.threads(),
                "kind": "port", "sample": f"{n} seeded-random pixels; oracle exact-SDF march, OpenMP"}



class SdfFrame:
    """The reference's shipped render path (render_sphere_trace behind
    cuda_render_frame): the terrain of TerrainSDF marched, then shaded with
    soft shadows toward the light and the atmosphere sky for misses, packed
    RGBA8.  Rays per frame: one primary ray per pixel plus one shadow ray per
    hit."""
    name = "sdf_frame"

    def __init__(self, torch):
        import rayengine_b200 as rb

        self.rb = rb
        self.fcfg = rb.configs.SdfFrameConfig()
        self.cfg = cfg = self.fcfg.terrain
        self.cam = cfg.camera()
        self.params = cfg.params()
        self.shade = self.fcfg.shade()
        W, H = cfg.width, cfg.height
        self.hits = torch.empty((H * W, 8), dtype=torch.int32, device="cuda")
        self.out = torch.empty(H * W, dtype=torch.int32, device="cuda")
        ev = torch.zeros(1, dtype=torch.int64, device="cuda")
        rb.sphere_trace(self.params, self.cam, W, H, self.hits)
        rb.shade_sdf(self.params, self.shade, self.cam, W, H, self.hits, self.out, evals=ev)
        o = self.hits.cpu().numpy()
        self.steps = int(o[:, 6].astype(np.int64).sum())
        self.nhits = int((o[:, 7] == 1).sum())
        self.shadow_evals = int(ev.item())
        self.rays_per_step = W * H + self.nhits
        # march, shadow pass, finish pass
        self.kernels_per_step = 3

    def config(self):
        sh = self.shade
        return {"workload": "shaded exact-SDF terrain frame d(p)=p.y-3fBm(0.25p), 1920x1080: march, "
                            "soft shadow toward the light, Phong-style light terms, atmosphere sky "
                            "for misses, RGBA8 (render_sphere_trace)",
                "field_evals_per_step": {"march": self.steps, "normals": 6 * self.nhits,
                                         "shadow": self.shadow_evals},
                "shade": {"light_pos": list(sh.light_pos), "light_intensity": sh.light_intensity,
                          "soft_shadow_k": sh.soft_shadow_k, "shadow_max_steps": sh.shadow_max_steps,
                          "flags": sh.flags},
                "rays_per_step": self.rays_per_step, "l2": "flushed between steps (256 MB write)"}

    def phases(self, stream):
        W, H = self.cfg.width, self.cfg.height
        rb = self.rb
        return [("sdf", lambda: rb.sphere_trace(self.params, self.cam, W, H, self.hits, stream)),
                ("shade", lambda: rb.shade_sdf(self.params, self.shade, self.cam, W, H, self.hits,
                                               self.out, stream=stream))]

    def roofline(self, phase_ms, peaks):
        evals = self.steps + 6 * self.nhits
        return fp32_roofline("sdf", evals * SDF_OPS_PER_EVAL, phase_ms["sdf"], peaks, self.name,
                             shade_kernels={"kernels": ["k_sdf_shadow", "k_sdf_finish"],
                                            "shadow_field_evals": self.shadow_evals,
                                            "ms": round(phase_ms["shade"], 4)})

    def e2e_compute(self, torch, stream):
        W, H = self.cfg.width, self.cfg.height
        self.rb.render_sdf_frame(self.params, self.shade, self.cam, W, H, self.hits, self.out,
                                 stream)

    def e2e_outputs(self):
        return [self.out]

    def e2e_bytes(self):
        import ctypes

        return (ctypes.sizeof(self.rb.RCamera) + ctypes.sizeof(self.params) +
                ctypes.sizeof(self.shade), self.cfg.width * self.cfg.height * 4)

    def cpu_baseline(self, budget_s=12.0):
        from oracle import pyoracle as po

        W, H = self.cfg.width, self.cfg.height
        rng = np.random.default_rng(0)
        n = 2000
        P = po.perm(self.cfg.seed)
        while True:
            pix = rng.choice(W * H, n, replace=False).astype(np.uint32)
            t0 = time.perf_counter()
            po.sdf_frame(P, self.cam, W, H, self.params, self.shade, pixels=pix)
            dt = time.perf_counter() - t0
            if dt > budget_s / 4 or n >= W * H:
                break
            n = min(W * H, int(n * min(8.0, budget_s / max(dt, 1e-3))))
        rays = n * self.rays_per_step / (W * H)
        return {"value": round(rays / dt / 1e6, 4), "unit": "Mrays/s", "cores": po.threads(),
                "kind": "port", "sample": f"{n} seeded-random pixels (primary + shadow rays "
                                          "scaled by the frame's hit fraction); oracle march + "
                                          "shading, OpenMP"}

    def parity(self):
        from oracle import pyoracle as po

        W, H = self.cfg.width, self.cfg.height
        got = self.out.cpu().numpy().view(np.uint32)
        pix = np.random.default_rng(12).choice(W * H, 3000, replace=False).astype(np.uint32)
        want = po.sdf_frame(po.perm(self.cfg.seed), self.cam, W, H, self.params, self.shade,
                            pixels=pix)
        return {"rgba8_vs_oracle": {"pixels": int(pix.size),
                                    "bitexact": int((got[pix] == want).sum())}}


class NeuralTerrainSDF:
    """The terrain of TerrainSDF traced through the neural surrogate: the
    network is trained at set-up (8M points, 20k Adam steps of 65,536), then
    a step = one 1920x1080 frame of network march + exact phase."""
    name = "nsdf_terrain"
    dtype = "bf16 (network, FP32 accumulate) + f32 (exact field)"

    def __init__(self, torch, train_steps=None):
        import rayengine_b200 as rb

        self.rb = rb
        self.ncfg = rb.configs.NeuralTerrainConfig()
        if train_steps:
            self.ncfg.train_steps = train_steps
        self.cfg = cfg = self.ncfg.terrain
        self.cam = cfg.camera()
        self.params = cfg.params()
        W, H = cfg.width, cfg.height
        t0 = time.perf_counter()
        self.model, self.tp, losses = self.ncfg.build()
        torch.cuda.synchronize()
        self.train_s = time.perf_counter() - t0
        self.final_loss = float(np.mean(losses[-100:]))
        self.out = torch.empty((H * W, 8), dtype=torch.int32, device="cuda")
        self.model.trace(self.params, self.tp, self.cam, W, H, self.out)
        self.stats = self.model.trace_status()
        if self.stats["error"]:
            raise RuntimeError("tensor-core wait bound reached in the network march")
        o = self.out.cpu().numpy()
        self.hits = int((o[:, 7] == 1).sum())
        # the exact tracer on the same frame, same run, for the ratio
        ex = torch.empty_like(self.out)
        for _ in range(3):
            rb.sphere_trace(self.params, self.cam, W, H, ex)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(20):
            rb.sphere_trace(self.params, self.cam, W, H, ex)
        b.record()
        torch.cuda.synchronize()
        self.exact_ms = a.elapsed_time(b) / 20
        self.rays_per_step = W * H
        # cone march, exact phase (+ the gradient-normal pass)
        self.kernels_per_step = 3 if self.ncfg.normal_taps == 1 else 2

    def config(self):
        n = self.ncfg
        st = self.stats
        R = self.rays_per_step
        return {"workload": "neural-SDF surrogate of d(p)=p.y-3fBm(0.25p) (8 octaves), 1920x1080: "
                            "Fourier features (16 freqs) -> 4x64 softplus MLP, BF16 tcgen05 inference; "
                            f"network phase: one cone per {n.cone_tile}x{n.cone_tile} pixel tile "
                            f"({n.cone_lanes} lanes per cone, speculative steps); exact phase from "
                            "the cone's stop (the exact tracer's steps, grown up to "
                            f"{n.relax}x along the secant; bracket + {n.root_steps} regula-falsi "
                            "steps) + the exact field's "
                            + ({4: "tetrahedral (compute_sdf_normal_tet) normal at radius 0.002 t",
                                1: "analytic-gradient normal"}.get(
                                   n.normal_taps, "central-difference normal at radius 0.002 t")),
                "training": {"points": n.num_points, "steps": n.train_steps, "batch": n.batch,
                             "lr": n.lr, "seconds": round(self.train_s, 2),
                             "final_l1_loss": round(self.final_loss, 5)},
                "trace_params": {"lipschitz": round(self.tp.lipschitz, 4),
                                 "lipschitz_quantile": n.lipschitz_quantile,
                                 "safety": n.cone_safety, "switch_dist": n.switch_dist,
                                 "min_step": n.min_step, "cone_max_passes": n.cone_max_passes,
                                 "root_steps": n.root_steps, "cone_tile": n.cone_tile,
                                 "cone_lanes": n.cone_lanes, "relax": n.relax,
                                 "root_tol": n.root_tol, "normal_taps": n.normal_taps},
                "per_ray": {"network_evals": round(st["network_evals"] / R, 3),
                            "network_rows": round(st["network_rows"] / R, 3),
                            "exact_evals": round(st["exact_evals"] / R, 3),
                            "normal_evals": round(st["normal_evals"] / R, 3)},
                "exact_sdf_same_run": {"ms_per_frame": round(self.exact_ms, 4),
                                       "mrays": round(R / self.exact_ms / 1e3, 3)},
                "rays_per_step": R, "l2": "flushed between steps (256 MB write)"}

    def phases(self, stream):
        W, H = self.cfg.width, self.cfg.height
        m = self.model
        return [("nsdf_network", lambda: m.trace(self.params, self.tp, self.cam, W, H, self.out,
                                                 stream, phase="network")),
                ("sdf_refine", lambda: m.trace(self.params, self.tp, self.cam, W, H, self.out, stream,
                                               phase="exact"))]

    def roofline(self, phase_ms, peaks):
        """The dominant phase's roofline (the exact phase: FP32 field
        evaluations against the measured FMA rate), with the network
        phase's tensor-core fraction beside it."""
        rows = self.stats["network_rows"]
        achieved = rows * NSDF_FLOPS_PER_EVAL / (phase_ms["nsdf_network"] / 1e3) / 1e12
        net = {"bound": "tensor", "kernel": "nsdf_network", "achieved": round(achieved, 2),
               "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
               "frac": round(achieved / peaks["bf16_tflops"], 4), "peak_source": peaks["source"],
               "alg_flops_per_launch": rows * NSDF_FLOPS_PER_EVAL,
               "ms": round(phase_ms["nsdf_network"], 4),
               "traffic": ncu_traffic(f"{self.name}:nsdf_network")}
        if phase_ms["nsdf_network"] >= phase_ms["sdf_refine"]:
            return net
        # normal_taps 1: each normal is one analytic gradient evaluation
        # (k_sdf_grad_normal, timed inside the exact phase)
        grad = self.ncfg.normal_taps == 1
        ops = (self.stats["exact_evals"] * SDF_OPS_PER_EVAL + self.stats["normal_evals"] *
               (SDF_GRAD_OPS_PER_EVAL if grad else SDF_OPS_PER_EVAL))
        return fp32_roofline("sdf_refine", ops, phase_ms["sdf_refine"], peaks, self.name,
                             network_phase=net,
                             exact_phase_kernels=["k_sdf_refine"] + (["k_sdf_grad_normal"]
                                                                     if grad else []))

    def e2e_compute(self, torch, stream):
        W, H = self.cfg.width, self.cfg.height
        self.model.trace(self.params, self.tp, self.cam, W, H, self.out, stream)

    def e2e_outputs(self):
        return [self.out]

    def e2e_bytes(self):
        import ctypes

        return (ctypes.sizeof(self.rb.RCamera) + ctypes.sizeof(self.params) +
                ctypes.sizeof(self.tp), self.cfg.width * self.cfg.height * 32)

    def cpu_baseline(self, budget_s=12.0):
        # the reference's method for this field on the host: the exact march
        return TerrainSDF.cpu_baseline(self, budget_s)

    def parity(self):
        """Hit error of the neural tracer's frame against the FP64 arbiter
        (target: median <= 1e-3 scene units), beside the exact tracer's."""
        from oracle import pyoracle as po

        W, H = self.cfg.width, self.cfg.height
        out = self.out.cpu().numpy()
        pix = np.random.default_rng(12).choice(W * H, 1500, replace=False).astype(np.uint32)
        P = po.perm(self.cfg.seed)
        jp, jh = po.sdf_arbiter(P, self.cam, W, H, pix)
        err, disagree, both = po.hit_errors(out, jp, jh, pix)
        # the whole frame's hit/miss against the exact tracer's frame
        ex = self.rb.sphere_trace(self.params, self.cam, W, H).cpu().numpy()
        frame_disagree = int(((out[:, 7] == 1) != (ex[:, 7] == 1)).sum())
        return {"vs_fp64_arbiter": {"pixels": int(pix.size), "hit_miss_disagree": disagree,
                                    "median_hit_error": float(np.median(err)) if both else None,
                                    "p95_hit_error": float(np.quantile(err, 0.95)) if both else None,
                                    "target": "median <= 1e-3 scene units"},
                "vs_exact_tracer_frame": {"pixels": W * H, "hit_miss_disagree": frame_disagree}}


class BatchWavefront:
    """32 seeded scenes (soups of 10k-2M triangles and volumetric terrains)
    at 640x360 / 1280x720 / 1920x1080, 1 spp path tracing to depth 4, one
    persistent launch per frame replayed from a CUDA graph, autotuned."""
    name = "batch32"

    scaling = "strong"  # with N GPUs the fixed batch is split by scenes
    parallelism = "scenes split"

    def __init__(self, torch, num_scenes=None, rank=0, world=1):
        import rayengine_b200 as rb

        self.rb = rb
        self.cfg = rb.configs.BatchConfig()
        if num_scenes:
            self.cfg.num_scenes = num_scenes
        t0 = time.perf_counter()
        self.batch, self.meshes = self.cfg.build(rank, world)
        self.build_s = time.perf_counter() - t0
        self.out = torch.empty(self.batch.total_pixels, dtype=torch.float32, device="cuda")
        self.tuning = self.batch.autotune(self.out)
        self.work = self.batch.counts(self.out)
        self.batch.render(self.out, graph=True)
        torch.cuda.synchronize()
        st = self.batch.stats()
        if st["error"]:
            raise RuntimeError("batch frame reported a wait-bound error")
        self.rays = st["rays"]
        self.rays_per_step = int(self.rays.sum())
        self.kernels_per_step = 1

    def config(self):
        sp = self.cfg.specs()
        return {"workload": f"batched wavefront path tracing: {len(sp)} seeded scenes "
                            f"({sum(s['kind'] == 'soup' for s in sp)} soups, "
                            f"{sum(s['kind'] == 'terrain' for s in sp)} fBm terrains), resolutions "
                            "from {640x360, 1280x720, 1920x1080}, 1 spp, depth 4 Lambertian; one "
                            "persistent launch per frame from a captured CUDA graph",
                "pixels": self.batch.total_pixels,
                "triangles": int(sum(s.get("num_tris", 0) for s in sp)),
                "rays_per_bounce": {"mesh": [int(x) for x in self.rays[:, 0]],
                                    "terrain": [int(x) for x in self.rays[:, 1]]},
                "work": self.work, "tuning": self.tuning,
                "scene_build_s": round(self.build_s, 2),
                "rays_per_step": self.rays_per_step, "l2": "flushed between steps (256 MB write)"}

    def phases(self, stream):
        return [("batch", lambda: self.batch.render(self.out, stream=stream, graph=True))]

    def alg_bytes(self):
        w = self.work
        cont = int(self.rays[1:].sum())
        return {"batch": traversal_bytes(int(self.rays.sum()), w["inner"], w["leaf"], w["tests"], cont)}

    def layout_bytes(self):
        w = self.work
        cont = int(self.rays[1:].sum())
        return {"batch": 16 * w["inner"] + 48 * w["leaf"] + 52 * w["tests"] + 64 * cont +
                4 * self.batch.total_pixels}

    def parity(self):
        from oracle import pyoracle as po

        scenes, offsets, _ = reference_batch_scenes(self.cfg)
        rad = self.out.cpu().numpy()
        g = np.sort(np.random.default_rng(12).choice(self.batch.total_pixels, 400,
                                                      replace=False)).astype(np.uint32)
        orad, _, _ = po.batch_path(scenes, offsets, g, self.cfg.max_depth, self.cfg.path_seed,
                                   self.cfg.mesh_bias)
        return {"vs_oracle_path_tracer": {
            "pixels": int(g.size),
            "radiance_bitexact": int((rad[g].view(np.uint32) == orad.view(np.uint32)).sum())}}

    def e2e_compute(self, torch, stream):
        self.batch.render(self.out, stream=stream, graph=True)

    def e2e_outputs(self):
        return [self.out]

    def e2e_bytes(self):
        return (0, 4 * self.batch.total_pixels)

    def cpu_baseline(self, budget_s=12.0):
        from oracle import pyoracle as po

        scenes, offsets, _ = reference_batch_scenes(self.cfg)
        rng = np.random.default_rng(0)
        n = 64
        while True:
            g = np.sort(rng.choice(self.batch.total_pixels, n, replace=False)).astype(np.uint32)
            t0 = time.perf_counter()
            _, _, nr = po.batch_path(scenes, offsets, g, self.cfg.max_depth, self.cfg.path_seed,
                                     self.cfg.mesh_bias)
            dt = time.perf_counter() - t0
            if dt > budget_s / 4 or n >= 1 << 16:
                break
            n = min(1 << 16, int(n * min(8.0, budget_s / max(dt, 1e-3))))
        return {"value": round(int(nr.sum()) / dt / 1e6, 6), "unit": "Mrays/s",
                "cores": po.threads(), "kind": "port",
                "sample": f"{n} seeded-random pixels of the batch ({int(nr.sum())} rays); oracle "
                          "path tracer with brute-force Moller-Trumbore (the reference's one-leaf "
                          "tree) and the exact SDF march, OpenMP"}


def reference_batch_scenes(cfg):
    """The batch's scenes for the CPU path (oracle generators only):
    (oracle scene dicts, first-pixel offsets, total pixels)."""
    from oracle import pyoracle as po
    import rayengine_b200.configs as C
    from rayengine_b200 import api

    scenes, offsets, off = [], [], 0
    for s in cfg.specs():
        w, h = s["width"], s["height"]
        offsets.append(off)
        off += w * h
        if s["kind"] == "soup":
            sc = C.SoupConfig(num_tris=s["num_tris"], seed=s["seed"], width=w, height=h)
            tri = po.soup(sc.seed, sc.num_tris)
            verts = tri.reshape(-1, 3)
            faces = np.arange(verts.shape[0], dtype=np.uint32).reshape(-1, 3)
            packed = api.pack_triangles(verts, faces)
            v = np.concatenate([packed[:, 0:3], packed[:, 0:3] + packed[:, 4:7],
                                packed[:, 0:3] + packed[:, 8:11]])
            cam = api.build_camera(sc.campos, sc.lookat, (60.0, api.vertical_fov(60.0, w, h)))
            scenes.append(dict(kind=0, tris=packed, bmin=v.min(0), bmax=v.max(0), cam=cam, w=w,
                               h=h, albedo=s["albedo"]))
        else:
            tc = C.TerrainConfig(seed=s["seed"], amplitude=s["amplitude"], width=w, height=h)
            scenes.append(dict(kind=1, seed=tc.seed, octaves=tc.octaves, scale=tc.scale,
                               amp=tc.amplitude, step_factor=tc.step_factor, eps=tc.eps,
                               tmax=tc.tmax, max_steps=tc.max_steps, cam=tc.camera(), w=w, h=h,
                               albedo=s["albedo"]))
    return scenes, np.array(offsets, np.uint64), off


# ---------------------------------------------------- the reference's path
def _cosine_dirs(n, rng, k):
    """k cosine-weighted directions around each unit normal n (m, 3) -> (m, k, 3)."""
    m = n.shape[0]
    t = np.where(np.abs(n[:, :1]) > np.abs(n[:, 1:2]),
                 np.stack([n[:, 2], np.zeros(m), -n[:, 0]], 1),
                 np.stack([np.zeros(m), -n[:, 2], n[:, 1]], 1))
    t /= np.maximum(np.linalg.norm(t, axis=1, keepdims=True), 1e-30)
    b = np.cross(n, t)
    u1, u2 = rng.random((m, k)), rng.random((m, k))
    r, phi = np.sqrt(u1), 2.0 * np.pi * u2
    x, y, z = r * np.cos(phi), np.sqrt(1.0 - u1), r * np.sin(phi)
    return x[..., None] * b[:, None] + y[..., None] * n[:, None] + z[..., None] * t[:, None]


def reference_workload(name):
    """(workload description, built-by note, kind, step(npix) -> rays traced,
    as-shipped variant or None) for the reference's own CPU path.

    Meshes: the reference's CPU ray query singleRayStacklessIntersect,
    compiled from its sources (oracle/_ref), over the same seeded scene
    (generated by the CPU oracle's generators) and an SAH tree of the
    configured parameters held as the reference's KDNodeCPU objects; as
    shipped the reference's tree is one leaf (every query tests every
    triangle), timed beside it.
    SDF and batch workloads: the reference's device march cannot be compiled
    for the host (texture hash, CUDA 10 texture references), so the arm
    times the oracle's restatement of it.  Nothing of this repository's
    engine runs on this path: the package is imported for its pure-Python
    workload descriptions only and its library is never loaded."""
    from oracle import pyoracle as po
    import rayengine_b200.configs as C
    from rayengine_b200 import api

    rng = np.random.default_rng(1)
    if name == "batch32":
        cfg = C.BatchConfig()
        scenes, offsets, total = reference_batch_scenes(cfg)

        def step(npix):
            g = np.sort(rng.choice(total, npix, replace=False)).astype(np.uint32)
            _, _, nr = po.batch_path(scenes, offsets, g, cfg.max_depth, cfg.path_seed,
                                     cfg.mesh_bias)
            return int(nr.sum())
        return ("batched path tracing of the 32-scene batch (depth 4, 1 spp), seeded-random "
                "pixels", "oracle restatement: single-leaf build (brute-force Moller-Trumbore) "
                "and the exact SDF march", "port", step, None)
    if name == "sdf_frame":
        fcfg = C.SdfFrameConfig()
        cfg = fcfg.terrain
        W, H = cfg.width, cfg.height
        P = po.perm(cfg.seed)
        cam = cfg.camera()
        field = cfg.params()
        shade = fcfg.shade()

        def step(npix):
            pix = rng.choice(W * H, npix, replace=False).astype(np.uint32)
            img, ev = po.sdf_frame(P, cam, W, H, field, shade, pixels=pix, evals=True)
            return npix + int((ev > 0).sum())
        return ("shaded exact-SDF terrain frame, 1920x1080 (march, soft shadow, sky, RGBA8)",
                "oracle restatement of render_sphere_trace (renderer.cu:143-285; the "
                "reference's device code does not compile for the host)", "port", step, None)
    if name in ("terrain_sdf", "nsdf_terrain"):
        cfg = C.TerrainConfig()
        W, H = cfg.width, cfg.height
        P = po.perm(cfg.seed)
        cam = cfg.camera()

        def step(npix):
            po.sdf_image(P, cam, W, H, pixels=rng.choice(W * H, npix, replace=False).astype(np.uint32))
            return npix
        return ("exact-SDF sphere tracing of d(p)=p.y-3fBm(0.25p), 8 octaves, 1920x1080",
                "oracle restatement of the exact-SDF march (sphere_tracing.cuh:183-216; the "
                "reference's device code does not compile for the host)", "port", step, None)
    if name.startswith("heightfield_ao"):
        cfg = C.HeightfieldConfig()
        verts, faces = po.heightfield(po.perm(cfg.seed), cfg.cells, cfg.lo, cfg.hi, cfg.octaves,
                                      cfg.amplitude)
        desc = ("heightfield 1024x1024 cells (2,097,152 tris); 1920x1080 primary + 1 shadow + 4 AO "
                "rays per hit")
    else:
        cfg = C.SoupConfig(num_tris=(1 << 20) if name.startswith("soup1m") else 65536)
        if name == "soup1m_2k":
            cfg.width = cfg.height = 2048
        tri = po.soup(cfg.seed, cfg.num_tris)
        verts = tri.reshape(-1, 3)
        faces = np.arange(verts.shape[0], dtype=np.uint32).reshape(-1, 3)
        desc = f"triangle soup {cfg.num_tris} tris; {cfg.width}x{cfg.height} primary rays"
    if po.ref_lib() is None:
        raise FileNotFoundError("oracle/_ref/libre_ref.so (the reference's compiled host code)")
    # The configured tree (SAH, depth <= 24, leaves of <= 8) cannot come from
    # the reference's builder (MAX_DEPTH = 1, its SAH code commented out), so
    # the checker's binned-SAH builder makes it and the reference's query
    # runs over it as the reference's own KDNodeCPU objects.  The reference
    # as shipped (one leaf: every query tests every triangle) is timed
    # beside it on a small sample.
    bonus = 0.15 if not name.startswith("heightfield_ao") else 0.1
    t0 = time.perf_counter()
    kdb = po.kdb_build(verts, faces, CONFIGURED_TREE["max_depth"], CONFIGURED_TREE["leaf_size"],
                       2.0, 1.0, bonus)
    kdb_s = time.perf_counter() - t0
    sah_tree = po.RefTree.from_kd(verts, faces, kdb)
    leaf_tree = po.RefTree(verts, faces)
    cam = cfg.camera()
    W, H = cfg.width, cfg.height
    built_by = ("the reference's CPU query RKDTreeCPU::singleRayStacklessIntersect "
                "(KDTree.cpp:993-1066: box test, leaf triangles, both children), compiled from "
                "its sources, OpenMP schedule(dynamic) over rays (RayTracer.cpp:154), over an SAH "
                f"kd-tree of the configured parameters (depth <= {CONFIGURED_TREE['max_depth']}, "
                f"leaves of <= {CONFIGURED_TREE['leaf_size']}, empty bonus {bonus}; "
                f"{len(kdb.nodes)} nodes, {len(kdb.index)} references, built in {kdb_s:.1f} s by "
                "the checker's builder and held as the reference's own KDNodeCPU objects: the "
                "reference's builder ships with MAX_DEPTH = 1)")

    def make_step(tree):
        def primary(npix):
            o, d = po.camera_rays(cam, W, H, rng.choice(W * H, npix, replace=False))
            t, nrm, _ = tree.trace(o, d)
            return o, d, t, nrm

        if name.startswith("heightfield_ao"):
            light = np.array(api.unit(cfg.light_dir), np.float64)

            def step(npix):
                o, d, t, nrm = primary(npix)
                hit = t < 1e19
                if not hit.any():
                    return npix
                n = nrm[hit].astype(np.float64)
                n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
                flip = np.einsum("ij,ij->i", n, d[hit]) > 0.0
                n[flip] = -n[flip]
                p = o[hit] + t[hit, None].astype(np.float64) * d[hit] + cfg.bias * n
                dirs = np.concatenate([np.broadcast_to(light, (n.shape[0], 1, 3)),
                                       _cosine_dirs(n, rng, 4)], 1).reshape(-1, 3)
                tree.trace(np.repeat(p, 5, axis=0), dirs)
                return npix + 5 * n.shape[0]
        else:
            def step(npix):
                primary(npix)
                return npix
        return step

    as_shipped = {"step": make_step(leaf_tree),
                  "what": "the reference as shipped: its RKDTreeCPU (one leaf, KDTree.cpp:12,347) "
                          "and the same query, i.e. every triangle per ray"}
    return desc, built_by, "reference", make_step(sah_tree), as_shipped


TREE_WORKLOADS = ("heightfield_ao", "soup", "soup1m", "soup1m_2k")

WORKLOADS = {
    "heightfield_ao": HeightfieldAO,
    "soup": SoupPrimary,
    "soup1m": lambda torch, **kw: SoupPrimary(torch, num_tris=1 << 20, **kw),
    # the same scene and camera at 2048x2048: a frame with enough rays to
    # fill the GPU (the 512x512 frame is shorter than its longest walks)
    "soup1m_2k": lambda torch, **kw: SoupPrimary(torch, num_tris=1 << 20, size=2048, **kw),
    "terrain_sdf": TerrainSDF,
    "sdf_frame": SdfFrame,
    "nsdf_terrain": NeuralTerrainSDF,
    "batch32": BatchWavefront,
}

METRIC = "Mrays/s on 1 B200: plain rope-kd/exact-SDF vs wavefront+neural SDF @<=1e-3 err"


# ------------------------------------------------------------------ arms
def run_reference(args):
    """--impl reference: rank 0 times the reference's CPU path; others exit."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    from oracle import pyoracle as po

    desc, built_by, kind, step, shipped = reference_workload(args.config)
    # size one step to about a second of work on all host cores, less when
    # many steps are asked for, so that the whole run stays within minutes
    target_s = min(1.0, 90.0 / max(1, args.steps + args.warmup))
    npix = 4
    for _ in range(2):  # the first call also pays one-time set-up
        t0 = time.perf_counter()
        step(npix)
        dt = time.perf_counter() - t0
        npix = max(4, min(200000, int(npix * target_s / max(dt, 1e-4))))
    for _ in range(args.warmup):
        step(npix)
    rays = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rays += step(npix)
    dt = time.perf_counter() - t0
    value = rays / dt / 1e6
    extra = {}
    if shipped is not None:
        # about a second of the as-shipped query on a small sample
        n2, r2, t2 = 4, 0, 0.0
        while t2 < 1.0 and n2 <= 4096:
            ta = time.perf_counter()
            r2 += shipped["step"](n2)
            t2 += time.perf_counter() - ta
            n2 *= 2
        extra["as_shipped"] = {"value": round(r2 / t2 / 1e6, 6), "unit": "Mrays/s",
                               "what": shipped["what"]}
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "Mrays/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": desc, "pixels_per_step": npix},
        "cpu_baseline": {"value": round(value, 6), "unit": "Mrays/s", "cores": po.threads(),
                         "kind": kind,
                         "sample": f"{npix} seeded-random pixels per step ({rays // args.steps} "
                                   f"rays per step); {built_by}"},
        "e2e": {"value": round(value, 6), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    line.update(extra)
    print(json.dumps(line), flush=True)
    return 0


def timed_steps(torch, phases, stream, flush, steps, world):
    """K steps bracketed by a barrier and a device synchronize on both sides,
    L2 flushed before each; CUDA events on the launching stream around every
    phase.  Returns (mean step ms, {phase: mean ms})."""
    n_ph = len(phases)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(n_ph + 1)] for _ in range(steps)]
    barrier(world)
    torch.cuda.synchronize()
    for k in range(steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(stream)
        for j, (_, fn) in enumerate(phases):
            fn()
            ev[k][j + 1].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    step_ms = [ev[k][0].elapsed_time(ev[k][n_ph]) for k in range(steps)]
    phase_ms = {name: statistics.mean(ev[k][j].elapsed_time(ev[k][j + 1]) for k in range(steps))
                for j, (name, _) in enumerate(phases)}
    return statistics.mean(step_ms), phase_ms


def configured_tree_line(torch, wl, stream, flush, args, world, dev):
    """The same workload over the tree the configuration names (depth 24,
    leaf 8), timed like the headline (same steps, warm-up and L2 flush)."""
    alt = wl.configured_variant(torch)
    if alt is None:
        return None
    phases = alt.phases(stream)
    for i in range(args.warmup):
        flush.fill_(i & 0xFF)
        for _, fn in phases:
            fn()
    ms, phase_ms = timed_steps(torch, phases, stream, flush, args.steps, world)
    ms_max = max_over_ranks(ms, world, dev)
    total = sum_over_ranks(alt.rays_per_step, world, dev)
    st = alt.scene.stats()
    out = {"value": round(total / (ms_max / 1e3) / 1e6, 3), "unit": "Mrays/s",
           "ms_per_step": round(ms_max, 4), "phases_ms": {k: round(v, 4) for k, v in phase_ms.items()},
           "kd_tree": alt.kd_desc, "kd_nodes": st["num_nodes"], "kd_refs": st["num_refs"],
           "kd_build_s": round(alt.build_s, 3), "rays_per_step": alt.rays_per_step,
           "note": "same rays and same hits as the headline; only the tree differs"}
    alt.scene.close()
    return out


def e2e_times(torch, wl, stream, flush, steps, world):
    """End-to-end step time through the library's public calls with host
    buffers, measured two ways on the wall clock:

    * latency: one frame at a time (render, read every output back into
      pinned host memory, synchronize); the L2 flush before each frame is
      outside the timed region;
    * throughput: frames back to back; frame k's outputs are snapshot on the
      device into one of two staging slots and read back into pinned host
      memory on a copy stream while frame k+1 renders.  The L2 flush before
      every frame and every read-back are inside the timed region.

    Returns (latency_ms, throughput_ms) per step."""
    outs = wl.e2e_outputs()
    host = [[torch.empty(o.shape, dtype=o.dtype, pin_memory=True) for o in outs] for _ in range(2)]
    stage = [[torch.empty_like(o) for o in outs] for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    ready = [torch.cuda.Event() for _ in range(2)]
    copied = [torch.cuda.Event() for _ in range(2)]

    def serial():
        wl.e2e_compute(torch, stream)
        for h, o in zip(host[0], outs):
            h.copy_(o, non_blocking=True)

    def pipelined(k):
        s = k & 1
        if k >= 2:
            stream.wait_event(copied[s])  # staging slot s is free again
        flush.fill_(k & 0xFF)
        wl.e2e_compute(torch, stream)
        for st, o in zip(stage[s], outs):
            st.copy_(o, non_blocking=True)
        ready[s].record(stream)
        copy_stream.wait_event(ready[s])
        with torch.cuda.stream(copy_stream):
            for h, st in zip(host[s], stage[s]):
                h.copy_(st, non_blocking=True)
            copied[s].record(copy_stream)

    for k in range(2):
        flush.fill_(k)
        serial()
    torch.cuda.synchronize()
    barrier(world)
    lat = []
    for k in range(steps):
        flush.fill_(k & 0xFF)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        serial()
        torch.cuda.synchronize()
        lat.append((time.perf_counter() - t0) * 1e3)
    barrier(world)
    for k in range(2):
        pipelined(k)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for k in range(steps):
        pipelined(k)
    torch.cuda.synchronize()
    thr = (time.perf_counter() - t0) * 1e3 / steps
    barrier(world)
    return statistics.mean(lat), thr


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    init_dist(world)
    dev = torch.device("cuda", local)
    opts = {}
    if args.config == "nsdf_terrain" and args.train_steps:
        opts["train_steps"] = args.train_steps
    if args.config == "batch32" and args.scenes:
        opts["num_scenes"] = args.scenes
    if args.config == "batch32" and world > 1:
        opts["rank"], opts["world"] = rank, world  # scenes split across ranks
    if args.config in TREE_WORKLOADS:
        opts["tree"] = args.tree
    wl = WORKLOADS[args.config](torch, **opts)
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    phases = wl.phases(stream)

    def step():
        for _, fn in phases:
            fn()

    if args.profile:
        # for ncu captures: one warm-up step, then one flushed step inside the
        # NVTX range "profile" (ncu --nvtx --nvtx-include "profile/"), no timing
        step()
        flush.fill_(1)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("profile")
        step()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        print(json.dumps({"profile": wl.name, "kernels_per_step": wl.kernels_per_step}))
        return 0

    for i in range(args.warmup):
        flush.fill_(i & 0xFF)
        step()
    torch.cuda.synchronize()

    cvd = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    clocks = ClockSampler(cvd.split(",")[local] if cvd else str(local))
    clocks.start()
    time.sleep(0.5)  # let nvidia-smi take its first samples before the timed region
    ms, phase_ms = timed_steps(torch, phases, stream, flush, args.steps, world)
    clk = clocks.stop()
    ms_max = max_over_ranks(ms, world, dev)
    total_rays = sum_over_ranks(wl.rays_per_step, world, dev)
    value = total_rays / (ms_max / 1e3) / 1e6

    # end to end through the C ABI with host buffers: every step's results are
    # read back into pinned host memory
    e_lat_ms, e_ms = e2e_times(torch, wl, stream, flush, args.steps, world)
    e_ms_max = max_over_ranks(e_ms, world, dev)
    e_lat_max = max_over_ranks(e_lat_ms, world, dev)
    scaling = getattr(wl, "scaling", "weak")
    h2d, d2h = wl.e2e_bytes()

    peaks = measured_peaks()
    peaks["l2_gbs"] = measure_l2_gbs(torch)
    peaks["fp32_tops"] = measure_fp32_tops(torch)
    roof = wl.roofline(phase_ms, peaks) if hasattr(wl, "roofline") else \
        hbm_roofline(wl, phase_ms, peaks)
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max, 4),
        "higher_is_better": True, "scaling": scaling, "vs_baseline": None,
        "dtype": getattr(wl, "dtype", "f32"),
        "data": "synthetic (seeded)", "config": dict(wl.config(), parallelism=f"{getattr(wl, 'parallelism', 'replica')} x{world}"),
        "phases_ms": {k: round(v, 4) for k, v in phase_ms.items()},
        "roofline": roof,
        "e2e": {"value": round(total_rays / (e_ms_max / 1e3) / 1e6, 3),
                "unit": "Mrays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": round(e_ms_max, 4),
                "mode": "frames back to back; frame k's read-back (device snapshot, then a "
                        "copy stream) overlaps frame k+1; wall clock over all steps",
                "latency_ms_per_step": round(e_lat_max, 4)},
        "gpu_launches": wl.kernels_per_step * args.steps,
        "clocks": clk,
    }
    if not args.no_configured_tree and hasattr(wl, "configured_variant"):
        ct = configured_tree_line(torch, wl, stream, flush, args, world, dev)
        if ct is not None:
            line["configured_tree"] = ct
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = wl.cpu_baseline()
        if hasattr(wl, "parity"):
            line["parity"] = wl.parity()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(WORKLOADS), default="heightfield_ao")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU baseline and the checker's parity summary")
    ap.add_argument("--tree", choices=["tuned", "configured"], default="tuned",
                    help="kd-tree of the mesh workloads: the B200-tuned library default, or "
                         "the configured SAH tree (depth <= 24, leaf <= 8)")
    ap.add_argument("--no-configured-tree", action="store_true",
                    help="do not also time the configured tree after the headline")
    ap.add_argument("--train-steps", type=int, default=0,
                    help="nsdf_terrain: training steps at set-up (default: the config's 20000)")
    ap.add_argument("--scenes", type=int, default=0,
                    help="batch32: number of scenes (default: the config's 32)")
    ap.add_argument("--profile", action="store_true",
                    help="one warm-up and one flushed step, untimed (for ncu captures)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
