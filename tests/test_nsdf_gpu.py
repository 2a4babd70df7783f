"""Neural SDF surrogate on the GPU against the CPU oracle (oracle/nsdf_oracle.py).

Tolerances: the device evaluates sin/cos with the special-function unit and
rounds features, weights and activations to BF16; the oracle rounds at the
same places from exact sin/cos, so a rounding boundary can flip one BF16 ulp
(2^-8 relative) of a feature.  Outputs are compared to 2e-2 of the output
scale, gradients by relative L2 error < 5e-2 and cosine > 0.998.
"""
import os
import tempfile

import numpy as np
import pytest
import torch

import rayengine_b200 as rb
from oracle import nsdf_oracle as no
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

BOX = ([-40.0, -6.0, -20.0], [40.0, 11.0, 60.0])
F0 = 0.5


def _model(seed=3):
    m = rb.NeuralSDF(BOX[0], BOX[1], F0, seed)
    return m


def _pts(n, seed=0):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(BOX[0][k], BOX[1][k], n) for k in range(3)], 1).astype(np.float32)


def test_tensor_core_eval_matches_reference_and_oracle(cuda):
    # trained weights (a short run), so every layer carries signal
    tc = rb.configs.TerrainConfig(width=192, height=108)
    lo, hi = rb.NeuralSDF.box_for_camera(tc.camera(), tc.width, tc.height, 60.0, -6.0, 11.0)
    with rb.NeuralSDF(lo, hi, F0, 3) as m:
        m.generate(tc.params(), tc.camera(), tc.width, tc.height, 1 << 17, seed=4)
        m.train(200, batch=8192, lr=2e-3)
        p = m.get_params()
        pts = m.data(5000)[:, :3].copy()
        d = torch.from_numpy(pts).cuda()
        tc_out = m.eval(d).cpu().numpy()
        ref = m.eval_reference(d).cpu().numpy()
        orc, _, _ = no.forward(p, pts, lo, hi, F0, bf16_round=True)
        scale = np.abs(orc).max() + 1e-6
        assert np.abs(ref - orc).max() / scale < 2e-2
        # the tensor-core path evaluates softplus in packed BF16 arithmetic
        # (pre-activation rounded to BF16 first): within 1 BF16 ulp per
        # activation of the training arithmetic
        assert np.abs(tc_out - ref).max() / scale < 2e-2
        assert np.corrcoef(tc_out, orc)[0, 1] > 0.9995
        # odd sizes: partial tiles and partly filled groups
        for n in (1, 127, 129, 1000, 4097):
            out = m.eval(d[:n].contiguous()).cpu().numpy()
            assert np.array_equal(out, tc_out[:n])


def test_loss_gradient_matches_oracle(cuda):
    with _model() as m:
        p = m.get_params()
        n = 1024
        pts = _pts(n, 1)
        labels = np.random.default_rng(2).normal(0, 1, n).astype(np.float32)
        xyzl = torch.from_numpy(np.concatenate([pts, labels[:, None]], 1)).cuda()
        g, pred = m.loss_grad(xyzl)
        g, pred = g.cpu().numpy().astype(np.float64), pred.cpu().numpy()
        loss, go, po_ = no.loss_grad(p, pts, labels, *BOX, F0, bf16_round=True)
        assert np.abs(pred - po_).max() < 2e-2 * (np.abs(po_).max() + 1e-6)
        # predictions that straddle the label can flip the sign of the L1
        # gradient; compare on the whole vector
        rel = np.linalg.norm(g - go) / np.linalg.norm(go)
        cos = g @ go / (np.linalg.norm(g) * np.linalg.norm(go))
        assert rel < 5e-2 and cos > 0.998, (rel, cos)


def test_training_reduces_loss_and_checkpoints(cuda):
    tc = rb.configs.TerrainConfig(width=192, height=108)
    cam = tc.camera()
    lo, hi = rb.NeuralSDF.box_for_camera(cam, tc.width, tc.height, 60.0, -6.0, 11.0)
    with rb.NeuralSDF(lo, hi, F0, 5) as m:
        m.generate(tc.params(), cam, tc.width, tc.height, 1 << 18, seed=9)
        data = m.data(4096)
        # labels: first-order distance of the exact field
        P = po.perm(tc.seed)
        dens = data[:, 1].astype(np.float64) - 3.0 * po.fbm_batch(P, data[:, :3], 8, scale=0.25)
        agree = np.sign(dens) == np.sign(data[:, 3])
        assert agree.mean() > 0.99
        near = np.abs(data[1::2, 3]) < 0.2
        assert near.mean() > 0.5  # the near-surface half is near the surface
        losses = m.train(300, batch=8192, lr=2e-3)
        assert np.all(np.isfinite(losses))
        assert losses[-20:].mean() < 0.5 * losses[:5].mean()
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "net.bin")
            m.save(path)
            p1 = m.get_params()
            m.train(5, batch=8192, lr=2e-3)
            assert not np.array_equal(m.get_params(), p1)
            m.load(path)
            assert np.array_equal(m.get_params(), p1)


def _sdf_errors(out, tc, pix):
    P = po.perm(tc.seed)
    jpos, jhit = po.sdf_arbiter(P, tc.camera(), tc.width, tc.height, pix)
    return po.hit_errors(out, jpos, jhit, pix)


def _normals_from_positions(out, cam, pix, taps):
    """The exact phase's normal recomputed on the host in FP64 from the
    returned hit positions: central differences (taps 6) or the tetrahedral
    stencil (taps 4), delta = 0.002 t with t = |p - camera|; taps 1: the
    field's gradient (FP64 central differences of radius 1e-5, whose error
    is far below FP32's).  Returns the angles in degrees."""
    tc = rb.configs.TerrainConfig()
    P = po.perm(tc.seed)
    f = out.view(np.float32)[pix]
    p = f[:, 0:3].astype(np.float64)
    t = np.linalg.norm(p - np.array(cam.campos, np.float64), axis=1)
    delta = (0.002 * t)[:, None] if taps != 1 else np.full((len(p), 1), 1e-5)
    if taps in (6, 1):
        n = np.zeros_like(p)
        for k in range(3):
            e = np.zeros(3)
            e[k] = 1.0
            n[:, k] = po.density_d(P, p + delta * e) - po.density_d(P, p - delta * e)
    else:
        n = np.zeros_like(p)
        c = 0.5773
        for e in ([c, -c, -c], [-c, -c, c], [-c, c, -c], [c, c, c]):
            e = np.array(e)
            n += e[None, :] * po.density_d(P, p + delta * e)[:, None]
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    got = f[:, 3:6].astype(np.float64)
    # the angle from atan2(|a x b|, a . b) of the renormalised vectors: an
    # arccos of the dot product would read FP32's normalisation error
    # (|n| = 1 +- 6e-8) as angles of ~0.02 degrees
    got /= np.linalg.norm(got, axis=1, keepdims=True)
    return np.degrees(np.arctan2(np.linalg.norm(np.cross(n, got), axis=1), (n * got).sum(1)))


def test_neural_trace_accuracy_and_exact_evaluations_saved(cuda):
    tc = rb.configs.TerrainConfig(width=480, height=270)
    ncfg = rb.configs.NeuralTerrainConfig(terrain=tc, num_points=1 << 21, train_steps=3000)
    m, tp, losses = ncfg.build()
    assert tp.cone_tile > 0  # the cone tracer is the configured method
    with m:
        assert np.all(np.isfinite(losses)) and losses[-100:].mean() < losses[:10].mean()
        W, H = tc.width, tc.height
        field, cam = tc.params(), tc.camera()
        ex = m.trace(field, rb.nsdf_trace_params(exact_only=True), cam, W, H).cpu().numpy()
        st_ex = m.trace_status()
        assert st_ex["network_evals"] == 0 and st_ex["handed_over"] == 0
        pix = np.random.default_rng(5).choice(W * H, 4000, replace=False).astype(np.uint32)
        err_e, mism_e, both_e = _sdf_errors(ex, tc, pix)
        assert np.median(err_e) <= 1e-3 and mism_e <= 0.01 * len(pix)
        exact_tracer = rb.sphere_trace(field, cam, W, H).cpu().numpy()
        lip = tp.lipschitz
        variants = {
            "cone": tp,
            "cone, one lane, tetrahedral normal": rb.nsdf_trace_params(
                lip, ncfg.safety, ncfg.switch_dist, ncfg.min_step, ncfg.max_network_steps, 0,
                ncfg.root_steps, 1.0, cone_tile=8, cone_lanes=1, normal_taps=4),
            "cone over a coarse level": rb.nsdf_trace_params(
                lip, ncfg.safety, ncfg.switch_dist, ncfg.min_step, ncfg.max_network_steps, 0,
                ncfg.root_steps, ncfg.relax, cone_tile=8, cone_coarse=32, cone_lanes=4),
            "per-ray march": ncfg.per_ray_params(lip),
        }
        for name, params in variants.items():
            net = m.trace(field, params, cam, W, H).cpu().numpy()
            st = m.trace_status()
            assert st["error"] == 0, name
            assert st["network_evals"] > 0, name
            # every pixel written with a valid status
            assert set(np.unique(net[:, 7])) <= {0, 1, 2}, name
            err_n, mism_n, both_n = _sdf_errors(net, tc, pix)
            # the target: median hit error <= 1e-3 scene units against the
            # FP64 root, few silhouette (hit / miss) disagreements
            assert np.median(err_n) <= 1e-3, (name, np.median(err_n))
            assert mism_n <= 0.01 * len(pix), (name, mism_n)
            assert (net[:, 7] != ex[:, 7]).mean() < 0.01, name
            assert ((net[:, 7] == 1) != (exact_tracer[:, 7] == 1)).mean() < 0.01, name
            # what the network gains: it replaces exact-field march steps
            assert st["exact_evals"] < 0.8 * st_ex["exact_evals"], (name, st, st_ex)
            # the normal is the stated stencil at the returned position
            hits = pix[net[pix, 7] == 1]
            ang = _normals_from_positions(net, cam, hits[:400], params.normal_taps or 6)
            assert np.quantile(ang, 0.99) < 0.05, (name, np.quantile(ang, 0.99))


def test_gradient_normal_pass(cuda):
    """normal_taps 1: the exact phase writes the same hits (position, step
    count, status) as with the tetrahedral normal, and the second pass adds
    the field's analytic gradient, which agrees with the FP64 gradient."""
    tc = rb.configs.TerrainConfig(width=320, height=180)
    with _model() as m:
        field, cam = tc.params(), tc.camera()
        W, H = tc.width, tc.height
        tet = m.trace(field, rb.nsdf_trace_params(exact_only=True, normal_taps=4), cam, W, H)
        tet = tet.cpu().numpy()
        st4 = m.trace_status()
        grad = m.trace(field, rb.nsdf_trace_params(exact_only=True, normal_taps=1), cam, W, H)
        grad = grad.cpu().numpy()
        st1 = m.trace_status()
        assert st1["error"] == 0
        for col in (0, 1, 2, 6, 7):
            assert np.array_equal(tet[:, col], grad[:, col]), col
        hits = np.nonzero(grad[:, 7] == 1)[0]
        assert len(hits) > 0.5 * W * H
        assert st1["exact_evals"] == st4["exact_evals"]
        assert st1["normal_evals"] == len(hits)  # one gradient per hit
        nrm = grad.view(np.float32)[hits, 3:6]
        assert np.allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-5)
        assert np.all(grad.view(np.float32)[grad[:, 7] != 1, 3:6] == 0)
        sample = np.random.default_rng(3).choice(hits, 3000, replace=False).astype(np.uint32)
        ang = _normals_from_positions(grad, cam, sample, 1)
        assert np.median(ang) < 1e-3 and np.quantile(ang, 0.99) < 1e-2, (
            np.median(ang), np.quantile(ang, 0.99), ang.max())
        # against it the finite-difference stencils at radius 0.002 t are
        # coarse (several degrees)
        tet_ang = _normals_from_positions(tet, cam, sample, 1)
        assert np.median(tet_ang) > 1.0


def test_trace_parameter_checks(cuda):
    tc = rb.configs.TerrainConfig(width=64, height=36)
    with _model() as m:
        field, cam = tc.params(), tc.camera()
        bad = [dict(cone_tile=8, cone_coarse=12), dict(cone_tile=8, cone_coarse=8),
               dict(cone_tile=0, cone_coarse=32), dict(cone_tile=300),
               dict(cone_tile=8, cone_lanes=3), dict(cone_tile=8, cone_lanes=32),
               dict(normal_taps=5)]
        for kw in bad:
            with pytest.raises(rb.RayEngineError):
                m.trace(field, rb.nsdf_trace_params(**kw), cam, tc.width, tc.height)
        # the exact phase needs the network phase of the same image and mode
        tp = rb.nsdf_trace_params(cone_tile=8, cone_lanes=2)
        out = m.trace(field, tp, cam, tc.width, tc.height)
        with pytest.raises(rb.RayEngineError):
            m.trace(field, rb.nsdf_trace_params(cone_tile=4), cam, tc.width, tc.height, out,
                    phase="exact")
        with pytest.raises(rb.RayEngineError):
            m.trace(field, tp, cam, tc.width + 8, tc.height, phase="exact")
