"""The learned confidence weight on the GPU: its kernels against the CPU
oracle (oracle/cnn.py), training, the raycaster, fusion with the learned
weight bit-exact against the restatement given the same confidence map, and
the gain of the trained network over the plain weight.

Tolerances: features and stored activations are BF16, so an element may
differ from the oracle by one BF16 step where FP32 and FP64 accumulation
round to different sides (<= 1 % of elements); layer outputs recomputed
from the GPU's own inputs agree to 1e-4 of their scale; parameter gradients
(FP32 sums over all pixels, atomics) to 1e-4 relative L2 per tensor.
"""
import numpy as np
import pytest

from oracle import cnn
from tests.helpers import SCALING

pytestmark = pytest.mark.gpu

W, H = 96, 72
K = np.array([525.0 * W / 640, 525.0 * W / 640, (W - 1) / 2.0, (H - 1) / 2.0])


def _depth_frames(n=2, w=W, h=H, noise=0.002, flying=0.1):
    """n rendered depth frames (int16 device tensors) of one scene."""
    import torch
    from fastfusion_b200 import scene
    seq = scene.room_circle_sequence(5, n_frames=100, width=w, height=h)
    out = []
    for k in range(n):
        R, t = seq.poses[10 * k]
        d, _ = scene.render_torch(seq.scene, R, t, w, h, seq.K, 5, k, noise_k=noise, flying_frac=flying)
        out.append(d)
    return torch.stack(out), seq.K


def _bf16_close(a, b, atol, frac=0.01):
    """Equal but for <= frac of the elements, which differ by at most one BF16
    step (2^-7 relative) plus atol (FP32 vs FP64 cancellation in sums and
    cross products)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    diff = a != b
    assert diff.mean() <= frac, diff.mean()
    tol = np.maximum(np.abs(b), np.abs(a)) * 2.0 ** -7 + atol
    bad = np.abs(a - b) > tol
    assert not bad.any(), (np.abs(a - b)[bad][:8], a[bad][:8], b[bad][:8])


def _net(seed=1):
    from fastfusion_b200.confidence import ConfidenceNet, init_params
    return ConfidenceNet(init_params(seed))


def test_features_match_oracle(lib_built):
    net = _net()
    d, Kd = _depth_frames()
    feat = net.features(d, Kd).float().cpu().numpy()
    dn = (d.cpu().numpy().astype(np.int32) & 0xFFFF).astype(np.uint16)
    ref = np.stack([cnn.features(x, SCALING, Kd) for x in dn])
    _bf16_close(feat, ref, atol=1e-3)
    assert (feat[..., 4] > 0).sum() > 0.9 * feat[..., 4].size


def test_forward_matches_oracle(lib_built):
    import torch
    net = _net()
    d, Kd = _depth_frames()
    feat_t = net.features(d, Kd)
    pred = net.forward(feat_t).cpu().numpy()
    b = net.bufs(*feat_t.shape[:3])
    a1 = b["a1"].float().cpu().numpy()
    a2 = b["a2"].float().cpu().numpy()
    feat = feat_t.float().cpu().numpy()
    params = net.state()
    P = {k: cnn.bf16(v) for k, v in cnn.unpack(params).items()}
    # layer by layer from the GPU's own inputs
    r1 = cnn.bf16(np.maximum(cnn.conv(feat[..., :5], P["W1"], P["b1"]), 0))
    _bf16_close(a1, r1, atol=1e-3 * np.abs(r1).max())
    assert (a1 > 0).mean() > 0.2
    r2 = cnn.bf16(np.maximum(cnn.conv(a1, P["W2"], P["b2"]), 0))
    _bf16_close(a2, r2, atol=1e-3 * np.abs(r2).max())
    r3 = cnn.conv(a2, P["W3"], P["b3"])[..., 0]
    assert np.max(np.abs(pred - r3)) <= 1e-4 * max(1.0, np.abs(r3).max())
    # the whole network from the features
    _, _, rp = cnn.forward(params, feat)
    assert np.percentile(np.abs(pred - rp), 99) <= 0.02 * max(1.0, np.abs(rp).max())
    # confidence mode
    conf = net.forward(feat_t, tau_m=0.03).cpu().numpy()
    assert np.max(np.abs(conf - cnn.confidence(pred, 3.0))) <= 1e-6
    torch.cuda.synchronize()


def test_backward_matches_oracle(lib_built):
    import torch
    net = _net(2)
    d, Kd = _depth_frames()
    feat_t = net.features(d, Kd)
    rng = np.random.default_rng(0)
    tgt = rng.uniform(0, 5, size=feat_t.shape[:3]).astype(np.float32)
    tgt[rng.random(tgt.shape) < 0.1] = -1.0
    tgt_t = torch.tensor(tgt, device="cuda")
    inv = 1.0 / float((tgt >= 0).sum())
    b = net.loss_and_grads(feat_t, tgt_t, inv)
    g = net.grads.cpu().numpy().astype(np.float64)
    loss = float(net.loss.item())
    pred = b["pred"].cpu().numpy()
    dpred = b["dpred"].cpu().numpy()
    rl, rd = cnn.mse(pred.astype(np.float64), tgt.astype(np.float64), inv)
    assert abs(loss - rl) <= 1e-6 * rl
    assert np.max(np.abs(dpred - rd)) <= 1e-6 * np.abs(rd).max()
    ref = cnn.backward(net.state(), feat_t.float().cpu().numpy(), b["a1"].float().cpu().numpy(),
                       b["a2"].float().cpu().numpy(), dpred)
    for name, (o, k) in zip(["W1", "b1", "W2", "b2", "W3", "b3"],
                            ((0, 2000), (2000, 16), (2016, 6400), (8416, 16), (8432, 400), (8832, 1))):
        e = np.linalg.norm(g[o:o + k] - ref[o:o + k]) / max(np.linalg.norm(ref[o:o + k]), 1e-30)
        assert e <= 1e-4, (name, e)
    assert np.linalg.norm(ref) > 0


def test_adam_step(lib_built):
    import torch
    net = _net(3)
    rng = np.random.default_rng(1)
    g = rng.normal(size=8833).astype(np.float32)
    w0 = net.state().astype(np.float64)
    net.grads.copy_(torch.tensor(g, device="cuda"))
    net.step_no = 0
    from fastfusion_b200 import fusion
    L = fusion.load_library()
    st = L.ff_cnn_adam(net.master.data_ptr(), net.params.data_ptr(), net.grads.data_ptr(), net.m.data_ptr(),
                       net.v.data_ptr(), 0.01, 0.9, 0.999, 1e-8, 1, torch.cuda.current_stream().cuda_stream)
    assert st == 0
    m = 0.1 * g.astype(np.float64)
    v = 0.001 * g.astype(np.float64) ** 2
    w1 = w0 - 0.01 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    got = net.state()
    assert np.max(np.abs(got - w1)) <= 1e-6
    assert np.array_equal(net.params.float().cpu().numpy(), cnn.bf16(got).astype(np.float32))
    assert float(net.grads.abs().max().item()) == 0.0


def test_training_reduces_loss(lib_built):
    from fastfusion_b200 import confidence
    net = confidence.ConfidenceNet()
    feats, targets = confidence.make_examples(net, [31, 32], n_views=10, label_views=(0, 5), width=160, height=120)
    assert feats.shape == (4, 120, 160, 8)
    lab = targets[targets >= 0]
    assert lab.numel() > 0.5 * targets.numel()
    # the same four images every step: the loss must fall
    losses = confidence.train(net, feats, targets, steps=200, batch=4, lr=3e-3)
    first, last = float(np.mean(losses[:3])), float(np.mean(losses[-20:]))
    print(f"\ntraining loss {first:.3f} -> {last:.3f}")
    assert last < 0.7 * first


def test_raycast_recovers_depth(lib_built):
    import torch
    from fastfusion_b200 import fusion, scene
    w, h = 320, 240
    seq = scene.room_circle_sequence(7, n_frames=100, width=w, height=h)
    f = fusion.FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True)
    f.set_stream(torch.cuda.current_stream().cuda_stream)
    frames = []
    for k in range(0, 100, 10):
        R, t = seq.poses[k]
        d, c, zt = scene.render_torch(seq.scene, R, t, w, h, seq.K, 7, k, noise_k=0.0012, hole_frac=0.0,
                                      return_true=True)
        f.addMapDevice(d.data_ptr(), c.data_ptr(), w, h, fusion.CameraInfo(seq.K, R, t), SCALING, 4.0)
        frames.append((d, zt, R, t))
    d, zt, R, t = frames[0]
    ray = torch.empty((h, w), dtype=torch.float32, device="cuda")
    f.raycast_depth(d.data_ptr(), w, h, fusion.CameraInfo(seq.K, R, t), ray.data_ptr(), SCALING, 0.15, 0.0025)
    ray = ray.cpu().numpy()
    zt = zt.cpu().numpy()
    ok = (ray > 0) & (zt < 4.0)
    print(f"\nraycast found a surface for {ok.mean():.3f} of the pixels")
    assert ok.mean() > 0.8
    err = np.abs(ray[ok] - zt[ok])
    print(f"raycast vs true depth: median {np.median(err) * 1e3:.2f} mm, p90 {np.percentile(err, 90) * 1e3:.2f} mm")
    # bricks are 1-2 cm voxels beyond 2-3 m (the reference's level rule) and
    # the depth noise there is ~5-10 mm per frame
    assert np.median(err) < 0.006 and np.percentile(err, 90) < 0.02
    f.close()


def test_learned_fusion_matches_restatement(lib_built, port_lib):
    """The update with a confidence map is bit-exact against the restatement
    given the same map (the map itself is checked against the oracle)."""
    from fastfusion_b200 import fusion, scene
    from fastfusion_b200.confidence import init_params
    w, h = 160, 120
    seq = scene.room_circle_sequence(3, n_frames=100, width=w, height=h)
    params = init_params(4)
    g = fusion.FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=65536, branches_max=1 << 20, rcp="exact")
    g.set_confidence(params, 0.03)
    p = port_lib.PortFusion(leaves_total=65536, branches_total=1 << 20, update_mode=1)
    any_partial = False
    for k in range(0, 50, 10):
        depth, bgr, R, t = seq.frame(k)
        cam = fusion.CameraInfo(seq.K, R, t)
        qg = g.addMap(depth, cam, bgr, SCALING, 4.0)
        conf = g.confidence_map()
        assert conf.shape == (h, w)
        _, _, rp = cnn.forward(params, cnn.features(depth, SCALING, seq.K)[None])
        rc = cnn.confidence(rp[0], 3.0)
        assert np.percentile(np.abs(conf - rc), 99) <= 0.05
        any_partial |= bool(((conf > 0) & (conf < 1)).any())
        p.set_confidence(conf)
        qp = p.add_map(depth, bgr, seq.K, R, t, SCALING, 4.0)
        assert qg == qp
    assert any_partial
    dg, wg, cg = g.bricks()
    dp, wp, cp = p.bricks()
    assert np.array_equal(dg.view(np.uint32), dp.view(np.uint32))
    assert np.array_equal(wg.view(np.uint32), wp.view(np.uint32))
    assert np.array_equal(cg, cp)
    # off again: the reference's weight
    g.set_confidence(None)
    g.close()


def test_learned_weight_beats_plain_weight(lib_built):
    """The committed trained network against the plain weight on held-out
    scenes (50 frames each, flying pixels and sigma = 0.002 z^2 noise)."""
    from fastfusion_b200 import confidence
    params, tau = confidence.load_weights()
    rows = [confidence.surface_rms(s, params, tau, n_frames=50) for s in
            range(confidence.EVAL_SEED0, confidence.EVAL_SEED0 + 3)]
    plain = np.mean([r["plain"] for r in rows])
    learned = np.mean([r["learned"] for r in rows])
    print(f"\nsurface RMS vs analytic SDF: plain {plain * 1e3:.3f} mm, learned {learned * 1e3:.3f} mm ({rows})")
    assert learned < plain
