"""Learned per-pixel confidence weight: training data, training on the GPU
with the library's own kernels, and evaluation against the plain weight.

The reference weights every pixel's voxel updates with the same distance
ramp (update_functions.cpp:1187-1444).  Here a 3-layer 5x5 CNN (16
channels, BF16 weights and activations, FP32 accumulation; the kernels are
in csrc/ff_cnn.cu) predicts each pixel's depth error r from its depth and
finite-difference normal, and the ramp's weight increment is multiplied by
(1 - r/tau)^2 (0 beyond tau).  The plain weight stays the fallback
(FusionMipMapCPU.set_confidence(None)).

Training data: seeded rooms as in the plain-method workload (4x4x3 m, 20
primitives, circle trajectory), rendered with sigma = 0.002 z^2 noise, 2 %
holes and 10 % of the depth-edge pixels displaced by +-0.1 m.  Each scene's
frames are fused with the plain weight; the target of a pixel is
|raw depth - depth raycast from that fused volume| (cm, capped at 15; 15
where no surface lies within 15 cm; no label where the pixel has no depth).

    python -m fastfusion_b200.confidence train [--scenes 500] [--steps 3000]
    python -m fastfusion_b200.confidence eval [--seeds 50]

`train` writes confidence_weights.npz next to this file (parameters and
tau); `eval` prints the surface RMS error against the analytic scene SDF of
the plain and the learned weight on held-out seeds.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from fastfusion_b200 import fusion, scene

N_PARAMS = 8833
PACKED_BYTES = 33280   # FF_CNN_PACKED_BYTES: the weights as tensor-core operands
LAYOUT = ((0, 2000), (2000, 16), (2016, 6400), (8416, 16), (8432, 400), (8832, 1))  # W1 b1 W2 b2 W3 b3
UNIT_M = 0.01          # the network predicts centimetres
CAP_CM = 15.0          # target cap and the raycast window
NOISE_K = 0.002        # depth noise sigma = NOISE_K z^2
FLYING = 0.10          # fraction of depth-edge pixels displaced
SCALING = 1.0 / 5000.0
MAXCAM = 4.0
VOXEL_M, THRESHOLD_M = 0.005, 0.01
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "confidence_weights.npz")
TRAIN_SEED0, EVAL_SEED0 = 10000, 20000


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases; the output bias starts at 1 cm."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[0:2000] = rng.normal(0.0, math.sqrt(2.0 / (5 * 25)), 2000)
    p[2016:8416] = rng.normal(0.0, math.sqrt(2.0 / (16 * 25)), 6400)
    p[8432:8832] = rng.normal(0.0, math.sqrt(1.0 / (16 * 25)), 400)
    p[8832] = 1.0
    return p


def load_weights(path: str = WEIGHTS_PATH) -> tuple[np.ndarray, float]:
    """(parameters, tau in metres) of a trained network."""
    z = np.load(path)
    return z["params"].astype(np.float32), float(z["tau_m"])


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


class ConfidenceNet:
    """The network on one GPU: FP32 master weights, their BF16 copy the
    kernels read, gradients and Adam moments (torch tensors as device
    memory; every step runs the library's kernels)."""

    def __init__(self, params: np.ndarray | None = None, device: str = "cuda"):
        import torch
        self.torch = torch
        self.L = fusion.load_library()
        self.dev = torch.device(device)
        p = init_params() if params is None else np.asarray(params, np.float32)
        assert p.size == N_PARAMS
        self.master = torch.tensor(p, dtype=torch.float32, device=self.dev)
        self.params = self.master.to(torch.bfloat16)
        self.grads = torch.zeros(N_PARAMS, dtype=torch.float32, device=self.dev)
        self.m = torch.zeros_like(self.grads)
        self.v = torch.zeros_like(self.grads)
        self.loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.packed = torch.empty(PACKED_BYTES, dtype=torch.uint8, device=self.dev)
        self.step_no = 0
        self._bufs = {}

    def _check(self, st):
        if st != fusion.FF_OK:
            raise fusion.FFError(st, self.L.ff_last_error(None).decode())

    def bufs(self, n: int, H: int, W: int) -> dict:
        key = (n, H, W)
        if key not in self._bufs:
            t, d = self.torch, self.dev
            self._bufs = {key: {
                "a1": t.empty((n, H, W, 16), dtype=t.bfloat16, device=d),
                "a2": t.empty((n, H, W, 16), dtype=t.bfloat16, device=d),
                "pred": t.empty((n, H, W), dtype=t.float32, device=d),
                "dpred": t.empty((n, H, W), dtype=t.float32, device=d),
                "g1": t.empty((n, H, W, 16), dtype=t.float32, device=d),
                "g2": t.empty((n, H, W, 16), dtype=t.float32, device=d),
            }}
        return self._bufs[key]

    def features(self, depth, K, scaling: float = SCALING):
        """depth: uint16 bit patterns as an int16 device tensor [n, H, W] or [H, W]."""
        t = self.torch
        d = depth if depth.dim() == 3 else depth[None]
        d = d.contiguous()
        n, H, W = d.shape
        feat = t.empty((n, H, W, 8), dtype=t.bfloat16, device=self.dev)
        Kd = np.ascontiguousarray(K, dtype=np.float64)
        self._check(self.L.ff_cnn_features(d.data_ptr(), n, W, H, float(scaling), Kd.ctypes.data, feat.data_ptr(),
                                           _stream()))
        return feat

    def forward(self, feat, tau_m: float = 0.0):
        """The prediction (cm), or the confidence when tau_m > 0: [n, H, W]."""
        n, H, W, _ = feat.shape
        b = self.bufs(n, H, W)
        out = self.torch.empty((n, H, W), dtype=self.torch.float32, device=self.dev)
        self._check(self.L.ff_cnn_forward(self.params.data_ptr(), self.packed.data_ptr(), feat.data_ptr(), n, W, H,
                                          b["a1"].data_ptr(), b["a2"].data_ptr(), out.data_ptr(), float(tau_m),
                                          _stream()))
        return out

    def loss_and_grads(self, feat, target, inv_count: float):
        """Forward, loss and backward; the gradient is added to self.grads."""
        n, H, W, _ = feat.shape
        b = self.bufs(n, H, W)
        self.loss.zero_()
        L, s = self.L, _stream()
        self._check(L.ff_cnn_forward(self.params.data_ptr(), self.packed.data_ptr(), feat.data_ptr(), n, W, H,
                                     b["a1"].data_ptr(), b["a2"].data_ptr(), b["pred"].data_ptr(), 0.0, s))
        self._check(L.ff_cnn_mse(b["pred"].data_ptr(), target.data_ptr(), n * H * W, float(inv_count),
                                 b["dpred"].data_ptr(), self.loss.data_ptr(), s))
        self._check(L.ff_cnn_backward(self.params.data_ptr(), feat.data_ptr(), b["a1"].data_ptr(), b["a2"].data_ptr(),
                                      b["dpred"].data_ptr(), n, W, H, b["g1"].data_ptr(), b["g2"].data_ptr(),
                                      self.grads.data_ptr(), s))
        return b

    def train_step(self, feat, target, inv_count: float, lr: float) -> None:
        self.loss_and_grads(feat, target, inv_count)
        self.step_no += 1
        self._check(self.L.ff_cnn_adam(self.master.data_ptr(), self.params.data_ptr(), self.grads.data_ptr(),
                                       self.m.data_ptr(), self.v.data_ptr(), float(lr), 0.9, 0.999, 1e-8,
                                       self.step_no, _stream()))

    def state(self) -> np.ndarray:
        return self.master.detach().cpu().numpy().copy()


# ------------------------------------------------------------------ data

def _render(seq, k: int, R, t, seed: int):
    return scene.render_torch(seq.scene, R, t, seq.width, seq.height, seq.K, seed, k, noise_k=NOISE_K,
                              hole_frac=0.02, flying_frac=FLYING)


def _new_map(storage: str = "fp32"):
    import torch
    f = fusion.FusionMipMapCPU(0, 0, 0, VOXEL_M, THRESHOLD_M, 0, True, leaves_max=271420, branches_max=4793488,
                               storage=storage)
    f.set_stream(torch.cuda.current_stream().cuda_stream)
    return f


def make_examples(net: ConfidenceNet, seeds, n_views: int = 20, label_views=(0, 10), width: int = 640,
                  height: int = 480):
    """(features bf16 [N, H, W, 8], targets f32 [N, H, W]) from the given
    scene seeds: each scene's n_views frames (evenly spaced on its circle)
    fused with the plain weight, targets raycast at label_views."""
    import torch
    feats, targets = [], []
    for seed in seeds:
        seq = scene.room_circle_sequence(int(seed), n_frames=100, width=width, height=height)
        step = max(1, 100 // n_views)
        fz = _new_map()
        kept = {}
        for j, k in enumerate(range(0, 100, step)[:n_views]):
            R, t = seq.poses[k]
            d, c = _render(seq, k, R, t, int(seed))
            fz.addMapDevice(d.data_ptr(), c.data_ptr(), width, height, fusion.CameraInfo(seq.K, R, t), SCALING,
                            MAXCAM)
            if j in label_views:
                kept[j] = (d, R, t)
        for j, (d, R, t) in kept.items():
            ray = torch.empty((height, width), dtype=torch.float32, device="cuda")
            fz.raycast_depth(d.data_ptr(), width, height, fusion.CameraInfo(seq.K, R, t), ray.data_ptr(), SCALING,
                             CAP_CM * UNIT_M, 0.5 * VOXEL_M)
            z = (d.to(torch.int32) & 0xFFFF).to(torch.float32) * SCALING
            res = torch.clamp((z - ray).abs() / UNIT_M, max=CAP_CM)
            tgt = torch.where(z <= 0, torch.full_like(z, -1.0), torch.where(ray < 0, torch.full_like(z, CAP_CM), res))
            feats.append(net.features(d, seq.K)[0])
            targets.append(tgt)
        fz.close()
    return torch.stack(feats), torch.stack(targets)


def train(net: ConfidenceNet, feats, targets, steps: int, batch: int = 4, lr: float = 2e-3, seed: int = 0,
          log=None) -> list:
    """Adam with cosine decay over random batches of whole images; returns
    the loss of every step (mean squared error in cm^2 over labelled pixels)."""
    import torch
    rng = np.random.default_rng(seed)
    N = feats.shape[0]
    counts = (targets >= 0).sum(dim=(1, 2)).cpu().numpy()
    losses = []
    for s in range(steps):
        idx = np.sort(rng.choice(N, size=min(batch, N), replace=False))
        it = torch.as_tensor(idx, device=feats.device)
        f = feats.index_select(0, it).contiguous()
        t = targets.index_select(0, it).contiguous()
        inv = 1.0 / max(1, int(counts[idx].sum()))
        cur = lr * 0.5 * (1.0 + math.cos(math.pi * s / max(1, steps)))
        net.train_step(f, t, inv, cur)
        losses.append(net.loss.clone())
        if log and (s % 200 == 0 or s == steps - 1):
            log(f"step {s} loss {float(net.loss.item()):.4f}")
    return torch.cat(losses).cpu().numpy().tolist() if losses else []


# ------------------------------------------------------------ evaluation

def surface_rms(seed: int, params=None, tau_m: float = 0.03, n_frames: int = 100, width: int = 640,
                height: int = 480, storage: str = "fp32") -> dict:
    """Fuse one held-out scene with the plain weight and (if params) the
    learned weight from the same frames; surface RMS (m) of each final mesh
    against the analytic scene SDF."""
    seq = scene.room_circle_sequence(int(seed), n_frames=100, width=width, height=height)
    plain = _new_map(storage)
    learned = None
    if params is not None:
        learned = _new_map(storage)
        learned.set_confidence(params, tau_m)
    step = max(1, 100 // n_frames)
    for k in range(0, 100, step)[:n_frames]:
        R, t = seq.poses[k]
        d, c = _render(seq, k, R, t, int(seed))
        cam = fusion.CameraInfo(seq.K, R, t)
        plain.addMapDevice(d.data_ptr(), c.data_ptr(), width, height, cam, SCALING, MAXCAM)
        if learned is not None:
            learned.addMapDevice(d.data_ptr(), c.data_ptr(), width, height, cam, SCALING, MAXCAM)
    out = {}
    for name, f in (("plain", plain), ("learned", learned)):
        if f is None:
            continue
        f.updateMeshes()
        v = f.getMeshInterleavedMarchingCubes().vertices.astype(np.float64)
        e = seq.scene.sdf(v) if len(v) else np.zeros(1)
        out[name] = float(np.sqrt(np.mean(e * e)))
        out[name + "_vertices"] = int(len(v))
        f.close()
    return out


def choose_tau(params, seeds, taus=(0.02, 0.03, 0.05, 0.08), n_frames: int = 50) -> tuple[float, dict]:
    """The tau with the lowest mean surface RMS on (training) seeds."""
    res = {}
    for tau in taus:
        r = [surface_rms(s, params, tau, n_frames=n_frames)["learned"] for s in seeds]
        res[tau] = float(np.mean(r))
    best = min(res, key=res.get)
    return best, res


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m fastfusion_b200.confidence")
    sub = ap.add_subparsers(dest="cmd", required=True)
    tr = sub.add_parser("train")
    tr.add_argument("--scenes", type=int, default=500)
    tr.add_argument("--steps", type=int, default=3000)
    tr.add_argument("--batch", type=int, default=4)
    tr.add_argument("--lr", type=float, default=2e-3)
    tr.add_argument("--out", default=WEIGHTS_PATH)
    tr.add_argument("--tau-seeds", type=int, default=4)
    ev = sub.add_parser("eval")
    ev.add_argument("--seeds", type=int, default=50)
    ev.add_argument("--frames", type=int, default=100)
    ev.add_argument("--weights", default=WEIGHTS_PATH)
    ev.add_argument("--storage", default="fp32")
    a = ap.parse_args(argv)
    import torch
    log = lambda m: print(m, flush=True)  # noqa: E731
    if a.cmd == "train":
        t0 = time.time()
        net = ConfidenceNet()
        feats, targets = make_examples(net, range(TRAIN_SEED0, TRAIN_SEED0 + a.scenes))
        torch.cuda.synchronize()
        lab = targets[targets >= 0]
        log(f"examples: {feats.shape[0]} images, {int(lab.numel())} labelled pixels, target mean "
            f"{float(lab.mean()):.3f} cm, capped {float((lab >= CAP_CM).float().mean()):.4f}, "
            f"{time.time() - t0:.1f} s")
        t1 = time.time()
        losses = train(net, feats, targets, a.steps, a.batch, a.lr, log=log)
        torch.cuda.synchronize()
        log(f"trained {a.steps} steps in {time.time() - t1:.1f} s; loss {losses[0]:.3f} -> "
            f"{np.mean(losses[-50:]):.3f}")
        params = net.state()
        tau, res = choose_tau(params, range(TRAIN_SEED0, TRAIN_SEED0 + a.tau_seeds))
        log(f"tau per mean surface RMS on training scenes: {res} -> {tau}")
        np.savez(a.out, params=params, tau_m=np.float32(tau), loss_first=np.float32(losses[0]),
                 loss_last=np.float32(np.mean(losses[-50:])), scenes=np.int32(a.scenes), steps=np.int32(a.steps))
        log(f"wrote {a.out}")
    else:
        params, tau = load_weights(a.weights)
        rows = []
        for s in range(EVAL_SEED0, EVAL_SEED0 + a.seeds):
            r = surface_rms(s, params, tau, n_frames=a.frames, storage=a.storage)
            r["seed"] = s
            rows.append(r)
        plain = np.array([r["plain"] for r in rows])
        learned = np.array([r["learned"] for r in rows])
        print(json.dumps({"metric": "surface RMS vs analytic SDF (m), held-out scenes", "seeds": a.seeds,
                          "frames": a.frames, "tau_m": tau, "storage": a.storage,
                          "plain_mean": float(plain.mean()), "learned_mean": float(learned.mean()),
                          "learned_better": int((learned < plain).sum()), "rows": rows}))


if __name__ == "__main__":
    main()
