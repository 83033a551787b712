"""One differentiable training step of a Gaussian scene on the GPU: render several
views, L1 + SSIM loss against target images, backward through the rasterizer, FP32
Adam on the Gaussians that were visible, densification statistics.

Mirrors LoG's training loop (LoG/render/renderer.py:260-273 for the loss,
LoG/model/sparse_optimizer.py for the optimizer, LoG/model/counter.py for the
statistics) with the rasterizer of this package.  Two paths compute the same step:

* BatchedTrainer -- every view's forward, the loss, the backward and the Adam update
  are enqueued without a host synchronisation and captured in one CUDA graph.
* PlainTrainer -- one view per call through the `_C` entry points (the reference's
  structure: a host synchronisation per view for the pair count), the gradients summed
  over the views, then the same Adam update.

Both give bit-identical parameters (the backward is deterministic and the views are
summed in the same order).
"""
import ctypes as C

import torch

from . import _lib
from ._C import rasterize_gaussians, rasterize_gaussians_backward
from ._lib import AdamArgs, call, lib

# LoG lr_dict of the training configs: means, SH, opacity, scale, rotation
DEFAULT_LR = (1.6e-4, 2.5e-3, 0.05, 5e-3, 1e-3)


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return None if t is None or t.numel() == 0 else C.c_void_p(t.data_ptr())


class TrainState:
    """Raw parameters, their activations, Adam moments, the device step counter and the
    densification statistics of one Gaussian set."""

    def __init__(self, xyz, log_scale, rot_raw, opac_logit, shs, lr=DEFAULT_LR, betas=(0.9, 0.999), eps=1e-15):
        c = lambda t: t.detach().float().contiguous().clone()  # noqa: E731
        self.xyz, self.log_scale, self.rot_raw = c(xyz), c(log_scale), c(rot_raw)
        self.opac_logit, self.shs = c(opac_logit).reshape(-1, 1), c(shs)
        self.P = int(self.xyz.shape[0])
        self.M = int(self.shs.shape[1])
        dev = self.xyz.device
        self.scale = torch.empty_like(self.log_scale)
        self.rot = torch.empty_like(self.rot_raw)
        self.opac = torch.empty_like(self.opac_logit)
        self.m = {k: torch.zeros_like(v) for k, v in self.raw().items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.raw().items()}
        self.step = torch.zeros(1, dtype=torch.int32, device=dev)
        self.grad_sum = torch.zeros(self.P, device=dev)
        self.vis_count = torch.zeros(self.P, dtype=torch.int32, device=dev)
        self.flag = torch.zeros(self.P, dtype=torch.uint8, device=dev)
        self.lr, self.betas, self.eps = tuple(float(x) for x in lr), betas, float(eps)
        self.activate()

    def raw(self):
        return dict(xyz=self.xyz, shs=self.shs, opacity=self.opac_logit, scale=self.log_scale, rotation=self.rot_raw)

    def activate(self):
        call("fgs_train_activate", self.P, _p(self.log_scale), _p(self.rot_raw), _p(self.opac_logit), _p(self.scale),
             _p(self.rot), _p(self.opac), _s())

    def adam(self, g_means3D, g_sh, g_opacity, g_scales, g_rotations):
        """Adam on the rows flagged visible in this step (gradients w.r.t. the rasterizer inputs)."""
        a = AdamArgs()
        a.P, a.M = self.P, self.M
        for i, x in enumerate(self.lr):
            a.lr[i] = x
        a.beta1, a.beta2, a.eps = float(self.betas[0]), float(self.betas[1]), self.eps
        a.xyz, a.shs, a.opac_logit, a.log_scale, a.rot_raw = (_p(self.xyz), _p(self.shs), _p(self.opac_logit),
                                                              _p(self.log_scale), _p(self.rot_raw))
        a.opac, a.scale, a.rot = _p(self.opac), _p(self.scale), _p(self.rot)
        a.g_xyz, a.g_shs, a.g_opac, a.g_scale, a.g_rot = (_p(g_means3D), _p(g_sh), _p(g_opacity), _p(g_scales),
                                                          _p(g_rotations))
        m, v = self.m, self.v
        a.m_xyz, a.m_shs, a.m_opac, a.m_scale, a.m_rot = (_p(m["xyz"]), _p(m["shs"]), _p(m["opacity"]), _p(m["scale"]),
                                                          _p(m["rotation"]))
        a.v_xyz, a.v_shs, a.v_opac, a.v_scale, a.v_rot = (_p(v["xyz"]), _p(v["shs"]), _p(v["opacity"]), _p(v["scale"]),
                                                          _p(v["rotation"]))
        self._adam_args = a  # kept alive: a captured graph does not re-read it, an eager call copies it
        call("fgs_adam_step", C.byref(a), _p(self.flag), _p(self.step), _s())


class Loss:
    """0.8 * L1 + 0.2 * (1 - SSIM) over a batch of [3,H,W] images (LoG/render/renderer.py:260-273);
    the per-view gradient is written into the caller's buffer, the sums stay on the device."""

    def __init__(self, sizes, device):
        self.sizes = [(int(w), int(h)) for w, h in sizes]
        self.n_l1 = sum(3 * w * h for w, h in self.sizes)
        self.n_ssim = sum(3 * (w - 10) * (h - 10) for w, h in self.sizes)
        nb = max(int(lib().fgs_loss_scratch_bytes(w, h)) for w, h in self.sizes)
        self.scratch = torch.empty(nb // 4 + 64, dtype=torch.float32, device=device)
        self.sums = torch.zeros(2, dtype=torch.float64, device=device)

    def __call__(self, preds, targets, grads):
        self.sums.zero_()
        for (w, h), x, y, g in zip(self.sizes, preds, targets, grads):
            call("fgs_loss_l1_ssim", w, h, _p(x), _p(y), _p(g), 0.8 / self.n_l1, 0.2 / self.n_ssim, _p(self.sums),
                 _p(self.scratch), _s())

    def value(self):
        s = self.sums.cpu()
        return float(0.8 * s[0] / self.n_l1 + 0.2 * (1.0 - s[1] / self.n_ssim))


class _Views:
    def __init__(self, cameras, targets):
        self.cams = list(cameras)
        self.targets = list(targets)


class BatchedTrainer:
    """The training step through the batched rasterizer, captured in one CUDA graph."""

    def __init__(self, state, cameras, targets, bg=None, graph=True):
        from .batched import BatchedRasterizer
        self.st = state
        self.v = _Views(cameras, targets)
        dev = state.xyz.device
        self.bg = bg if bg is not None else torch.zeros(3, device=dev)
        self.br = BatchedRasterizer(state.xyz, state.opac, state.scale, state.rot, self.v.cams, shs=state.shs,
                                    sh_degree=3, bg=self.bg, graph=False)
        call("fgs_batch_set_densify", self.br.handle, _p(state.grad_sum), _p(state.vis_count), _p(state.flag))
        self.loss = Loss([(c.W, c.H) for c in self.v.cams], dev)
        self.use_graph = graph
        self.graph = None

    def _enqueue(self):
        st, br = self.st, self.br
        st.flag.zero_()
        br.forward()
        self.loss(br.images, self.v.targets, br.dL)
        br.backward()
        g = br.grad
        st.adam(g["means3D"], g["sh"], g["opacity"], g["scales"], g["rotations"])

    def step(self):
        if not self.use_graph:
            self._enqueue()
            return
        if self.graph is None:
            s = torch.cuda.Stream(device=self.st.xyz.device)
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self._enqueue()             # eager once (module loading), then capture
            torch.cuda.current_stream().wait_stream(s)
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                self._enqueue()
            self.graph = g
            return
        self.graph.replay()

    def check(self):
        self.br.check()


class PlainTrainer:
    """The same step, one view per call through the `_C` entry points."""

    def __init__(self, state, cameras, targets, bg=None):
        self.st = state
        self.v = _Views(cameras, targets)
        dev = state.xyz.device
        self.bg = bg if bg is not None else torch.zeros(3, device=dev)
        self.loss = Loss([(c.W, c.H) for c in self.v.cams], dev)
        P, M = state.P, state.M
        self.g = dict(means3D=torch.zeros(P, 3, device=dev), sh=torch.zeros(P, M, 3, device=dev),
                      opacity=torch.zeros(P, 1, device=dev), scales=torch.zeros(P, 3, device=dev),
                      rotations=torch.zeros(P, 4, device=dev))
        self.dL = [torch.empty(3, c.H, c.W, device=dev) for c in self.v.cams]

    def step(self):
        st = self.st
        st.flag.zero_()
        for t in self.g.values():
            t.zero_()
        e = torch.empty(0, device=st.xyz.device)
        self.loss.sums.zero_()
        for cam, y, dl in zip(self.v.cams, self.v.targets, self.dL):
            out = rasterize_gaussians(self.bg, st.xyz, e, st.opac, st.scale, st.rot, 1.0, e, cam.viewmatrix,
                                      cam.projmatrix, cam.tanfovx, cam.tanfovy, cam.H, cam.W, st.shs, 3, cam.campos,
                                      False, True, False, 0.2, 0.2, 0.05, 0.7, False)
            K, color, _pid, _pwp, _pw, radii, geom, binning, img, _st = out
            call("fgs_loss_l1_ssim", cam.W, cam.H, _p(color), _p(y), _p(dl), 0.8 / self.loss.n_l1,
                 0.2 / self.loss.n_ssim, _p(self.loss.sums), _p(self.loss.scratch), _s())
            g = rasterize_gaussians_backward(self.bg, st.xyz, radii, e, st.scale, st.rot, 1.0, e, cam.viewmatrix,
                                             cam.projmatrix, cam.tanfovx, cam.tanfovy, dl, st.shs, 3, cam.campos,
                                             geom, K, binning, img, False)
            dmean2D, _dcol, dopac, dmean3D, _dcov, dsh, dscale, drot = g
            self.g["means3D"] += dmean3D
            self.g["sh"] += dsh
            self.g["opacity"] += dopac
            self.g["scales"] += dscale
            self.g["rotations"] += drot
            call("fgs_densify_dense", st.P, _p(radii), _p(dmean2D), _p(st.grad_sum), _p(st.vis_count), _p(st.flag),
                 _s())
        st.adam(self.g["means3D"], self.g["sh"], self.g["opacity"], self.g["scales"], self.g["rotations"])
