"""Batched multi-view rasterization with CUDA-graph capture.

Renders V cameras of one Gaussian set per step: forward for every view, then
backward with the views' gradients summed into shared dense buffers.  The
per-view front end keeps its pair counts on the device and compositing is
one persistent launch per direction over all views' tiles (C ABI
fgs_batch_*), so a whole forward + backward step has no host
synchronisation and is captured once into two CUDA graphs (forward, backward)
and replayed; `step()` can mark the end of the forward with an event and hold
the backward on another, so callers overlap image downloads and gradient
uploads with compute.

Pair capacities are planned from the views' exact pair counts (one plain
preprocess per view) with headroom; a replay that overflows a capacity is
reported by `check()` and re-planned with `replan()`.
"""
import ctypes as C

import torch

from . import _lib
from ._C import BACKWARD_MODES, _args
from ._lib import call, lib


class _ViewArgs(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("tan_fovx", C.c_float), ("tan_fovy", C.c_float),
                ("viewmatrix", C.c_void_p), ("projmatrix", C.c_void_p), ("campos", C.c_void_p),
                ("pair_capacity", C.c_longlong), ("out_color", C.c_void_p), ("out_radii", C.c_void_p),
                ("dL_dout_color", C.c_void_p)]


def _L():
    return lib()


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return None if t is None or t.numel() == 0 else C.c_void_p(t.data_ptr())


class Camera:
    """One view: image size, tan of the half field of view, 4x4 column-major matrices, centre (device tensors)."""

    def __init__(self, width, height, tanfovx, tanfovy, viewmatrix, projmatrix, campos):
        self.W, self.H = int(width), int(height)
        self.tanfovx, self.tanfovy = float(tanfovx), float(tanfovy)
        self.viewmatrix, self.projmatrix, self.campos = viewmatrix, projmatrix, campos


class BatchedRasterizer:
    """Forward + backward of V views per step, sharing one set of Gaussians."""

    def __init__(self, means3D, opacities, scales, rotations, cameras, shs=None, sh_degree=0, colors_precomp=None,
                 bg=None, use_filter=True, ogfs=(0.2, 0.2, 0.05, 0.7), filter3d_scale=0.0,
                 backward_mode="ref_compat", headroom=1.15, graph=True, full_outputs=False):
        dev = means3D.device
        self.dev = dev
        self.P = int(means3D.shape[0])
        self.means3D, self.opacities = means3D.contiguous(), opacities.contiguous()
        self.scales, self.rotations = scales.contiguous(), rotations.contiguous()
        self.shs = shs.contiguous() if shs is not None else None
        self.colors = colors_precomp.contiguous() if colors_precomp is not None else None
        self.sh_degree = int(sh_degree)
        self.bg = bg if bg is not None else torch.zeros(3, device=dev)
        self.use_filter, self.ogfs, self.filter3d = bool(use_filter), tuple(ogfs), float(filter3d_scale)
        self.mode = BACKWARD_MODES[backward_mode]
        self.cams = list(cameras)
        self.V = len(self.cams)
        self.headroom = float(headroom)
        self.images = [torch.empty(3, c.H, c.W, device=dev) for c in self.cams]
        self.dL = [torch.zeros(3, c.H, c.W, device=dev) for c in self.cams]
        self.radii = [torch.empty(self.P, dtype=torch.int32, device=dev) for _ in self.cams]
        # the rest of the reference's forward outputs per view (point_id, point_weight_pixel, point_weight)
        self.full_outputs = bool(full_outputs)
        if self.full_outputs:
            self.point_id = [torch.empty(c.H, c.W, dtype=torch.int32, device=dev) for c in self.cams]
            self.point_weight_pixel = [torch.empty(c.H, c.W, device=dev) for c in self.cams]
            self.point_weight = [torch.empty(self.P, device=dev) for _ in self.cams]
        M = int(self.shs.shape[1]) if self.shs is not None else 0
        self.grad = dict(means3D=torch.zeros(self.P, 3, device=dev), opacity=torch.zeros(self.P, 1, device=dev),
                         sh=torch.zeros(self.P, M, 3, device=dev), scales=torch.zeros(self.P, 3, device=dev),
                         rotations=torch.zeros(self.P, 4, device=dev))
        self.use_graph = graph
        self.handle = None
        self.graph = None      # (forward graph, backward graph) once captured
        self.capacity = self._plan_capacity()
        self._build()

    # ------------------------------------------------------------------ planning
    def _shared_args(self):
        M = int(self.shs.shape[1]) if self.shs is not None else 0
        e = None
        return _args(self.P, self.sh_degree, M, 16, 16, self.bg, self.means3D, self.shs if self.colors is None else e,
                     self.colors, self.opacities, self.scales, 1.0, self.rotations, e, self.cams[0].viewmatrix,
                     self.cams[0].projmatrix, self.cams[0].campos, 1.0, 1.0, False, self.use_filter, *self.ogfs, False,
                     self.filter3d)

    def _plan_capacity(self):
        """Exact pair counts of every view from one preprocess each, plus headroom."""
        L = lib()
        caps = []
        geom = torch.empty(int(L.fgs_geom_bytes(self.P)), dtype=torch.uint8, device=self.dev)
        for c in self.cams:
            a = self._shared_args()
            a.width, a.height, a.tan_fovx, a.tan_fovy = c.W, c.H, c.tanfovx, c.tanfovy
            a.viewmatrix, a.projmatrix, a.campos = _p(c.viewmatrix), _p(c.projmatrix), _p(c.campos)
            img = torch.empty(int(L.fgs_image_bytes(c.W, c.H)), dtype=torch.uint8, device=self.dev)
            K = C.c_longlong(0)
            call("fgs_forward_preprocess", C.byref(a), _p(geom), _p(img), None, C.byref(K), _s())
            caps.append(int(K.value * self.headroom) + 4096)
        return caps

    def _build(self):
        L = _L()
        if self.handle:
            L.fgs_batch_destroy(self.handle)
            self.handle = None
        self.graph = None
        va = (_ViewArgs * self.V)()
        for i, c in enumerate(self.cams):
            va[i] = _ViewArgs(c.W, c.H, c.tanfovx, c.tanfovy, _p(c.viewmatrix), _p(c.projmatrix), _p(c.campos),
                              self.capacity[i], _p(self.images[i]), _p(self.radii[i]), _p(self.dL[i]))
        self._va = va
        nbytes = int(L.fgs_batch_workspace_bytes(self.P, self.V, C.cast(va, C.c_void_p)))
        if nbytes == 0:
            raise RuntimeError("fgs_batch_workspace_bytes rejected the views")
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=self.dev)
        st = C.c_int(0)
        self._shared = self._shared_args()
        g = self.grad
        h = L.fgs_batch_create(C.byref(self._shared), self.V, C.cast(va, C.c_void_p), _p(self.workspace), nbytes,
                               self.mode, _p(g["means3D"]), _p(g["opacity"]), _p(g["sh"]) if g["sh"].numel() else None,
                               _p(g["scales"]), _p(g["rotations"]), C.byref(st), _s())
        if not h:
            _lib.check(st.value, "fgs_batch_create")
        self.handle = h
        if self.full_outputs:
            n = self.V
            ids = (C.c_int * n)(*range(n))
            pid = (C.c_void_p * n)(*[t.data_ptr() for t in self.point_id])
            pwp = (C.c_void_p * n)(*[t.data_ptr() for t in self.point_weight_pixel])
            pw = (C.c_void_p * n)(*[t.data_ptr() for t in self.point_weight])
            _lib.check(L.fgs_batch_set_view_outputs(h, n, C.cast(ids, C.c_void_p), C.cast(pid, C.c_void_p),
                                                    C.cast(pwp, C.c_void_p), C.cast(pw, C.c_void_p), _s()),
                       "fgs_batch_set_view_outputs")

    def _capture(self):
        L = _L()
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):           # warm-up outside capture (lazy module loading)
            self._enqueue(L, s)
        torch.cuda.current_stream(self.dev).wait_stream(s)
        torch.cuda.synchronize(self.dev)
        gf, gb = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
        ptr = C.c_void_p(s.cuda_stream)
        with torch.cuda.graph(gf, stream=s):
            _lib.check(L.fgs_batch_forward(self.handle, ptr), "fgs_batch_forward")
        with torch.cuda.graph(gb, stream=s):
            _lib.check(L.fgs_batch_backward(self.handle, ptr), "fgs_batch_backward")
        self.graph = (gf, gb)

    def _enqueue(self, L, s):
        ptr = C.c_void_p(s.cuda_stream)
        _lib.check(L.fgs_batch_forward(self.handle, ptr), "fgs_batch_forward")
        _lib.check(L.fgs_batch_backward(self.handle, ptr), "fgs_batch_backward")

    # ------------------------------------------------------------------ use
    def step(self, forward_done=None, backward_ready=None):
        """One forward + backward of all views (graph replays when enabled), on the current stream.
        forward_done (a torch.cuda.Event) is recorded once the images are final, so that a copy
        stream can download them while the backward runs; the backward waits for backward_ready
        when given (e.g. the upload of the upstream gradients, which the forward does not read)."""
        s = torch.cuda.current_stream(self.dev)
        L = _L()
        if self.use_graph:
            if self.graph is None:
                self._capture()
            self.graph[0].replay()
        else:
            _lib.check(L.fgs_batch_forward(self.handle, C.c_void_p(s.cuda_stream)), "fgs_batch_forward")
        if forward_done is not None:
            forward_done.record(s)
        if backward_ready is not None:
            s.wait_event(backward_ready)
        if self.use_graph:
            self.graph[1].replay()
        else:
            _lib.check(L.fgs_batch_backward(self.handle, C.c_void_p(s.cuda_stream)), "fgs_batch_backward")

    def forward(self):
        _lib.check(_L().fgs_batch_forward(self.handle, _s()), "fgs_batch_forward")
        return self.images

    def backward(self):
        _lib.check(_L().fgs_batch_backward(self.handle, _s()), "fgs_batch_backward")
        return self.grad

    def set_io(self, view, image, dL=None):
        """Point view `view` at another image buffer (and upstream gradient) for the steps that follow
        on the current stream; a captured graph follows without re-capture (double-buffered I/O)."""
        self.set_io_many([view], [image], [dL])

    def set_io_many(self, views, images, dLs=None):
        dLs = dLs if dLs is not None else [None] * len(views)
        for v, img, d in zip(views, images, dLs):
            c = self.cams[v]
            for t in (img, d):
                if t is not None and (tuple(t.shape) != (3, c.H, c.W) or t.dtype != torch.float32 or
                                      not t.is_contiguous() or t.device != self.dev):
                    raise ValueError(f"view {v}: expected a contiguous float32 [3,{c.H},{c.W}] tensor on {self.dev}")
        n = len(views)
        ids = (C.c_int * n)(*[int(v) for v in views])
        outs = (C.c_void_p * n)(*[t.data_ptr() for t in images])
        dls = (C.c_void_p * n)(*[(t.data_ptr() if t is not None else None) for t in dLs])
        _lib.check(_L().fgs_batch_set_view_io(self.handle, n, C.cast(ids, C.c_void_p), C.cast(outs, C.c_void_p),
                                              C.cast(dls, C.c_void_p), _s()), "fgs_batch_set_view_io")
        for v, img, d in zip(views, images, dLs):
            self.images[v] = img
            if d is not None:
                self.dL[v] = d

    def pair_counts(self):
        out = (C.c_longlong * self.V)()
        _lib.check(_L().fgs_batch_pair_counts(self.handle, C.cast(out, C.c_void_p), _s()), "fgs_batch_pair_counts")
        return list(out)

    def check(self):
        """Synchronise; raise FgsError on a device-side error (FGS_ERR_OVERFLOW: a capacity was exceeded)."""
        _lib.check(_L().fgs_batch_check(self.handle, _s()), "fgs_batch_check")

    def replan(self):
        self.capacity = self._plan_capacity()
        self._build()

    def __del__(self):
        try:
            if self.handle:
                _L().fgs_batch_destroy(self.handle)
        except Exception:
            pass
