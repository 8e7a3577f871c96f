"""Learned Poisson preconditioner inside flexible CG (no counterpart in the reference).

Network (4 levels, 32 channels, 3x3 convolutions, BF16 weights and activations,
FP32 accumulation, 65,025 parameters):

    a0  = relu(conv 1->32 (r / ||r||))                      level 0 (CUDA cores)
    a0b = relu(conv 32->32 (a0))                            level 0 (tensor cores)
    a1  = relu(conv 32->32 (pool a0b))                      level 1
    a2  = relu(conv 32->32 (pool a1))                       level 2
    a3  = relu(conv 32->32 (pool a2))                       level 3
    d2  = relu(conv 32->32 (up a3 + a2))                    level 2
    d1  = relu(conv 32->32 (up d2 + a1))                    level 1
    d0  = relu(conv 32->32 (up d1 + a0b))                   level 0
    out = conv 32->1 (d0)                                   level 0 (CUDA cores)

Every layer output is multiplied by the fluid mask of its level. The 32->32
layers run on tcgen05 (``cfd2d_lpc_conv32``); the 1-channel layers, pooling,
upsampling and the whole backward pass are hand-written CUDA-core kernels of the
same library (``net_forward`` / ``net_backward``); the optimiser (Adam) is
PyTorch's, on FP32 master weights.

The network works on the dimensionless operator Ah = h^2 A (h^2 = 2 / (1/dx^2 +
1/dy^2)), so one set of weights serves every grid spacing: for a residual r it
approximates Ah^-1 (r / ||r||). Training minimises the energy-norm error of that
approximation, (e - o)^T Ah (e - o) with e = Ah^-1 r_hat, i.e. o^T Ah o - 2 o.r_hat
(the constant e^T Ah e dropped), over residuals harvested from the plain solver's
own iterations. Inside flexible CG (Notay's form, one stored direction) the preconditioner is
M(r) = h^2 ||r|| net(r / ||r||) + omega D^-1 r; the loop runs on the device inside
one CUDA graph (a WHILE node) and falls back to the plain Jacobi-PCG from the
current iterate when it stalls.
"""

from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _lib

CH = 32
LAYERS = [  # name, cin, cout, level, relu
    ("a0", 1, CH, 0, True), ("a0b", CH, CH, 0, True), ("a1", CH, CH, 1, True), ("a2", CH, CH, 2, True),
    ("a3", CH, CH, 3, True), ("d2", CH, CH, 2, True), ("d1", CH, CH, 1, True), ("d0", CH, CH, 0, True),
    ("out", CH, 1, 0, False),
]
NLEVELS = 4


def _t():
    return _lib.torch()


def level_shapes(H, W):
    shapes = [(H, W)]
    for _ in range(NLEVELS - 1):
        h, w = shapes[-1]
        shapes.append(((h + 1) // 2, (w + 1) // 2))
    return shapes


class LPCNet:
    """Weights (FP32 masters) and the packed BF16 tensor-core images of the 32->32 layers.

    With ``bias=False`` (the default) the biases stay zero and are not trained: the
    network is then positively homogeneous, net(a r) = a net(r) for a > 0, and with
    sign-flipped training samples close to odd, as a preconditioner inside CG must
    be (a trained bias adds a fixed field to every preconditioned residual, and the
    flexible CG stalls on it)."""

    def __init__(self, seed: int = 0, bias: bool = False):
        t = _t()
        self.bias = bias
        g = t.Generator().manual_seed(seed)
        self.w, self.b = {}, {}
        for name, cin, cout, _lvl, relu in LAYERS:
            # uniform in +-1/sqrt(fan_in), the output layer ten times smaller: the
            # network starts close to zero and the Jacobi term leads the first steps
            bound = 1.0 / math.sqrt(cin * 9)
            if not relu:
                bound *= 0.1
            self.w[name] = ((t.rand((cout, cin, 3, 3), generator=g) * 2.0 - 1.0) * bound).to(_lib.device())
            self.b[name] = t.zeros(cout, device=_lib.device())
        self._images = {}
        self._wq = {}
        self.repack()

    @property
    def n_params(self) -> int:
        return sum(v.numel() for v in self.w.values()) + sum(v.numel() for v in self.b.values())

    def parameters(self):
        out = []
        for name, *_ in LAYERS:
            out += [self.w[name], self.b[name]] if self.bias else [self.w[name]]
        return out

    def repack(self):
        """BF16 weights: round the masters and pack the tensor-core images. The
        images and the rounded CUDA-core weights are updated in place, so graphs
        captured with them stay valid."""
        t = _t()
        L = _lib.lib()
        nbytes = int(L.cfd2d_lpc_w32_bytes())
        for name, cin, cout, _lvl, _relu in LAYERS:
            if not (cin == CH and cout == CH):
                q = self.wq(name)
                if name in self._wq:
                    self._wq[name].copy_(q)
                else:
                    self._wq[name] = q
            if cin == CH and cout == CH:
                img = self._images.get(name)
                if img is None:
                    img = t.zeros(nbytes // 2, dtype=t.bfloat16, device=_lib.device())
                    self._images[name] = img
                w = self.w[name].detach().float().contiguous()
                _lib.check(L.cfd2d_lpc_pack_w32(_lib.ptr(w), _lib.ptr(img), _lib.stream_ptr()), "pack_w32")

    def wq(self, name):
        """The BF16-rounded weights the kernels use, as FP32 (for the CUDA-core layers)."""
        return self.w[name].detach().to(_t().bfloat16).float().contiguous()

    def state_dict(self):
        return {f"{k}.w": v.detach().cpu() for k, v in self.w.items()} | \
               {f"{k}.b": v.detach().cpu() for k, v in self.b.items()}

    def load_state_dict(self, d):
        self.bias = any(float(d[f"{name}.b"].abs().max()) > 0.0 for name, *_ in LAYERS)
        for name, *_ in LAYERS:
            self.w[name].copy_(d[f"{name}.w"].to(self.w[name].device))
            self.b[name].copy_(d[f"{name}.b"].to(self.b[name].device))
        self.repack()


def _take_net_error(ws) -> bool:
    """Read and clear the error flag the tensor-core convolutions set when their bounded
    wait for the MMAs gives up (the flag lives in the workspace)."""
    if int(ws.err.item()) == 0:
        return False
    ws.err.zero_()
    return True


class Workspace:
    """Activation buffers of one grid size (reused across applications)."""

    def __init__(self, H: int, W: int, mask):
        t = _t()
        dev = _lib.device()
        L = _lib.lib()
        self.H, self.W = H, W
        self.shapes = level_shapes(H, W)
        self.masks = [t.zeros(s, dtype=t.uint8, device=dev) for s in self.shapes]
        self.mask_src = None
        self.set_mask(mask)
        act = lambda lvl: t.zeros(self.shapes[lvl] + (CH,), dtype=t.bfloat16, device=dev)  # noqa: E731
        self.a = {name: act(lvl) for name, cin, cout, lvl, _ in LAYERS if cout == CH}
        self.pool = {lvl: act(lvl) for lvl in (1, 2, 3)}
        self.up = {lvl: act(lvl) for lvl in (0, 1, 2)}
        self.out = t.zeros((H, W), dtype=t.float32, device=dev)
        self.err = t.zeros(1, dtype=t.int32, device=dev)


def _ws_set_mask(self, mask):
    """Fluid mask of level 0 (H, W) and its pooled masks (any child fluid)."""
    t = _t()
    L = _lib.lib()
    m0 = mask if isinstance(mask, t.Tensor) else _lib.to_dev(np.asarray(mask, dtype=np.uint8))
    self.masks[0].copy_(m0.reshape(self.H, self.W).to(t.uint8))
    for lvl in range(1, NLEVELS):
        h, w = self.shapes[lvl - 1]
        _lib.check(L.cfd2d_lpc_pool_mask(_lib.ptr(self.masks[lvl - 1]), _lib.ptr(self.masks[lvl]), h, w,
                                         _lib.stream_ptr()), "pool_mask")
    self.mask_src = mask


Workspace.set_mask = _ws_set_mask


def net_forward(net: LPCNet, ws: Workspace, x_in):
    """out = net(x_in) on the device (x_in: FP32 (H, W)); activations stay in ``ws``."""
    L = _lib.lib()
    s = _lib.stream_ptr()
    P = _lib.ptr
    sh = ws.shapes

    def conv32(name, src, lvl, skip=None):
        h, w = sh[lvl]
        rc = L.cfd2d_lpc_conv32(P(src), P(net._images[name]), P(net.b[name]), P(skip), P(ws.masks[lvl]),
                                P(ws.a[name]), h, w, 1, P(ws.err), s)
        _lib.check(rc, "lpc_conv32")

    H, W = sh[0]
    _lib.check(L.cfd2d_lpc_conv(1, CH, P(x_in), 0, P(net._wq["a0"]), P(net.b["a0"]), P(ws.masks[0]), P(ws.a["a0"]),
                                1, H, W, 1, 0, s), "lpc_conv a0")
    conv32("a0b", ws.a["a0"], 0)
    prev = ws.a["a0b"]
    for lvl, name in ((1, "a1"), (2, "a2"), (3, "a3")):
        h, w = sh[lvl - 1]
        _lib.check(L.cfd2d_lpc_pool2(P(prev), P(ws.pool[lvl]), h, w, s), "pool2")
        conv32(name, ws.pool[lvl], lvl)
        prev = ws.a[name]
    for lvl, name, skip in ((2, "d2", "a2"), (1, "d1", "a1"), (0, "d0", "a0b")):
        h, w = sh[lvl]
        _lib.check(L.cfd2d_lpc_upadd(P(prev), P(ws.a[skip]), P(ws.up[lvl]), h, w, s), "upadd")
        conv32(name, ws.up[lvl], lvl)
        prev = ws.a[name]
    _lib.check(L.cfd2d_lpc_conv(CH, 1, P(prev), 1, P(net._wq["out"]), P(net.b["out"]), P(ws.masks[0]), P(ws.out),
                                0, H, W, 0, 0, s), "lpc_conv out")
    return ws.out


def net_backward(net: LPCNet, ws: Workspace, x_in, dout):
    """Gradients of sum(out * dout) w.r.t. every weight and bias (FP32), from the
    activations left in ``ws`` by net_forward(x_in)."""
    t = _t()
    L = _lib.lib()
    s = _lib.stream_ptr()
    P = _lib.ptr
    sh = ws.shapes
    dev = _lib.device()
    grads = {}

    def zeros(lvl, ch=CH):
        return t.zeros(sh[lvl] + (ch,), dtype=t.float32, device=dev)

    def dw(name, cin, cout, x, xbf, g, lvl):
        h, w = sh[lvl]
        ppb = 256
        part = t.empty(int(L.cfd2d_lpc_conv_dw_partial_floats(cin, cout, h, w, ppb)), dtype=t.float32, device=dev)
        out = t.empty(cout * cin * 9 + cout, dtype=t.float32, device=dev)
        _lib.check(L.cfd2d_lpc_conv_dw(cin, cout, P(x), xbf, P(g), h, w, ppb, P(part), P(out), s), "conv_dw")
        grads[name] = (out[:cout * cin * 9].view(cout, cin, 3, 3), out[cout * cin * 9:])

    def relu_g(dy, y, lvl, relu=True, ch=CH):
        h, w = sh[lvl]
        g = t.empty_like(dy)
        _lib.check(L.cfd2d_lpc_relu_bwd(P(dy), P(y), P(ws.masks[lvl]), P(g), h * w, ch, int(relu), s), "relu_bwd")
        return g

    def conv_t(name, cin_f, cout_f, g, lvl):
        # data gradient of a forward layer (cin_f -> cout_f): adjoint conv of g (cout_f channels)
        h, w = sh[lvl]
        dx = zeros(lvl, cin_f)
        _lib.check(L.cfd2d_lpc_conv(cout_f, cin_f, P(g), 0, P(net.wq(name)), None, None, P(dx), 0, h, w, 0, 1, s),
                   "conv transposed")
        return dx

    H, W = sh[0]
    g = relu_g(dout.contiguous(), None, 0, relu=False, ch=1)
    dw("out", CH, 1, ws.a["d0"], 1, g, 0)
    dd = conv_t("out", CH, 1, g, 0)
    skip_grad = {}
    for lvl, name, skip, inp in ((0, "d0", "a0b", ws.up[0]), (1, "d1", "a1", ws.up[1]), (2, "d2", "a2", ws.up[2])):
        g = relu_g(dd, ws.a[name], lvl)
        dw(name, CH, CH, inp, 1, g, lvl)
        du = conv_t(name, CH, CH, g, lvl)
        skip_grad[skip] = du
        h, w = sh[lvl]
        dc = zeros(lvl + 1)
        _lib.check(L.cfd2d_lpc_upadd_bwd(P(du), P(dc), h, w, s), "upadd_bwd")
        dd = dc
    # encoder, deepest first: da3 = dd
    da = dd
    for lvl, name in ((3, "a3"), (2, "a2"), (1, "a1")):
        g = relu_g(da, ws.a[name], lvl)
        dw(name, CH, CH, ws.pool[lvl], 1, g, lvl)
        dp = conv_t(name, CH, CH, g, lvl)
        below = {3: "a2", 2: "a1", 1: "a0b"}[lvl]
        nxt = skip_grad[below].clone()
        h, w = sh[lvl - 1]
        _lib.check(L.cfd2d_lpc_pool_bwd(P(dp), P(nxt), h, w, s), "pool_bwd")
        da = nxt
    g = relu_g(da, ws.a["a0b"], 0)
    dw("a0b", CH, CH, ws.a["a0"], 1, g, 0)
    da0 = conv_t("a0b", CH, CH, g, 0)
    g = relu_g(da0, ws.a["a0"], 0)
    dw("a0", 1, CH, x_in.contiguous(), 0, g, 0)
    return grads


def torch_reference_forward(net: LPCNet, x_in, masks):
    """The same network in PyTorch (CPU, FP32 on BF16-rounded weights and activations):
    the reference computation for the CUDA kernels and their gradients."""
    t = _t()
    F = t.nn.functional

    def bf(a):
        return a.to(t.bfloat16).float()

    def conv(name, a, relu, lvl, round_out=True):
        bias = net.b[name]
        bias = bias.detach().cpu() if bias.is_cuda else bias
        y = F.conv2d(a, net.wq(name).cpu(), bias, padding=1)
        if relu:
            y = t.relu(y)
        y = y * masks[lvl]
        return bf(y) if round_out else y

    def pool(a):
        # mean over the in-range children of each coarse cell
        h, w = a.shape[-2:]
        ap = F.pad(a, (0, w % 2, 0, h % 2))
        cnt = F.avg_pool2d(F.pad(t.ones((1, 1, h, w)), (0, w % 2, 0, h % 2)), 2) * 4
        return bf(F.avg_pool2d(ap, 2) * 4 / cnt)

    def up(a, skip):
        h, w = skip.shape[-2:]
        u = a.repeat_interleave(2, -2).repeat_interleave(2, -1)[..., :h, :w]
        return bf(u + skip)

    x = x_in.cpu().float()[None, None]
    a0 = conv("a0", x, True, 0)
    a0b = conv("a0b", a0, True, 0)
    a1 = conv("a1", pool(a0b), True, 1)
    a2 = conv("a2", pool(a1), True, 2)
    a3 = conv("a3", pool(a2), True, 3)
    d2 = conv("d2", up(a3, a2), True, 2)
    d1 = conv("d1", up(d2, a1), True, 1)
    d0 = conv("d0", up(d1, a0b), True, 0)
    return conv("out", d0, False, 0, round_out=False)[0, 0]


# ------------------------------------------------------------------ flexible CG
def h2_of(pressure) -> float:
    """h^2 of the dimensionless operator: 2 / (1/dx^2 + 1/dy^2)."""
    return 2.0 / (pressure.dx2 + pressure.dy2)


class LearnedPCG:
    """Flexible CG with the learned preconditioner for one PressureSolver's operator.

    solve(rhs) mirrors PressureSolver.solve on domains with an outflow (Dirichlet)
    boundary: same operator, warm start (the solver's x0, updated in place), stop
    test ||r|| < tol ||b||. If the residual fails to fall by ``stall_factor`` over
    ``stall_window`` iterations, the solve continues with the plain Jacobi-PCG from
    the current iterate. The window is long on purpose: the residual norm of a
    flexible CG can sit on a plateau for tens of iterations while the error keeps
    falling in the energy norm.
    """

    def __init__(self, pressure, net: LPCNet, omega: float = 0.5, stall_window: int = 200,
                 stall_factor: float = 0.9, maxiter: int = 3000):
        t = _t()
        if pressure.neumann_components:
            raise ValueError("the learned preconditioner path needs an outflow (Dirichlet) boundary")
        self.ps, self.net = pressure, net
        self.omega, self.stall_window, self.stall_factor = omega, stall_window, stall_factor
        self.maxiter = maxiter
        self.h2 = h2_of(pressure)
        g = pressure.grid
        self.nx, self.ny = g.nx, g.ny
        n = self.nx * self.ny
        dev = _lib.device()
        z = lambda: t.zeros(n, dtype=t.float64, device=dev)  # noqa: E731
        self.b, self.r, self.p, self.q, self.z = z(), z(), z(), z(), z()
        self.rhs_buf = z()
        self.net_in = t.zeros((self.nx, self.ny), dtype=t.float32, device=dev)
        self.partial = t.zeros(int(_lib.lib().cfd2d_fcg_partial_doubles(n)), dtype=t.float64, device=dev)
        self.scal = t.zeros(C.sizeof(_lib.FcgScalars) // 8, dtype=t.float64, device=dev)
        self.mask = pressure._d_nbr.view(self.nx, self.ny) >= 0x80
        self.mask_u8 = self.mask.to(t.uint8).contiguous()
        self.ws = Workspace(self.nx, self.ny, self.mask_u8)
        self.hist = t.zeros(maxiter + 1, dtype=t.float64, device=dev)
        self.ctl = t.zeros(C.sizeof(_lib.FcgControl), dtype=t.uint8, device=dev)
        self._graphs = {}
        self.iters_out = 0  # device address that also receives the iteration count (0: none)
        self.last_iterations = 0
        self.last_total_iterations = 0
        self.last_fallback = False
        self.last_reason = 0
        self.last_net_error = False
        self.history = []

    # ---------------------------------------------------------------- pieces
    def _scalars(self):
        raw = self.scal.cpu().numpy().tobytes()
        return _lib.FcgScalars.from_buffer_copy(raw)

    def precondition(self):
        L = _lib.lib()
        s = _lib.stream_ptr()
        P = _lib.ptr
        n = self.nx * self.ny
        _lib.check(L.cfd2d_fcg_net_in(n, P(self.r), P(self.scal), P(self.mask_u8), P(self.net_in), s), "net_in")
        out = net_forward(self.net, self.ws, self.net_in)
        _lib.check(L.cfd2d_fcg_net_out(n, P(out), P(self.r), P(self.ps._d_dinv), P(self.mask_u8), P(self.scal),
                                       self.h2, self.omega, P(self.z), s), "net_out")

    def _init(self, rhs=None, F=None, G=None, dx=1.0, dy=1.0, dt_ptr=None):
        P = _lib.ptr
        _lib.check(_lib.lib().cfd2d_fcg_init(C.byref(self.ps.op), P(F), P(G), P(rhs), dx, dy, dt_ptr, P(self.b),
                                             P(self.ps._d_x0.view(-1)), P(self.r), P(self.p), P(self.scal),
                                             P(self.partial), _lib.stream_ptr()), "fcg_init")

    def _body(self, handle: int):
        """One iteration: z = M(r), beta = -(z . A p_old) / (p_old . A p_old), p = z + beta p,
        q = A p, alpha = (p . r) / (p . q), x and r update, gate."""
        L = _lib.lib()
        s = _lib.stream_ptr()
        P = _lib.ptr
        n = self.nx * self.ny
        op = C.byref(self.ps.op)
        self.precondition()
        _lib.check(L.cfd2d_fcg_zr(n, P(self.z), P(self.q), -1, P(self.scal), P(self.partial), s), "zr")
        _lib.check(L.cfd2d_fcg_dir(n, P(self.z), P(self.p), P(self.scal), s), "dir")
        _lib.check(L.cfd2d_fcg_pq(op, P(self.p), P(self.q), P(self.r), P(self.scal), P(self.partial), s), "pq")
        _lib.check(L.cfd2d_fcg_update(n, P(self.ps._d_x0.view(-1)), P(self.r), P(self.p), P(self.q), P(self.scal),
                                      P(self.partial), s), "update")
        _lib.check(L.cfd2d_fcg_gate(P(self.scal), P(self.ctl), handle, s), "gate")

    def _set_control(self, tol):
        t = _t()
        c = _lib.FcgControl(rtol=tol, stall_factor=self.stall_factor, stall_window=self.stall_window,
                            maxiter=self.maxiter, reason=0, iters=0, calls=0, pad=0, hist=self.hist.data_ptr(),
                            iters_out=self.iters_out or None)
        host = t.frombuffer(bytearray(bytes(c)), dtype=t.uint8)
        self.ctl.copy_(host)

    def _control(self):
        return _lib.FcgControl.from_buffer_copy(self.ctl.cpu().numpy().tobytes())

    # ---------------------------------------------------------------- solves
    def solve_into_x_host(self, rhs=None, F=None, G=None, dx=1.0, dy=1.0, dt_ptr=None, tol=None):
        """The same iteration driven from the host (one launch sequence and one scalar
        read per iteration); kept as the reference for the graph-driven loop."""
        tol = self.ps.rtol if tol is None else tol
        self._set_control(tol)
        self._init(rhs, F, G, dx, dy, dt_ptr)
        _lib.check(_lib.lib().cfd2d_fcg_gate(_lib.ptr(self.scal), _lib.ptr(self.ctl), 0, _lib.stream_ptr()), "gate")
        while self._control().reason == _lib.FCG_RUNNING:
            self._body(0)
        return self._finish()

    def _graph(self, key, rhs=None, F=None, G=None, dx=1.0, dy=1.0, dt_ptr=None):
        """Graph of one whole solve: init, gate, WHILE(body), zero-rhs fix."""
        g = self._graphs.get(key)
        if g is not None:
            return g
        t = _t()
        L = _lib.lib()
        main, body = t.cuda.Stream(), t.cuda.Stream()
        main.wait_stream(t.cuda.current_stream())
        n = self.nx * self.ny
        graph = C.c_void_p()
        with t.cuda.stream(main):
            mp = C.c_void_p(main.cuda_stream)
            _lib.check(L.cfd2d_capture_begin(mp), "capture_begin")
            try:
                self._init(rhs, F, G, dx, dy, dt_ptr)
                h = C.c_uint64()
                _lib.check(L.cfd2d_capture_condition(mp, C.byref(h)), "capture_condition")
                _lib.check(L.cfd2d_fcg_gate(_lib.ptr(self.scal), _lib.ptr(self.ctl), h.value, mp), "gate")
                _lib.check(L.cfd2d_capture_while_begin(mp, C.c_void_p(body.cuda_stream), h.value), "while_begin")
                with t.cuda.stream(body):
                    self._body(h.value)
                _lib.check(L.cfd2d_capture_while_end(C.c_void_p(body.cuda_stream)), "while_end")
                _lib.check(L.cfd2d_fcg_zero_rhs(n, _lib.ptr(self.b), _lib.ptr(self.ps._d_x0.view(-1)),
                                                _lib.ptr(self.scal), mp), "zero_rhs")
                _lib.check(L.cfd2d_capture_end(mp, C.byref(graph)), "capture_end")
            except Exception:
                L.cfd2d_capture_abort(C.c_void_p(body.cuda_stream))
                L.cfd2d_capture_abort(mp)
                raise
        self._graphs[key] = graph
        return graph

    def solve_into_x(self, rhs=None, F=None, G=None, dx=1.0, dy=1.0, dt_ptr=None, tol=None, key=None):
        """Run the graph-driven FCG on x = pressure x0 (in place). Returns the iteration count."""
        tol = self.ps.rtol if tol is None else tol
        self._set_control(tol)
        graph = self._graph(key if key is not None else ("rhs", _lib.ptr(rhs).value if rhs is not None else 0),
                            rhs, F, G, dx, dy, dt_ptr)
        _lib.check(_lib.lib().cfd2d_graph_launch(graph, _lib.stream_ptr()), "graph_launch")
        return self._finish()

    def _finish(self):
        c = self._control()
        self.last_net_error = _take_net_error(self.ws)
        if self.last_net_error:
            import warnings

            warnings.warn("learned preconditioner: a tensor-core convolution gave up waiting for its MMAs; "
                          "its output rows were zeroed (the solve still stops on the true residual test, "
                          "and the plain solver finishes it if the flexible CG did not converge)")
        self.last_reason = c.reason
        self.last_iterations = c.iters
        self.last_fallback = c.reason == _lib.FCG_STALLED
        self.history = self.hist[: c.iters + 1].cpu().numpy().tolist()
        if c.reason == _lib.FCG_NONFINITE:
            raise FloatingPointError("flexible CG produced a non-finite residual")
        return c.iters

    def solve(self, rhs, graph: bool = True):
        """Lap(p) = rhs (same conventions as PressureSolver.solve); host or device rhs."""
        t = _t()
        host = not isinstance(rhs, t.Tensor)
        self.rhs_buf.copy_(_lib.to_dev(rhs, t.float64).reshape(-1))
        if graph:
            self.solve_into_x(rhs=self.rhs_buf)
        else:
            self.solve_into_x_host(rhs=self.rhs_buf)
        extra = 0
        if self.last_reason in (_lib.FCG_STALLED, _lib.FCG_MAXITER):
            # continue with the plain Jacobi-PCG from the current iterate
            self.ps.solve(rhs)
            extra = self.ps.last_iterations
        out = self.ps._d_x0.clone()
        out[~self.mask] = 0.0
        self.last_total_iterations = self.last_iterations + extra
        return out.cpu().numpy() if host else out

    def close(self):
        for g in self._graphs.values():
            _lib.lib().cfd2d_graph_destroy(g)
        self._graphs.clear()


# ------------------------------------------------------------------ data and training
def random_obstacles(rng, lx: float = 2.0, ly: float = 1.0, nmin: int = 2, nmax: int = 12):
    """The obstacle-flow generator's obstacle list (``cases.random_obstacles``)."""
    from . import cases

    return cases.random_obstacles(rng, lx, ly, nmin, nmax)


def obstacle_case(rng, nx: int, ny: int, pressure_solver: str = "cg", lx: float = 2.0, ly: float = 1.0):
    """One seeded obstacle flow (``cases.random_obstacle_flow``)."""
    from . import cases

    return cases.random_obstacle_flow(rng, nx, ny, lx=lx, ly=ly, pressure_solver=pressure_solver)


class TrainingSet:
    """Normalised residuals r_k / ||r_k|| (FP32, (N, H, W), on the device), the case
    each one belongs to, and per case the pressure operator (for Ah o in the loss),
    its h^2 and its fluid mask."""

    def __init__(self, R, case_of, solvers, masks):
        self.R, self.case_of, self.solvers, self.masks = R, case_of, solvers, masks
        self.h2 = [h2_of(ps) for ps in solvers]

    def __len__(self):
        return int(self.R.shape[0])


def harvest_residuals(n_cases: int = 24, nx: int = 256, ny: int = 128, seed: int = 0, steps: int = 3,
                      every: int = 8, max_snaps: int = 100, rtol: float = 1e-11) -> TrainingSet:
    """Residuals from the solver's own runs.

    For each seeded obstacle case: a few projection steps, then the pressure system
    of the next predictor solved from zero by the plain Jacobi-PCG (grid solver) with
    iterate snapshots; each snapshot x_k gives the residual r_k = A (x* - x_k) of an
    iterate the preconditioner will meet. Later snapshots are dominated by the smooth
    error modes Jacobi-PCG is slow on.
    """
    import os

    from .pressure import PressureSolver

    t = _t()
    L = _lib.lib()
    rng = np.random.default_rng(seed)
    Rs, case_of, solvers, masks = [], [], [], []
    for ci in range(n_cases):
        case = obstacle_case(rng, nx, ny)
        sim = case.sim
        sim.pressure.tol = 1e-8
        sim.advance(steps)
        F, G, dt = sim.F, sim.G, sim.dt
        g = sim.grid
        rhs = ((F[1:, 1:-1] - F[:-1, 1:-1]) / g.dx + (G[1:-1, 1:] - G[1:-1, :-1]) / g.dy) / dt
        old = os.environ.get("CFD2D_PCG_VARIANT")
        os.environ["CFD2D_PCG_VARIANT"] = "grid"
        try:
            ps = PressureSolver(g, sim.boundary, method="cg", tol=rtol)
        finally:
            if old is None:
                os.environ.pop("CFD2D_PCG_VARIANT")
            else:
                os.environ["CFD2D_PCG_VARIANT"] = old
        n = nx * ny
        snap = t.zeros((max_snaps, n), dtype=t.float64, device=_lib.device())
        rd = _lib.to_dev(rhs)
        p = t.empty_like(rd)
        st = t.zeros(1, dtype=t.int32, device=_lib.device())
        _lib.check(L.cfd2d_pressure_solve_snapshots(C.byref(ps.op), _lib.ptr(rd), _lib.ptr(p), rtol, 20000,
                                                    _lib.ptr(snap), every, max_snaps, _lib.ptr(ps._d_iters),
                                                    _lib.ptr(st), _lib.stream_ptr()), "snapshots")
        its = int(ps._d_iters[0].item())
        xstar = ps._d_x0.view(-1).clone()
        mask = (ps._d_nbr >= 0x80).to(t.uint8).contiguous().view(nx, ny)
        k = min(max_snaps, its // every)
        for s_ in range(k):
            e = xstar - snap[s_]
            r = t.empty_like(e)
            _lib.check(L.cfd2d_poisson_matvec(C.byref(ps.op), _lib.ptr(e), _lib.ptr(r), _lib.stream_ptr()),
                       "matvec")
            rn = float(t.linalg.vector_norm(r))
            if rn == 0.0 or not math.isfinite(rn):
                continue
            Rs.append((r / rn).float().view(nx, ny))
            case_of.append(ci)
        solvers.append(ps)
        masks.append(mask)
    return TrainingSet(t.stack(Rs), case_of, solvers, masks)


def energy_loss_grad(ps, h2: float, out, r_hat):
    """Energy-norm loss o^T Ah o - 2 o.r_hat of one sample and its gradient
    2 (Ah o - r_hat), with Ah = h^2 A applied by the solver's FP64 operator."""
    t = _t()
    o = out.reshape(-1).double()
    Ao = t.empty_like(o)
    _lib.check(_lib.lib().cfd2d_poisson_matvec(C.byref(ps.op), _lib.ptr(o), _lib.ptr(Ao), _lib.stream_ptr()),
               "matvec")
    Ao.mul_(h2)
    rh = r_hat.reshape(-1).double()
    loss = t.dot(o, Ao) - 2.0 * t.dot(o, rh)
    grad = (2.0 * (Ao - rh)).float().view_as(out)
    return loss, grad


def train(net: LPCNet, data: TrainingSet, steps: int = 1000, batch: int = 4, lr: float = 1e-3, seed: int = 0,
          log_every: int = 100, time_budget_s: float | None = None, clip: float = 1.0):
    """Minimise the energy-norm error of net(r_hat) ~ Ah^-1 r_hat with the project's
    forward and backward kernels; Adam with a cosine learning-rate decay on FP32
    master weights, gradient-norm clipping, BF16 copies repacked every step.
    Returns the per-step mean loss."""
    t = _t()
    params = net.parameters()
    for p_ in params:
        p_.requires_grad_(False)
    opt = t.optim.Adam(params, lr=lr)
    H, W = data.R.shape[1:]
    ws = Workspace(H, W, data.masks[0])
    cur_mask = 0
    gen = np.random.default_rng(seed)
    log = []
    t0 = time.time()
    for step in range(steps):
        # cosine decay over the step count or the time budget, whichever ends first
        frac = step / max(1, steps)
        if time_budget_s:
            frac = max(frac, (time.time() - t0) / time_budget_s)
        for grp in opt.param_groups:
            grp["lr"] = lr * 0.5 * (1.0 + math.cos(math.pi * min(1.0, frac)))
        idx = gen.integers(0, len(data), batch)
        acc = {name: (t.zeros_like(net.w[name]), t.zeros_like(net.b[name])) for name, *_ in LAYERS}
        loss = t.zeros((), dtype=t.float64, device=_lib.device())
        for k in idx:
            ci = data.case_of[k]
            if ci != cur_mask:
                ws.set_mask(data.masks[ci])
                cur_mask = ci
            x = data.R[k].contiguous()
            if gen.random() < 0.5:
                x = -x  # residuals of both signs: the target is odd in r
            out = net_forward(net, ws, x)
            lk, g = energy_loss_grad(data.solvers[ci], data.h2[ci], out, x)
            loss += lk / batch
            grads = net_backward(net, ws, x, (g / batch).contiguous())
            for name in grads:
                acc[name][0].add_(grads[name][0])
                acc[name][1].add_(grads[name][1])
        opt.zero_grad(set_to_none=False)
        for name, *_ in LAYERS:
            net.w[name].grad = acc[name][0]
            if net.bias:
                net.b[name].grad = acc[name][1]
        if clip:
            t.nn.utils.clip_grad_norm_(params, clip)
        opt.step()
        net.repack()
        log.append(float(loss))
        if _take_net_error(ws):
            raise RuntimeError("a tensor-core convolution gave up waiting for its MMAs during training")
        if log_every and step % log_every == 0:
            print(f"train step {step}: loss {np.mean(log[-log_every:]):.4f}", flush=True)
        if time_budget_s is not None and time.time() - t0 > time_budget_s:
            break
    return log


def save_weights(net: LPCNet, path) -> None:
    np.savez(path, **{k: v.numpy() for k, v in net.state_dict().items()})


def load_weights(path, net: LPCNet | None = None) -> LPCNet:
    t = _t()
    net = net or LPCNet()
    d = np.load(path)
    net.load_state_dict({k: t.from_numpy(d[k]) for k in d.files})
    return net


def pretrained():
    """The shipped network: trained on 1920 residuals of 24 seeded 256 x 128
    obstacle flows (plain Jacobi-PCG iterates), 1500 Adam steps of batch 4 with a
    cosine learning rate from 1e-3, by ``train`` (``python -m cfd2d_b200.learned``
    with ``--steps 1500`` reproduces the recipe)."""
    from pathlib import Path

    return load_weights(Path(__file__).resolve().parent / "data" / "lpc_weights.npz")


def main(argv=None):
    """Harvest residuals, train, save the weights: python -m cfd2d_b200.learned OUT.npz"""
    import argparse

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("out")
    ap.add_argument("--cases", type=int, default=24)
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--ny", type=int, default=128)
    ap.add_argument("--seconds", type=float, default=0.0, help="time budget (0: none)")
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    data = harvest_residuals(n_cases=a.cases, nx=a.nx, ny=a.ny, seed=a.seed, every=8, max_snaps=80)
    print(f"residuals {tuple(data.R.shape)}", flush=True)
    net = LPCNet(seed=a.seed)
    log = train(net, data, steps=a.steps, batch=a.batch, lr=a.lr, seed=a.seed, log_every=200,
                time_budget_s=a.seconds or None)
    print(f"steps {len(log)} loss first {np.mean(log[:50]):.4f} last {np.mean(log[-50:]):.4f}", flush=True)
    save_weights(net, a.out)


if __name__ == "__main__":
    main()
