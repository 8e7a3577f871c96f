"""Learned Poisson preconditioner inside flexible CG (no counterpart in the reference).

Network: a U-Net over as many levels as the grid needs for its coarsest level to
be at most ``coarsest`` cells on a side (8 by default: 7 levels at 256 x 256, 8 at
1024 x 512, 9 at 2048 x 1024), 32 channels, 3x3 convolutions, BF16 weights and
activations, FP32 accumulation. Nine weight tensors (65,088 parameters), the
deepest encoder and decoder shared by every level from ``shared`` (3) down, so one
set of weights serves every grid size:

    a_0 = f(conv_a0 (r / ||r||))                              level 0 (1 -> 32)
    a_l = f(conv_e(l) (pool a_{l-1}))   (nrep times at l >= 3) levels 1 .. L-1
    d_{L-1} = a_{L-1}
    d_l = f(conv_d(l) (scale * up d_{l+1} + a_l))  (nrep times at l >= 3)
    out = conv_out (d_0)                                      level 0 (32 -> 1)

with e(l) = e1, e2, e3, e3, ... and d(l) = d0, d1, d2, d3, d3, ...; every layer
output is multiplied by the fluid mask of its level (a coarse cell is fluid if any
child is). f is the identity by default (``act="linear"``: the network is then a
fixed linear operator, odd and homogeneous by construction, as a preconditioner
must be) or ReLU. ``scale`` = 4 makes a coarse level contribute in the units of the
finer one: the network approximates Ah^-1 with Ah = h^2 A, and the same
dimensionless operator on a grid of twice the spacing is 4 times weaker, so a
correction computed on level l counts 4^l times on level 0.

The 32->32 layers run on tcgen05 (``cfd2d_lpc_conv32``); the 1-channel layers,
pooling, upsampling and the whole backward pass are hand-written CUDA-core kernels
of the same library (``net_forward`` / ``net_backward``, replaying one op list per
grid size); the optimiser (Adam) is PyTorch's, on FP32 master weights.

Training minimises the energy-norm error of net(r_hat) against Ah^-1 r_hat,
o^T Ah o - 2 o.r_hat (the constant e^T Ah e dropped), over residuals harvested from
the plain solver's own iterations. Inside flexible CG (Notay's form, one stored
direction) the preconditioner is M(r) = h^2 ||r|| net(r / ||r||) + omega D^-1 r; the
loop runs on the device inside one CUDA graph (a WHILE node) and falls back to the
plain Jacobi-PCG from the current iterate when it stalls.
"""

from __future__ import annotations

import ctypes as C
import json
import math
import time

import numpy as np

from . import _lib

CH = 32
# weight tensors: name -> (cin, cout)
WEIGHTS = {"a0": (1, CH), "e1": (CH, CH), "e2": (CH, CH), "e3": (CH, CH), "d0": (CH, CH), "d1": (CH, CH),
           "d2": (CH, CH), "d3": (CH, CH), "out": (CH, 1)}
DEFAULT_ARCH = {"act": "linear", "scale": 4.0, "nrep": 2, "coarsest": 8, "shared": 3}


def _t():
    return _lib.torch()


def nlevels(H: int, W: int, coarsest: int) -> int:
    """Levels of an H x W grid: halve (rounding up) until both sides are <= coarsest."""
    L = 1
    while max(H, W) > coarsest:
        H, W = (H + 1) // 2, (W + 1) // 2
        L += 1
    return L


def level_shapes(H, W, L):
    shapes = [(H, W)]
    for _ in range(L - 1):
        h, w = shapes[-1]
        shapes.append(((h + 1) // 2, (w + 1) // 2))
    return shapes


def op_list(L: int, arch: dict):
    """The network as a list of ops over named buffers, in execution order:
    ("conv", weight, level, src, dst), ("pool", level, src, dst) (src on level - 1),
    ("upadd", level, coarse, skip, dst)."""
    S, nrep = arch["shared"], arch["nrep"]
    ops = [("conv", "a0", 0, "in", "a0.0")]
    cur = "a0.0"
    for lvl in range(1, L):
        ops.append(("pool", lvl, cur, f"p{lvl}"))
        cur = f"p{lvl}"
        w = f"e{min(lvl, S)}"
        for k in range(nrep if lvl >= S else 1):
            ops.append(("conv", w, lvl, cur, f"a{lvl}.{k}"))
            cur = f"a{lvl}.{k}"
    skips = {}
    for op in ops:
        if op[0] == "conv" and op[1] != "out":
            skips[op[2]] = op[4]  # last conv output of each level
    for lvl in range(L - 2, -1, -1):
        ops.append(("upadd", lvl, cur, skips[lvl], f"u{lvl}"))
        cur = f"u{lvl}"
        w = f"d{min(lvl, S)}"
        for k in range(nrep if lvl >= S else 1):
            ops.append(("conv", w, lvl, cur, f"d{lvl}.{k}"))
            cur = f"d{lvl}.{k}"
    ops.append(("conv", "out", 0, cur, "out"))
    return ops


class LPCNet:
    """Weights (FP32 masters) and the packed BF16 tensor-core images of the 32->32 layers.

    With ``bias=False`` (the default) the biases stay zero and are not trained: the
    network is then positively homogeneous, net(a r) = a net(r) for a > 0 (and, with
    the linear activation, linear), as a preconditioner inside CG must be (a trained
    bias adds a fixed field to every preconditioned residual, and the flexible CG
    stalls on it)."""

    def __init__(self, seed: int = 0, bias: bool = False, arch: dict | None = None):
        t = _t()
        self.bias = bias
        self.arch = dict(DEFAULT_ARCH, **(arch or {}))
        g = t.Generator().manual_seed(seed)
        self.w, self.b = {}, {}
        for name, (cin, cout) in WEIGHTS.items():
            # uniform in +-1/sqrt(fan_in) (the linear form: scaled so that a layer
            # roughly keeps the norm), the output layer ten times smaller: the network
            # starts close to zero and the Jacobi term leads the first steps
            bound = 1.0 / math.sqrt(cin * 9)
            if self.arch["act"] == "linear":
                bound *= math.sqrt(3.0) / math.sqrt(3.0 if cin > 1 else 1.0)
            if name == "out":
                bound *= 0.1
            self.w[name] = ((t.rand((cout, cin, 3, 3), generator=g) * 2.0 - 1.0) * bound).to(_lib.device())
            self.b[name] = t.zeros(cout, device=_lib.device())
        self._images = {}
        self._adj_images = {}
        self._wq = {}
        self.repack()

    @property
    def relu(self) -> int:
        return 1 if self.arch["act"] == "relu" else 0

    @property
    def n_params(self) -> int:
        return sum(v.numel() for v in self.w.values()) + sum(v.numel() for v in self.b.values())

    def parameters(self):
        out = []
        for name in WEIGHTS:
            out += [self.w[name], self.b[name]] if self.bias else [self.w[name]]
        return out

    def repack(self):
        """BF16 weights: round the masters and pack the tensor-core images. The
        images and the rounded CUDA-core weights are updated in place, so graphs
        captured with them stay valid."""
        t = _t()
        L = _lib.lib()
        nbytes = int(L.cfd2d_lpc_w32_bytes())
        for name, (cin, cout) in WEIGHTS.items():
            if not (cin == CH and cout == CH):
                q = self.wq(name)
                if name in self._wq:
                    self._wq[name].copy_(q)
                else:
                    self._wq[name] = q
                continue
            img = self._images.get(name)
            if img is None:
                img = t.zeros(nbytes // 2, dtype=t.bfloat16, device=_lib.device())
                self._images[name] = img
                self._adj_images[name] = t.zeros(nbytes // 2, dtype=t.bfloat16, device=_lib.device())
            w = self.w[name].detach().float().contiguous()
            _lib.check(L.cfd2d_lpc_pack_w32(_lib.ptr(w), _lib.ptr(img), _lib.stream_ptr()), "pack_w32")
            # the data-gradient convolution of the same layer, for the backward pass
            _lib.check(L.cfd2d_lpc_pack_w32_adjoint(_lib.ptr(w), _lib.ptr(self._adj_images[name]),
                                                    _lib.stream_ptr()), "pack_w32_adjoint")

    def wq(self, name):
        """The BF16-rounded weights the kernels use, as FP32."""
        return self.w[name].detach().to(_t().bfloat16).float().contiguous()

    def state_dict(self):
        t = _t()
        d = {f"{k}.w": v.detach().cpu() for k, v in self.w.items()} | \
            {f"{k}.b": v.detach().cpu() for k, v in self.b.items()}
        d["arch"] = t.tensor(list(json.dumps(self.arch).encode()), dtype=t.uint8)
        return d

    def load_state_dict(self, d):
        if "arch" in d:
            self.arch = dict(DEFAULT_ARCH, **json.loads(bytes(d["arch"].tolist()).decode()))
        self.bias = any(float(d[f"{name}.b"].abs().max()) > 0.0 for name in WEIGHTS)
        for name in WEIGHTS:
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
    """Masks and activation buffers of one grid size and architecture (reused across
    applications): one BF16 buffer per op output, named as in ``op_list``."""

    def __init__(self, H: int, W: int, mask, arch: dict | None = None):
        t = _t()
        dev = _lib.device()
        self.arch = dict(DEFAULT_ARCH, **(arch or {}))
        self.H, self.W = H, W
        self.L = nlevels(H, W, self.arch["coarsest"])
        self.shapes = level_shapes(H, W, self.L)
        self.ops = op_list(self.L, self.arch)
        self.masks = [t.zeros(s, dtype=t.uint8, device=dev) for s in self.shapes]
        self.mask_src = None
        self.set_mask(mask)
        self.buf = {}
        for op in self.ops:
            lvl, dst = (op[2], op[4]) if op[0] == "conv" else (op[1], op[-1])
            if dst == "out":
                continue
            self.buf[dst] = t.zeros(self.shapes[lvl] + (CH,), dtype=t.bfloat16, device=dev)
        self.out = t.zeros((H, W), dtype=t.float32, device=dev)
        self.err = t.zeros(1, dtype=t.int32, device=dev)

    def set_mask(self, mask):
        """Fluid mask of level 0 (H, W) and its pooled masks (any child fluid)."""
        t = _t()
        L = _lib.lib()
        m0 = mask if isinstance(mask, t.Tensor) else _lib.to_dev(np.asarray(mask, dtype=np.uint8))
        self.masks[0].copy_(m0.reshape(self.H, self.W).to(t.uint8))
        for lvl in range(1, self.L):
            h, w = self.shapes[lvl - 1]
            _lib.check(L.cfd2d_lpc_pool_mask(_lib.ptr(self.masks[lvl - 1]), _lib.ptr(self.masks[lvl]), h, w,
                                             _lib.stream_ptr()), "pool_mask")
        self.mask_src = mask


def net_forward(net: LPCNet, ws: Workspace, x_in):
    """out = net(x_in) on the device (x_in: FP32 (H, W)); activations stay in ``ws``."""
    L = _lib.lib()
    s = _lib.stream_ptr()
    P = _lib.ptr
    sh = ws.shapes
    relu = net.relu
    scale = float(net.arch["scale"])
    for op in ws.ops:
        if op[0] == "conv":
            _, name, lvl, src, dst = op
            h, w = sh[lvl]
            cin, cout = WEIGHTS[name]
            if cin == CH and cout == CH:
                rc = L.cfd2d_lpc_conv32(P(ws.buf[src]), P(net._images[name]), P(net.b[name]), None, P(ws.masks[lvl]),
                                        P(ws.buf[dst]), h, w, relu, P(ws.err), s)
                _lib.check(rc, "lpc_conv32")
            elif cin == 1:
                _lib.check(L.cfd2d_lpc_conv(1, CH, P(x_in), 0, P(net._wq[name]), P(net.b[name]), P(ws.masks[lvl]),
                                            P(ws.buf[dst]), 1, h, w, relu, 0, s), "lpc_conv in")
            else:
                _lib.check(L.cfd2d_lpc_conv(CH, 1, P(ws.buf[src]), 1, P(net._wq[name]), P(net.b[name]),
                                            P(ws.masks[lvl]), P(ws.out), 0, h, w, 0, 0, s), "lpc_conv out")
        elif op[0] == "pool":
            _, lvl, src, dst = op
            h, w = sh[lvl - 1]
            _lib.check(L.cfd2d_lpc_pool2(P(ws.buf[src]), P(ws.buf[dst]), h, w, s), "pool2")
        else:
            _, lvl, coarse, skip, dst = op
            h, w = sh[lvl]
            _lib.check(L.cfd2d_lpc_upadd(P(ws.buf[coarse]), P(ws.buf[skip]), P(ws.buf[dst]), h, w, scale, s),
                       "upadd")
    return ws.out


def net_backward(net: LPCNet, ws: Workspace, x_in, dout, tc_dgrad: bool = True):
    """Gradients of sum(out * dout) w.r.t. every weight and bias (FP32), from the
    activations left in ``ws`` by net_forward(x_in): the op list replayed in reverse
    with the hand-written backward kernels; shared weights sum their gradients over
    the levels that use them. With ``tc_dgrad`` the data gradient of every 32->32 layer
    runs on the tensor cores (the forward tcgen05 convolution with the adjoint weight
    image: channels swapped, taps mirrored; the gradient rounded to BF16 on the way
    in and out, FP32 accumulation); else on the CUDA-core transposed convolution in
    FP32. Weight gradients are CUDA-core reductions over the pixels."""
    t = _t()
    L = _lib.lib()
    s = _lib.stream_ptr()
    P = _lib.ptr
    sh = ws.shapes
    dev = _lib.device()
    relu = net.relu
    scale = float(net.arch["scale"])
    grads = {name: (t.zeros((cout, cin, 3, 3), device=dev), t.zeros(cout, device=dev))
             for name, (cin, cout) in WEIGHTS.items()}
    g = {"out": dout.contiguous()}  # gradient of every buffer, FP32
    zero_bias = t.zeros(CH, dtype=t.float32, device=dev)

    def add(name, val):
        if name in g:
            g[name].add_(val)
        else:
            g[name] = val

    for op in reversed(ws.ops):
        if op[0] == "conv":
            _, name, lvl, src, dst = op
            h, w = sh[lvl]
            cin, cout = WEIGHTS[name]
            gy = g.pop(dst)
            # through the mask (and the ReLU) of the layer output
            gp = t.empty_like(gy)
            yb = ws.buf[dst] if dst != "out" else None
            r = relu if dst != "out" else 0
            _lib.check(L.cfd2d_lpc_relu_bwd(P(gy), P(yb), P(ws.masks[lvl]), P(gp), h * w, cout, r, s), "relu_bwd")
            xsrc, xbf = (x_in.contiguous(), 0) if src == "in" else (ws.buf[src], 1)
            ppb = 256
            part = t.empty(int(L.cfd2d_lpc_conv_dw_partial_floats(cin, cout, h, w, ppb)), dtype=t.float32, device=dev)
            dwb = t.empty(cout * cin * 9 + cout, dtype=t.float32, device=dev)
            _lib.check(L.cfd2d_lpc_conv_dw(cin, cout, P(xsrc), xbf, P(gp), h, w, ppb, P(part), P(dwb), s), "conv_dw")
            grads[name][0].add_(dwb[:cout * cin * 9].view(cout, cin, 3, 3))
            grads[name][1].add_(dwb[cout * cin * 9:])
            if src != "in":
                if tc_dgrad and cin == CH and cout == CH:
                    gb = gp.to(t.bfloat16)
                    dxb = t.empty(sh[lvl] + (cin,), dtype=t.bfloat16, device=dev)
                    _lib.check(L.cfd2d_lpc_conv32(P(gb), P(net._adj_images[name]), P(zero_bias), None, None, P(dxb),
                                                  h, w, 0, P(ws.err), s), "conv32 data gradient")
                    dx = dxb.float()
                else:
                    dx = t.zeros(sh[lvl] + (cin,), dtype=t.float32, device=dev)
                    _lib.check(L.cfd2d_lpc_conv(cout, cin, P(gp), 0, P(net.wq(name)), None, None, P(dx), 0, h, w, 0,
                                                1, s), "conv transposed")
                add(src, dx)
        elif op[0] == "pool":
            _, lvl, src, dst = op
            h, w = sh[lvl - 1]
            gy = g.pop(dst)
            dfine = g[src] if src in g else t.zeros(sh[lvl - 1] + (CH,), dtype=t.float32, device=dev)
            _lib.check(L.cfd2d_lpc_pool_bwd(P(gy), P(dfine), h, w, s), "pool_bwd")
            g[src] = dfine
        else:
            _, lvl, coarse, skip, dst = op
            h, w = sh[lvl]
            gy = g.pop(dst)
            dc = t.empty(sh[lvl + 1] + (CH,), dtype=t.float32, device=dev)
            _lib.check(L.cfd2d_lpc_upadd_bwd(P(gy), P(dc), h, w, scale, s), "upadd_bwd")
            add(coarse, dc)
            add(skip, gy.clone())
    return grads


def torch_reference_forward(net, x_in, masks, arch: dict | None = None):
    """The same network in PyTorch (CPU, FP32 on BF16-rounded weights and activations):
    the reference computation for the CUDA kernels and their gradients."""
    t = _t()
    F = t.nn.functional
    arch = dict(DEFAULT_ARCH, **(arch or getattr(net, "arch", {}) or {}))
    relu = arch["act"] == "relu"
    scale = float(arch["scale"])

    def bf(a):
        return a.to(t.bfloat16).float()

    def conv(name, a, lvl, act, round_out=True):
        bias = net.b[name]
        bias = bias.detach().cpu() if bias.is_cuda else bias
        y = F.conv2d(a, net.wq(name).cpu(), bias, padding=1)
        if act:
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
        return bf(scale * u + skip)

    Lv = len(masks)
    buf = {"in": x_in.cpu().float()[None, None]}
    for op in op_list(Lv, arch):
        if op[0] == "conv":
            _, name, lvl, src, dst = op
            last = dst == "out"
            buf[dst] = conv(name, buf[src], lvl, relu and not last, round_out=not last)
        elif op[0] == "pool":
            _, lvl, src, dst = op
            buf[dst] = pool(buf[src])
        else:
            _, lvl, coarse, skip, dst = op
            buf[dst] = up(buf[coarse], buf[skip])
    return buf["out"][0, 0]


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
        self.ws = Workspace(self.nx, self.ny, self.mask_u8, net.arch)
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
    """Normalised residuals r_k / ||r_k|| (FP32 (H, W) tensors on the device, grids of
    any size), the case each one belongs to, and per case the pressure operator (for
    Ah o in the loss), its h^2 and its fluid mask."""

    def __init__(self, R, case_of, solvers, masks, rhs=None):
        self.R, self.case_of, self.solvers, self.masks = list(R), list(case_of), list(solvers), list(masks)
        self.rhs = list(rhs) if rhs is not None else [None] * len(self.solvers)
        self.h2 = [h2_of(ps) for ps in solvers]

    def __len__(self):
        return len(self.R)

    def merge(self, other: "TrainingSet") -> "TrainingSet":
        """The samples of both sets (case indices of ``other`` shifted after this one's)."""
        n = len(self.solvers)
        return TrainingSet(self.R + other.R, self.case_of + [c + n for c in other.case_of],
                           self.solvers + other.solvers, self.masks + other.masks, self.rhs + other.rhs)

    def with_samples(self, R, case_of) -> "TrainingSet":
        """This set plus more residuals of its own cases."""
        return TrainingSet(self.R + list(R), self.case_of + list(case_of), self.solvers, self.masks, self.rhs)


def harvest_residuals(n_cases: int = 24, nx: int = 256, ny: int = 128, seed: int = 0, steps: int = 3,
                      every: int = 8, max_snaps: int = 100, rtol: float = 1e-11, lx: float = 2.0,
                      ly: float = 1.0) -> TrainingSet:
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
    Rs, case_of, solvers, masks, rhss = [], [], [], [], []
    for ci in range(n_cases):
        case = obstacle_case(rng, nx, ny, lx=lx, ly=ly)
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
        rhss.append(rd)
    return TrainingSet(Rs, case_of, solvers, masks, rhss)


def harvest_fcg_residuals(net: LPCNet, data: TrainingSet, iters: int = 300, every: int = 10,
                          tol: float = 1e-10):
    """Residuals the flexible CG with ``net`` meets on the cases of ``data`` (each
    case's pressure system from zero, ``iters`` iterations at most, one residual every
    ``every``): the residuals the preconditioner handles worst are the ones that
    survive its own iterations, and the plain solver's iterates do not contain them.
    Returns (residuals, case indices) to add to ``data``."""
    t = _t()
    Rs, case_of = [], []
    for ci, ps in enumerate(data.solvers):
        rhs = data.rhs[ci]
        if rhs is None:
            continue
        fcg = LearnedPCG(ps, net, maxiter=iters + 1, stall_window=iters + 1)
        nx, ny = fcg.nx, fcg.ny
        fcg.rhs_buf.copy_(rhs.reshape(-1))
        ps._d_x0.zero_()
        fcg._set_control(tol)
        fcg._init(rhs=fcg.rhs_buf)
        _lib.check(_lib.lib().cfd2d_fcg_gate(_lib.ptr(fcg.scal), _lib.ptr(fcg.ctl), 0, _lib.stream_ptr()), "gate")
        for it in range(iters):
            fcg._body(0)
            if (it + 1) % every == 0:
                if fcg._control().reason != _lib.FCG_RUNNING:
                    break
                r = fcg.r.view(nx, ny) * fcg.mask
                rn = float(t.linalg.vector_norm(r))
                if rn > 0.0 and math.isfinite(rn):
                    Rs.append((r / rn).float().contiguous())
                    case_of.append(ci)
        fcg.close()
    return Rs, case_of


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
    wss = {}  # one workspace per grid size, with the mask of the case it last served
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
        acc = {name: (t.zeros_like(net.w[name]), t.zeros_like(net.b[name])) for name in WEIGHTS}
        loss = t.zeros((), dtype=t.float64, device=_lib.device())
        for k in idx:
            ci = data.case_of[k]
            x = data.R[k].contiguous()
            H, W = x.shape
            if (H, W) not in wss:
                wss[(H, W)] = [Workspace(H, W, data.masks[ci], net.arch), ci]
            ws, cur = wss[(H, W)]
            if cur != ci:
                ws.set_mask(data.masks[ci])
                wss[(H, W)][1] = ci
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
        for name in WEIGHTS:
            net.w[name].grad = acc[name][0]
            if net.bias:
                net.b[name].grad = acc[name][1]
        if clip:
            t.nn.utils.clip_grad_norm_(params, clip)
        opt.step()
        net.repack()
        log.append(float(loss))
        if any(_take_net_error(w_[0]) for w_ in wss.values()):
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
    """The shipped network (``data/lpc_weights.npz``). First trained by ``train`` on the
    "channel" recipe: residuals of the plain Jacobi-PCG's iterates on 60 seeded
    obstacle flows of the generator at 256 x 128 and 20 at 512 x 256 (the benchmark's
    2 x 1 channel, square cells), 6000 Adam steps, then one on-policy round (the
    residuals the flexible CG with the trained network meets on the same cases, about
    2.4k, added; 3000 more steps at half the learning rate):
    ``python -m cfd2d_b200.learned train OUT.npz --cases 60``. Then fine-tuned by
    ``finetune`` on larger grids, where the deeper levels of the U-Net first meet real
    data: 20 channel-recipe cases replayed plus 3 seeded obstacle flows each at
    1024 x 512 and 2048 x 1024 (their plain iterates' residuals), one round of the
    flexible CG's own residuals, 2000 steps at 2e-4 (``finetune A.npz``); then from
    that, 4 flows per size, two such rounds (``finetune B.npz --init A.npz --cases 4
    --rounds 2 --seed 200``); then 6 flows per size, two rounds of 3000 steps
    (``finetune C.npz --init B.npz --cases 6 --rounds 2 --steps 3000 --seed 300``);
    then the same with other flows at a lower rate (``finetune D.npz --init C.npz
    --cases 6 --rounds 2 --steps 3000 --lr 1.5e-4 --seed 500``). The benchmark's flow
    (generator seed 13) is held out of every set."""
    from pathlib import Path

    return load_weights(Path(__file__).resolve().parent / "data" / "lpc_weights.npz")


def harvest_recipe(cases: int = 50, snaps: int = 100, seed: int = 0, kind: str = "channel") -> TrainingSet:
    """Training sets. "channel": ``cases`` seeded obstacle flows of the generator on the
    2 x 1 channel at 256 x 128 and a third as many at 512 x 256 (square cells, as the
    benchmark grids); "mixed": ``cases`` on 256 x 256 (unit square) and as many at
    256 x 128. Up to ``snaps`` residuals of the plain solver's iterates per case."""
    if kind == "mixed":
        sq = harvest_residuals(n_cases=cases, nx=256, ny=256, seed=seed, every=12, max_snaps=snaps, lx=1.0, ly=1.0)
        ch = harvest_residuals(n_cases=cases, nx=256, ny=128, seed=seed + 1000, every=8, max_snaps=snaps)
        return sq.merge(ch)
    small = harvest_residuals(n_cases=cases, nx=256, ny=128, seed=seed + 1000, every=8, max_snaps=snaps)
    big = harvest_residuals(n_cases=max(1, cases // 3), nx=512, ny=256, seed=seed + 2000, every=16,
                            max_snaps=snaps)
    return small.merge(big)


def main(argv=None):
    """python -m cfd2d_b200.learned train OUT.npz [options]: harvest residuals, train,
    save the weights. python -m cfd2d_b200.learned finetune OUT.npz [options]: go on
    training a network (the shipped one by default) with residuals of larger obstacle
    flows added, the flexible CG's own among them. python -m cfd2d_b200.learned apply NX NY [--reps N]: one
    obstacle flow (generator seed 13) of NX x NY, N applications of the shipped
    network's preconditioner, event-timed (the command the network's profiles use)."""
    import argparse

    ap = argparse.ArgumentParser(description=main.__doc__)
    sub = ap.add_subparsers(dest="cmd", required=True)
    tr = sub.add_parser("train")
    tr.add_argument("out")
    tr.add_argument("--cases", type=int, default=50)
    tr.add_argument("--snaps", type=int, default=100)
    tr.add_argument("--seconds", type=float, default=0.0, help="time budget (0: none)")
    tr.add_argument("--steps", type=int, default=6000)
    tr.add_argument("--batch", type=int, default=4)
    tr.add_argument("--lr", type=float, default=1e-3)
    tr.add_argument("--seed", type=int, default=0)
    tr.add_argument("--recipe", choices=["channel", "mixed"], default="channel")
    tr.add_argument("--arch", default="{}", help="JSON overrides of the architecture (e.g. '{\"nrep\": 1}')")
    tr.add_argument("--onpolicy", type=int, default=1,
                    help="rounds of adding the flexible CG's own residuals and training on")
    ft = sub.add_parser("finetune")
    ft.add_argument("out")
    ft.add_argument("--init", default="", help="weights to start from (default: the shipped network)")
    ft.add_argument("--sizes", default="1024x512,2048x1024", help="grids of the added obstacle flows")
    ft.add_argument("--cases", type=int, default=3, help="seeded obstacle flows per size")
    ft.add_argument("--replay", type=int, default=20, help="cases of the channel recipe kept in the set")
    ft.add_argument("--steps", type=int, default=2000)
    ft.add_argument("--batch", type=int, default=4)
    ft.add_argument("--lr", type=float, default=2e-4)
    ft.add_argument("--seed", type=int, default=100)
    ft.add_argument("--rounds", type=int, default=1,
                    help="rounds of adding the flexible CG's own residuals and training on")
    apl = sub.add_parser("apply")
    apl.add_argument("nx", type=int)
    apl.add_argument("ny", type=int)
    apl.add_argument("--reps", type=int, default=5)
    a = ap.parse_args(argv)
    if a.cmd == "train":
        t0 = time.time()
        data = harvest_recipe(cases=a.cases, snaps=a.snaps, seed=a.seed, kind=a.recipe)
        print(f"residuals {len(data)} from {len(data.solvers)} cases in {time.time() - t0:.0f}s", flush=True)
        net = LPCNet(seed=a.seed, arch=json.loads(a.arch))
        log = train(net, data, steps=a.steps, batch=a.batch, lr=a.lr, seed=a.seed, log_every=500,
                    time_budget_s=a.seconds or None)
        print(f"steps {len(log)} loss first {np.mean(log[:50]):.4f} last {np.mean(log[-50:]):.4f}", flush=True)
        for rnd in range(a.onpolicy):
            R, co = harvest_fcg_residuals(net, data)
            data = data.with_samples(R, co)
            print(f"round {rnd + 1}: {len(R)} residuals of the flexible CG added ({len(data)} in all)", flush=True)
            log = train(net, data, steps=a.steps // 2, batch=a.batch, lr=a.lr / 2, seed=a.seed + rnd + 1,
                        log_every=500)
            print(f"steps {len(log)} loss last {np.mean(log[-50:]):.4f}", flush=True)
        save_weights(net, a.out)
        return
    if a.cmd == "finetune":
        t0 = time.time()
        net = load_weights(a.init) if a.init else pretrained()
        data = harvest_recipe(cases=a.replay, snaps=50, seed=a.seed, kind="channel")
        for k, size in enumerate(a.sizes.split(",")):
            nx, ny = (int(v) for v in size.lower().split("x"))
            # seeds apart from the benchmark's generator seed (13), which stays held out
            big = harvest_residuals(n_cases=a.cases, nx=nx, ny=ny, seed=a.seed + 3000 + k, every=max(8, nx // 10),
                                    max_snaps=40)
            data = data.merge(big)
        print(f"residuals {len(data)} from {len(data.solvers)} cases in {time.time() - t0:.0f}s", flush=True)
        for rnd in range(a.rounds):
            R, co = harvest_fcg_residuals(net, data)
            data = data.with_samples(R, co)
            print(f"round {rnd + 1}: {len(R)} residuals of the flexible CG added ({len(data)} in all)", flush=True)
            log = train(net, data, steps=a.steps, batch=a.batch, lr=a.lr, seed=a.seed + rnd, log_every=500)
            print(f"steps {len(log)} loss last {np.mean(log[-50:]):.4f}", flush=True)
        save_weights(net, a.out)
        return
    from . import cases

    t = _t()
    case = cases.obstacle_flow(13, a.nx, a.ny, pressure_solver="cg")
    sim = case.sim
    sim.advance(1)
    fcg = LearnedPCG(sim.pressure, pretrained())
    fcg.r.copy_(t.randn_like(fcg.r))
    ev = [t.cuda.Event(enable_timing=True) for _ in range(2)]
    fcg.precondition()
    t.cuda.synchronize()
    ev[0].record()
    for _ in range(a.reps):
        fcg.precondition()
    ev[1].record()
    t.cuda.synchronize()
    print(json.dumps({"grid": [a.nx, a.ny], "levels": fcg.ws.L, "ms_per_application": ev[0].elapsed_time(ev[1]) / a.reps}))
    fcg.close()


if __name__ == "__main__":
    main()
