"""Learned Poisson preconditioner: kernels against PyTorch CPU, training, flexible CG (GPU).

The CPU checker is PyTorch on the same BF16-rounded weights and activations: the
forward pass must agree to BF16 resolution and every weight gradient of the
hand-written backward kernels to a few percent (the kernels keep activations in
BF16 and accumulate in FP32, the PyTorch computation in FP32 throughout).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu]


@pytest.fixture(scope="module")
def L(cuda_lib):
    import torch

    from cfd2d_b200 import _lib, learned

    torch.manual_seed(0)
    return torch, _lib, learned


def relerr(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


# one full and one partial 128-pixel segment per row; the sizes select 1, 2 and 2 rows
# per CTA (the last two with a partial block of rows)
@pytest.mark.parametrize("H,W", [(7, 200), (601, 300), (1201, 300)])
def test_conv32_tensor_cores_match_torch(L, H, W):
    torch, _lib, learned = L
    F = torch.nn.functional
    g = torch.Generator().manual_seed(1)
    x = torch.randn((H, W, 32), generator=g).to(torch.bfloat16)
    w = torch.randn((32, 32, 3, 3), generator=g) * 0.1
    b = torch.randn(32, generator=g) * 0.1
    skip = torch.randn((H, W, 32), generator=g).to(torch.bfloat16)
    mask = (torch.rand((H, W), generator=g) > 0.2).to(torch.uint8)
    dev = _lib.device()
    img = torch.zeros(int(_lib.lib().cfd2d_lpc_w32_bytes()) // 2, dtype=torch.bfloat16, device=dev)
    wd = w.to(dev).contiguous()
    _lib.check(_lib.lib().cfd2d_lpc_pack_w32(_lib.ptr(wd), _lib.ptr(img), _lib.stream_ptr()), "pack")
    xd, sd, md = x.to(dev), skip.to(dev), mask.to(dev)
    y = torch.zeros((H, W, 32), dtype=torch.bfloat16, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    bd = b.to(dev)
    _lib.check(_lib.lib().cfd2d_lpc_conv32(_lib.ptr(xd), _lib.ptr(img), _lib.ptr(bd), _lib.ptr(sd), _lib.ptr(md),
                                           _lib.ptr(y), H, W, 1, _lib.ptr(err), _lib.stream_ptr()), "conv32")
    assert int(err.item()) == 0
    xin = x.float().permute(2, 0, 1)[None]
    ref = F.conv2d(xin, w.to(torch.bfloat16).float(), b, padding=1)[0].permute(1, 2, 0)
    ref = torch.relu(ref + skip.float()) * mask[..., None]
    assert relerr(y.float().cpu(), ref.to(torch.bfloat16).float()) < 1e-2


@pytest.mark.parametrize("cin,cout", [(1, 32), (32, 1), (32, 32)])
def test_cuda_core_conv_and_adjoint(L, cin, cout):
    torch, _lib, learned = L
    F = torch.nn.functional
    H, W = 9, 13
    g = torch.Generator().manual_seed(cin * 100 + cout)
    x = torch.randn((H, W, cin), generator=g)
    w = torch.randn((cout, cin, 3, 3), generator=g) * 0.2
    b = torch.randn(cout, generator=g)
    dev = _lib.device()
    y = torch.zeros((H, W, cout), device=dev)
    xd, wd, bd = x.to(dev).contiguous(), w.to(dev).contiguous(), b.to(dev)
    _lib.check(_lib.lib().cfd2d_lpc_conv(cin, cout, _lib.ptr(xd), 0, _lib.ptr(wd), _lib.ptr(bd), None, _lib.ptr(y), 0,
                                         H, W, 0, 0, _lib.stream_ptr()), "conv")
    ref = F.conv2d(x.permute(2, 0, 1)[None], w, b, padding=1)[0].permute(1, 2, 0)
    assert relerr(y.cpu(), ref) < 1e-5
    # adjoint: <conv(x), d> == <x, conv^T(d)>
    d = torch.randn((H, W, cout), generator=g)
    dx = torch.zeros((H, W, cin), device=dev)
    dd = d.to(dev).contiguous()
    _lib.check(_lib.lib().cfd2d_lpc_conv(cout, cin, _lib.ptr(dd), 0, _lib.ptr(wd), None, None, _lib.ptr(dx), 0,
                                         H, W, 0, 1, _lib.stream_ptr()), "conv^T")
    lhs = float(((ref - b) * d).sum())
    rhs = float((x * dx.cpu()).sum())
    assert abs(lhs - rhs) <= 1e-4 * max(abs(lhs), 1.0)


def test_forward_fast_paths_match_the_generic_kernel(L):
    """The forward 1 -> 32 (FP32 in, BF16 out) and 32 -> 1 (BF16 in, FP32 out) layers
    take their own vectorised kernels; they give the generic kernel's bits and agree
    with torch."""
    torch, _lib, learned = L
    F = torch.nn.functional
    H, W = 37, 141
    g = torch.Generator().manual_seed(7)
    dev = _lib.device()
    lib = _lib.lib()
    m = torch.from_numpy(_random_mask(H, W, 3)).to(dev)
    # 1 -> 32, ReLU, mask
    x = torch.randn((H, W, 1), generator=g).to(dev)
    w = (torch.randn((32, 1, 3, 3), generator=g) * 0.3).to(dev).contiguous()
    b = (torch.randn(32, generator=g) * 0.1).to(dev)
    fast = torch.zeros((H, W, 32), dtype=torch.bfloat16, device=dev)
    gen = torch.zeros((H, W, 32), device=dev)
    P = _lib.ptr
    _lib.check(lib.cfd2d_lpc_conv(1, 32, P(x), 0, P(w), P(b), P(m), P(fast), 1, H, W, 1, 0, _lib.stream_ptr()), "1to32")
    _lib.check(lib.cfd2d_lpc_conv(1, 32, P(x), 0, P(w), P(b), P(m), P(gen), 0, H, W, 1, 0, _lib.stream_ptr()), "gen")
    assert torch.equal(fast, gen.to(torch.bfloat16))
    ref = torch.relu(F.conv2d(x.cpu().permute(2, 0, 1)[None], w.cpu(), b.cpu(), padding=1)[0].permute(1, 2, 0))
    ref = ref * m.cpu()[..., None]
    assert relerr(fast.float().cpu(), ref) < 1e-2
    # 32 -> 1, no ReLU, mask
    xb = torch.randn((H, W, 32), generator=g).to(torch.bfloat16).to(dev)
    w1 = (torch.randn((1, 32, 3, 3), generator=g) * 0.1).to(dev).contiguous()
    b1 = (torch.randn(1, generator=g) * 0.1).to(dev)
    fast1 = torch.zeros((H, W, 1), device=dev)
    gen1 = torch.zeros((H, W, 1), device=dev)
    xf = xb.float().contiguous()
    _lib.check(lib.cfd2d_lpc_conv(32, 1, P(xb), 1, P(w1), P(b1), P(m), P(fast1), 0, H, W, 0, 0, _lib.stream_ptr()),
               "32to1")
    _lib.check(lib.cfd2d_lpc_conv(32, 1, P(xf), 0, P(w1), P(b1), P(m), P(gen1), 0, H, W, 0, 0, _lib.stream_ptr()),
               "gen")
    assert torch.equal(fast1, gen1)
    ref1 = F.conv2d(xf.cpu().permute(2, 0, 1)[None], w1.cpu(), b1.cpu(), padding=1)[0].permute(1, 2, 0)
    ref1 = ref1 * m.cpu()[..., None]
    assert relerr(fast1.cpu(), ref1) < 1e-5


def _random_mask(H, W, seed):
    rng = np.random.default_rng(seed)
    m = np.ones((H, W), dtype=np.uint8)
    for _ in range(4):
        i, j = rng.integers(0, H - 4), rng.integers(0, W - 4)
        m[i:i + 4, j:j + 3] = 0
    return m


def test_network_forward_matches_torch(L):
    torch, _lib, learned = L
    H, W = 40, 37
    net = learned.LPCNet(seed=3)
    for name in net.b:
        net.b[name].copy_(torch.randn_like(net.b[name]) * 0.05)
    net.repack()
    mask = _random_mask(H, W, 0)
    ws = learned.Workspace(H, W, mask)
    g = torch.Generator().manual_seed(4)
    x = (torch.randn((H, W), generator=g) * torch.from_numpy(mask)).float()
    out = learned.net_forward(net, ws, x.to(_lib.device()).contiguous()).cpu()
    masks = [m.cpu().float()[None, None] for m in ws.masks]
    ref = learned.torch_reference_forward(net, x, masks)
    assert relerr(out, ref) < 3e-2


@pytest.mark.parametrize("tc_dgrad", [True, False])
def test_backward_kernels_match_autograd(L, tc_dgrad):
    """Every weight gradient of the hand-written backward kernels against PyTorch
    autograd, with the data gradients of the 32->32 layers on the tensor cores (BF16
    in and out) and on the CUDA cores (FP32); 72 x 65 has five levels, so the shared
    deepest encoder and decoder (applied twice on level 3 and below) are used and
    checked as well."""
    torch, _lib, learned = L
    H, W = 72, 65
    net = learned.LPCNet(seed=5)
    mask = _random_mask(H, W, 1)
    ws = learned.Workspace(H, W, mask)
    g = torch.Generator().manual_seed(6)
    x = (torch.randn((H, W), generator=g) * torch.from_numpy(mask)).float()
    dout = torch.randn((H, W), generator=g) * torch.from_numpy(mask)
    learned.net_forward(net, ws, x.to(_lib.device()).contiguous())
    grads = learned.net_backward(net, ws, x.to(_lib.device()).contiguous(), dout.to(_lib.device()).contiguous(),
                                 tc_dgrad=tc_dgrad)
    # autograd on the CPU reference with leaf copies of the BF16-rounded weights
    masks = [m.cpu().float()[None, None] for m in ws.masks]
    saved = {k: (v.clone(), net.b[k].clone()) for k, v in net.w.items()}
    leaf_w = {k: net.wq(k).cpu().requires_grad_(True) for k in net.w}
    leaf_b = {k: net.b[k].detach().cpu().clone().requires_grad_(True) for k in net.b}

    class Shim:
        w = leaf_w
        b = leaf_b

        @staticmethod
        def wq(name):
            return leaf_w[name]

    out = learned.torch_reference_forward(Shim, x, masks)
    (out * dout).sum().backward()
    for name in net.w:
        gw, gb = grads[name]
        assert leaf_w[name].grad is not None, name
        assert relerr(gw.cpu(), leaf_w[name].grad) < 5e-2, name
        if leaf_b[name].grad.abs().max() > 0:
            assert relerr(gb.cpu(), leaf_b[name].grad) < 5e-2, name
    for k, (w_, b_) in saved.items():
        assert torch.equal(net.w[k], w_) and torch.equal(net.b[k], b_)


def test_flexible_cg_reaches_tolerance_and_matches_plain_cg(L):
    torch, _lib, learned = L
    rng = np.random.default_rng(7)
    case = learned.obstacle_case(rng, 256, 128)
    sim = case.sim
    sim.advance(2)
    g = sim.grid
    F, G = sim.F, sim.G
    rhs = ((F[1:, 1:-1] - F[:-1, 1:-1]) / g.dx + (G[1:-1, 1:] - G[1:-1, :-1]) / g.dy) / sim.dt
    ps = sim.pressure
    # both solvers from a cold start (the warm start after a step already solves
    # this right-hand side) to a tight relative residual
    ps.tol = 1e-9
    zero = np.zeros(int(ps.fluid.sum()))
    ps._x0 = zero
    p_plain = ps.solve(rhs)
    assert ps.last_iterations > 0
    net = learned.LPCNet(seed=0)
    fcg = learned.LearnedPCG(ps, net)
    # the graph-driven loop and the host-driven loop run the same kernels in the
    # same order: identical iterates
    ps._x0 = zero
    p_host = fcg.solve(rhs, graph=False)
    its_host, hist_host = fcg.last_total_iterations, list(fcg.history)
    ps._x0 = zero
    p_fcg = fcg.solve(rhs)
    assert fcg.last_total_iterations > 0
    assert fcg.last_total_iterations == its_host and fcg.history == hist_host
    assert np.array_equal(p_fcg, p_host)
    assert relerr(p_fcg, p_plain) < 1e-4
    # the stop test is the plain solver's, ||r|| < tol ||b|| on the recursively
    # updated residual; the true residual of the final iterate is within 2x of it
    A = ps.A
    b = -rhs[ps.fluid]
    x = ps._x0
    assert np.linalg.norm(b - A @ x) <= 2e-9 * np.linalg.norm(b)
    fcg.close()


def test_training_lowers_the_energy_loss(L):
    torch, _lib, learned = L
    data = learned.harvest_residuals(n_cases=3, nx=128, ny=64, seed=1, every=6, max_snaps=40)
    assert len(data) >= 20 and tuple(data.R[0].shape) == (128, 64)
    net = learned.LPCNet(seed=1)
    log = learned.train(net, data, steps=150, batch=2, lr=2e-3, log_every=0)
    assert np.all(np.isfinite(log))
    assert np.mean(log[-20:]) < np.mean(log[:20]) and np.mean(log[-20:]) < 0.0


def test_trained_network_reduces_iterations(L):
    """What the shipped network gains over the method without it: the same solve
    from zero to 1e-8 by flexible CG with the learned preconditioner against the
    plain Jacobi-PCG, on held-out obstacle flows (seeds not in the training set)."""
    torch, _lib, learned = L
    net = learned.pretrained()
    for seed in (11, 12):
        rng = np.random.default_rng(seed)
        case = learned.obstacle_case(rng, 256, 128)
        sim = case.sim
        sim.pressure.tol = 1e-8
        sim.advance(2)
        g = sim.grid
        F, G = sim.F, sim.G
        rhs = ((F[1:, 1:-1] - F[:-1, 1:-1]) / g.dx + (G[1:-1, 1:] - G[1:-1, :-1]) / g.dy) / sim.dt
        ps = sim.pressure
        zero = np.zeros(int(ps.fluid.sum()))
        ps._x0 = zero
        p_plain = ps.solve(rhs)
        its_plain = ps.last_iterations
        fcg = learned.LearnedPCG(ps, net)
        ps._x0 = zero
        p = fcg.solve(rhs)
        assert fcg.last_reason == _lib.FCG_CONVERGED, (seed, fcg.last_reason, fcg.last_iterations)
        assert fcg.last_total_iterations <= 0.7 * its_plain, (seed, fcg.last_total_iterations, its_plain)
        assert relerr(p, p_plain) < 1e-4
        fcg.close()


def test_learned_solve_is_faster_on_the_1024x512_obstacle_flow(L):
    """The time the shipped network gains: one pressure system of the seeded 1024x512
    obstacle flow (its fourth step, from the previous step's pressure) solved to 1e-8 by
    the plain Jacobi-PCG and by flexible CG with the learned preconditioner, each timed
    with CUDA events after one untimed solve of the same system. The learned solve must
    converge without falling back and take at most 85 % of the plain solve's time."""
    torch, _lib, learned = L
    from cfd2d_b200 import cases

    sim = cases.obstacle_flow(13, 1024, 512, pressure_solver="cg").sim
    ps = sim.pressure
    ps.tol = 1e-8
    sim.advance(3)
    xprev = ps._d_x0.clone()
    sim.advance(1)
    g = sim.grid
    F, G = sim.F, sim.G
    rhs = torch.from_numpy(((F[1:, 1:-1] - F[:-1, 1:-1]) / g.dx + (G[1:-1, 1:] - G[1:-1, :-1]) / g.dy)
                           / sim.dt).cuda()
    fcg = learned.LearnedPCG(ps, learned.pretrained())
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ms, sol = {}, {}
    for name, solve in (("plain", lambda: ps.solve(rhs)), ("learned", lambda: fcg.solve(rhs))):
        for _timed in (False, True):
            ps._d_x0.copy_(xprev)
            torch.cuda.synchronize()
            ev[0].record()
            out = solve()
            ev[1].record()
            torch.cuda.synchronize()
        ms[name] = ev[0].elapsed_time(ev[1])
        sol[name] = np.asarray(out.cpu() if hasattr(out, "cpu") else out)
    assert fcg.last_reason == _lib.FCG_CONVERGED, (fcg.last_reason, fcg.last_iterations)
    assert fcg.last_total_iterations < 0.1 * ps.last_iterations, (fcg.last_total_iterations, ps.last_iterations)
    assert ms["learned"] <= 0.85 * ms["plain"], ms
    assert relerr(sol["learned"], sol["plain"]) < 1e-4
    fcg.close()


def test_learned_pressure_solve_inside_the_step(L):
    """Simulation.set_pressure_preconditioner: the same steps from the same state
    with the plain and the learned pressure solve agree to the solver tolerance."""
    torch, _lib, learned = L
    net = learned.pretrained()
    out = {}
    for mode in ("plain", "learned"):
        rng = np.random.default_rng(31)
        case = learned.obstacle_case(rng, 256, 128)
        sim = case.sim
        sim.pressure.tol = 1e-8
        sim.advance(20)
        if mode == "learned":
            sim.set_pressure_preconditioner(net)
        sim.advance(4)
        out[mode] = (sim.u.copy(), sim.v.copy(), list(sim.history.extra["cg_iterationen"][-4:]))
        sim.set_pressure_preconditioner(None)
    (up, vp, ip), (ul, vl, il) = out["plain"], out["learned"]
    assert relerr(ul, up) < 1e-6 and relerr(vl, vp) < 1e-6
    assert all(a > 0 for a in il) and sum(il) < sum(ip), (il, ip)
