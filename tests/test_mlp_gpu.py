"""The learned initial guess: tcgen05 BF16 GEMMs (FP32 accumulation) checked
against a NumPy FP64 evaluation of the same quantised network, gradients
checked against the CPU oracle's FP64 backward, the fused guess kernel
against the layer-by-layer forward, the hinted locate against drb_locate
with the same guesses, and a short training run showing the gain over the
element-centre guess."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16(a):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1 + np.tanh(0.7978845608028654 * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(0.7978845608028654 * (x + 0.044715 * x ** 3))
    du = 0.7978845608028654 * (1 + 3 * 0.044715 * x * x)
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * du


def unpack(p):
    from devil_ray_b200 import learned as LG
    p = np.asarray(p, np.float64)
    W1 = p[LG.W1:LG.B1].reshape(128, 84)
    b1 = p[LG.B1:LG.W2]
    W2 = p[LG.W2:LG.B2].reshape(128, 128)
    b2 = p[LG.B2:LG.W3]
    W3 = p[LG.W3:LG.B3].reshape(3, 128)
    b3 = p[LG.B3:LG.N_PARAMS]
    return W1, b1, W2, b2, W3, b3


def oracle_forward(p, X):
    """FP64 forward of the network as the kernels quantise it: bf16 inputs,
    W1, W2 and first-layer activations; fp32-exact head."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    Xq = bf16(X)[:, :84]
    Z1 = Xq @ bf16(W1).T + b1
    H1 = bf16(gelu(Z1))
    Z2 = H1 @ bf16(W2).T + b2
    H2 = gelu(Z2)
    y = H2 @ W3.T + b3
    return Xq, Z1, H1, Z2, H2, y


def oracle_grad(p, X, T, w, n):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    Xq, Z1, H1, Z2, H2, y = oracle_forward(p, X)
    dY = 2 * w[:, None] * (y - T) / n
    g = {}
    g["W3"] = dY.T @ H2
    g["b3"] = dY.sum(0)
    dZ2 = bf16((dY @ W3) * gelu_grad(Z2))
    g["b2"] = dZ2.sum(0)
    g["W2"] = dZ2.T @ H1
    dZ1 = bf16((dZ2 @ bf16(W2)) * gelu_grad(Z1))
    g["b1"] = dZ1.sum(0)
    g["W1"] = dZ1.T @ Xq
    loss = float((w[:, None] * (y - T) ** 2).sum() / n)
    return g, loss


@pytest.fixture(scope="module")
def setup(cuda):
    import torch
    from devil_ray_b200 import api, meshgen
    from devil_ray_b200 import learned as LG
    m = meshgen.trilinear_distorted_mesh(12, 2, 0.15, seed=31)
    mesh = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    model = LG.GuessMLP(cuda, seed=7)
    # perturb the biases so every parameter block matters
    g = torch.Generator(device="cpu").manual_seed(3)
    model.params += (torch.rand(model.params.shape, generator=g) - 0.5).cuda() * 0.02
    model.prepare()
    n = 1000
    elem, pts, label, w = LG.training_set(mesh, n, seed=5)
    X = model.features(mesh, elem, pts)
    torch.cuda.synchronize()
    return mesh, model, elem, pts, label, w, X, n


def test_tcgen05_forward_matches_fp64(setup):
    import torch
    mesh, model, elem, pts, label, w, X, n = setup
    y = model.forward(X, n)
    torch.cuda.synchronize()
    model.check_err()
    p = model.params.cpu().numpy()
    Xn = X.float().cpu().numpy()[:n]
    *_, yo = oracle_forward(p, Xn)
    err = np.abs(y.cpu().numpy() - yo).max()
    scale = np.abs(yo).max()
    print(f"forward: max |y - y_fp64| {err:.3e} (|y| <= {scale:.2f})")
    assert err < 2e-3 * max(1.0, scale)


def test_tcgen05_gradients_match_fp64(setup):
    import torch
    mesh, model, elem, pts, label, w, X, n = setup
    grad, loss = model.grad(X, label, n, w)
    torch.cuda.synchronize()
    model.check_err()
    from devil_ray_b200 import learned as LG
    p = model.params.cpu().numpy()
    og, oloss = oracle_grad(p, X.float().cpu().numpy()[:n], label.cpu().numpy().astype(np.float64),
                            w.cpu().numpy().astype(np.float64), n)
    gg = grad.cpu().numpy()
    blocks = {"W1": gg[LG.W1:LG.B1].reshape(128, 84), "b1": gg[LG.B1:LG.W2],
              "W2": gg[LG.W2:LG.B2].reshape(128, 128), "b2": gg[LG.B2:LG.W3],
              "W3": gg[LG.W3:LG.B3].reshape(3, 128), "b3": gg[LG.B3:LG.N_PARAMS]}
    for k, v in blocks.items():
        ref = og[k]
        rel = np.abs(v - ref).max() / max(np.abs(ref).max(), 1e-12)
        print(f"grad {k}: max rel err {rel:.2e}")
        assert rel < 3e-2, k
    assert abs(float(loss.item()) - oloss) <= 1e-3 * max(1.0, oloss)


def test_fused_guess_matches_forward(setup):
    import torch
    mesh, model, elem, pts, label, w, X, n = setup
    y = model.forward(X, n).clamp(0, 1)
    gss = model.guess(mesh, elem, pts)
    torch.cuda.synchronize()
    model.check_err()
    assert torch.allclose(gss, y, atol=2e-3), (gss - y).abs().max()
    # visiting the rows in another order (as the Morton order does) changes nothing
    perm = torch.randperm(elem.numel(), generator=torch.Generator().manual_seed(9)).to(
        device=elem.device, dtype=torch.int32)
    gp = model.guess(mesh, elem, pts, order=perm)
    torch.cuda.synchronize()
    model.check_err()
    assert torch.equal(gp, gss)


def test_hinted_locate_equals_plain_given_guess(cuda, setup):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import learned as LG
    from devil_ray_b200 import meshgen
    mesh, model, *_ = setup
    q = torch.as_tensor(meshgen.uniform_queries(50000, 17), device=cuda)
    ll = LG.LearnedLocator(mesh, model, tol=1e-5, max_steps=20)
    # recompute the guesses exactly as LearnedLocator does, then run plain
    order = ll._order.order(q)
    bvh = mesh.get_bvh()
    fl = torch.empty(q.shape[0], dtype=torch.int32, device=cuda)
    fe = torch.empty_like(fl)
    import ctypes as C
    L.check(LG._lib().drb_first_candidates(C.byref(bvh.desc()), C.c_void_p(q.data_ptr()),
                                           q.shape[0], C.c_void_p(order.data_ptr()),
                                           C.c_void_p(fl.data_ptr()), C.c_void_p(fe.data_ptr()),
                                           None), "first")
    guess = model.guess(mesh, fe, q)
    c0, r0, it0, ca0, nd0 = mesh.locate(q, tol=1e-5, max_steps=20, guess_mode=L.GUESS_GIVEN,
                                        guess=guess, stats=True)
    c1, r1, it1, ca1, nd1 = ll.locate(q, order=order, stats=True)
    torch.cuda.synchronize()
    assert torch.equal(c0, c1)
    assert torch.equal(r0, r1)
    assert torch.equal(it0, it1) and torch.equal(ca0, ca1)


def test_training_reduces_newton_iterations(cuda):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    from devil_ray_b200 import learned as LG
    m = meshgen.trilinear_distorted_mesh(16, 2, 0.15, seed=41)
    mesh = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    model = LG.GuessMLP(cuda, seed=1)
    losses = LG.train(model, mesh, samples=1 << 20, batch=16384, epochs=4, lr=3e-3)
    assert losses[-1] < 0.05 * losses[0], losses
    # guessed vs centre solves on held-out (element, point) pairs
    he, hp, hl, hw = LG.training_set(mesh, 100000, seed=77)
    guess = model.guess(mesh, he, hp)
    rg, fg, ig = LG.newton_pairs(mesh, he, hp, 1e-5, 20, guess)
    rc, fc, ic = LG.newton_pairs(mesh, he, hp, 1e-5, 20)
    ok = fc
    err = (guess[ok] - rc[ok]).abs().max(dim=1).values
    print(f"held-out guess error: median {err.median().item():.3e}, "
          f"p99 {err.quantile(0.99).item():.3e}; guessed solve converged "
          f"{fg[ok].float().mean().item():.5f}; iterations {ig[ok].float().mean().item():.3f} "
          f"vs centre {ic[ok].float().mean().item():.3f}")
    assert ig[ok].float().mean() < ic[ok].float().mean()
    q = torch.as_tensor(meshgen.uniform_queries(200000, 99), device=cuda)
    c0, r0, it0, *_ = api.BatchedLocator(mesh, 1e-5, 20).locate(q, stats=True)
    ll = LG.LearnedLocator(mesh, model, 1e-5, 20)
    c1, r1, it1, *_ = ll.locate(q, stats=True)
    torch.cuda.synchronize()
    hit = (c0 >= 0) & (c1 >= 0)
    agree = (c0 == c1).float().mean().item()
    mi0 = it0[hit].float().mean().item()
    mi1 = it1[hit].float().mean().item()
    print(f"learned guess: mean Newton iterations {mi1:.3f} vs centre {mi0:.3f}, "
          f"cell agreement {agree:.5f}, final loss {losses[-1]:.2e}")
    assert agree > 0.999
    assert (r0[hit] - r1[hit]).abs().max().item() < 1e-5
    assert mi1 < mi0
