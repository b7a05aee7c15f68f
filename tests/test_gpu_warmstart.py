"""Learned warm start on the GPU.

1. The network's forward pass, loss and every parameter gradient (tcgen05 convolutions,
   pooling, upsampling, ReLU masks) against the CPU oracle with the same bf16 roundings.
2. The warm start inside the model: pairs collected during spin-up, training on the GPU,
   then V-cycles per step with the trained guess against the plain solve (which starts from
   the previous pressure, as the reference's does), on identical states; and the solution
   still meets the unchanged stopping test.
"""
import numpy as np
import pytest

from conftest import make_setup, rel_l2
from oracle import nn_oracle as no

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import pawsim_b200
    return pawsim_b200


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("B,H,W", [(2, 16, 24), (1, 32, 32)])
def test_network_gradients_match_oracle(torch_cuda, lib, B, H, W):
    torch = torch_cuda
    net = lib.Net(H, W, Bmax=B, seed=3)
    assert net.param_count == no.param_count()
    rng = np.random.default_rng(B * 100 + H)
    p = net.get_params().astype(np.float64)
    # non-zero biases so that every ReLU mask is exercised
    for l, (w, b) in enumerate(no.unflatten(p)):
        b[:] = 0.05 * rng.standard_normal(b.size)
    p = no.flatten(no.unflatten(p)).astype(np.float32)
    net.set_params(p)
    x = np.zeros((B, H, W, 16))
    x[..., :3] = rng.standard_normal((B, H, W, 3))
    t = rng.standard_normal((B, H, W)).astype(np.float32)
    xd = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).cuda().contiguous()
    td = torch.tensor(t).cuda()
    out = net.forward(xd.data_ptr(), B, H, W)
    ref_out, _ = no.net_forward(p, x, quant=True)
    assert rel_l2(out, ref_out) < 5e-3, rel_l2(out, ref_out)
    loss = net.backward(xd.data_ptr(), td.data_ptr(), B)
    ref_loss, ref_g = no.net_loss_grad(p, x, t, quant=True)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    g = net.get_grads().astype(np.float64)
    # The bf16 roundings of the backward pass amplify FP32 accumulation-order differences
    # (a flip of one rounding moves a value by one bf16 ulp). The oracle measures that noise
    # floor on itself: the same gradient with the weights perturbed at the FP32 ulp level.
    # Three draws; the floor of a vector is the largest of its three deviations.
    noise = [no.net_loss_grad(p * (1 + 2e-7 * rng.standard_normal(p.size)), x, t, quant=True)[1]
             for _ in range(3)]
    o = 0
    for ci, co, _, _ in no.LAYERS:
        for n in (co * 9 * ci, co):
            a, r = g[o:o + n], ref_g[o:o + n]
            if np.linalg.norm(r) > 0:
                floor = max(rel_l2(z[o:o + n], r) for z in noise)
                assert rel_l2(a, r) <= 2.5 * floor + 1e-2, (o, rel_l2(a, r), floor)
                assert np.dot(a, r) / (np.linalg.norm(a) * np.linalg.norm(r)) > 0.99
            o += n


def test_adam_reduces_loss(torch_cuda, lib):
    torch = torch_cuda
    B, H, W = 4, 16, 16
    net = lib.Net(H, W, Bmax=B, seed=5)
    rng = np.random.default_rng(9)
    x = np.zeros((B, H, W, 16))
    x[..., :3] = rng.standard_normal((B, H, W, 3))
    t = (0.5 * x[..., 0] - 0.25 * x[..., 1]).astype(np.float32)
    xd = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).cuda().contiguous()
    td = torch.tensor(t).cuda()
    first = net.backward(xd.data_ptr(), td.data_ptr(), B)
    for _ in range(60):
        net.adam(2e-3)
        last = net.backward(xd.data_ptr(), td.data_ptr(), B)
    assert last < 0.2 * first, (first, last)


def test_trained_warm_start_saves_vcycles(tmp_path, lib):
    kw = dict(N=128, solver=1, tol=1e-11, dt=450.0)
    _, cfg, f = make_setup(tmp_path, "gyre", **kw)
    plain = lib.Model(cfg, f)
    learn = lib.Model(cfg, f)
    learn.nn_setup(collect=True, use=False, max_pairs=256, batch=8, seed=11)
    plain.prelim()
    learn.prelim()
    n_spin, n_eval = 120, 40
    for n in range(1, n_spin + 1):
        a, b = plain.step(n), learn.step(n)
        assert a["iters"] == b["iters"]
    assert learn.nn_pairs() == n_spin - 1   # pairs need two earlier solves (prelim, step 1)
    loss = learn.nn_train(epochs=40, lr=1e-3)
    assert np.isfinite(loss)
    learn.nn_setup(collect=False, use=True)
    it_plain, it_learn, used = [], [], 0
    for n in range(n_spin + 1, n_spin + n_eval + 1):
        a, b = plain.step(n), learn.step(n)
        it_plain.append(a["iters"])
        it_learn.append(b["iters"])
        used += b["warm_start"] == 1
        assert b["warm_start"] in (1, 2)
        assert b["stop_measure"] <= 1e-11
    s_p, s_l = plain.state(), learn.state()
    for v in ("u", "v", "h"):
        assert rel_l2(s_l[v], s_p[v]) < 1e-8
    print(f"V-cycles per step: plain {np.mean(it_plain):.2f}, learned {np.mean(it_learn):.2f}; "
          f"guess used in {used}/{n_eval} steps; training loss {loss:.3e}")
    assert np.mean(it_learn) < np.mean(it_plain)
