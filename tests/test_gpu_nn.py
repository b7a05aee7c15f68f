"""Tensor-core convolutions of the learned warm start against the CPU oracle.

The 3x3 convolution (forward, input gradient through flipped weights, and weight/bias
gradients) runs on tcgen05 with bf16 operands and FP32 accumulation; the oracle computes the
same sums in float64 from the same bf16 values, so only the FP32 accumulation order differs.
Sizes include a pixel count that is not a multiple of the 128-row tile and images smaller
than the 3x3 halo would suggest.
"""
import numpy as np
import pytest

from oracle import nn_oracle as no

pytestmark = pytest.mark.gpu

SHAPES = [(16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 32), (48, 16), (32, 48)]


def _dev(torch, a, dtype):
    return torch.tensor(np.asarray(a, dtype=np.float32)).to(dtype).cuda().contiguous()


def _ptr(t):
    import ctypes
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pawsim_b200
    return torch, pawsim_b200.load_library()


@pytest.mark.parametrize("cin,cout", SHAPES)
@pytest.mark.parametrize("B,H,W", [(2, 20, 20), (1, 7, 45), (3, 32, 16)])
def test_conv_forward(env, cin, cout, B, H, W):
    torch, lib = env
    rng = np.random.default_rng(cin * 100 + cout + H)
    x = no.bf16(rng.standard_normal((B, H, W, cin)))
    w = no.bf16(rng.standard_normal((cout, 3, 3, cin)) / np.sqrt(9 * cin))
    b = rng.standard_normal(cout).astype(np.float32)
    for relu in (0, 1):
        ref = no.conv3x3(x, w, b.astype(np.float64), relu=bool(relu))
        xd, wd = _dev(torch, x, torch.bfloat16), _dev(torch, w, torch.bfloat16)
        bd = torch.tensor(b).cuda()
        of = torch.zeros((B, H, W, cout), dtype=torch.float32, device="cuda")
        ob = torch.zeros((B, H, W, cout), dtype=torch.bfloat16, device="cuda")
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        rc = lib.pawsim_nn_conv3x3(_ptr(xd), B, H, W, cin, _ptr(wd), _ptr(bd), cout, relu, _ptr(ob), _ptr(of),
                                   _ptr(err), None)
        torch.cuda.synchronize()
        assert rc == 0 and int(err.item()) == 0
        got = of.cpu().numpy().astype(np.float64)
        assert np.max(np.abs(got - ref)) <= 1e-5 * (1 + np.max(np.abs(ref))), np.max(np.abs(got - ref))
        # the bf16 output is the FP32 result rounded to nearest even
        gb = ob.float().cpu().numpy().astype(np.float64)
        assert np.array_equal(gb, no.bf16(got))


@pytest.mark.parametrize("cin,cout", SHAPES)
def test_conv_gradients(env, cin, cout):
    torch, lib = env
    B, H, W = 2, 24, 40           # 1920 pixels: a partial pixel chunk for the weight gradient
    rng = np.random.default_rng(7 * cin + cout)
    x = no.bf16(rng.standard_normal((B, H, W, cin)))
    w = no.bf16(rng.standard_normal((cout, 3, 3, cin)) / np.sqrt(9 * cin))
    g = no.bf16(rng.standard_normal((B, H, W, cout)))
    xd, wd, gd = _dev(torch, x, torch.bfloat16), _dev(torch, w, torch.bfloat16), _dev(torch, g, torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    # weight and bias gradients
    dw = torch.zeros((cout, 3, 3, cin), dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    assert lib.pawsim_nn_conv3x3_wgrad(_ptr(xd), _ptr(gd), B, H, W, cin, cout, _ptr(dw), _ptr(db), _ptr(err),
                                       None) == 0
    # input gradient: forward convolution of g with the flipped weights
    wt = torch.zeros((cin, 3, 3, cout), dtype=torch.bfloat16, device="cuda")
    assert lib.pawsim_nn_flip_weights(_ptr(wd), cout, cin, _ptr(wt), None) == 0
    dx = torch.zeros((B, H, W, cin), dtype=torch.float32, device="cuda")
    assert lib.pawsim_nn_conv3x3(_ptr(gd), B, H, W, cout, _ptr(wt), None, cin, 0, None, _ptr(dx), _ptr(err),
                                 None) == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    rdw, rdb = no.conv3x3_wgrad(x, g)
    rdx = no.conv3x3_dgrad(g, w)
    for got, ref in ((dw, rdw), (db, rdb), (dx, rdx)):
        got = got.cpu().numpy().astype(np.float64)
        assert np.max(np.abs(got - ref)) <= 2e-5 * (1 + np.max(np.abs(ref))), np.max(np.abs(got - ref))
    assert np.array_equal(wt.float().cpu().numpy(), no.flip(w))
