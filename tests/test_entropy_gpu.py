"""The autofocus loss kernels (sarbp_image_entropy and its gradient) against
the same formula written with torch operations, on CUDA images."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("shape", [(1,), (7,), (1, 40, 33), (1, 512, 512), (3, 129, 257)])
def test_entropy_and_gradient_match_the_torch_formula(torch_cuda, shape):
    torch = torch_cuda
    from uncc_sar_focusing_b200 import autograd as A

    g = torch.Generator(device="cuda").manual_seed(sum(shape))
    img = torch.randn(shape, dtype=torch.complex64, device="cuda", generator=g)
    # a few exact zeros and a bright point, as focused images have
    flat = img.view(-1)
    flat[: min(3, flat.numel() - 1)] = 0
    flat[-1] *= 40
    x = img.clone().requires_grad_(True)
    y = img.clone().requires_grad_(True)
    e = A.image_entropy(x)
    e_ref = A.image_entropy_torch(y)
    assert e.dtype == torch.float32 and e.shape == ()
    assert abs(float(e.detach()) - float(e_ref.detach())) <= 2e-5 * max(1.0, abs(float(e_ref.detach())))
    (3.0 * e).backward()
    (3.0 * e_ref).backward()
    gx, gy = x.grad, y.grad
    assert gx.shape == img.shape and gx.dtype == torch.complex64
    # the gradient's natural scale: 2 |I| / sum |I|^2 per unit of log p
    w = img.abs().pow(2)
    scale = float(2.0 * img.abs().max() / w.sum())
    diff = float((gx - gy).abs().max())
    if img.numel() == 1:
        # E = 0 for every value of a one-pixel image: both gradients are rounding noise
        assert float(gx.abs().max()) < 1e-5 * scale and diff < 1e-5 * scale
    else:
        rel = float((gx - gy).abs().pow(2).sum().sqrt() / gy.abs().pow(2).sum().sqrt())
        assert rel < 1e-4, rel


def test_entropy_is_repeatable_and_captures_in_a_graph(torch_cuda):
    torch = torch_cuda
    from uncc_sar_focusing_b200 import autograd as A

    img = torch.randn((1, 256, 256), dtype=torch.complex64, device="cuda")
    a = A.image_entropy(img)
    b = A.image_entropy(img)
    assert float(a) == float(b)  # sums in a fixed order
    x = img.clone().requires_grad_(True)
    static_out = torch.empty((), dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(2):  # warm-up outside the capture
            x.grad = None
            A.image_entropy(x).backward()
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    x.grad = None
    with torch.cuda.graph(graph):
        e = A.image_entropy(x)
        e.backward()
        static_out.copy_(e.detach())
    x.grad.zero_()
    graph.replay()
    torch.cuda.synchronize()
    assert float(static_out) == float(a)
    ref = img.clone().requires_grad_(True)
    A.image_entropy(ref).backward()
    assert torch.equal(x.grad, ref.grad)


def test_entropy_of_a_focused_point_is_low(torch_cuda):
    torch = torch_cuda
    from uncc_sar_focusing_b200 import autograd as A

    point = torch.zeros((1, 64, 64), dtype=torch.complex64, device="cuda")
    point[0, 10, 20] = 1.0 + 1.0j
    flat = torch.ones((1, 64, 64), dtype=torch.complex64, device="cuda")
    assert float(A.image_entropy(point)) == pytest.approx(0.0, abs=1e-6)
    assert float(A.image_entropy(flat)) == pytest.approx(np.log(64 * 64), rel=1e-6)
