"""X' W X on the tensor cores (split BF16, `hdfe_gram_bf16x3`) against a
plain PyTorch reference of the same product in FP32 and in FP64: within
2e-5 relative (max |difference| / max |entry|) of both; row counts that fill
no chunk, part of a chunk and more chunks than SMs; weights; widths up to
the 128-column limit."""

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.mark.parametrize("N,c,weighted", [(1, 3, False), (50, 8, True), (64, 16, False),
                                          (1_000, 37, True), (200_003, 64, False),
                                          (300_000, 128, True)])
def test_gram_matches_torch(device, N, c, weighted):
    import torch
    from hdfe_stream_b200.gram import xtx
    g = torch.Generator(device="cpu").manual_seed(N + c)
    X = (torch.randn((N, c), generator=g, dtype=torch.float64) * 3.0 + 1.0).to(device)
    w = torch.rand(N, generator=g, dtype=torch.float64).to(device) * 1.5 + 0.5 if weighted \
        else None
    got = xtx(X, w)
    Xw = X if w is None else X * torch.sqrt(w)[:, None]
    ref64 = Xw.T @ Xw
    ref32 = (Xw.float().T @ Xw.float()).double()
    scale = float(ref64.abs().max())
    err = float((got - ref64).abs().max()) / scale
    err32 = float((got - ref32).abs().max()) / scale
    assert err < 2e-5, (err, err32)
    assert err32 < 2e-5, (err, err32)
    assert torch.allclose(got, got.T, rtol=0, atol=1e-6 * scale)


def test_gram_rejects_too_many_columns(device):
    import torch
    from hdfe_stream_b200.gram import xtx
    with pytest.raises(ValueError):
        xtx(torch.zeros((10, 129), dtype=torch.float64, device=device))
