"""The surrogate MLP's tcgen05 training kernels: forward and gradients against
the CPU oracle (oracle/mlp_oracle.py, float64 with the GPU's BF16 roundings),
and a training run that fits a smooth function."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mlp():
    from crysplight_b200.surrogate import MLP
    m = MLP(0, max_batch=1024, seed=3)
    yield m
    m.close()


def _batch(B, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, size=(B, 3)).astype(np.float32)
    t = (np.sin(2 * x[:, :1]) * np.cos(x[:, 1:2]) + 0.3 * x[:, 2:3]
         + 0.1 * rng.standard_normal((B, 192))).astype(np.float32)
    return x, t


def test_forward_matches_oracle(mlp):
    import torch
    from oracle import mlp_oracle
    x, _ = _batch(384, 1)
    p = mlp.get_params().astype(np.float64)
    out = mlp.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    ref, _ = mlp_oracle.forward(p, x)
    err = np.abs(out - ref).max()
    print("forward max abs err", err, "scale", np.abs(ref).max())
    assert err < 2e-3 * max(1.0, np.abs(ref).max())


def test_gradients_match_oracle(mlp):
    import torch
    from oracle import mlp_oracle
    x, t = _batch(512, 2)
    p = mlp.get_params().astype(np.float64)
    loss, g = mlp.gradient(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    rloss, rg = mlp_oracle.gradient(p, x, t)
    assert loss == pytest.approx(rloss, rel=1e-2)
    from oracle.mlp_oracle import SHAPES
    o = 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        a, b = g[o:o + n].astype(np.float64), rg[o:o + n]
        cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
        rel = float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30))
        print(name, "cos", cos, "rel", rel)
        # the oracle rounds at the same points as the GPU: only FP32 summation order differs
        assert cos > 0.99999 and rel < 2e-3
        o += n


@pytest.mark.parametrize("B,ctas", [(4096, 5), (2048, 3), (65536, 0)])
def test_gradients_persistent_tiles(B, ctas):
    """Few CTAs walking many 128-row tiles: exercises the stage ring across
    tiles and both TMEM accumulators being reused."""
    import torch
    from crysplight_b200.surrogate import MLP
    from oracle import mlp_oracle
    from oracle.mlp_oracle import SHAPES
    m = MLP(0, max_batch=B, seed=8)
    m.set_max_ctas(ctas)      # 0: one CTA per SM; 65536 rows = the training batch, 64 K-splits
    x, t = _batch(B, 4)
    p = m.get_params().astype(np.float64)
    loss, g = m.gradient(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    out = m.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    m.close()
    rloss, rg = mlp_oracle.gradient(p, x, t)
    ref, _ = mlp_oracle.forward(p, x)
    assert np.abs(out - ref).max() < 2e-3 * max(1.0, np.abs(ref).max())
    assert loss == pytest.approx(rloss, rel=1e-3)
    o = 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        a, b = g[o:o + n].astype(np.float64), rg[o:o + n]
        rel = float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30))
        print(name, "rel", rel)
        assert rel < 2e-3
        o += n


def test_training_reduces_loss():
    import torch
    from crysplight_b200.surrogate import MLP
    m = MLP(0, max_batch=4096, seed=5)
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, size=(20000, 3)).astype(np.float32)
    base = np.sin(2 * x[:, 0]) * np.cos(x[:, 1]) + 0.5 * x[:, 2] ** 2
    t = np.stack([base * (1 + 0.01 * j) for j in range(192)], axis=1).astype(np.float32)
    xt, tt = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    m.set_data(xt, tt)
    first = m.train(20, batch=4096, lr=1e-3, seed=1)
    last = m.train(400, batch=4096, lr=1e-3, seed=1)
    print("loss", first, "->", last)
    assert last < 0.05 * first
    m.close()
