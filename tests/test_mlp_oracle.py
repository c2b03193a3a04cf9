"""The MLP oracle pinned on the CPU: analytic gradients against central finite
differences, and its bf16 rounding against torch's conversion."""
import numpy as np
import torch

from oracle import mlp_ref as R


def test_oracle_gradients_match_finite_differences():
    for seed in (0, 1):
        assert R.fd_check(seed, n=8, n_probe=60, h=1e-3) < 1e-3


def test_oracle_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(0, 1, 100000), rng.normal(0, 1e-30, 1000),
                        [0.0, -0.0, 1.0, 3.0e38, -3.0e38, 1.00390625, 1.01171875]]).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(R.bf16(x), want)


def test_oracle_layout():
    assert R.N_PARAMS == 259076
    flat = R.init(0)
    p = R.unpack(flat)
    assert np.array_equal(R.pack(p), flat)
    assert p["W1"].shape == (256, 493) and p["b4"].shape == (4,)
