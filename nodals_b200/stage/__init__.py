"""The learned pressure stage: training (train.py) and its parameters
(mpnn_params.bin, float32, NDS_MPNN_NPARAM values)."""
from pathlib import Path

import numpy as np

PARAMS = Path(__file__).resolve().parent / "mpnn_params.bin"


def load_params(path=None) -> np.ndarray:
    p = np.fromfile(path or PARAMS, dtype=np.float32)
    if p.size != 25026:
        raise ValueError(f"{path or PARAMS}: expected 25026 parameters, found {p.size}")
    return p


def init_params(seed: int = 0) -> np.ndarray:
    """Initial parameters of training: He-normal dense weights (fan-in 2 for
    the encoder, 128 for the layers), 1/sqrt(64) for the decoder, zero
    biases, skip coefficient cs = 1 (the stage starts as a scaled Jacobi step
    plus a small learned term)."""
    H = 64
    rng = np.random.default_rng(seed)
    p = np.zeros(25026)
    p[0:128] = rng.normal(0.0, 1.0, 128)
    for l in range(3):
        o = 192 + l * (H * 2 * H + H)
        p[o:o + H * 2 * H] = rng.normal(0.0, np.sqrt(2.0 / (2 * H)), H * 2 * H)
    o = 192 + 3 * (H * 2 * H + H)
    p[o:o + H] = rng.normal(0.0, 0.1 / np.sqrt(H), H)
    p[o + H + 1] = 1.0
    return p.astype(np.float32)
