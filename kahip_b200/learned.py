"""The trained learned-edge-rating model shipped with the package."""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MODEL = os.path.join(HERE, "data", "rating_mpnn")
PARAMS = 27137


def load_model(path: str = MODEL):
    """(params float32[27137], metadata dict) or None when the files are absent."""
    if not os.path.exists(path + ".f32"):
        return None
    P = np.fromfile(path + ".f32", dtype="<f4").astype(np.float32)
    if P.size != PARAMS:
        raise ValueError(f"{path}.f32 holds {P.size} floats, expected {PARAMS}")
    meta = {}
    if os.path.exists(path + ".json"):
        with open(path + ".json") as f:
            meta = json.load(f)
    return P, meta
