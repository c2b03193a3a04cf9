"""Recall / ghost rate against generator ground truth, and output-to-output matching."""
import numpy as np
from scipy.spatial import cKDTree


def recall_ghost(found: np.ndarray, truth: np.ndarray, radius: float):
    if len(found) == 0:
        return 0.0, 0.0
    d_gt, _ = cKDTree(found).query(truth)
    d_f, _ = cKDTree(truth).query(found)
    return float(np.mean(d_gt <= radius)), float(np.mean(d_f > radius))


def match(a: np.ndarray, b: np.ndarray):
    """Distance from every point of a to its nearest point of b."""
    if len(a) == 0 or len(b) == 0:
        return np.full(len(a), np.inf)
    d, _ = cKDTree(b).query(a)
    return d
