"""Track-list comparison for the STB parity tests: rows (track id, frame, x, y, z) in
list order, compared exactly on the ids and frames and within a stated tolerance on
the positions; every difference is reported with its size."""
import numpy as np


def compare(ref_rows, gpu_rows, pos_tol: float, label: str = ""):
    """Returns (ok, max position difference, messages)."""
    a = np.asarray(ref_rows, dtype=np.float64).reshape(-1, 5)
    b = np.asarray(gpu_rows, dtype=np.float64).reshape(-1, 5)
    msgs = []
    if a.shape != b.shape:
        msgs.append(f"{label}: {len(a)} reference rows, {len(b)} rows here")
        n = min(len(a), len(b))
    else:
        n = len(a)
    ids_ok = np.array_equal(a[:n, :2], b[:n, :2])
    if not ids_ok:
        bad = np.flatnonzero(np.any(a[:n, :2] != b[:n, :2], axis=1))
        i = int(bad[0])
        msgs.append(f"{label}: first (track id, frame) difference at row {i}: reference "
                    f"{a[i, :2].astype(int).tolist()} here {b[i, :2].astype(int).tolist()} "
                    f"({len(bad)} rows differ)")
    dmax = float(np.max(np.abs(a[:n, 2:] - b[:n, 2:]))) if n else 0.0
    if dmax > pos_tol:
        i = int(np.argmax(np.max(np.abs(a[:n, 2:] - b[:n, 2:]), axis=1)))
        msgs.append(f"{label}: position difference {dmax:.3e} mm at row {i} (track "
                    f"{int(a[i, 0])}, frame {int(a[i, 1])})")
    return (a.shape == b.shape and ids_ok and dmax <= pos_tol), dmax, msgs
