"""Field-by-field proof comparison (test helper)."""
import numpy as np


def diff(a, b, path="proof"):
    if isinstance(a, dict):
        if set(a) != set(b):
            return f"{path}: keys {sorted(set(a) ^ set(b))}"
        for k in a:
            d = diff(a[k], b[k], f"{path}.{k}")
            if d:
                return d
        return None
    if isinstance(a, (list, tuple)) and not isinstance(a, np.ndarray):
        if len(a) != len(b):
            return f"{path}: length {len(a)} != {len(b)}"
        for i, (x, y) in enumerate(zip(a, b)):
            d = diff(x, y, f"{path}[{i}]")
            if d:
                return d
        return None
    if isinstance(a, np.ndarray) or isinstance(b, np.ndarray):
        x, y = np.asarray(a), np.asarray(b)
        if x.shape != y.shape or not np.array_equal(x.astype(np.uint64) if x.dtype != np.uint8 else x,
                                                    y.astype(np.uint64) if y.dtype != np.uint8 else y):
            return f"{path}: arrays differ"
        return None
    if isinstance(a, bytes) or isinstance(b, bytes):
        return None if bytes(a) == bytes(b) else f"{path}: bytes differ"
    return None if int(a) == int(b) else f"{path}: {a} != {b}"
