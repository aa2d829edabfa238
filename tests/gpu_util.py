"""Helpers shared by the GPU tests (device <-> numpy in column-major form)."""
import numpy as np


def to_np_colmajor(t, m, n, ld):
    """Torch 1-D device tensor holding an m x n column-major matrix (ld) -> numpy (m, n) F-order."""
    return t.view(-1)[: ld * n].view(n, ld)[:, :m].cpu().numpy().T


def from_np_colmajor(torch, a, ld=None, dtype=None, device="cuda"):
    m, n = a.shape
    ld = m if ld is None else ld
    buf = np.zeros((n, ld), dtype=a.dtype if dtype is None else dtype)
    buf[:, :m] = a.T
    return torch.from_numpy(buf.reshape(-1)).to(device)


def rel_fro(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
