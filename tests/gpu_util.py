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


class _DevBuf:
    """A raw device allocation seen through __cuda_array_interface__ (bytes)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1",
                                         "data": (int(ptr), False), "version": 3}


def device_bytes(torch, ptr, nbytes):
    """Copy nbytes of device memory at ptr to a numpy uint8 array."""
    return torch.as_tensor(_DevBuf(ptr, nbytes), device="cuda").cpu().numpy().copy()


def panel_slot(torch, view, slot, row0, rows, kext):
    """Rows row0 .. row0+rows of panel slot `slot` (kext elements of K each) of
    a workspace panel view, as raw bytes (rows x kext*esize), plus the FP8
    scale bytes of those rows' tiles (or None)."""
    es, ld = view["esize"], view["ld"]
    nbytes = (row0 + rows) * ld * es
    raw = device_bytes(torch, view["data"], nbytes).reshape(row0 + rows, ld * es)
    k0 = slot * view["slot_k"] * es
    out = raw[row0:row0 + rows, k0:k0 + kext * es]
    sc = None
    if view["scales"]:
        mt = -(-(row0 + rows) // 128)
        allsc = device_bytes(torch, view["scales"], mt * view["sc_ld"]).reshape(mt, view["sc_ld"])
        kt = -(-kext // 128)
        sc = allsc[row0 // 128:mt, slot * view["sc_slot"]:slot * view["sc_slot"] + kt]
    return out, sc
