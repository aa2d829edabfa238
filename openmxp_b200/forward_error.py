"""FP64 reference solutions for forward-error statements.

A checker, not part of the solve path: it factors the FP64 system that the
refinement solves (off-diagonals regenerated in FP64, diagonal d, built by
mxp_matgen_f64) with a blocked right-looking no-pivot LU made of library FP64
calls (cuSOLVER getrf without pivoting on the diagonal blocks, cuBLAS TRSM and
DGEMM through torch), then solves with blocked substitution.  The matrix is
diagonally dominant, so the no-pivot LU is stable.  Everything is in place on
one n x n FP64 buffer (8 n^2 bytes: 121 GB at n = 122880); the temporaries are
bounded by `block` x n.

Storage: column-major A (element (i, j) at i + j*lda) viewed row-major is
M = A^T.  M = L U (no pivoting) gives A = U^T L^T, so A x = b is solved as
U^T y = b (lower, non-unit) then L^T x = y (upper, unit).
"""
from __future__ import annotations


def lu_nopiv_inplace(M, block: int = 8192, chunk: int = 16384) -> None:
    """In-place no-pivot LU of the square (row-major) torch FP64 view M."""
    import torch
    n = M.shape[0]
    for k0 in range(0, n, block):
        k1 = min(k0 + block, n)
        D = M[k0:k1, k0:k1]
        LUd, _ = torch.linalg.lu_factor(D, pivot=False)
        D.copy_(LUd)
        if k1 == n:
            break
        L11 = torch.tril(LUd, -1) + torch.eye(k1 - k0, dtype=M.dtype, device=M.device)
        U11 = torch.triu(LUd)
        del LUd
        for c0 in range(k1, n, chunk):   # U12 = L11^{-1} A12, a column chunk at a time
            c1 = min(c0 + chunk, n)
            M[k0:k1, c0:c1] = torch.linalg.solve_triangular(L11, M[k0:k1, c0:c1], upper=False,
                                                            unitriangular=True)
        for r0 in range(k1, n, chunk):   # L21 = A21 U11^{-1}, a row chunk at a time
            r1 = min(r0 + chunk, n)
            M[r0:r1, k0:k1] = torch.linalg.solve_triangular(U11, M[r0:r1, k0:k1], upper=True,
                                                            left=False)
        del L11, U11
        L21 = M[k1:, k0:k1]
        U12 = M[k0:k1, k1:].contiguous()
        for r0 in range(k1, n, chunk):   # A22 -= L21 U12, a row chunk at a time, in place
            r1 = min(r0 + chunk, n)
            M[r0:r1, k1:].addmm_(L21[r0 - k1:r1 - k1], U12, alpha=-1.0)
        del U12


def solve_factored(M, b, block: int = 8192):
    """x with A x = b from the in-place factors M = L U of M = A^T (see module doc)."""
    import torch
    n = M.shape[0]
    y = b.clone()
    for i0 in range(0, n, block):               # U^T y = b  (forward)
        i1 = min(i0 + block, n)
        Uii = torch.triu(M[i0:i1, i0:i1])
        y[i0:i1] = torch.linalg.solve_triangular(Uii.t(), y[i0:i1, None], upper=False)[:, 0]
        if i1 < n:
            y[i1:] -= M[i0:i1, i1:].t() @ y[i0:i1]
    x = y
    for i0 in reversed(range(0, n, block)):     # L^T x = y  (backward, unit diagonal)
        i1 = min(i0 + block, n)
        Lii = torch.tril(M[i0:i1, i0:i1], -1) + torch.eye(i1 - i0, dtype=M.dtype, device=M.device)
        x[i0:i1] = torch.linalg.solve_triangular(Lii.t(), x[i0:i1, None], upper=True,
                                                 unitriangular=True)[:, 0]
        if i0 > 0:
            x[:i0] -= M[i0:i1, :i0].t() @ x[i0:i1]
    return x


def reference_solution(n: int, seed: int, diag_rule: int, rhs, block: int = 8192):
    """FP64 solution of the generated system for right-hand side rhs (torch FP64, device)."""
    import torch

    from . import matgen_f64
    A = matgen_f64(n, seed, diag_rule)
    M = A.view(n, n)            # row-major view of column-major A: M = A^T
    lu_nopiv_inplace(M, block=block)
    x = solve_factored(M, rhs.to(torch.float64), block=block)
    del A, M
    return x


def forward_error(x, x_ref) -> float:
    """||x - x_ref||_inf / ||x_ref||_inf."""
    return float((x - x_ref).abs().max() / x_ref.abs().max())
