"""CPU stand-in for openmxp_b200.grid.CudaBackend, for the multi-process gloo
tests of the 2D block-cyclic driver.  Test infrastructure only: every step is
the oracle's restatement (oracle/mxp_oracle.c) on torch CPU tensors, so the
driver's schedule, ownership and collectives run unchanged across CPU ranks.
Panels stay FP32 here (4-byte elements) in the product's panel layout (row i
of a panel holds its K values contiguously, ld = b), so the driver's row
offsets into them work unchanged; the Schur update quantises them to the form
(orc_schur_update), exactly as the oracle's single-process LU does.  The
panel products of the TRSM by inverse are the same routine on a zero C
(C = -quant(P) quant(X), negated back exactly): the operands quantised as the
tensor-core products quantise them (BF16, or hi|hi|lo x hi|lo|hi split BF16)
and summed in FP32 in a fixed order, so every element's value depends only
on its own row or column, whatever the grid.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from oracle import oracle as O
from oracle.blocked import FORM_BF16


class OracleBackend:
    def __init__(self, b: int, form: int):
        if form not in (O.FORM_FP16, O.FORM_BF16X2, O.FORM_FP8):
            raise ValueError("CPU backend: FP16, BF16X2 and FP8 forms")
        if form == O.FORM_FP8 and b % 128:
            # the E4M3 scales are per 128 x 128 tile of the operand the
            # routine is given: with b a multiple of 128 those tiles are whole
            # blocks, the same on every grid and in the one-process LU
            raise ValueError("CPU backend: the FP8 form needs b % 128 == 0")
        self.b, self.form = b, form
        self.L = O.lib()
        self._full = {}

    def empty(self, numel, dtype):
        return torch.empty(max(int(numel), 1), dtype=dtype)

    def zeros(self, numel, dtype):
        return torch.zeros(max(int(numel), 1), dtype=dtype)

    @staticmethod
    def _p(t, off=0):
        return C.c_void_p(t.data_ptr() + int(off) * t.element_size())

    def panel_layout(self, rows, b):
        return b, 4, 0

    def _matrix(self, n, seed, rule):
        key = (n, seed, rule)
        if key not in self._full:
            A, d, _, rhs = O.matgen(n, seed, rule)
            self._full[key] = (A, d, rhs, O.matgen_f64(n, seed, d))
        return self._full[key]

    def vectors(self, n, seed, rule):
        self._rule = rule
        _, d, rhs, _ = self._matrix(n, seed, rule)
        return torch.from_numpy(d.copy()), torch.from_numpy(rhs.copy())

    @staticmethod
    def _rows(n, b, nproc, me):
        return np.concatenate([np.arange(I * b, (I + 1) * b) for I in range(me, n // b, nproc)] or
                              [np.zeros(0, np.int64)])

    def matgen_local(self, g, n, b, seed, d, A, lda):
        full, _, _, _ = self._matrix(n, seed, self._rule)
        rows, cols = self._rows(n, b, g.nprow, g.myrow), self._rows(n, b, g.npcol, g.mycol)
        loc = full[np.ix_(rows, cols)]
        A.numpy()[: lda * len(cols)].reshape(len(cols), lda)[:, : len(rows)] = loc.T

    def getrf_inv(self, b, A, off, lda, XU, XL):
        assert self.L.orc_getrf_nopiv(b, b, self._p(A, off), lda) == 0
        self.L.orc_tri_inverses(b, self._p(A, off), lda, self._p(XU), self._p(XL), b, 0)

    def trsm_right_upper(self, m, b, U, ldu, A, off, lda):
        self.L.orc_trsm_runn(m, b, self._p(U), ldu, self._p(A, off), lda)

    def trsm_left_lower_unit(self, b, ncols, Lm, ldl, A, off, lda):
        self.L.orc_trsm_llnu(b, ncols, self._p(Lm), ldl, self._p(A, off), lda)

    def _product(self, m, ncols, P, ldp, X, ldx, single, A, off, lda):
        """A block (m x ncols at off) = P (m x K) X (K x ncols), K = b, both
        quantised as the TRSM by inverse quantises them."""
        tform = FORM_BF16 if single else O.FORM_BF16X2
        C = np.zeros((ncols, m), np.float32)  # column-major m x ncols
        self.L.orc_schur_update(tform, m, ncols, self.b, P, ldp, X, ldx, C.ctypes.data, m)
        A.as_strided((ncols, m), (lda, 1), off).numpy()[:] = -C

    def trsm_inv_right_upper(self, m, b, XU, ldx, A, off, lda, single):
        P = np.array(self._block(A, off, lda, m, b))  # [k, i]: column-major m x b, ld = m
        self._product(m, b, P.ctypes.data, m, self._p(XU), ldx, single, A, off, lda)

    def trsm_inv_left_lower(self, b, ncols, XL, ldx, A, off, lda, single):
        B = np.array(self._block(A, off, lda, b, ncols))  # [j, k]: column-major b x ncols, ld = b
        self._product(b, ncols, self._p(XL), ldx, B.ctypes.data, b, single, A, off, lda)

    def _block(self, A, off, lda, m, ncols):
        return A.as_strided((ncols, m), (lda, 1), off).numpy()  # [c, r]

    def cast_left(self, m, b, A, off, lda, out, ldk, scales):
        # row i of the L panel: its b values of K
        out.view(torch.float32)[: m * b].numpy().reshape(m, b)[:] = self._block(A, off, lda, m, b).T

    def cast_right(self, ncols, b, A, off, lda, out, ldk, scales):
        # row j of the R panel: column j of the U panel, its b values of K
        out.view(torch.float32)[: ncols * b].numpy().reshape(ncols, b)[:] = self._block(A, off, lda, b, ncols)

    def schur(self, m, ncols, b, Lp, ldl, ls, Rp, ldr, rs, A, off, lda):
        # orc_schur_update takes L column-major (m x b) and U as K x ncols
        # column-major, which is the R panel's layout (ld = b)
        Lcm = np.asfortranarray(Lp.view(torch.float32)[: m * b].numpy().reshape(m, b))
        self.L.orc_schur_update(self.form, m, ncols, b, Lcm.ctypes.data, m,
                                self._p(Rp.view(torch.float32)), b, self._p(A, off), lda)

    def otf_gemv_local(self, g, n, b, seed, d, alpha, x, y):
        _, _, _, A64 = self._matrix(n, seed, self._rule)
        rows, cols = self._rows(n, b, g.nprow, g.myrow), self._rows(n, b, g.npcol, g.mycol)
        yn, xn = y.numpy(), x.numpy()
        yn[rows] += alpha * (A64[np.ix_(rows, cols)] @ xn[cols])

    def block_gemv(self, m, ncols, alpha, A, off, lda, x, xoff, beta, y, yoff):
        Ab = A.as_strided((m, ncols), (1, lda), off).numpy().astype(np.float64)
        yn = y.numpy()
        acc = Ab @ x.numpy()[xoff:xoff + ncols]
        yn[yoff:yoff + m] = alpha * acc if beta == 0.0 else alpha * acc + beta * yn[yoff:yoff + m]

    def close(self):
        pass
