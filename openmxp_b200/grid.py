"""2D block-cyclic multi-GPU solve: one system of order n factored and refined
by a P x Q grid of processes, one per GPU.

This is the reference's production layout (panel_trf.hpp:470-867 over a Grid,
grid.hpp:25-80; its gdirect look-ahead variant is panel_trf_gdirect.hpp:
593-1192) rebuilt on this library's kernels, with torch.distributed (NCCL
between GPUs, gloo for the CPU tests) in place of MPI:

* layout (Panels, panel.hpp:189-215): global b x b block (I, J) lives on the
  process at grid coordinates (I mod P, J mod Q), which keeps its blocks in one
  column-major local matrix at local block (I div P, J div Q); ranks are laid
  out column-major on the grid (the reference's default "Global Column Major"
  map: row = rank mod P, column = rank div P);
* generation (panel_matgen_dev, matgen.hpp:84-117): every process fills its
  own blocks (mxp_matgen_local), d and the right-hand side are whole-length
  vectors on every process;
* LU step k (panel_lu_async_wGPU's loop body): the owner of block (k, k)
  factors it (mxp_getrf_nopiv_inv, keeping both triangular inverses for the
  refinement).  Panel solves by inverse (trsm "split" or "single", the
  reference's -alt path, panel_trf_gdirect.hpp:73-142): inv(U_kk) goes along
  the owner's process column and inv(L_kk) along its process row, and the
  processes of column k mod Q form their rows of the L panel as A21 inv(U_kk)
  and those of row k mod P their columns of the U panel as inv(L_kk) A12 on
  the tensor cores (mxp_trsm_inv_*); with trsm "strsm" the factored block goes
  along both (broadcast_pivlu, panel_trf.hpp:60-107) for SIMT STRSMs.  The
  panels are cast, the low-precision L panel is broadcast along each process
  row and the R panel along each process column (broadcast_left/right_panels,
  panel_trf.hpp:127-170), and every process applies the tcgen05 Schur update
  to its trailing local blocks.  A received panel lands in the process's own
  device memory before the Schur kernel reads it (no kernel reads another
  GPU's memory);
* look-ahead (depth 1, panel_trf.hpp:470-867 and the gdirect driver's
  panel_trf_gdirect.hpp:777-1172): step k's update is applied first to block
  column k+1 and block row k+1, panel k+1 is formed and its broadcasts are
  started, and only then is the rest of step k's trailing update applied, so
  the panel broadcasts run beside it (asynchronous collectives on the
  communication stream; two sets of panel buffers).  Every element still
  receives its updates in step order, so the factors are the same bit for bit
  with and without it;
* refinement (iterative_refinement.hpp:141-171): x, r and the corrections are
  whole-length FP64 vectors on every process; the residual is the local
  regenerating GEMV (mxp_otf_gemv_local) summed over all processes
  (panel_gemv.hpp:177 sums over the process row; here every process adds its
  rows' partial sums into one whole-length vector); the triangular solves are
  block substitutions over the grid (trsvL_h / trsvU_h, panel_trsv.hpp:
  308-597): per block, the partial sums of the owner's process row are reduced
  to the owner, which applies the stored inverse of the diagonal block with
  one refinement step, and the new block of the solution is broadcast.

Every process issues the same collectives in the same order; a collective
runs only inside the row or column group whose members all take part
(membership and message sizes are uniform across each group by construction).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

FORM_FP16, FORM_BF16X2, FORM_FP8 = 0, 1, 2
EPS64 = 2.0 ** -53


def local_extent(n: int, b: int, nproc: int, me: int) -> int:
    """Rows (or columns) of the local matrix of grid coordinate `me` among
    `nproc`: b times the number of block indices I < n/b with I mod nproc == me
    (mirrors mxp_local_extent)."""
    if n <= 0 or b <= 0 or n % b or nproc <= 0 or not 0 <= me < nproc:
        raise ValueError("local_extent: bad arguments")
    nb = n // b
    return (nb - me + nproc - 1) // nproc * b if nb > me else 0


def blocks_upto(k: int, nproc: int, me: int) -> int:
    """Number of block indices I <= k with I mod nproc == me (so the local
    blocks of global index > k start at local block blocks_upto(k))."""
    return 0 if k < me else (k - me) // nproc + 1


@dataclass
class ProcessGrid:
    """P x Q process grid over torch.distributed ranks (column-major), with
    one group per process row (hcomm in grid.hpp) and one per process column
    (vcomm).  With a single process no collective is issued."""
    nprow: int
    npcol: int
    rank: int = 0
    dist: object = None
    row_group: object = None
    col_group: object = None

    def __post_init__(self):
        if self.nprow <= 0 or self.npcol <= 0:
            raise ValueError("grid dimensions must be positive")
        size = self.nprow * self.npcol
        if self.dist is not None and self.dist.is_initialized():
            if self.dist.get_world_size() != size:
                raise ValueError(f"grid {self.nprow}x{self.npcol} needs {size} ranks, "
                                 f"world has {self.dist.get_world_size()}")
            self.rank = self.dist.get_rank()
            # every rank creates every group, in the same order
            rows = [self.dist.new_group([self.rank_of(r, c) for c in range(self.npcol)])
                    for r in range(self.nprow)]
            cols = [self.dist.new_group([self.rank_of(r, c) for r in range(self.nprow)])
                    for c in range(self.npcol)]
            self.row_group, self.col_group = rows[self.myrow], cols[self.mycol]
        elif size != 1:
            raise ValueError("a grid of more than one process needs torch.distributed")

    @property
    def myrow(self) -> int:
        return self.rank % self.nprow

    @property
    def mycol(self) -> int:
        return self.rank // self.nprow

    @property
    def size(self) -> int:
        return self.nprow * self.npcol

    def rank_of(self, prow: int, pcol: int) -> int:
        return prow + pcol * self.nprow

    # collectives (no-ops on a one-process grid or a one-member group).  With
    # async_op the broadcast is only started: the returned handles (a list,
    # empty when nothing was issued) are waited on before the tensor is used.
    def bcast_row(self, t, root_col: int, async_op: bool = False):
        if self.npcol > 1:
            w = self.dist.broadcast(t, src=self.rank_of(self.myrow, root_col), group=self.row_group,
                                    async_op=async_op)
            return [w] if async_op else []
        return []

    def bcast_col(self, t, root_row: int, async_op: bool = False):
        if self.nprow > 1:
            w = self.dist.broadcast(t, src=self.rank_of(root_row, self.mycol), group=self.col_group,
                                    async_op=async_op)
            return [w] if async_op else []
        return []

    def reduce_row(self, t, root_col: int) -> None:
        if self.npcol > 1:
            self.dist.reduce(t, dst=self.rank_of(self.myrow, root_col), op=self.dist.ReduceOp.SUM,
                             group=self.row_group)

    def bcast_all(self, t, root: int) -> None:
        if self.size > 1:
            self.dist.broadcast(t, src=root)

    def sum_all(self, t) -> None:
        if self.size > 1:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)


class CudaBackend:
    """The product backend: every step on this library's kernels through the
    C ABI, on the current CUDA device and stream."""

    def __init__(self, b: int, form: int):
        import torch

        from . import FORMS, Workspace, lib  # noqa: F401  (fails loudly without libmxp.so)
        self.torch = torch
        self.lib = lib()
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.form = form
        # on this process's GPU (one process per GPU: the current device)
        self.ws = Workspace(b, b, form, device=self.dev.index)

    # storage
    def empty(self, numel: int, dtype):
        return self.torch.empty(max(int(numel), 1), dtype=dtype, device=self.dev)

    def zeros(self, numel: int, dtype):
        return self.torch.zeros(max(int(numel), 1), dtype=dtype, device=self.dev)

    def _p(self, t, off: int = 0) -> int:
        return t.data_ptr() + int(off) * t.element_size()

    def _s(self) -> int:
        return self.torch.cuda.current_stream().cuda_stream

    def _ck(self, status: int) -> None:
        from . import check
        check(status)

    def panel_layout(self, rows: int, b: int):
        """(row pitch in elements, element bytes, scale bytes) of a cast panel."""
        kmul = 3 if self.form == FORM_BF16X2 else 1
        es = 1 if self.form == FORM_FP8 else 2
        per = 16 // es
        ldk = -(-b * kmul // per) * per
        sc = (-(-rows // 128)) * (-(-b // 128)) if self.form == FORM_FP8 else 0
        return ldk, es, sc

    # generation
    def vectors(self, n: int, seed: int, diag_rule: int):
        d = self.empty(n, self.torch.float64)
        rhs = self.empty(n, self.torch.float64)
        self._ck(self.lib.mxp_matgen(n, seed, diag_rule, None, n, self._p(d), None, self._p(rhs), self._s()))
        return d, rhs

    def matgen_local(self, g: ProcessGrid, n: int, b: int, seed: int, d, A, lda: int) -> None:
        self._ck(self.lib.mxp_matgen_local(n, b, seed, g.nprow, g.npcol, g.myrow, g.mycol, self._p(d),
                                           self._p(A), lda, self._s()))

    # LU pieces
    def getrf_inv(self, b: int, A, off: int, lda: int, XU, XL) -> None:
        self._ck(self.lib.mxp_getrf_nopiv_inv(b, self._p(A, off), lda, self._p(XU), self._p(XL), b,
                                              self.ws.handle, self._s()))

    def reserve(self, rows: int) -> None:
        """Make the workspace hold panel products of up to `rows` rows (the
        TRSM by inverse stages its operands there)."""
        if rows > self.ws.n - self.ws.b:
            from . import Workspace
            b = self.ws.b
            self.ws.close()
            self.ws = Workspace(rows + b, b, self.form, device=self.dev.index)

    def trsm_right_upper(self, m: int, b: int, U, ldu: int, A, off: int, lda: int) -> None:
        self._ck(self.lib.mxp_trsm_right_upper(m, b, self._p(U), ldu, self._p(A, off), lda, self._s()))

    def trsm_inv_right_upper(self, m: int, b: int, XU, ldx: int, A, off: int, lda: int, single: bool) -> None:
        self._ck(self.lib.mxp_trsm_inv_right_upper(m, b, self._p(XU), ldx, self._p(A, off), lda, int(single),
                                                   self.ws.handle, self._s()))

    def trsm_inv_left_lower(self, b: int, ncols: int, XL, ldx: int, A, off: int, lda: int, single: bool) -> None:
        self._ck(self.lib.mxp_trsm_inv_left_lower(b, ncols, self._p(XL), ldx, self._p(A, off), lda, int(single),
                                                  self.ws.handle, self._s()))

    def trsm_left_lower_unit(self, b: int, ncols: int, L, ldl: int, A, off: int, lda: int) -> None:
        self._ck(self.lib.mxp_trsm_left_lower_unit(b, ncols, self._p(L), ldl, self._p(A, off), lda, self._s()))

    def cast_left(self, m: int, b: int, A, off: int, lda: int, out, ldk: int, scales) -> None:
        self._ck(self.lib.mxp_panel_cast_left(self.form, m, b, self._p(A, off), lda, self._p(out), ldk,
                                              self._p(scales) if scales is not None else None, self._s()))

    def cast_right(self, ncols: int, b: int, A, off: int, lda: int, out, ldk: int, scales) -> None:
        self._ck(self.lib.mxp_panel_cast_right(self.form, ncols, b, self._p(A, off), lda, self._p(out), ldk,
                                               self._p(scales) if scales is not None else None, self._s()))

    def schur(self, m: int, ncols: int, b: int, Lp, ldl: int, ls, Rp, ldr: int, rs, A, off: int, lda: int) -> None:
        self._ck(self.lib.mxp_schur_update(self.form, m, ncols, b, self._p(Lp), ldl,
                                           self._p(ls) if ls is not None else None, self._p(Rp), ldr,
                                           self._p(rs) if rs is not None else None, self._p(A, off), lda,
                                           self.ws.handle, self._s()))

    # refinement pieces
    def otf_gemv_local(self, g: ProcessGrid, n: int, b: int, seed: int, d, alpha: float, x, y) -> None:
        self._ck(self.lib.mxp_otf_gemv_local(n, b, seed, g.nprow, g.npcol, g.myrow, g.mycol, self._p(d), alpha,
                                             self._p(x), self._p(y), self._s()))

    def block_gemv(self, m: int, ncols: int, alpha: float, A, off: int, lda: int, x, xoff: int, beta: float, y,
                   yoff: int) -> None:
        self._ck(self.lib.mxp_block_gemv(m, ncols, alpha, self._p(A, off), lda, self._p(x, xoff), beta,
                                         self._p(y, yoff), self._s()))

    def close(self) -> None:
        self.ws.close()


@dataclass
class GridStats:
    iterations: int = 0
    converged: bool = False
    hpl_harness: float = math.inf
    residual: float = math.inf
    history: list = field(default_factory=list)


class BlockCyclicSolver:
    """One system of order n over a P x Q grid: generation, LU, classic
    refinement.  `backend` supplies the per-process kernels (CudaBackend on
    GPUs); torch tensors hold every buffer."""

    TRSMS = ("split", "single", "strsm")

    def __init__(self, grid: ProcessGrid, n: int, b: int, seed: int, backend, form: int = FORM_FP16,
                 diag_rule: int = 0, trsm: str = "split", lookahead: bool = True):
        """trsm: the panel solves, "split" (three split-BF16 products against
        the FP32 inverse, near FP32), "single" (one BF16 product) or "strsm"
        (FP32 SIMT triangular solves); lookahead: depth-1 look-ahead (needs
        b % 128 == 0 in the FP8 form, whose panel scales are per 128 rows;
        off otherwise)."""
        if n <= 0 or b <= 0 or n % b:
            raise ValueError("n must be a positive multiple of b")
        if trsm not in self.TRSMS:
            raise ValueError(f"trsm must be one of {self.TRSMS}")
        import torch
        self.torch = torch
        self.g, self.n, self.b, self.seed, self.form = grid, n, b, seed, form
        self.diag_rule = diag_rule
        self.trsm = trsm
        self.lookahead = bool(lookahead) and (form != FORM_FP8 or b % 128 == 0)
        self.be = backend
        self.nb = n // b
        self.mloc = local_extent(n, b, grid.nprow, grid.myrow)
        self.nloc = local_extent(n, b, grid.npcol, grid.mycol)
        self.lda = max(self.mloc, 1)
        if trsm != "strsm" and hasattr(backend, "reserve"):
            backend.reserve(max(self.mloc, self.nloc))
        self.A = backend.empty(self.lda * self.nloc, torch.float32)
        self.d, self.rhs = backend.vectors(n, seed, diag_rule)
        if self.mloc and self.nloc:
            backend.matgen_local(grid, n, b, seed, self.d, self.A, self.lda)
        ldk, es, nsc = backend.panel_layout(self.mloc, b)
        self.ldk_l, self.es = ldk, es
        ldk_r, _, nsc_r = backend.panel_layout(self.nloc, b)
        self.ldk_r = ldk_r
        self.sct = -(-b // 128)  # FP8 scale bytes per 128 panel rows
        nbuf = 2 if self.lookahead else 1
        self.Lp = [backend.empty(self.mloc * ldk * es, torch.uint8) for _ in range(nbuf)]
        self.Ls = [backend.empty(nsc, torch.uint8) if nsc else None for _ in range(nbuf)]
        self.Rp = [backend.empty(self.nloc * ldk_r * es, torch.uint8) for _ in range(nbuf)]
        self.Rs = [backend.empty(nsc_r, torch.uint8) if nsc_r else None for _ in range(nbuf)]
        self.D = backend.empty(b * b, torch.float32)
        self.XUb = backend.empty(b * b, torch.float32)  # inv(U_kk) on the owner's process column
        self.XLb = backend.empty(b * b, torch.float32)  # inv(L_kk) on the owner's process row
        self.diag = {}  # k -> (unit-lower L_kk, U_kk, inv(L_kk), inv(U_kk)) on the owner

    def regenerate(self) -> None:
        """Refill the local blocks (the factorisation overwrites them)."""
        if self.mloc and self.nloc:
            self.be.matgen_local(self.g, self.n, self.b, self.seed, self.d, self.A, self.lda)
        self.diag.clear()

    # --- ownership -------------------------------------------------------
    def owner(self, k: int) -> tuple[int, int]:
        return k % self.g.nprow, k % self.g.npcol

    def _off(self, lrow: int, lcol: int) -> int:
        return lrow + lcol * self.lda

    # --- LU ----------------------------------------------------------------
    def _start(self, k: int) -> tuple[int, int, int, int]:
        """(first local row of the blocks below k, first local column of the
        blocks right of k, their counts of rows and columns)."""
        g, b = self.g, self.b
        r0 = blocks_upto(k, g.nprow, g.myrow) * b
        c0 = blocks_upto(k, g.npcol, g.mycol) * b
        return r0, c0, self.mloc - r0, self.nloc - c0

    def _form_panel(self, k: int, buf: int) -> list:
        """Step k's panels into panel buffer `buf`: diagonal factor (and
        inverses) on the owner, the triangle or its inverse along the owner's
        row and column, the panel solves, the casts; then the panel
        broadcasts are started.  Returns their handles."""
        torch, g, b, be = self.torch, self.g, self.b, self.be
        io, jo = self.owner(k)
        lik, ljk = k // g.nprow, k // g.npcol
        r0, c0, mb, nr = self._start(k)
        inv = self.trsm != "strsm"
        single = self.trsm == "single"
        if g.myrow == io and g.mycol == jo:
            off = self._off(lik * b, ljk * b)
            XU, XL = be.empty(b * b, torch.float32), be.empty(b * b, torch.float32)
            be.getrf_inv(b, self.A, off, self.lda, XU, XL)
            blk = self.A.as_strided((b, b), (1, self.lda), off)  # [r, c] of the factored block
            self.D.view(b, b).copy_(blk.t())                     # D column-major, ld = b
            Dm = self.D.view(b, b).t()                           # Dm[r, c]
            Lf = torch.tril(Dm, -1) + torch.eye(b, dtype=Dm.dtype, device=Dm.device)
            Uf = torch.triu(Dm)
            # column-major copies for the block GEMVs
            self.diag[k] = (Lf.t().contiguous().view(-1), Uf.t().contiguous().view(-1), XL, XU)
            if inv:
                self.XUb.copy_(XU)
                self.XLb.copy_(XL)
        if inv:
            if g.mycol == jo:
                g.bcast_col(self.XUb, io)  # inv(U_kk) to the L-panel products of this process column
            if g.myrow == io:
                g.bcast_row(self.XLb, jo)  # inv(L_kk) to the U-panel products of this process row
        else:
            if g.myrow == io:
                g.bcast_row(self.D, jo)    # L_kk to the U-panel solves of this process row
            if g.mycol == jo:
                g.bcast_col(self.D, io)    # U_kk to the L-panel solves of this process column
        Lp, Ls, Rp, Rs = self.Lp[buf], self.Ls[buf], self.Rp[buf], self.Rs[buf]
        if g.mycol == jo and mb > 0:
            off = self._off(r0, ljk * b)
            if inv:
                be.trsm_inv_right_upper(mb, b, self.XUb, b, self.A, off, self.lda, single)
            else:
                be.trsm_right_upper(mb, b, self.D, b, self.A, off, self.lda)
            be.cast_left(mb, b, self.A, off, self.lda, Lp, self.ldk_l, Ls)
        if g.myrow == io and nr > 0:
            off = self._off(lik * b, c0)
            if inv:
                be.trsm_inv_left_lower(b, nr, self.XLb, b, self.A, off, self.lda, single)
            else:
                be.trsm_left_lower_unit(b, nr, self.D, b, self.A, off, self.lda)
            be.cast_right(nr, b, self.A, off, self.lda, Rp, self.ldk_r, Rs)
        works = []
        if mb > 0:  # uniform across the process row
            works += g.bcast_row(Lp[: mb * self.ldk_l * self.es], jo, async_op=True)
            if Ls is not None:
                works += g.bcast_row(Ls[: (-(-mb // 128)) * self.sct], jo, async_op=True)
        if nr > 0:  # uniform across the process column
            works += g.bcast_col(Rp[: nr * self.ldk_r * self.es], io, async_op=True)
            if Rs is not None:
                works += g.bcast_col(Rs[: (-(-nr // 128)) * self.sct], io, async_op=True)
        return works

    def _schur(self, k: int, buf: int, dr: int, dc: int, m: int, ncols: int) -> None:
        """Step k's update of the trailing rows [r0 + dr, r0 + dr + m) x
        columns [c0 + dc, c0 + dc + ncols) (r0, c0: the first trailing local
        row and column), from panel rows dr.. and dc.. of buffer `buf`."""
        if m <= 0 or ncols <= 0:
            return
        r0, c0, _, _ = self._start(k)
        es = self.es
        Ls, Rs = self.Ls[buf], self.Rs[buf]
        self.be.schur(m, ncols, self.b, self.Lp[buf][dr * self.ldk_l * es:], self.ldk_l,
                      None if Ls is None else Ls[(dr // 128) * self.sct:],
                      self.Rp[buf][dc * self.ldk_r * es:], self.ldk_r,
                      None if Rs is None else Rs[(dc // 128) * self.sct:],
                      self.A, self._off(r0 + dr, c0 + dc), self.lda)

    def factor(self) -> None:
        g, b = self.g, self.b
        works = self._form_panel(0, 0)
        for k in range(self.nb):
            for w in works:
                w.wait()
            works = []
            buf = k % 2 if self.lookahead else 0
            _, _, mb, nr = self._start(k)
            nxt = k + 1 < self.nb
            if nxt and self.lookahead:
                # block column k+1 and block row k+1 first (those of this
                # process, when it owns them), then panel k+1, then the rest
                ac = b if g.mycol == (k + 1) % g.npcol else 0
                ar = b if g.myrow == (k + 1) % g.nprow else 0
                self._schur(k, buf, 0, 0, mb, ac)
                self._schur(k, buf, 0, ac, ar, nr - ac)
                works = self._form_panel(k + 1, (k + 1) % 2)
                self._schur(k, buf, ar, ac, mb - ar, nr - ac)
            else:
                self._schur(k, buf, 0, 0, mb, nr)
                if nxt:
                    works = self._form_panel(k + 1, 0)

    # --- triangular solves over the grid ----------------------------------
    def _diag_solve(self, k: int, t, lower: bool):
        """x = T_kk^{-1} t with the stored inverse X and one refinement step,
        x = x1 + X (t - T x1) (T unit lower for L, upper for U)."""
        be, b = self.be, self.b
        Lf, Uf, XL, XU = self.diag[k]
        T, X = (Lf, XL) if lower else (Uf, XU)
        x = be.zeros(b, self.torch.float64)
        be.block_gemv(b, b, 1.0, X, 0, b, t, 0, 0.0, x, 0)
        w = t.clone()
        be.block_gemv(b, b, -1.0, T, 0, b, x, 0, 1.0, w, 0)
        be.block_gemv(b, b, 1.0, X, 0, b, w, 0, 1.0, x, 0)
        return x

    def _trsv(self, r, lower: bool):
        torch, g, b, be = self.torch, self.g, self.b, self.be
        z = be.zeros(self.n, torch.float64)
        s = be.zeros(self.mloc, torch.float64)   # this process's partial sums, by local row
        order = range(self.nb) if lower else range(self.nb - 1, -1, -1)
        for k in order:
            io, jo = self.owner(k)
            lik, ljk = k // g.nprow, k // g.npcol
            zk = z[k * b:(k + 1) * b]
            if g.myrow == io:
                part = s[lik * b:(lik + 1) * b].clone()
                g.reduce_row(part, jo)
                if g.mycol == jo:
                    zk.copy_(self._diag_solve(k, r[k * b:(k + 1) * b] - part, lower))
            g.bcast_all(zk, g.rank_of(io, jo))
            if g.mycol == jo:
                if lower:   # rows of the blocks below k: s += L(:, k) z_k
                    r0 = blocks_upto(k, g.nprow, g.myrow) * b
                    if self.mloc > r0:
                        be.block_gemv(self.mloc - r0, b, 1.0, self.A, self._off(r0, ljk * b), self.lda, z, k * b,
                                      1.0, s, r0)
                else:       # rows of the blocks above k: s += U(:, k) z_k
                    ra = blocks_upto(k - 1, g.nprow, g.myrow) * b
                    if ra > 0:
                        be.block_gemv(ra, b, 1.0, self.A, self._off(0, ljk * b), self.lda, z, k * b, 1.0, s, 0)
        return z

    def lu_solve(self, r):
        """z = U^{-1} L^{-1} r over the grid (r, z whole-length on every process)."""
        return self._trsv(self._trsv(r, True), False)

    # --- refinement ----------------------------------------------------------
    def residual(self, x):
        """r = b - A x with A regenerated (every process gets all of r)."""
        y = self.be.zeros(self.n, self.torch.float64)
        if self.mloc and self.nloc:
            self.be.otf_gemv_local(self.g, self.n, self.b, self.seed, self.d, 1.0, x, y)
        self.g.sum_all(y)
        return self.rhs - y

    def refine(self, maxit: int = 50) -> tuple[object, GridStats]:
        """Classic refinement (iterative_refinement.hpp:141-171): x0 = b ./ d,
        stop at scaled residual ||r|| / ((||A|| ||x|| + ||b||) n eps) < 16 with
        ||A|| = 2 max d (panel_norm.hpp:129-135)."""
        st = GridStats()
        x = self.rhs / self.d
        norma = 2.0 * float(self.d.abs().max())
        normb = float(self.rhs.abs().max())
        for it in range(maxit + 1):
            r = self.residual(x)
            resid = float(r.abs().max())
            hpl = resid / ((norma * float(x.abs().max()) + normb) * self.n * EPS64)
            st.history.append(hpl)
            st.residual, st.hpl_harness, st.iterations = resid, hpl, it
            if hpl < 16.0:
                st.converged = True
                break
            if it == maxit:
                break
            x = x + self.lu_solve(r)
        return x, st

    def gather_factors(self, root: int = 0):
        """The whole factored matrix on `root` (column-major n x n tensor on
        the backend's device), None elsewhere; for checks, not on the solve
        path."""
        torch, g, b = self.torch, self.g, self.b
        n = self.n
        full = self.be.zeros(n * n, torch.float32) if g.rank == root else None
        for pr in range(g.nprow):
            for pc in range(g.npcol):
                src = g.rank_of(pr, pc)
                ml, nl = local_extent(n, b, g.nprow, pr), local_extent(n, b, g.npcol, pc)
                if ml == 0 or nl == 0:
                    continue
                if src == g.rank:
                    buf = self.A[: ml * nl].clone() if self.lda == ml else None
                else:
                    buf = self.be.empty(ml * nl, torch.float32)
                if g.size > 1:
                    if src == g.rank and g.rank != root:
                        g.dist.send(buf, dst=root)
                    elif g.rank == root and src != root:
                        g.dist.recv(buf, src=src)
                if g.rank == root:
                    Lm = buf.view(nl, ml)  # Lm[lc, lr]
                    F = full.view(n, n)    # F[c, r]
                    for lcb in range(nl // b):
                        J = lcb * g.npcol + pc
                        for lrb in range(ml // b):
                            I = lrb * g.nprow + pr
                            F[J * b:(J + 1) * b, I * b:(I + 1) * b] = Lm[lcb * b:(lcb + 1) * b, lrb * b:(lrb + 1) * b]
        return full
