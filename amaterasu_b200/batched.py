"""Block Davidson for every k-point at once (lockstep), on per-k packed device storage.

Per k-point this is the reference's algorithm (amaterasu ``scf/eigen/davidson.py:48-111``:
Rayleigh-Ritz, residuals, Teter-Payne-Allan corrections of the active bands, two
projections off the basis, drop directions below 1e-7, orthonormalise, extend, collapse at
subspace_factor * nbands). All k-points advance together: every step is one launch over all
k (ragged plane-wave counts), H.psi runs on every k's new block in one engine call, the
small per-k problems are solved by the batched Jacobi eigensolver, and the host synchronises
for the whole set instead of per k. ``BatchedDavidson.run`` runs the loop inside the library
(``ama_davidson``, csrc/davidson.cu: two synchronisations per iteration, the segments between
them replayed as CUDA graphs once they recur); ``run_python`` is the same loop with its host
logic written here over the same kernels (three synchronisations), kept as its check.

Storage: the basis of k-point k is a (cap, npw_k) block at cap * pw_off[k]; every k carries
the same number of rows. When a k-point has fewer new directions than the others (fewer
active bands, or directions dropped as dependent), its surplus rows are zero and marked
invalid: their Rayleigh-Ritz diagonal is set just above that k's Gershgorin bound of the
valid block, which decouples them without inflating the matrix norm (the Jacobi solver's
stopping rule is relative to it).
Orthonormalisation: the initial block and the rank-revealing pass over the new directions
use the Gram eigendecomposition, which spans the same space as the reference's SVD; the
second pass (the reference's Cholesky) is a Newton-Schulz symmetric orthonormalisation on
FP64 GEMMs, the overlap being the identity to within rounding there. The Ritz pairs agree.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from ._lib import AMA_C64, AMA_C128, AmaKOperand, call
from .engine import engine_for, ptr, stream_ptr

_GAP = 1.0            # Ha, invalid Rayleigh-Ritz rows sit this far above the Gershgorin bound
_JACOBI_MAX = 80
_TC_MIN_NPW = 8192


class _KOp:
    """An operand inside per-k packed storage."""

    def __init__(self, t: torch.Tensor, rows_per_k=0, row0=0, ragged=True, ld=0, kstride=0):
        self.t = t
        self.c = AmaKOperand(ct.c_void_p(t.data_ptr()), int(rows_per_k), int(row0), 1 if ragged else 0,
                             int(ld), int(kstride))


def graph_stats(reset: bool = False) -> dict:
    """ama_davidson's iteration segments on this thread and the current device: captured as
    CUDA graphs, replayed from a graph, launched kernel by kernel."""
    c, r, n = ct.c_int64(0), ct.c_int64(0), ct.c_int64(0)
    call("ama_davidson_graph_stats", ct.byref(c), ct.byref(r), ct.byref(n), 1 if reset else 0)
    return {"captured": int(c.value), "replayed": int(r.value), "launched": int(n.value)}


class BatchedDavidson:
    def __init__(self, system, nbands: int, dtype=torch.complex128, tensor_cores: bool = True,
                 tc_min_npw: int = _TC_MIN_NPW, graphs: bool = True):
        self.eng = engine_for(system)
        self.system = system
        self.nk = self.eng.nk
        self.nb = nbands
        self.dtype = dtype
        self.prec = AMA_C64 if dtype == torch.complex64 else AMA_C128
        dev = self.eng.device
        self.dev = dev
        self.npw = torch.from_numpy(self.eng.npw.astype(np.int32)).to(dev)
        self.pw_off = torch.from_numpy(self.eng.pw_off[:-1].astype(np.int64)).to(dev)
        self.max_npw = int(self.eng.npw.max())
        self.total_pw = int(self.eng.pw_off[-1])
        self.kin = torch.from_numpy(np.concatenate([s.kinetic_energy for s in system.wave_spheres])).to(dev)
        self.max_sub = min(4 * nbands, int(self.eng.npw.min()))
        self.cap = self.max_sub + nbands
        # complex64 plane-wave products on the tensor cores (split-TF32) once the spheres are
        # long enough for the staged tiles to pay; shorter ones stay on the SIMT kernels
        self.tensor_cores = bool(tensor_cores) and dtype == torch.complex64 and self.max_npw >= tc_min_npw
        self.tc_min_npw = int(tc_min_npw)
        self.graphs = bool(graphs)  # ama_davidson replays recurring iteration segments as CUDA graphs
        self.trace = []  # per iteration of the last run: (iteration, active directions, subspace size, max norm)

    # ---------------------------------------------------------------- kernels
    def _gemm(self, form, m, n, k, a: _KOp, b: _KOp, c: _KOp, alpha=1.0, beta=0.0, max_m=None, max_n=None):
        al = (ct.c_double * 2)(float(np.real(alpha)), float(np.imag(alpha)))
        be = (ct.c_double * 2)(float(np.real(beta)), float(np.imag(beta)))
        if self.tensor_cores and ((form == 1 and k < 0 and m > 0 and n > 0) or (form == 0 and n < 0 and m > 0 and k > 0)):
            call("ama_kbatch_zgemm_tc", form, self.nk, m, n, k, ptr(self.npw), ptr(self.pw_off),
                 ct.byref(a.c), ct.byref(b.c), ct.byref(c.c), al, be, self.max_npw, stream_ptr())
            return
        mm = max_m if max_m is not None else (self.max_npw if m < 0 else m)
        nn = max_n if max_n is not None else (self.max_npw if n < 0 else n)
        call("ama_kbatch_zgemm", self.prec, form, self.nk, m, n, k, ptr(self.npw), ptr(self.pw_off),
             ct.byref(a.c), ct.byref(b.c), ct.byref(c.c), al, be, mm, nn, stream_ptr())

    def _blocks(self, rows):
        return torch.zeros(rows * self.total_pw, dtype=self.dtype, device=self.dev)

    def _small(self, rows, cols):
        return torch.zeros((self.nk, rows, cols), dtype=self.dtype, device=self.dev)

    def _gram(self, blk: torch.Tensor, rows: int, rows_per_k: int, row0: int = 0) -> torch.Tensor:
        """G[k] = X_k X_k^H for `rows` rows of a packed block (FP64, Hermitised)."""
        g = self._small(rows, rows)
        op = _KOp(blk, rows_per_k, row0)
        self._gemm(1, rows, rows, -1, op, op, _KOp(g, ragged=False, ld=rows, kstride=rows * rows))
        g = g.to(torch.complex128)
        return 0.5 * (g + g.conj().transpose(1, 2))

    def _heev(self, mats: torch.Tensor, lowest: int | None = None):
        """Batched FP64 Hermitian eigensolve: (w ascending [nk][n], V columns [nk][n][n]).
        With ``lowest``, only the first ``lowest`` eigenpairs are valid (large n only)."""
        n = mats.shape[1]
        m = mats.contiguous().clone()
        w = torch.empty((self.nk, n), dtype=torch.float64, device=self.dev)
        if n <= _JACOBI_MAX:
            call("ama_heev_small", n, ptr(m), ptr(w), self.nk, stream_ptr())
        elif lowest is not None and lowest < n:
            call("ama_heev_lowest", n, int(lowest), ptr(m), ptr(w), self.nk, stream_ptr())
        else:
            call("ama_heev", n, ptr(m), ptr(w), self.nk, stream_ptr())
        return w, m

    def _rotate(self, rot: torch.Tensor, src: torch.Tensor, src_rows_per_k: int, k_rows: int, out_rows: int):
        """out[k] = rot[k] (out_rows x k_rows) . src[k][:k_rows]  -> packed (out_rows, npw_k)."""
        out = self._blocks(out_rows)
        r = rot.to(self.dtype).contiguous()
        self._gemm(0, out_rows, -1, k_rows, _KOp(r, ragged=False, ld=k_rows, kstride=out_rows * k_rows),
                   _KOp(src, src_rows_per_k, 0), _KOp(out, out_rows, 0))
        return out

    def _copy(self, src, src_rows_per_k, src_row0, dst, dst_rows_per_k, dst_row0, nrows):
        call("ama_kbatch_copy_rows", self.prec, self.nk, nrows, ptr(self.npw), ptr(self.pw_off), ptr(src),
             src_rows_per_k, src_row0, ptr(dst), dst_rows_per_k, dst_row0, stream_ptr())

    def _orthonormal_rows(self, blk: torch.Tensor, rows: int, threshold: float, drop_small: bool):
        """Orthonormal rows spanning the dominant part of each k's block (Gram eigh),
        zero rows where directions are dropped. Returns (block, valid [nk][rows] numpy)."""
        g = self._gram(blk, rows, rows)
        if drop_small:  # rows whose norm is <= threshold are removed before the SVD
            diag = torch.diagonal(g, dim1=1, dim2=2).real
            small = diag <= threshold * threshold
            g = g * (~small)[:, :, None] * (~small)[:, None, :]
        w, u = self._heev(g)
        s = torch.sqrt(torch.clamp(w, min=0.0))
        smax = s.max(dim=1, keepdim=True).values
        keep = s > threshold * torch.clamp(smax, min=1e-300)
        inv = torch.where(keep, 1.0 / torch.where(keep, s, torch.ones_like(s)), torch.zeros_like(s))
        rot = (u.conj().transpose(1, 2) * inv[:, :, None])  # rows: u_j^H / s_j
        out = self._rotate(rot, blk, rows, rows, rows)
        return out, keep.cpu().numpy()

    def _small_gemm(self, a, b, out, rows):
        """out[k] = a[k] b[k] for the nk small (rows x rows) complex128 matrices (FP64 tensor cores)."""
        one = (ct.c_double * 2)(1.0, 0.0)
        zero = (ct.c_double * 2)(0.0, 0.0)
        st = rows * rows
        call("ama_zgemm", AMA_C128, 0, rows, rows, rows, one, ptr(a), rows, st, ptr(b), rows, st, zero, ptr(out),
             rows, st, self.nk, stream_ptr())
        return out

    def _lowdin_rows(self, blk: torch.Tensor, rows: int, keep: np.ndarray):
        """Rows of each k's block re-orthonormalised by the Newton-Schulz iteration for
        S^{-1/2} (S = the rows' overlap, coupled form Y <- Y T, Z <- T Z, T = (3I - Z Y)/2):
        a symmetric (Loewdin) orthonormalisation on FP64 GEMMs, for rows that are already
        orthonormal to within rounding (the second pass after the rank-revealing one).
        Invalid (zero) rows are decoupled and stay zero. Returns None when the overlap is too
        far from the identity for the iteration (the caller then decomposes it)."""
        g = self._gram(blk, rows, rows)
        inval = torch.from_numpy(~keep[:, :rows]).to(self.dev)
        eye = torch.eye(rows, dtype=torch.complex128, device=self.dev).expand(self.nk, rows, rows)
        g = g * (~inval)[:, :, None] * (~inval)[:, None, :] + torch.diag_embed(inval.to(torch.complex128))
        dev = float(torch.linalg.matrix_norm(g - eye).max())  # Frobenius, >= spectral norm
        if not dev < 0.5:
            return None
        iters = 0
        err = max(dev, 1e-300)
        while err > 1e-18 and iters < 6:
            err *= err
            iters += 1
        y = g.contiguous()
        z = eye.contiguous().clone()
        t = torch.empty_like(y)
        tmp = torch.empty_like(y)
        for _ in range(iters):
            self._small_gemm(z, y, t, rows)
            t = 1.5 * eye - 0.5 * t
            self._small_gemm(y, t, tmp, rows)
            y, tmp = tmp, y
            self._small_gemm(t, z, tmp, rows)
            z, tmp = tmp, z
        return self._rotate(z, blk, rows, rows, rows)

    def _rr(self, B, HB, m, valid):
        p = self._small(m, m)
        self._gemm(1, m, m, -1, _KOp(B, self.cap, 0), _KOp(HB, self.cap, 0),
                   _KOp(p, ragged=False, ld=m, kstride=m * m))
        p = p.to(torch.complex128).conj()
        p = 0.5 * (p + p.conj().transpose(1, 2))
        inval = torch.from_numpy(~valid[:, :m]).to(self.dev)
        p = p * (~inval)[:, :, None] * (~inval)[:, None, :]
        bound = p.abs().sum(dim=2).max(dim=1, keepdim=True).values + _GAP  # per-k Gershgorin bound
        p = p + torch.diag_embed(inval.to(torch.float64) * bound).to(torch.complex128)
        w, v = self._heev(p, lowest=self.nb)  # only the nb lowest Ritz pairs are kept
        rot = v[:, :, :self.nb].transpose(1, 2)  # (nb x m) per k: X_n = sum_i V[i, n] b_i
        X = self._rotate(rot, B, self.cap, m, self.nb)
        HX = self._rotate(rot, HB, self.cap, m, self.nb)
        return w[:, :self.nb].contiguous(), X, HX

    def _apply(self, H, blk, rows, spin):
        out = torch.empty_like(blk)
        self.eng.hpsi(blk, out, k_first=0, k_count=self.nk, nbands=rows, spin=spin)
        return out

    # -------------------------------------------------------------------- run
    def run(self, H, guess_packed: torch.Tensor, *, tolerance=1e-8, max_iterations=40, spin=0):
        """Lowest nbands eigenpairs at every k through the library's own loop
        (``ama_davidson``: the iteration below, orchestrated in C++). ``guess_packed`` packs
        one (nbands, npw_k) block per k; returns (eigenvalues [nk][nb] numpy, X packed,
        norms numpy, iterations)."""
        H._bind()
        guess = guess_packed.to(self.dtype).contiguous()
        eps = torch.empty((self.nk, self.nb), dtype=torch.float64, device=self.dev)
        norms = torch.empty_like(eps)
        X = torch.empty_like(guess)
        it = ct.c_int32(0)
        tc_min = self.tc_min_npw if self.tensor_cores else 0
        self.eng.set_davidson_graphs(self.graphs)
        call("ama_davidson", self.eng.handle, self.prec, int(spin), self.nb, ptr(guess), float(tolerance),
             int(max_iterations), int(tc_min), ptr(eps), ptr(X), ptr(norms), ct.byref(it), stream_ptr())
        return eps.cpu().numpy(), X, norms.cpu().numpy(), int(it.value)

    def run_python(self, H, guess_packed: torch.Tensor, *, tolerance=1e-8, max_iterations=40, spin=0):
        """The same iteration with its host logic in Python over the same kernels; kept to
        check ``ama_davidson`` against (tests/test_eigen_gpu.py). Records ``trace``."""
        nb, cap = self.nb, self.cap
        self.trace = []
        H._bind()
        guess = guess_packed.to(self.dtype).contiguous()
        # the guess is usually the previous step's orthonormal orbitals: polish them without a
        # decomposition, else decompose the overlap (and reject a rank-deficient start)
        X0 = self._lowdin_rows(guess, nb, np.ones((self.nk, nb), dtype=bool))
        if X0 is None:
            X0, ok = self._orthonormal_rows(guess, nb, 1e-10, False)
            if not ok.all():
                raise ValueError("the starting block of some k-point is rank deficient")
        B, HB = self._blocks(cap), self._blocks(cap)
        HX0 = self._apply(H, X0, nb, spin)
        self._copy(X0, nb, 0, B, cap, 0, nb)
        self._copy(HX0, nb, 0, HB, cap, 0, nb)
        valid = np.zeros((self.nk, cap), dtype=bool)
        valid[:, :nb] = True
        m = nb
        eps, X, HX = self._rr(B, HB, m, valid)
        norms = np.full((self.nk, nb), np.inf)
        it = 0
        for it in range(1, max_iterations + 1):
            nrm = torch.empty((self.nk, nb), dtype=torch.float64, device=self.dev)
            call("ama_kbatch_residual", self.prec, self.nk, nb, ptr(self.npw), ptr(self.pw_off), ptr(X), ptr(HX),
                 ptr(eps), ptr(self.kin), ptr(nrm), None, 0, None, stream_ptr())
            norms = nrm.cpu().numpy()
            active = norms > tolerance
            counts = active.sum(axis=1)
            nn = int(counts.max())
            self.trace.append((it, nn, m, float(norms.max())))
            if nn == 0:
                break
            # row of each active band in its k-point's correction block (-1: inactive)
            rows = np.where(active, np.cumsum(active, axis=1) - 1, -1).astype(np.int32)
            rows_t = torch.from_numpy(rows).to(self.dev)
            C = self._blocks(nn)
            call("ama_kbatch_residual", self.prec, self.nk, nb, ptr(self.npw), ptr(self.pw_off), ptr(X), ptr(HX),
                 ptr(eps), ptr(self.kin), ptr(nrm), ptr(rows_t), nn, ptr(C), stream_ptr())
            for _ in range(2):
                t = self._small(nn, m)
                self._gemm(1, nn, m, -1, _KOp(C, nn, 0), _KOp(B, cap, 0), _KOp(t, ragged=False, ld=m, kstride=nn * m))
                self._gemm(0, nn, -1, m, _KOp(t, ragged=False, ld=m, kstride=nn * m), _KOp(B, cap, 0), _KOp(C, nn, 0),
                           alpha=-1.0, beta=1.0)
            new, keep1 = self._orthonormal_rows(C, nn, 1e-7, True)
            if not keep1.any():
                self.trace.append((it, 0, m, -1.0))  # every new direction was dependent
                break
            polished = self._lowdin_rows(new, nn, keep1)
            if polished is not None:
                new, keep = polished, keep1
            else:
                new, keep = self._orthonormal_rows(new, nn, 0.5, False)
            HN = self._apply(H, new, nn, spin)
            self._copy(new, nn, 0, B, cap, m, nn)
            self._copy(HN, nn, 0, HB, cap, m, nn)
            valid[:, m:m + nn] = keep
            m += nn
            eps, X, HX = self._rr(B, HB, m, valid)
            if m + nb > self.max_sub:
                self._copy(X, nb, 0, B, cap, 0, nb)
                self._copy(HX, nb, 0, HB, cap, 0, nb)
                valid[:] = False
                valid[:, :nb] = True
                m = nb
        return eps.cpu().numpy(), X, norms, it
