"""Device-resident FDFD wave operator (the plan behind every solve).

``GridOperator`` uploads one problem definition -- ``omega``, ``dxes``,
``epsilon`` and the optional ``mu`` / ``pec`` / ``pmc`` of the reference's
``operators.e_full`` (``meanas/fdfd/operators.py:40-96``) -- builds a
``libmeanas_fdfd`` plan over it and exposes the matrix-free products and the
solver.  No sparse matrix is assembled: the plan holds 1D cell-width tables,
``1/mu``, one mask byte per cell and (for mixed precision) complex64 copies.

PyTorch is only the device-memory and stream carrier here; all arithmetic runs
in the library's CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Any

import numpy
import torch

from . import _lib

_OPS = {'A0': _lib.OP_A0, 'sym': _lib.OP_SYM, 'sym_h': _lib.OP_SYM_H}
_PREC = {'c128': _lib.C128, 'c64': _lib.C64}
_METHODS = {'cocg': _lib.METHOD_COCG, 'fp64': _lib.METHOD_COCG, 'mixed': _lib.METHOD_MIXED,
            'bicgstab': _lib.METHOD_BICGSTAB}
_CRITS = {'true': _lib.CRIT_TRUE, 'precond': _lib.CRIT_PRECOND, 'preconditioned': _lib.CRIT_PRECOND}


@dataclasses.dataclass
class SolveInfo:
    """Outcome of one solve (the reference discards scipy's ``info``; this keeps it)."""
    status: str
    iterations: int
    outer_iterations: int
    residual: float        # ||b0 - A0 E|| / ||b0||  (FP64, recomputed on the result)
    residual_pc: float     # residual of the symmetrised system generic() builds
    kernel_launches: int
    method: str
    history: numpy.ndarray | None = None
    kernel_ms: tuple = ()      # with profile=True: device ms of the iteration kernels by kind
    kernel_count: tuple = ()   # (COCG stencil, COCG pointwise, BiCGSTAB P, BiCGSTAB S)

    @property
    def converged(self) -> bool:
        return self.status == 'converged'


def _device(device: Any | None) -> torch.device:
    if device is None:
        device = torch.device('cuda', torch.cuda.current_device())
    device = torch.device(device)
    if device.type != 'cuda':
        raise ValueError('meanas_b200 runs on CUDA devices only')
    return device


def as_device(a: Any, dtype: torch.dtype, device: torch.device, n: int | None = None,
              name: str = 'array') -> torch.Tensor:
    """Contiguous device tensor of ``dtype`` (copies host arrays; converts device tensors)."""
    if isinstance(a, torch.Tensor):
        t = a.to(device=device, dtype=dtype)
    else:
        arr = numpy.asarray(a)
        if dtype.is_complex:
            arr = arr.astype(numpy.complex128 if dtype == torch.complex128 else numpy.complex64, copy=False)
        else:
            if numpy.iscomplexobj(arr):
                raise ValueError(f'{name} must be real')
            arr = arr.astype(numpy.float64, copy=False)
        t = torch.from_numpy(numpy.ascontiguousarray(arr)).to(device=device, dtype=dtype)
    t = t.reshape(-1).contiguous()
    if n is not None and t.numel() != n:
        raise ValueError(f'{name} has {t.numel()} elements, expected {n}')
    return t


# x planes per CTA chosen by GridOperator.autotune, per (device, grid shape, precision):
# later operators of the same size (a generic() call, a serving slot) start from them.
_TUNED: dict[tuple[int, tuple[int, int, int], str], int] = {}


def _stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


class GridOperator:
    """``A0 = pe (ch pm mu^-1 ce - omega^2 eps) pe`` on the device, with its solver."""

    def __init__(self, omega: complex, dxes, epsilon, mu=None, pec=None, pmc=None, *,
                 device: Any | None = None, fp32: bool = True):
        self.lib = _lib.load()
        self.device = _device(device)
        self.omega = complex(omega)
        self.shape = tuple(int(numpy.size(d)) for d in dxes[0])
        if len(self.shape) != 3 or any(s < 1 for s in self.shape):
            raise ValueError(f'bad grid shape {self.shape}')
        if tuple(int(numpy.size(d)) for d in dxes[1]) != self.shape:
            raise ValueError('dxes[0] and dxes[1] disagree on the grid shape')
        self.n_cells = int(numpy.prod(self.shape))
        self.n = 3 * self.n_cells
        dev = self.device
        with torch.cuda.device(dev):
            self._keep: list[torch.Tensor] = []
            dxe = [as_device(d, torch.complex128, dev, s, 'dx_e') for d, s in zip(dxes[0], self.shape)]
            dxh = [as_device(d, torch.complex128, dev, s, 'dx_h') for d, s in zip(dxes[1], self.shape)]
            # 1/dx as numpy computes it (the values the reference's sparse operators hold)
            inv_e = [as_device(1 / numpy.asarray(d, dtype=complex), torch.complex128, dev) for d in dxes[0]]
            inv_h = [as_device(1 / numpy.asarray(d, dtype=complex), torch.complex128, dev) for d in dxes[1]]
            self.epsilon = as_device(epsilon, torch.float64, dev, self.n, 'epsilon')
            self.mu = None if mu is None else as_device(mu, torch.float64, dev, self.n, 'mu')
            self.pec = None if pec is None else as_device(pec, torch.float64, dev, self.n, 'pec')
            self.pmc = None if pmc is None else as_device(pmc, torch.float64, dev, self.n, 'pmc')
            self._keep += dxe + dxh + inv_e + inv_h
            self._dxe, self._dxh, self._inv_e, self._inv_h = dxe, dxh, inv_e, inv_h
            d = _lib.GridDesc()
            d.shape[:] = self.shape
            d.flags = _lib.GRID_FP32 if fp32 else 0
            d.omega[:] = (self.omega.real, self.omega.imag)
            for a in range(3):
                d.dxe[a] = dxe[a].data_ptr()
                d.dxh[a] = dxh[a].data_ptr()
                d.inv_dxe[a] = inv_e[a].data_ptr()
                d.inv_dxh[a] = inv_h[a].data_ptr()
            d.epsilon = self.epsilon.data_ptr()
            d.mu = self.mu.data_ptr() if self.mu is not None else None
            d.pec = self.pec.data_ptr() if self.pec is not None else None
            d.pmc = self.pmc.data_ptr() if self.pmc is not None else None
            self._desc = d
            nbytes = C.c_size_t()
            _lib.check(self.lib.fdfd_plan_workspace_bytes(C.byref(d), C.byref(nbytes)))
            self._plan_ws = torch.empty(max(int(nbytes.value), 256), dtype=torch.uint8, device=dev)
            plan = C.c_void_p()
            _lib.check(self.lib.fdfd_plan_create(C.byref(d), self._plan_ws.data_ptr(), nbytes.value,
                                                 _stream_handle(), C.byref(plan)))
            self._plan = plan
            self.fp32 = fp32
        self._solve_ws: dict[tuple, torch.Tensor] = {}
        for prec in ('c128', 'c64'):
            xc = _TUNED.get((self.device.index, self.shape, prec))
            if xc is not None and (prec == 'c128' or fp32):
                self.set_xchunk(prec, xc)

    def update(self, omega: complex, dxes, epsilon, mu=None, pec=None, pmc=None) -> None:
        """Load a new problem of the same shape (and the same optional arrays) into this
        operator's device buffers and refill the plan in place (``fdfd_plan_update``), so
        workspaces and captured iteration graphs are reused.  Host inputs are copied on the
        current stream (asynchronously from pinned tensors)."""
        if tuple(int(numpy.size(d)) for d in dxes[0]) != self.shape:
            raise ValueError('update() needs a problem of the same shape')
        if (mu is None) != (self.mu is None) or (pec is None) != (self.pec is None) or \
                (pmc is None) != (self.pmc is None):
            raise ValueError('update() needs the same set of optional arrays (mu, pec, pmc)')

        def put(dst: torch.Tensor, src, dtype, name):
            if isinstance(src, torch.Tensor):
                dst.copy_(src.reshape(-1).to(dtype=dtype), non_blocking=src.is_pinned())
            else:
                dst.copy_(as_device(src, dtype, self.device, dst.numel(), name))
        self.omega = complex(omega)
        with torch.cuda.device(self.device):
            for a in range(3):
                put(self._dxe[a], numpy.asarray(dxes[0][a], dtype=complex), torch.complex128, 'dx_e')
                put(self._dxh[a], numpy.asarray(dxes[1][a], dtype=complex), torch.complex128, 'dx_h')
                put(self._inv_e[a], 1 / numpy.asarray(dxes[0][a], dtype=complex), torch.complex128, 'dx_e')
                put(self._inv_h[a], 1 / numpy.asarray(dxes[1][a], dtype=complex), torch.complex128, 'dx_h')
            put(self.epsilon, epsilon, torch.float64, 'epsilon')
            for t, src, name in ((self.mu, mu, 'mu'), (self.pec, pec, 'pec'), (self.pmc, pmc, 'pmc')):
                if t is not None:
                    put(t, src, torch.float64, name)
            self._desc.omega[:] = (self.omega.real, self.omega.imag)
            _lib.check(self.lib.fdfd_plan_update(self.plan, C.byref(self._desc), _stream_handle()))

    # ------------------------------------------------------------------ lifetime
    def close(self) -> None:
        if getattr(self, '_plan', None):
            torch.cuda.synchronize(self.device)
            self.lib.fdfd_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def plan(self) -> C.c_void_p:
        if not self._plan:
            raise RuntimeError('GridOperator is closed')
        return self._plan

    def set_xchunk(self, precision: str, xchunk: int) -> None:
        """Override the x planes per CTA (autotuning hook; for complex128 rounded up to
        whole blocks of the reductions' fixed plane partition: 8 planes, 4 below 2M cells);
        0 restores the default."""
        _lib.check(self.lib.fdfd_plan_set_xchunk(self.plan, _PREC[precision], int(xchunk)))

    # ------------------------------------------------------------------ products
    def apply(self, x, op: str = 'A0', precision: str = 'c128', out: torch.Tensor | None = None) -> torch.Tensor:
        """``y = op(x)``: ``'A0'``, ``'sym'`` (Pl A0 Pr) or ``'sym_h'`` ((Pl A0 Pr)^H)."""
        dt = torch.complex128 if precision == 'c128' else torch.complex64
        xt = as_device(x, dt, self.device, self.n, 'x')
        y = out if out is not None else torch.empty_like(xt)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.fdfd_apply(self.plan, _OPS[op], _PREC[precision], xt.data_ptr(),
                                           y.data_ptr(), _stream_handle()))
        return y

    def residual(self, E, J) -> dict[str, float]:
        """FP64 ``||b0 - A0 E||`` and ``||Pl (b0 - A0 E)||`` (absolute and relative)."""
        Et = as_device(E, torch.complex128, self.device, self.n, 'E')
        Jt = as_device(J, torch.complex128, self.device, self.n, 'J')
        nbytes = C.c_size_t()
        _lib.check(self.lib.fdfd_residual_workspace_bytes(self.plan, C.byref(nbytes)))
        ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        out = (C.c_double * 4)()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.fdfd_residual(self.plan, Et.data_ptr(), Jt.data_ptr(), out, ws.data_ptr(),
                                              nbytes.value, _stream_handle()))
        r, rpc, b, bpc = list(out)
        return dict(abs=r, rel=r / b if b else r, abs_pc=rpc, rel_pc=rpc / bpc if bpc else rpc, b=b, b_pc=bpc)

    def eps_gradient(self, E: torch.Tensor, E_adj: torch.Tensor) -> torch.Tensor:
        """``Re(omega^2 conj(E_adj) E)`` per component (zero on PEC): dL/deps given the adjoint field."""
        Et = as_device(E, torch.complex128, self.device, self.n, 'E')
        Ea = as_device(E_adj, torch.complex128, self.device, self.n, 'E_adj')
        g = torch.empty(self.n, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.fdfd_eps_gradient(self.plan, Et.data_ptr(), Ea.data_ptr(), g.data_ptr(),
                                                  _stream_handle()))
        return g

    # ------------------------------------------------------------------ after the solve
    def e2h(self, E, out: torch.Tensor | None = None) -> torch.Tensor:
        """``H = pm diag(1/mu) ce(E) / (-i omega)``: the reference's sparse
        ``operators.e2h(omega, dxes, mu, pmc) @ E`` (``meanas/fdfd/operators.py:253-282``)."""
        Et = as_device(E, torch.complex128, self.device, self.n, 'E')
        H = out if out is not None else torch.empty_like(Et)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.fdfd_e2h(self.plan, Et.data_ptr(), H.data_ptr(), None, 0, _stream_handle()))
        return H

    def poynting(self, E, H=None, *, conj: bool = True) -> tuple[torch.Tensor, torch.Tensor]:
        """``(S, H)`` with ``S = E x conj(H)`` (``conj=False``: ``E x H``) on the Yee grid of
        ``meanas/fdfd/functional.py:187-221`` -- the ``poynting_e_cross(E) @ H.conj()`` of
        ``meanas/test/test_fdfd.py:38-40``; ``Re(S)/2`` is the time-averaged Poynting vector.
        With ``H=None``, H is ``e2h(E)`` and both come from one pass over E."""
        Et = as_device(E, torch.complex128, self.device, self.n, 'E')
        S = torch.empty_like(Et)
        flags = _lib.E2H_CONJ if conj else 0
        if H is None:
            Ht = torch.empty_like(Et)
        else:
            Ht = as_device(H, torch.complex128, self.device, self.n, 'H')
            flags |= _lib.E2H_H_IN
        with torch.cuda.device(self.device):
            _lib.check(self.lib.fdfd_e2h(self.plan, Et.data_ptr(), Ht.data_ptr(), S.data_ptr(), flags,
                                         _stream_handle()))
        return S, Ht

    def tfsf_source(self, E, tf_region, *, edges: bool = False, periodic: bool = False,
                    out: torch.Tensor | None = None) -> torch.Tensor:
        """``J = (A0 Q - Q A0) E / (-i omega)`` with ``Q = diag(tf_region)``
        (``meanas/fdfd/operators.py:366-393``); ``edges`` keeps J only where shifting Q by one
        cell changes it (``e_boundary_source``, ``:396-450``; ``periodic`` =
        ``periodic_mask_edges``).  The operator must have no PEC/PMC."""
        Et = as_device(E, torch.complex128, self.device, self.n, 'E')
        q = as_device(tf_region, torch.float64, self.device, self.n, 'tf_region')
        J = out if out is not None else torch.empty_like(Et)
        flags = (_lib.SRC_EDGES if edges else 0) | (_lib.SRC_PERIODIC if periodic else 0)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.fdfd_tfsf_source(self.plan, Et.data_ptr(), q.data_ptr(), J.data_ptr(), flags,
                                                 _stream_handle()))
        return J

    # ------------------------------------------------------------------ solve
    def solve_opts(self, *, method: str = 'cocg', rtol: float = 1e-8, atol: float = 0.0,
                   maxiter: int | None = None, criterion: str = 'true', adjoint: bool = False,
                   chunk: int = 0, use_graph: bool = True, inner_rtol: float = 0.0, max_outer: int = 0,
                   history: torch.Tensor | None = None, has_guess: bool = False,
                   profile: bool = False) -> _lib.SolveOpts:
        o = _lib.SolveOpts()
        o.method = _METHODS[method]
        o.criterion = _CRITS[criterion]
        o.adjoint = int(bool(adjoint))
        o.maxiter = int(maxiter if maxiter is not None else 10 * self.n)
        o.maxiter = min(o.maxiter, 2 ** 31 - 1)
        o.rtol = float(rtol)
        o.atol = float(atol)
        o.has_guess = int(bool(has_guess))
        o.chunk = int(chunk)
        o.use_graph = int(bool(use_graph))
        o.max_outer = int(max_outer)
        o.inner_rtol = float(inner_rtol)
        o.history = history.data_ptr() if history is not None else None
        o.profile = int(bool(profile))
        return o

    def workspace(self, opts: _lib.SolveOpts) -> torch.Tensor:
        key = (opts.method,)
        nbytes = C.c_size_t()
        _lib.check(self.lib.fdfd_solve_workspace_bytes(self.plan, C.byref(opts), C.byref(nbytes)))
        ws = self._solve_ws.get(key)
        if ws is None or ws.numel() < nbytes.value:
            ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
            self._solve_ws[key] = ws
        return ws

    def autotune(self, methods=('cocg', 'mixed'), iters: int = 40, candidates=None) -> dict:
        """Pick the x planes per CTA (the tiling's free parameter: CTA count vs the
        per-CTA prologue of two extra planes and the tail wave) for each precision by timing
        ``iters`` iterations of the real solver passes on dense data (a random initial
        guess), with per-kernel CUDA events; the figure compared is the median of three
        such runs.  The choice is kept for the process: later operators of the same grid
        size on the same device start from it.  Returns {precision: (xchunk, us/iteration, all)}."""
        X = self.shape[0]
        cands = {}
        if candidates is None:
            # complex128: whole blocks of the reductions' plane partition (8 planes, 4 below
            # 2M cells; the library rounds up to them); complex64: any chunk
            step = 8 if self.n_cells >= 1 << 21 else 4
            cands['c128'] = sorted({c for c in range(step, 65, step) if c <= max(step, X)} | {min(X, 64)})
            cands['c64'] = sorted({c for c in (4, 5, 6, 8, 10, 11, 12, 14, 16, 20, 24, 28, 32, 40, 48, 64)
                                   if c <= max(4, X)} | {min(X, 64)})
        else:
            cands['c128'] = cands['c64'] = list(candidates)
        g = torch.Generator(device=self.device).manual_seed(1)
        J = torch.zeros(self.n, dtype=torch.complex128, device=self.device)
        J[self.n // 2] = 1.0
        guess = torch.randn(self.n, dtype=torch.complex128, device=self.device, generator=g)
        best = {}
        for method in methods:
            prec = 'c64' if method == 'mixed' else 'c128'
            if method == 'mixed' and not self.fp32:
                continue
            kinds = (2, 3) if method == 'mixed' else (0, 1)
            timing = {}
            for xc in cands[prec]:
                self.set_xchunk(prec, xc)
                # one batch of exactly `iters` iterations, so few no-op launches follow the cap
                kw = dict(method=method, rtol=1e-30, maxiter=iters, criterion='true', profile=True,
                          max_outer=1, chunk=iters)
                self.solve(J, E_guess=guess, **kw)            # warm-up
                runs = []
                for _ in range(3):
                    _, info = self.solve(J, E_guess=guess, **kw)
                    # per real iteration (the no-op launches of the batch after the cap are
                    # timed too and add the same small amount to every candidate)
                    n = max(1, info.iterations)
                    runs.append(1e3 * sum(info.kernel_ms[k] for k in kinds) / n)
                timing[xc] = float(numpy.median(runs))
            xc = min(timing, key=timing.get)
            self.set_xchunk(prec, xc)
            _TUNED[(self.device.index, self.shape, prec)] = xc
            best[prec] = (xc, timing[xc], timing)
        return best

    def release_workspaces(self) -> None:
        self._solve_ws.clear()

    def solve(self, J, *, E_guess=None, out: torch.Tensor | None = None, record_history: bool = False,
              **kw) -> tuple[torch.Tensor, SolveInfo]:
        """Solve ``A0 E = -i omega J`` (or the adjoint) on the device; returns ``(E, info)``."""
        Jt = as_device(J, torch.complex128, self.device, self.n, 'J')
        E = out if out is not None else torch.empty(self.n, dtype=torch.complex128, device=self.device)
        has_guess = E_guess is not None
        if has_guess:
            E.copy_(as_device(E_guess, torch.complex128, self.device, self.n, 'E_guess'))
        hist = None
        if record_history:
            maxiter = kw.get('maxiter') or 10 * self.n
            hist = torch.zeros(int(maxiter) + 1, dtype=torch.float64, device=self.device)
        opts = self.solve_opts(history=hist, has_guess=has_guess, **kw)
        ws = self.workspace(opts)
        info = _lib.SolveInfo()
        with torch.cuda.device(self.device):
            rc = _lib.check(self.lib.fdfd_solve(self.plan, C.byref(opts), Jt.data_ptr(), E.data_ptr(),
                                                ws.data_ptr(), ws.numel(), C.byref(info), _stream_handle()))
        del rc
        h = None
        if hist is not None:
            h = hist[:info.iterations + 1].cpu().numpy()
        si = SolveInfo(status=_lib.STATUS_NAMES.get(info.status, str(info.status)), iterations=info.iterations,
                       outer_iterations=info.outer_iterations, residual=info.residual,
                       residual_pc=info.residual_pc, kernel_launches=info.kernel_launches,
                       method=kw.get('method', 'cocg'), history=h,
                       kernel_ms=tuple(info.kernel_ms), kernel_count=tuple(info.kernel_count))
        return E, si
