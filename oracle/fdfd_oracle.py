"""CPU restatement (numpy / scipy) of the reference FDFD solve path.

TEST INFRASTRUCTURE ONLY: this module is the parity checker and the timed CPU
baseline.  The product path (``meanas_b200``) never imports it.

Parity pinning: ``tests/golden/make_golden.py`` runs the reference itself
(``meanas.fdfd.operators.e_full``, ``e_full_preconditioners``,
``solvers.generic`` and ``scpml``) on small grids and stores inputs/outputs as
``tests/golden/*.npz``; ``tests/test_oracle.py`` checks every function below
against those vectors.

What each function restates:

* ``e_full_apply``   matrix-free ``A0 @ E`` with the semantics of the sparse
  ``meanas/fdfd/operators.py:40-96``: ``pe (ch pm diag(1/mu) ce - omega^2 diag(eps)) pe``,
  using the periodic ``roll`` derivatives of ``meanas/fdmath/functional.py:16-122``.
  (Note the sparse form divides by ``mu``; the functional
  ``meanas/fdfd/functional.py:45`` multiplies.  ``generic()`` uses the sparse form,
  so this follows it.)
* ``e_full_csr``     the same operator assembled as CSR in complex128, built from
  periodic shift matrices like ``meanas/fdmath/operators.py:15-52,99-171,222-251``.
* ``precond_p2``     ``p^2`` of ``meanas/fdfd/operators.py:116-118`` (per component
  products of 1D widths); ``Pl = sqrt(p^2)``, ``Pr = 1/Pl`` (``:120-122``).
* ``generic_qmr``    ``meanas/fdfd/solvers.py:66-141`` with the default
  ``_scipy_qmr`` (``:21-63``): the symmetrised CSR system handed to
  ``scipy.sparse.linalg.qmr``.  QMR itself is third-party (scipy; the reference
  pins ``scipy~=1.14`` in ``pyproject.toml:44``, ``uv.lock`` locks 1.16.3); it
  is called, not restated.  The adjoint branch (``:119-137``) is written with
  explicit conjugate transposes, since ``csr_array.H`` is gone in SciPy >= 1.14.
* ``e2h``            ``H = pm diag(1/mu) ce(E) / (-i omega)``, the sparse
  ``meanas/fdfd/operators.py:253-282`` (its functional twin
  ``meanas/fdfd/functional.py:89-117`` has no PMC argument).
* ``poynting_e_cross_h``  ``E x H`` with the one-cell shift of E and the cell-width
  weights of ``meanas/fdfd/functional.py:187-221`` (the same product as
  ``operators.poynting_e_cross(E) @ H``, ``meanas/fdfd/operators.py:310-336``).
* ``tfsf_source``    ``(A0 Q - Q A0) E / (-i omega)`` with ``A0`` unmasked
  (``meanas/fdfd/operators.py:366-393``) and, with ``edges``, the edge mask of
  ``e_boundary_source`` (``:396-450``; mirrored or periodic one-cell shifts,
  ``meanas/fdmath/operators.py:55-98``).
* ``expand_e`` / ``mode_source``  the unidirectional waveguide-mode source:
  ``meanas/fdfd/waveguide_3d.py:206-257`` (the source-plane cross-section repeated along the
  axis with the phase ``exp(-i polarity k r)``) and ``:113-156`` (the boundary source of that
  field on the half-space mask from the source plane onward).
* ``fdtd_plain_step`` / ``CpmlUpdates``  the FDTD Yee updates: ``maxwell_h`` /
  ``maxwell_e`` (``meanas/fdtd/base.py:13-125``) and ``updates_with_cpml``
  (``meanas/fdtd/pml.py:115-230``, which divides its forward differences by the H-grid
  widths ``dxes[1]``) with psi and the PML sums held in the psi dtype, as there.
* ``cocg``           complex-symmetric CG in the E-space with the ``p^2``-weighted
  bilinear form: algebraically the COCG iteration on ``Pl A0 Pr`` (the system
  ``generic()`` builds) rewritten with ``x = Pl E``; the GPU solver runs the same
  recurrence.
"""
from __future__ import annotations

import numpy
from numpy.typing import NDArray
from scipy import sparse
import scipy.sparse.linalg


def _shape_of(dxes) -> tuple[int, int, int]:
    return tuple(int(numpy.size(d)) for d in dxes[0])


def _bcast(a: NDArray, axis: int) -> NDArray:
    idx = [None, None, None]
    idx[axis] = slice(None)
    return numpy.asarray(a)[tuple(idx)]


def _dfwd(f: NDArray, dx: NDArray, axis: int) -> NDArray:
    return (numpy.roll(f, -1, axis=axis) - f) / _bcast(dx, axis)


def _dback(f: NDArray, dx: NDArray, axis: int) -> NDArray:
    return (f - numpy.roll(f, 1, axis=axis)) / _bcast(dx, axis)


def curl_forward(dx_e, e: NDArray) -> NDArray:
    """Forward curl of a (3,X,Y,Z) field, ``meanas/fdmath/functional.py:67-91``."""
    out = numpy.empty_like(e)
    out[0] = _dfwd(e[2], dx_e[1], 1) - _dfwd(e[1], dx_e[2], 2)
    out[1] = _dfwd(e[0], dx_e[2], 2) - _dfwd(e[2], dx_e[0], 0)
    out[2] = _dfwd(e[1], dx_e[0], 0) - _dfwd(e[0], dx_e[1], 1)
    return out


def curl_back(dx_h, h: NDArray) -> NDArray:
    """Backward curl of a (3,X,Y,Z) field, ``meanas/fdmath/functional.py:94-122``."""
    out = numpy.empty_like(h)
    out[0] = _dback(h[2], dx_h[1], 1) - _dback(h[1], dx_h[2], 2)
    out[1] = _dback(h[0], dx_h[2], 2) - _dback(h[2], dx_h[0], 0)
    out[2] = _dback(h[1], dx_h[0], 0) - _dback(h[0], dx_h[1], 1)
    return out


def e_full_apply(omega, dxes, epsilon, E, mu=None, pec=None, pmc=None) -> NDArray:
    """``A0 @ E`` for 1D C-order vectors (length 3XYZ); returns complex128 (3XYZ,)."""
    shape = _shape_of(dxes)
    f3 = (3, *shape)
    e = numpy.asarray(E, dtype=complex).reshape(f3)
    eps = numpy.asarray(epsilon).reshape(f3)
    if pec is not None:
        e = e * numpy.where(numpy.asarray(pec).reshape(f3), 0, 1)
    h = curl_forward(dxes[0], e)
    if mu is not None:
        h = h / numpy.asarray(mu).reshape(f3)
    if pmc is not None:
        h = h * numpy.where(numpy.asarray(pmc).reshape(f3), 0, 1)
    y = curl_back(dxes[1], h) - omega ** 2 * eps * e
    if pec is not None:
        y = y * numpy.where(numpy.asarray(pec).reshape(f3), 0, 1)
    return y.ravel()


def e2h(omega, dxes, E, mu=None, pmc=None) -> NDArray:
    """``H = pm diag(1/mu) ce(E) / (-i omega)`` for 1D C-order vectors, complex128 (3XYZ,)
    (``meanas/fdfd/operators.py:253-282``)."""
    shape = _shape_of(dxes)
    f3 = (3, *shape)
    h = curl_forward(dxes[0], numpy.asarray(E, dtype=complex).reshape(f3)) / (-1j * omega)
    if mu is not None:
        h = h / numpy.asarray(mu).reshape(f3)
    if pmc is not None:
        h = h * numpy.where(numpy.asarray(pmc).reshape(f3), 0, 1)
    return h.ravel()


def poynting_e_cross_h(dxes, E, H) -> NDArray:
    """``E x H`` on the Yee grid (``meanas/fdfd/functional.py:187-221``): components of E
    weighted by ``dx_e``, of H by ``dx_h``, E shifted by one cell along the cross axis.
    Pass ``H.conj()`` for the complex Poynting vector; complex128 (3XYZ,)."""
    shape = _shape_of(dxes)
    f3 = (3, *shape)
    e = numpy.asarray(E, dtype=complex).reshape(f3)
    h = numpy.asarray(H, dtype=complex).reshape(f3)
    ex, ey, ez = (e[a] * _bcast(dxes[0][a], a) for a in range(3))
    hx, hy, hz = (h[a] * _bcast(dxes[1][a], a) for a in range(3))
    s = numpy.empty_like(e)
    s[0] = numpy.roll(ey, -1, axis=0) * hz - numpy.roll(ez, -1, axis=0) * hy
    s[1] = numpy.roll(ez, -1, axis=1) * hx - numpy.roll(ex, -1, axis=1) * hz
    s[2] = numpy.roll(ex, -1, axis=2) * hy - numpy.roll(ey, -1, axis=2) * hx
    return s.ravel()


def _edge_mask(q: NDArray, periodic: bool) -> NDArray:
    """Cells of a (3,X,Y,Z) array where a one-cell shift along a non-singleton axis changes it."""
    m = numpy.zeros(q.shape, dtype=bool)
    for axis in (1, 2, 3):
        n = q.shape[axis]
        if n == 1:
            continue
        for s in (-1, 1):
            idx = numpy.arange(n) + s
            idx = idx % n if periodic else numpy.clip(idx, 0, n - 1)
            m |= numpy.take(q, idx, axis=axis) != q
    return m


def tfsf_source(omega, dxes, epsilon, E, tf_region, mu=None, *, edges=False, periodic=False) -> NDArray:
    """``J = (A0 Q E - Q A0 E) / (-i omega)``, optionally on the edges of Q only; (3XYZ,)."""
    q = numpy.asarray(tf_region, dtype=float)
    e = numpy.asarray(E, dtype=complex)
    j = (e_full_apply(omega, dxes, epsilon, q * e, mu) - q * e_full_apply(omega, dxes, epsilon, e, mu)) / (-1j * omega)
    if edges:
        shape = _shape_of(dxes)
        j = j * _edge_mask(q.reshape(3, *shape), periodic).ravel()
    return j


def expand_e(E, wavenumber, dxes, axis: int, polarity: int, slices) -> NDArray:
    """(3,X,Y,Z) field: the cross-section of ``E`` at ``slices`` repeated along ``axis``
    with phase ``exp(-i polarity wavenumber r)`` (``meanas/fdfd/waveguide_3d.py:232-257``)."""
    E = numpy.asarray(E, dtype=complex)
    slices = tuple(slices)
    pos = numpy.cumsum(numpy.real(numpy.asarray(dxes[0][axis])))
    dist = pos - pos[slices[axis]]
    ph = numpy.exp(polarity * -1j * wavenumber * dist)
    bshape = [1, 1, 1, 1]
    bshape[axis + 1] = -1
    out = numpy.zeros_like(E)
    dst = [slice(None), *slices]
    dst[axis + 1] = slice(None)
    out[tuple(dst)] = ph.reshape(bshape) * E[(slice(None), *slices)]
    return out


def mode_source(E, wavenumber, omega, dxes, axis: int, polarity: int, slices, epsilon, mu=None) -> NDArray:
    """(3,X,Y,Z) current of the unidirectional mode source (``meanas/fdfd/waveguide_3d.py:113-156``):
    the boundary source (``tfsf_source(..., edges=True)``) of ``expand_e`` on the half-space
    from ``slices[axis].start`` onward (``polarity > 0``) or up to ``slices[axis].stop``."""
    Ee = expand_e(E, wavenumber, dxes, axis, polarity, slices)
    sl = tuple(slices)[axis]
    q = numpy.zeros(Ee.shape)
    half = [slice(None)] * 4
    half[axis + 1] = slice(sl.start, None) if polarity > 0 else slice(None, sl.stop)
    q[tuple(half)] = 1.0
    eps = numpy.asarray(epsilon).ravel()
    mu = None if mu is None else numpy.asarray(mu).ravel()
    J = tfsf_source(omega, dxes, eps, Ee.ravel(), q.ravel(), mu, edges=True)
    return J.reshape(Ee.shape)


def fdtd_plain_step(e: NDArray, h: NDArray, epsilon: NDArray, dt: float, dxes) -> None:
    """One ``maxwell_h`` then ``maxwell_e`` update of (3,X,Y,Z) fields, in place."""
    h -= dt * curl_forward(dxes[0], e)
    e += dt * curl_back(dxes[1], h) / epsilon


class CpmlUpdates:
    """``updates_with_cpml``: ``update_E(e, h, epsilon)`` / ``update_H(e, h, mu)`` in place.
    ``params[axis][pp]`` is None or ``(param_e, param_h)`` with each a (3, th) array of
    ``p0, p1, p2`` per layer (``pp = 0``: the low face, ``1``: the high face)."""

    def __init__(self, params, dt: float, dxes, shape, dtype=numpy.float32):
        self.dt = dt
        self.dx = [numpy.asarray(d, dtype=float) for d in dxes[1]]
        self.shape = tuple(shape)
        self.dtype = dtype
        self.params = params
        self.psi_e = [[None, None] for _ in range(3)]
        self.psi_h = [[None, None] for _ in range(3)]
        for a in range(3):
            for pp in range(2):
                if params[a][pp] is not None:
                    th = params[a][pp][0].shape[1]
                    rs = list(self.shape)
                    rs[a] = th
                    self.psi_e[a][pp] = [numpy.zeros(rs, dtype) for _ in range(2)]
                    self.psi_h[a][pp] = [numpy.zeros(rs, dtype) for _ in range(2)]

    def _region(self, a, pp, th):
        sl = [slice(None)] * 3
        sl[a] = slice(None, th) if pp == 0 else slice(-th, None)
        return tuple(sl)

    def _bcast(self, v, a):
        idx = [None, None, None]
        idx[a] = slice(None)
        return v[tuple(idx)]

    def _pml(self, d, psi, side):
        p = numpy.zeros((3, *self.shape), dtype=self.dtype)
        for a in range(3):
            se = (-1, 1, -1)[a]
            u, v = [b for b in range(3) if b != a]
            du, dv = d[a]
            for pp in range(2):
                if self.params[a][pp] is None:
                    continue
                tab = self.params[a][pp][0 if side == 'e' else 1]
                p0, p1, p2 = (self._bcast(tab[i], a) for i in range(3))
                reg = self._region(a, pp, tab.shape[1])
                du[reg] *= p2
                dv[reg] *= p2
                pu, pv = psi[a][pp]
                pu *= p0
                pv *= p0
                pu += p1 * dv[reg]
                pv += p1 * du[reg]
                p[u][reg] += +se * pu
                p[v][reg] += -se * pv
        return p

    def update_E(self, e, h, epsilon):
        b = [lambda f, a=a: (f - numpy.roll(f, 1, axis=a)) / self._bcast(self.dx[a], a) for a in range(3)]
        dyHx, dzHx = b[1](h[0]), b[2](h[0])
        dxHy, dzHy = b[0](h[1]), b[2](h[1])
        dxHz, dyHz = b[0](h[2]), b[1](h[2])
        p = self._pml(((dxHy, dxHz), (dyHx, dyHz), (dzHx, dzHy)), self.psi_e, 'e')
        e[0] += self.dt / epsilon[0] * (dyHz - dzHy + p[0])
        e[1] += self.dt / epsilon[1] * (dzHx - dxHz + p[1])
        e[2] += self.dt / epsilon[2] * (dxHy - dyHx + p[2])

    def update_H(self, e, h, mu=(1, 1, 1)):
        f = [lambda g, a=a: (numpy.roll(g, -1, axis=a) - g) / self._bcast(self.dx[a], a) for a in range(3)]
        dyEx, dzEx = f[1](e[0]), f[2](e[0])
        dxEy, dzEy = f[0](e[1]), f[2](e[1])
        dxEz, dyEz = f[0](e[2]), f[1](e[2])
        p = self._pml(((dxEy, dxEz), (dyEx, dyEz), (dzEx, dzEy)), self.psi_h, 'h')
        h[0] -= self.dt / mu[0] * (dyEz - dzEy + p[0])
        h[1] -= self.dt / mu[1] * (dzEx - dxEz + p[1])
        h[2] -= self.dt / mu[2] * (dxEy - dyEx + p[2])


def precond_p2(dxes) -> NDArray:
    """(3,X,Y,Z) complex ``p^2``: x: dxe_x dxh_y dxh_z, y: dxh_x dxe_y dxh_z, z: dxh_x dxh_y dxe_z."""
    (ex, ey, ez), (hx, hy, hz) = dxes
    ex, ey, ez, hx, hy, hz = (numpy.asarray(v, dtype=complex) for v in (ex, ey, ez, hx, hy, hz))
    return numpy.stack([
        ex[:, None, None] * hy[None, :, None] * hz[None, None, :],
        hx[:, None, None] * ey[None, :, None] * hz[None, None, :],
        hx[:, None, None] * hy[None, :, None] * ez[None, None, :],
    ])


def precond_pl(dxes) -> NDArray:
    """1D ``Pl`` diagonal: principal-branch ``sqrt(p^2)`` (``Pr = 1/Pl``)."""
    return numpy.sqrt(precond_p2(dxes).ravel())


def _shift_matrix(shape, axis: int) -> sparse.csr_array:
    """``(S f)[..i..] = f[..(i+1) mod n..]`` along ``axis``."""
    n = int(numpy.prod(shape))
    idx = numpy.arange(n).reshape(shape)
    cols = numpy.roll(idx, -1, axis=axis).ravel()
    return sparse.csr_array((numpy.ones(n), (numpy.arange(n), cols)), shape=(n, n))


def _cell_widths(dx1d, shape, axis) -> NDArray:
    return numpy.broadcast_to(_bcast(numpy.asarray(dx1d), axis), shape).ravel()


def e_full_csr(omega, dxes, epsilon, mu=None, pec=None, pmc=None) -> sparse.csr_array:
    """CSR ``A0`` (complex128, 3XYZ x 3XYZ)."""
    shape = _shape_of(dxes)
    n = int(numpy.prod(shape))
    eye = sparse.eye_array(n, format='csr')
    Df, Db = [], []
    for a in range(3):
        S = _shift_matrix(shape, a)
        Df.append(sparse.diags_array(1 / _cell_widths(dxes[0][a], shape, a)) @ (S - eye))
        Db.append(sparse.diags_array(1 / _cell_widths(dxes[1][a], shape, a)) @ (eye - S.T))

    def cross(D):
        z = sparse.csr_array((n, n))
        return sparse.block_array([[z, -D[2], D[1]], [D[2], z, -D[0]], [-D[1], D[0], z]])
    ce = cross(Df)
    ch = cross(Db)
    N3 = 3 * n
    pe = sparse.diags_array(numpy.where(pec, 0.0, 1.0) if pec is not None else numpy.ones(N3))
    pm = sparse.diags_array(numpy.where(pmc, 0.0, 1.0) if pmc is not None else numpy.ones(N3))
    md = sparse.diags_array(1 / numpy.asarray(mu) if mu is not None else numpy.ones(N3))
    ed = sparse.diags_array(numpy.asarray(epsilon))
    return (pe @ (ch @ pm @ md @ ce - omega ** 2 * ed) @ pe).tocsr()


def true_residual(omega, dxes, epsilon, E, J, mu=None, pec=None, pmc=None) -> float:
    """``||A0 E - b0|| / ||b0||`` with ``b0 = -i omega J`` (``meanas/test/test_fdfd.py:15-18``)."""
    b0 = -1j * omega * numpy.asarray(J)
    r = e_full_apply(omega, dxes, epsilon, E, mu, pec, pmc) - b0
    return float(numpy.linalg.norm(r) / numpy.linalg.norm(b0))


def generic_qmr(omega, dxes, J, epsilon, mu=None, *, pec=None, pmc=None, adjoint=False,
                rtol=1e-8, atol=0.0, maxiter=None, E_guess=None, counter=None, matrix_solver=None):
    """Reference ``generic()`` + ``_scipy_qmr`` on the CPU: assemble, symmetrise, scipy QMR.
    ``matrix_solver(A, b, **opts) -> x`` replaces QMR as the reference's hook of that name
    does (``meanas/fdfd/solvers.py:97-103,134``); it then returns ``(E, None)``."""
    b0 = -1j * omega * numpy.asarray(J)
    A0 = e_full_csr(omega, dxes, epsilon, mu, pec, pmc)
    pl = precond_pl(dxes)
    Pl = sparse.diags_array(pl)
    Pr = sparse.diags_array(1 / pl)
    if adjoint:
        A = (Pl @ A0 @ Pr).conj().T
        b = Pr.conj().T @ b0
    else:
        A = Pl @ A0 @ Pr
        b = Pl @ b0
    kw = dict(rtol=rtol, atol=atol)
    if maxiter is not None:
        kw['maxiter'] = maxiter
    if E_guess is not None:
        kw['x0'] = (Pr.conj().T if adjoint else Pl) @ numpy.asarray(E_guess)
    if counter is not None:
        def cb(_xk):
            counter[0] += 1
        kw['callback'] = cb
    if matrix_solver is not None:
        kw.pop('callback', None)
        x, info = matrix_solver(A.tocsr(), b, **kw), None
    else:
        x, info = scipy.sparse.linalg.qmr(A.tocsr(), b, **kw)
    E = (Pl.conj().T @ x) if adjoint else (Pr @ x)
    return E, info


BREAKDOWN_RATIO = 1e-14


def cocg(omega, dxes, epsilon, b0, mu=None, pec=None, pmc=None, *, rtol=1e-8, maxiter=100000,
         x0=None, history=None):
    """E-space COCG: solves ``A0 E = b0`` with bilinear form ``<u, v> = sum(u * p^2 * v)``.

    Stops when the true residual ``||b0 - A0 E||`` (recurrence value) is
    ``<= rtol ||b0||``.  Returns ``(E, iterations, status)`` with status 0 =
    converged, 1 = maxiter, 2 = breakdown.
    """
    W = precond_p2(dxes).ravel()
    mask = numpy.where(pec, 0, 1) if pec is not None else None
    b0 = numpy.asarray(b0, dtype=complex)
    if mask is not None:
        b0 = b0 * mask

    def A(v):
        return e_full_apply(omega, dxes, epsilon, v, mu, pec, pmc)
    x = numpy.zeros_like(b0) if x0 is None else numpy.array(x0, dtype=complex)
    r = b0 - A(x) if x0 is not None else b0.copy()
    p = numpy.zeros_like(b0)
    bnorm = numpy.linalg.norm(b0)
    aW = numpy.abs(W)
    rho = numpy.sum(r * W * r)
    beta = 0.0
    for it in range(maxiter):
        if numpy.linalg.norm(r) <= rtol * bnorm:
            return x, it, 0
        # (near) breakdown: the unconjugated form cancelled below 1e-14 of its bound
        if abs(rho) <= BREAKDOWN_RATIO * numpy.sum(aW * abs(r) ** 2):
            return x, it, 2
        p = r + beta * p
        q = A(p)
        sigma = numpy.sum(p * W * q)
        bound = numpy.sqrt(numpy.sum(aW * abs(p) ** 2) * numpy.sum(aW * abs(q) ** 2))
        if not numpy.isfinite(sigma) or abs(sigma) <= BREAKDOWN_RATIO * bound:
            return x, it, 2
        alpha = rho / sigma
        x = x + alpha * p
        r = r - alpha * q
        rho_new = numpy.sum(r * W * r)
        beta = rho_new / rho
        rho = rho_new
        if history is not None:
            history.append(numpy.linalg.norm(r) / bnorm)
    return x, maxiter, 1
