"""Generate tests/golden/*.npz by running the reference meanas itself.

Run from the repository root with the path of a reference checkout:

    python tests/golden/make_golden.py <path to the meanas checkout>

The reference is pure Python (numpy/scipy) and imports directly; this script is
the only place that reads it.  Outputs:

* ``scpml.npz``     ``stretch_with_scpml`` / ``uniform_grid_scpml`` cell widths.
* ``operator.npz``  random small problems (PML, non-uniform widths, eps, mu, PEC,
                    PMC) with ``e_full @ x``, ``(Pl e_full Pr) @ x``, its conjugate
                    transpose applied to x, and ``Pl``.
* ``solve.npz``     reference ``generic()`` solutions: the grids and fixtures of
                    ``meanas/test/test_fdfd.py`` / ``conftest.py`` (rtol 1e-11,
                    atol 1e-15), the 1D PML cases of ``meanas/test/test_fdfd_pml.py``
                    (their unidirectional sources included), and 3D PML problems
                    with mu, PEC and PMC, forward and adjoint.
* ``e2h.npz``       ``operators.e2h @ x`` (mu, PMC) and the Poynting products
                    ``operators.poynting_e_cross(x) @ conj(H)`` and
                    ``functional.poynting_e_cross_h(dxes)(x, conj(H))`` on random
                    small problems.
* ``sources.npz``   ``operators.e_tfsf_source(Q, ...) @ x`` and
                    ``operators.e_boundary_source(Q, ..., periodic_mask_edges) @ x`` for
                    box-shaped and random total-field regions.
* ``fdtd.npz``      reference FDTD trajectories: ``maxwell_h`` / ``maxwell_e`` steps with a
                    current injected at steps 0, 4, 8 (the loop of
                    ``meanas/test/test_fdtd.py:203-235``), and ``updates_with_cpml`` with
                    ``cpml_params`` on every face (float32 and float64 fields), plus the
                    CPML parameter tables.
* ``dipole48.npz``  reference ``generic()`` on the 48^3 dipole-in-core problem
                    (rtol 1e-8, scipy QMR): field stored as complex64.
* ``modesrc.npz``   ``waveguide_3d.expand_e`` and ``waveguide_3d.compute_source`` with their
                    inputs: the mode fields of ``meanas/test/test_fdfd_pml.py`` on its 1D
                    grids, and random cross-section fields on 3D grids (PML, non-uniform
                    widths, mu, partial transverse windows, complex wavenumbers, every axis
                    and both polarities).
* ``grad96.npz``    the adjoint gradient of the 96x96x64 design problem from the reference's
                    own solves: ``generic()`` for E, ``generic(adjoint=True)`` with
                    ``-i omega J_adj = 2 E`` on the monitor plane, ``dL/deps =
                    Re(omega^2 conj(E_adj) E)`` over the 40x40x8 design region (not part of
                    the default set: two QMR solves of 1.77M unknowns take hours; the QMR
                    tolerance comes from GRAD96_RTOL, default 1e-10, and is stored).
* ``grad48.npz``    the same on the design problem scaled to 48x48x40 (``GRAD48``), whose two
                    QMR solves take minutes.
"""
from __future__ import annotations

import os
import sys
import time
from pathlib import Path

import numpy

if len(sys.argv) < 2:
    sys.exit('usage: python tests/golden/make_golden.py <path to the meanas checkout> [names...]')
REF = sys.argv[1]
sys.path.insert(0, REF)
sys.path.insert(0, str(Path(__file__).resolve().parents[2]))

import scipy.sparse  # noqa: E402
from meanas.fdfd import functional, operators, scpml, solvers, waveguide_3d  # noqa: E402
from meanas import fdtd  # noqa: E402
from meanas.fdmath import vec, unvec  # noqa: E402

# generic(adjoint=True) uses csr_array.H, which SciPy >= 1.14 removed.
if not hasattr(scipy.sparse.csr_array, 'H'):
    scipy.sparse.csr_array.H = property(lambda s: s.conj().T)
    scipy.sparse.dia_array.H = property(lambda s: s.conj().T)

OUT = Path(__file__).resolve().parent


def pack_dxes(prefix: str, dxes, out: dict) -> None:
    for g in range(2):
        for a in range(3):
            out[f'{prefix}dx{g}{a}'] = numpy.asarray(dxes[g][a], dtype=complex)


def gen_scpml() -> None:
    out = {}
    cases = [((48, 48, 48), 2 * numpy.pi / 30, 10, 1.0, -16, 3.5),
             ((20, 17, 9), 0.7, 4, 1.3, -12, 4.0),
             ((30, 1, 1), 1 / 1500, 10, 2.5, -16, 4.0),
             ((64, 40, 33), 2 * numpy.pi / 26, 7, 2.1, -20, 3.0)]
    for n, (shape, om, th, eff, lnr, m) in enumerate(cases):
        dxes = [[numpy.ones(s) for s in shape] for _ in range(2)]
        sf = scpml.prepare_s_function(ln_R=lnr, m=m)
        for ax in range(3):
            if shape[ax] <= 2 * th:
                continue
            for pol in (-1, 1):
                dxes = scpml.stretch_with_scpml(dxes, axis=ax, polarity=pol, omega=om,
                                                epsilon_effective=eff, thickness=th, s_function=sf)
        out[f'c{n}_params'] = numpy.array([om, th, eff, lnr, m])
        out[f'c{n}_shape'] = numpy.array(shape)
        pack_dxes(f'c{n}_', dxes, out)
        u = scpml.uniform_grid_scpml(shape, [min(th, s // 3) for s in shape], om, eff)
        pack_dxes(f'c{n}_u', u, out)
        out[f'c{n}_uth'] = numpy.array([min(th, s // 3) for s in shape])
    out['n'] = numpy.array(len(cases))
    numpy.savez_compressed(OUT / 'scpml.npz', **out)


def gen_operator() -> None:
    rng = numpy.random.default_rng(2024)
    out = {}
    cases = [((6, 5, 4), True, True, True, 2),
             ((7, 6, 1), False, True, False, 2),
             ((1, 6, 7), True, False, True, 0),
             ((9, 8, 7), False, False, False, 3),
             ((12, 10, 8), True, True, True, 3),
             ((5, 1, 5), False, False, False, 0),
             ((21, 9, 34), True, True, True, 4),
             ((4, 37, 1), True, True, True, 1)]
    for n, (shape, use_mu, use_pec, use_pmc, th) in enumerate(cases):
        om = complex(2 * numpy.pi / rng.uniform(6, 12), 0.0) if n != 3 else complex(0.9, 0.05)
        dxes = [[rng.uniform(0.8, 1.3, s) for s in shape] for _ in range(2)]
        sf = scpml.prepare_s_function(ln_R=-16, m=3.5)
        for ax in range(3):
            if shape[ax] > 2 * th + 1 and th > 0:
                for pol in (-1, 1):
                    dxes = scpml.stretch_with_scpml(dxes, axis=ax, polarity=pol, omega=om.real,
                                                    thickness=th, s_function=sf)
        N3 = 3 * int(numpy.prod(shape))
        eps = rng.uniform(1, 12.1, N3)
        mu = rng.uniform(1, 1.5, N3) if use_mu else None
        pec = (rng.random(N3) < 0.08).astype(float) if use_pec else None
        pmc = (rng.random(N3) < 0.05).astype(float) if use_pmc else None
        x = rng.standard_normal(N3) + 1j * rng.standard_normal(N3)
        A0 = operators.e_full(om, dxes, eps, mu, pec, pmc).tocsr()
        Pl, Pr = operators.e_full_preconditioners(dxes)
        S = (Pl @ A0 @ Pr).tocsr()
        p = f'c{n}_'
        out[p + 'shape'] = numpy.array(shape)
        out[p + 'omega'] = numpy.array(om)
        pack_dxes(p, dxes, out)
        out[p + 'eps'] = eps
        for name, arr in (('mu', mu), ('pec', pec), ('pmc', pmc)):
            if arr is not None:
                out[p + name] = arr
        out[p + 'x'] = x
        out[p + 'A0x'] = A0 @ x
        out[p + 'Sx'] = S @ x
        out[p + 'SHx'] = S.conj().T @ x
        out[p + 'pl'] = Pl.diagonal()
    out['n'] = numpy.array(len(cases))
    numpy.savez_compressed(OUT / 'operator.npz', **out)


def gen_e2h() -> None:
    rng = numpy.random.default_rng(77)
    out = {}
    cases = [((6, 5, 4), True, True, 2),
             ((7, 6, 1), False, True, 2),
             ((1, 6, 7), True, False, 0),
             ((9, 8, 7), False, False, 3),
             ((21, 9, 34), True, True, 4),
             ((4, 37, 1), True, True, 1)]
    for n, (shape, use_mu, use_pmc, th) in enumerate(cases):
        om = complex(2 * numpy.pi / rng.uniform(6, 12), 0.0) if n != 3 else complex(0.9, 0.05)
        dxes = [[rng.uniform(0.8, 1.3, s) for s in shape] for _ in range(2)]
        sf = scpml.prepare_s_function(ln_R=-16, m=3.5)
        for ax in range(3):
            if shape[ax] > 2 * th + 1 and th > 0:
                for pol in (-1, 1):
                    dxes = scpml.stretch_with_scpml(dxes, axis=ax, polarity=pol, omega=om.real,
                                                    thickness=th, s_function=sf)
        N3 = 3 * int(numpy.prod(shape))
        mu = rng.uniform(1, 1.5, N3) if use_mu else None
        pmc = (rng.random(N3) < 0.05).astype(float) if use_pmc else None
        x = rng.standard_normal(N3) + 1j * rng.standard_normal(N3)
        H = operators.e2h(om, dxes, mu, pmc) @ x
        p = f'c{n}_'
        out[p + 'shape'] = numpy.array(shape)
        out[p + 'omega'] = numpy.array(om)
        pack_dxes(p, dxes, out)
        for name, arr in (('mu', mu), ('pmc', pmc)):
            if arr is not None:
                out[p + name] = arr
        out[p + 'x'] = x
        out[p + 'H'] = H
        out[p + 'S_op'] = operators.poynting_e_cross(x, dxes) @ H.conj()
        out[p + 'S_fn'] = vec(functional.poynting_e_cross_h(dxes)(unvec(x, shape), unvec(H.conj(), shape)))
    out['n'] = numpy.array(len(cases))
    numpy.savez_compressed(OUT / 'e2h.npz', **out)


def gen_sources() -> None:
    rng = numpy.random.default_rng(5)
    out = {}
    cases = [((10, 9, 8), True, 'box', 2),
             ((12, 7, 1), False, 'box', 2),
             ((1, 9, 11), True, 'random', 0),
             ((8, 8, 8), False, 'random', 3),
             ((16, 11, 13), True, 'box', 3)]
    for n, (shape, use_mu, kind, th) in enumerate(cases):
        om = complex(2 * numpy.pi / rng.uniform(6, 12), 0.0)
        dxes = [[rng.uniform(0.8, 1.3, s) for s in shape] for _ in range(2)]
        sf = scpml.prepare_s_function(ln_R=-16, m=3.5)
        for ax in range(3):
            if shape[ax] > 2 * th + 1 and th > 0:
                for pol in (-1, 1):
                    dxes = scpml.stretch_with_scpml(dxes, axis=ax, polarity=pol, omega=om.real,
                                                    thickness=th, s_function=sf)
        N3 = 3 * int(numpy.prod(shape))
        eps = rng.uniform(1, 12.1, N3)
        mu = rng.uniform(1, 1.5, N3) if use_mu else None
        if kind == 'box':
            q = numpy.zeros((3, *shape))
            sl = tuple(slice(s // 4, max(s // 4 + 1, 3 * s // 4)) for s in shape)
            q[(slice(None), *sl)] = 1.0
            q = q.ravel()
        else:
            q = (rng.random(N3) < 0.3).astype(float)
        x = rng.standard_normal(N3) + 1j * rng.standard_normal(N3)
        p = f'c{n}_'
        out[p + 'shape'] = numpy.array(shape)
        out[p + 'omega'] = numpy.array(om)
        pack_dxes(p, dxes, out)
        out[p + 'eps'] = eps
        if mu is not None:
            out[p + 'mu'] = mu
        out[p + 'q'] = q
        out[p + 'x'] = x
        out[p + 'tfsf'] = operators.e_tfsf_source(q, om, dxes, eps, mu) @ x
        out[p + 'edge_mirror'] = operators.e_boundary_source(q, om, dxes, eps, mu) @ x
        out[p + 'edge_periodic'] = operators.e_boundary_source(q, om, dxes, eps, mu,
                                                               periodic_mask_edges=True) @ x
    out['n'] = numpy.array(len(cases))
    numpy.savez_compressed(OUT / 'sources.npz', **out)


def gen_fdtd() -> None:
    rng = numpy.random.default_rng(99)
    out = {}
    n = 0
    # plain Yee updates (maxwell_h then maxwell_e, current added at steps 0, 4, 8)
    for shape, dt, kind in (((5, 5, 1), 0.3, 'center'), ((6, 7, 5), 0.3, 'random'), ((9, 4, 6), 0.25, 'random')):
        f3 = (3, *shape)
        dxes = [[numpy.full(s, 1.5) for s in shape] for _ in range(2)]
        for g in range(2):
            for a in range(3):
                dxes[g][a][dxes[g][a].size // 2] *= 1.1
        eps = rng.uniform(1.0, 2.5, f3)
        j = numpy.zeros(f3)
        if kind == 'center':
            j[:, shape[0] // 2, shape[1] // 2, shape[2] // 2] = 1.0
        else:
            j[:] = rng.uniform(-1, 1, f3)
        e = numpy.zeros(f3)
        h = numpy.zeros(f3)
        eh2h = fdtd.maxwell_h(dt=dt, dxes=dxes)
        eh2e = fdtd.maxwell_e(dt=dt, dxes=dxes)
        es, hs = [], []
        for tt in range(10):
            e = e.copy()
            h = h.copy()
            eh2h(e, h)
            eh2e(e, h, eps)
            if tt in (0, 4, 8):
                e += j / eps
            es.append(e)
            hs.append(h)
        p = f'c{n}_'
        out[p + 'kind'] = numpy.array('plain')
        out[p + 'shape'] = numpy.array(shape)
        out[p + 'dt'] = numpy.array(dt)
        for g in range(2):
            for a in range(3):
                out[f'{p}dx{g}{a}'] = dxes[g][a]
        out[p + 'eps'] = eps
        out[p + 'j'] = j
        out[p + 'es'] = numpy.array(es)
        out[p + 'hs'] = numpy.array(hs)
        n += 1
    # CPML updates on all six faces
    for shape, dt, th, ftype in (((20, 16, 14), 0.3, 4, numpy.float32), ((12, 18, 1), 0.3, 5, numpy.float64),
                                 ((16, 12, 22), 0.25, 6, numpy.float64)):
        f3 = (3, *shape)
        dxes = [[rng.uniform(0.9, 1.1, s) for s in shape] for _ in range(2)]
        eps = rng.uniform(1.0, 4.0, f3)
        params = [[None, None] for _ in range(3)]
        for a in range(3):
            if shape[a] > 2 * th:
                for pp, pol in enumerate((-1, 1)):
                    params[a][pp] = fdtd.cpml_params(axis=a, polarity=pol, dt=dt, thickness=th,
                                                     epsilon_eff=1.5, cfs_alpha=0.05)
        upd_e, upd_h = fdtd.updates_with_cpml(cpml_params=params, dt=dt, dxes=dxes, epsilon=eps, dtype=numpy.float32)
        e = numpy.zeros(f3, dtype=ftype)
        h = numpy.zeros(f3, dtype=ftype)
        src = tuple(s // 2 for s in shape)
        es, hs = [], []
        for tt in range(40):
            upd_h(e, h)
            upd_e(e, h, eps)
            e[(2, *src)] += numpy.sin(0.35 * tt) * numpy.exp(-((tt - 12) / 6) ** 2)
            if tt % 8 == 7:
                es.append(e.copy())
                hs.append(h.copy())
        p = f'c{n}_'
        out[p + 'kind'] = numpy.array('cpml')
        out[p + 'shape'] = numpy.array(shape)
        out[p + 'dt'] = numpy.array(dt)
        out[p + 'th'] = numpy.array(th)
        out[p + 'ftype'] = numpy.array(numpy.dtype(ftype).name)
        for g in range(2):
            for a in range(3):
                out[f'{p}dx{g}{a}'] = dxes[g][a]
        out[p + 'eps'] = eps
        out[p + 'es'] = numpy.array(es)
        out[p + 'hs'] = numpy.array(hs)
        for a in range(3):
            for pp in range(2):
                if params[a][pp] is not None:
                    for side in ('e', 'h'):
                        tab = numpy.stack([numpy.ravel(v) for v in params[a][pp]['param_' + side]])
                        out[f'{p}pml{a}{pp}{side}'] = tab
        n += 1
    out['n'] = numpy.array(n)
    numpy.savez_compressed(OUT / 'fdtd.npz', **out)


def gen_solve() -> None:
    """Reference generic() solutions."""
    rng = numpy.random.RandomState(12345)
    out = {}
    n = 0
    om = 1 / 1500

    def store(tag, shape, dxes, eps, J, E, om, mu=None, pec=None, pmc=None, adjoint=False, extra=None):
        nonlocal n
        p = f'c{n}_'
        out[p + 'tag'] = numpy.array(tag)
        out[p + 'shape'] = numpy.array(shape)
        out[p + 'omega'] = numpy.array(complex(om))
        pack_dxes(p, dxes, out)
        out[p + 'eps'] = eps
        out[p + 'J'] = J
        out[p + 'E'] = E
        out[p + 'adjoint'] = numpy.array(adjoint)
        for name, arr in (('mu', mu), ('pec', pec), ('pmc', pmc)):
            if arr is not None:
                out[p + name] = arr
        for k, v in (extra or {}).items():
            out[p + k] = v
        n += 1

    # meanas/test/test_fdfd.py fixtures (test_residual / test_poynting_planes)
    for shape in [(5, 5, 1), (5, 1, 5), (5, 5, 5)]:
        is3d = 1 not in shape
        for eps_kind in ['center', '000', 'random']:
            for bg in [1.0, 1.5]:
                for fg in [1.0, 2.5]:
                    if is3d and (eps_kind == '000' or bg != 1 or fg not in (1.0, 2.0)):
                        continue
                    for dxk in ['uniform', 'centerbig']:
                        for dx in [1.0, 1.5]:
                            eps = numpy.full((3, *shape), bg)
                            if eps_kind == 'center':
                                eps[:, shape[0] // 2, shape[1] // 2, shape[2] // 2] = fg
                            elif eps_kind == '000':
                                eps[:, 0, 0, 0] = fg
                            else:
                                eps[:] = rng.uniform(low=min(bg, fg), high=max(bg, fg), size=(3, *shape))
                            dxes = [[numpy.full(s, dx) for s in shape] for _ in range(2)]
                            if dxk == 'centerbig':
                                for eh in (0, 1):
                                    for ax in (0, 1, 2):
                                        dxes[eh][ax][dxes[eh][ax].size // 2] *= 1.1
                            j = numpy.zeros((3, *shape), dtype=complex)
                            cm = numpy.zeros((3, *shape), dtype=bool)
                            cm[:, shape[0] // 2, shape[1] // 2, shape[2] // 2] = True
                            j[numpy.roll(cm, [1, 1, 1], axis=(1, 2, 3))] = 1 + 1j
                            j[numpy.roll(cm, [-1, -1, -1], axis=(1, 2, 3))] = 1 - 1j
                            E = solvers.generic(J=vec(j), omega=om, dxes=dxes, epsilon=vec(eps),
                                                matrix_solver_opts=dict(atol=1e-15, rtol=1e-11))
                            store('test_fdfd', shape, dxes, vec(eps), vec(j), E, om)

    # meanas/test/test_fdfd_pml.py (test_pml): 1D grids, PML on the propagation axis
    for shape in [(30, 1, 1), (1, 30, 1), (1, 1, 30)]:
        for pol in (+1, -1):
            for fg in (1.0, 2.5):
                for dx in (1.0, 1.5):
                    sh3 = (3, *shape)
                    eps = numpy.full(sh3, fg)
                    dxes = [[numpy.full(s, dx) for s in shape] for _ in range(2)]
                    dim = numpy.where(numpy.array(shape) > 1)[0][0]
                    for p_ in (-1, 1):
                        dxes = scpml.stretch_with_scpml(dxes, axis=dim, polarity=p_, omega=om,
                                                        epsilon_effective=fg, thickness=10)
                    other = [0, 1, 2]
                    other.remove(dim)
                    dx_prop = (dxes[0][dim][shape[dim] // 2] + dxes[1][dim][shape[dim] // 2]) / 2
                    cm = numpy.zeros(sh3, dtype=bool)
                    cm[other, shape[0] // 2, shape[1] // 2, shape[2] // 2] = True
                    k = om * numpy.sqrt(eps[cm].mean())
                    kc = 2 / dx_prop * numpy.arcsin(k * dx_prop / 2)
                    e = numpy.zeros_like(eps, dtype=complex)
                    e[cm] = 1 / numpy.linalg.norm(cm[:])
                    sl = [slice(None)] * 3
                    sl[dim] = slice(shape[dim] // 2, shape[dim] // 2 + 1)
                    j = waveguide_3d.compute_source(E=e, wavenumber=kc, omega=om, dxes=dxes, axis=dim,
                                                    polarity=pol, slices=sl, epsilon=eps)
                    E = solvers.generic(J=vec(j), omega=om, dxes=dxes, epsilon=vec(eps),
                                        matrix_solver_opts={'atol': 1e-15, 'rtol': 1e-11})
                    store('test_pml', shape, [list(d) for d in dxes], vec(eps), vec(j), E, om,
                          extra=dict(src_polarity=numpy.array(pol)))

    # 3D PML problems with mu / PEC / PMC, forward and adjoint
    r2 = numpy.random.default_rng(7)
    for shape, th, use_mu, use_masks in [((12, 10, 8), 3, True, True), ((10, 9, 7), 2, False, True),
                                         ((14, 12, 1), 3, True, False), ((11, 8, 9), 2, True, True)]:
        om2 = 2 * numpy.pi / 8
        dxes = [[r2.uniform(0.9, 1.1, s) for s in shape] for _ in range(2)]
        for ax in range(3):
            if shape[ax] > 2 * th + 1:
                for p_ in (-1, 1):
                    dxes = scpml.stretch_with_scpml(dxes, axis=ax, polarity=p_, omega=om2, thickness=th)
        N3 = 3 * int(numpy.prod(shape))
        eps = r2.uniform(1, 12, N3)
        mu = r2.uniform(1, 1.5, N3) if use_mu else None
        pec = (r2.random(N3) < 0.05).astype(float) if use_masks else None
        pmc = (r2.random(N3) < 0.03).astype(float) if use_masks else None
        J = numpy.zeros((3, *shape), dtype=complex)
        c = tuple(s // 2 for s in shape)
        J[(2, *c)] = 1.0
        J[(0, *c)] = 0.5j
        Jv = vec(J)
        if pec is not None:
            Jv = Jv * (pec == 0)
        for adjoint in (False, True):
            E = solvers.generic(omega=om2, dxes=dxes, J=Jv, epsilon=eps, mu=mu, pec=pec, pmc=pmc,
                                adjoint=adjoint, matrix_solver_opts=dict(rtol=1e-12, atol=0))
            store('pml3d', shape, dxes, eps, Jv, E, om2, mu, pec, pmc, adjoint=adjoint)
    out['n'] = numpy.array(n)
    numpy.savez_compressed(OUT / 'solve.npz', **out)


def gen_dipole48() -> None:
    from meanas_b200 import workloads
    p = workloads.dipole_core(48)
    it = [0]

    def qmr_counting(A, b, **kw):
        def cb(_):
            it[0] += 1
        return scipy.sparse.linalg.qmr(A, b, callback=cb, **kw)[0]
    t0 = time.perf_counter()
    E = solvers.generic(p.omega, p.dxes, p.J, p.epsilon, matrix_solver=qmr_counting,
                        matrix_solver_opts=dict(rtol=1e-8, atol=0))
    t1 = time.perf_counter()
    A0 = operators.e_full(p.omega, p.dxes, p.epsilon).tocsr()
    b0 = -1j * p.omega * p.J
    res = numpy.linalg.norm(A0 @ E - b0) / numpy.linalg.norm(b0)
    numpy.savez_compressed(OUT / 'dipole48.npz', E=E.astype(numpy.complex64), qmr_iterations=it[0],
                           seconds=t1 - t0, residual=res)
    print('dipole48', it[0], t1 - t0, res)


def gen_modesrc() -> None:
    out = {}
    n = 0

    def store(shape, dxes, eps, mu, E, k, om, axis, pol, sl):
        nonlocal n
        p = f'c{n}_'
        Ee = waveguide_3d.expand_e(E=E, wavenumber=k, dxes=dxes, axis=axis, polarity=pol, slices=sl)
        J = waveguide_3d.compute_source(E=E, wavenumber=k, omega=om, dxes=dxes, axis=axis, polarity=pol,
                                        slices=sl, epsilon=eps, mu=mu)
        out[p + 'shape'] = numpy.array(shape)
        out[p + 'omega'] = numpy.array(complex(om))
        out[p + 'k'] = numpy.array(complex(k))
        out[p + 'axis'] = numpy.array(axis)
        out[p + 'polarity'] = numpy.array(pol)
        out[p + 'slices'] = numpy.array([[s_.start if s_.start is not None else -(10 ** 9),
                                          s_.stop if s_.stop is not None else 10 ** 9] for s_ in sl])
        pack_dxes(p, dxes, out)
        out[p + 'eps'] = eps
        if mu is not None:
            out[p + 'mu'] = mu
        out[p + 'E'] = E
        out[p + 'E_expanded'] = numpy.asarray(Ee)
        out[p + 'J'] = numpy.asarray(J)
        n += 1

    # meanas/test/test_fdfd_pml.py: the hand-built mode on 1D grids (fixtures there)
    om = 1 / 1500
    for shape in [(30, 1, 1), (1, 30, 1), (1, 1, 30)]:
        for pol in (+1, -1):
            for fg in (1.0, 2.5):
                dx = 1.0 if fg == 1.0 else 1.5
                sh3 = (3, *shape)
                eps = numpy.full(sh3, fg)
                dxes = [[numpy.full(s_, dx) for s_ in shape] for _ in range(2)]
                dim = int(numpy.where(numpy.array(shape) > 1)[0][0])
                for p_ in (-1, 1):
                    dxes = scpml.stretch_with_scpml(dxes, axis=dim, polarity=p_, omega=om,
                                                    epsilon_effective=fg, thickness=10)
                other = [0, 1, 2]
                other.remove(dim)
                dx_prop = (dxes[0][dim][shape[dim] // 2] + dxes[1][dim][shape[dim] // 2]) / 2
                cm = numpy.zeros(sh3, dtype=bool)
                cm[other, shape[0] // 2, shape[1] // 2, shape[2] // 2] = True
                k = om * numpy.sqrt(eps[cm].mean())
                kc = 2 / dx_prop * numpy.arcsin(k * dx_prop / 2)
                e = numpy.zeros_like(eps, dtype=complex)
                e[cm] = 1 / numpy.linalg.norm(cm[:])
                sl = [slice(None)] * 3
                sl[dim] = slice(shape[dim] // 2, shape[dim] // 2 + 1)
                store(shape, [list(d) for d in dxes], eps, None, e, kc, om, dim, pol, sl)

    # 3D grids: random cross-section fields in partial windows, PML, mu, complex wavenumbers
    rng = numpy.random.default_rng(77)
    for shape, axis, pol, th, use_mu in [((14, 11, 9), 0, 1, 3, False), ((14, 11, 9), 0, -1, 3, True),
                                         ((9, 16, 10), 1, 1, 2, True), ((9, 16, 10), 1, -1, 0, False),
                                         ((10, 9, 17), 2, 1, 3, True), ((10, 9, 17), 2, -1, 3, False),
                                         ((12, 13, 1), 0, 1, 3, False), ((1, 12, 13), 2, -1, 2, True)]:
        om3 = 2 * numpy.pi / rng.uniform(6, 10)
        dxes = [[rng.uniform(0.8, 1.2, s_) for s_ in shape] for _ in range(2)]
        for ax in range(3):
            if th and shape[ax] > 2 * th + 1:
                for p_ in (-1, 1):
                    dxes = scpml.stretch_with_scpml(dxes, axis=ax, polarity=p_, omega=om3, thickness=th)
        sh3 = (3, *shape)
        eps = rng.uniform(1, 12, sh3)
        mu = rng.uniform(1, 1.5, sh3) if use_mu else None
        s0 = int(rng.integers(2, shape[axis] - 2)) if shape[axis] > 4 else 0
        sl = []
        for a, n_a in enumerate(shape):
            if a == axis:
                sl.append(slice(s0, s0 + 1))
            elif n_a > 4:
                lo = int(rng.integers(0, n_a // 3))
                sl.append(slice(lo, n_a - int(rng.integers(0, n_a // 3))))
            else:
                sl.append(slice(None))
        E = numpy.zeros(sh3, dtype=complex)
        E[(slice(None), *sl)] = rng.standard_normal((3, *E[(0, *sl)].shape)) + \
            1j * rng.standard_normal((3, *E[(0, *sl)].shape))
        k = om3 * rng.uniform(1.2, 3.0) * (1 - 0.01j)
        store(shape, dxes, eps, mu, E, k, om3, axis, pol, sl)
    out['n'] = numpy.array(n)
    numpy.savez_compressed(OUT / 'modesrc.npz', **out)


def gen_grad96() -> None:
    from meanas_b200 import workloads
    _grad_fixture(workloads.adjoint_design(), os.environ.get('GRAD96_FILE', 'grad96.npz'))


def gen_grad48() -> None:
    from meanas_b200 import workloads
    _grad_fixture(workloads.adjoint_design(**GRAD48), 'grad48.npz')


# the 96x96x64 design problem scaled down (the reference's QMR solves take minutes)
GRAD48 = dict(shape=(48, 48, 40), pml=8, wavelength=26.0, design=(16, 16, 6), source_x=12, monitor_x=36)


def _grad_fixture(p, name: str) -> None:
    its = []

    t_start = time.perf_counter()

    def qmr_counting(A, b, **kw):
        it = [0]

        def cb(_):
            it[0] += 1
            if it[0] % 1000 == 0:
                print(f'{name}: solve {len(its) + 1}, QMR iteration {it[0]}, '
                      f'{time.perf_counter() - t_start:.0f} s', flush=True)
        x = scipy.sparse.linalg.qmr(A, b, callback=cb, **kw)[0]
        its.append(it[0])
        return x
    # GRAD96_RTOL: the QMR tolerance of both solves (default 1e-10)
    opts = dict(rtol=float(os.environ.get('GRAD96_RTOL', '1e-10')), atol=0)
    t0 = time.perf_counter()
    E = solvers.generic(p.omega, p.dxes, p.J, p.epsilon, matrix_solver=qmr_counting,
                        matrix_solver_opts=opts)
    mon = p.extra['monitor']
    G = 2 * E * mon                     # dL/dE* convention of torch: L = sum |E|^2 on the plane
    J_adj = G / (-1j * p.omega)
    E_adj = solvers.generic(p.omega, p.dxes, J_adj, p.epsilon, adjoint=True,
                            matrix_solver=qmr_counting, matrix_solver_opts=opts)
    t1 = time.perf_counter()
    grad = numpy.real(p.omega ** 2 * numpy.conj(E_adj) * E).reshape(3, *p.shape)
    dsl = p.extra['design_slices']
    A0 = operators.e_full(p.omega, p.dxes, p.epsilon).tocsr()
    b0 = -1j * p.omega * p.J
    res = numpy.linalg.norm(A0 @ E - b0) / numpy.linalg.norm(b0)
    ba = -1j * p.omega * J_adj
    res_adj = numpy.linalg.norm(A0.conj().T @ E_adj - ba) / numpy.linalg.norm(ba)
    numpy.savez_compressed(OUT / name, grad_design=grad[(slice(None), *dsl)],
                           eps_design=p.epsilon.reshape(3, *p.shape)[(slice(None), *dsl)],
                           loss=float(numpy.sum(numpy.abs(E[mon]) ** 2)), qmr_iterations=numpy.array(its),
                           seconds=t1 - t0, residual=res, residual_adjoint=res_adj, rtol=opts['rtol'])
    print(name, its, t1 - t0, res, res_adj)


if __name__ == '__main__':
    which = sys.argv[2:] or ['scpml', 'operator', 'e2h', 'sources', 'fdtd', 'solve', 'dipole48', 'modesrc']
    for w in which:
        t = time.perf_counter()
        globals()[f'gen_{w}']()
        print(w, f'{time.perf_counter() - t:.1f}s')
