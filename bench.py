"""Benchmark: FDFD solves/s at FP64 residual 1e-8 (mixed vs FP64 GPU), p50/p99 latency.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one full solve from a zero initial guess to a true FP64
relative residual ||b0 - A0 E|| / ||b0|| <= 1e-8): the 160x160x128 grid with a
12-cell SC-PML (stretch_with_scpml, ln_R = -16, m = 3.5), omega = 2 pi / 24,
diagonal anisotropic eps in {1, 2.1, 12.1} on seeded random 8-20 cell blocks
(30% of the interior), and a Gaussian (sigma = 6 cells) Jy plane source at z = 20.
Synthetic, seeded data; every input array (eps, J, tables) is larger than the
L2 cache in total and the solve streams several 150 MB vectors per iteration, so
no L2 flush is added between steps.

Both GPU solvers are timed: the complex128 COCG solver (the plain FP64 drop-in)
and the mixed-precision solver (complex64 BiCGSTAB inner solves refined in
complex128).  `value` is the faster one's solves/s; both are reported.

Multi-GPU (torchrun, N > 1): replicas only -- each rank solves its own copy; the
job's solves/s is N*K over the slowest rank's time (weak scaling).

`--impl reference` times the reference algorithm on the host CPU: the oracle port
of meanas' generic() (CSR assembly + scipy.sparse.linalg.qmr on the symmetrised
system) on a bounded sample (operator assembly + a fixed number of QMR
iterations), extrapolated to a full solve with the iteration count stated in the
JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = 'FDFD solves/s at FP64 residual 1e-8, mixed vs FP64 GPU; p50/p99 latency'
WORKLOADS = {
    'aniso_blocks': 'aniso_blocks 160x160x128, 12-cell SC-PML, omega=2pi/24, '
                    'diag-anisotropic eps blocks {1,2.1,12.1}, Gaussian Jy plane z=20',
    'dipole_core': 'dipole_core 48^3, 10-cell SC-PML, omega=2pi/30, eps=12.1 core, unit Jz dipole',
    'masked_large': 'masked_large 320x320x200, 16-cell SC-PML, omega=2pi/20, eps in [1,12.1], '
                    'mu in [1,1.5], PEC 5% / PMC 2% slabs, 3 dipoles',
}


def workload_config(name: str, p) -> dict:
    return dict(workload=WORKLOADS[name], shape=list(p.shape), unknowns=p.n_unknowns, rtol=1e-8,
                criterion='true FP64 residual ||b0-A0 E||/||b0||',
                l2=('inputs and per-iteration vectors larger than L2 (no flush)' if p.n_cells * 456 > 126e6
                    else 'working set fits in L2 (small reference case)'))
RTOL = 1e-8
# Algorithmic bytes per cell of each iteration kernel (complex128 = 16 B, complex64 = 8 B
# per component, eps 3 reals; the stencil's halo and neighbour-plane re-reads are served
# from L2 and not counted):
#   COCG stencil pass (c128): read r, p_old, x, eps; write p, x, q   = 6*48 + 24 = 312
#   COCG pointwise pass (c128): read r, q; write r                  = 3*48      = 144
#   BiCGSTAB P pass (c64): read r, v, t, p, x, eps; write r, p, v, x = 9*24 + 12 = 228
#   BiCGSTAB S pass (c64): read r, v, eps; write t                   = 3*24 + 12 = 84
KERNEL_BYTES_PER_CELL = {0: 312, 1: 144, 2: 228, 3: 84}
METHOD_NAMES = {'cocg': 'fp64 (complex128 COCG)', 'mixed': 'mixed (complex64 inner, complex128 refinement)'}
KERNEL_NAMES = {0: 'cocg_stencil_c128', 1: 'cocg_point_c128', 2: 'bicgstab_P_c64', 3: 'bicgstab_S_c64'}


def peaks() -> tuple[float, str]:
    p = ROOT / 'MEASURED_PEAKS.json'
    if p.exists():
        try:
            return float(json.loads(p.read_text())['hbm_gbs']), 'measured'
        except Exception:
            pass
    return 6650.0, 'fallback'


PROFILE_TAGS = {'aniso_blocks': 'aniso160', 'dipole_core': 'dipole48', 'masked_large': 'masked320'}


def profile_traffic(kernel: str, workload: str) -> tuple[float | None, str | None]:
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu summary
    profiles/<kernel>_<workload tag>.md, and where that number comes from (the file and the
    source commit it records for the capture).  (None, None) when no capture exists: ncu
    cannot run inside the timed program, so the figure is the one of the last capture."""
    f = ROOT / 'profiles' / f'{kernel}_{PROFILE_TAGS[workload]}.md'
    if f.exists():
        text = f.read_text()
        m = re.search(r'traffic_bytes_per_launch:\s*([0-9.eE+]+)', text)
        if m:
            c = re.search(r'captured_source_commit:\s*([0-9a-f]+)', text)
            return float(m.group(1)), f'profiles/{f.name}' + (f' (capture of commit {c.group(1)})' if c else '')
    return None, None


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(f'/tmp/fdfd_clocks_{os.getpid()}.csv')

    def __enter__(self):
        try:
            self.fh = open(self.path, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.Q}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self) -> dict:
        if self.proc is None or not self.path.exists():
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        sm, smax, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        self.path.unlink(missing_ok=True)
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': smax,
                'reasons': sorted(reasons), 'samples': len(sm)}


def dist_setup(n_gpus: int):
    import torch
    import torch.distributed as dist
    rank, world = int(os.environ.get('RANK', 0)), int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def _collective_device() -> str:
    import torch
    import torch.distributed as dist
    return 'cuda' if dist.is_initialized() and dist.get_backend() == 'nccl' and torch.cuda.is_available() else 'cpu'


def barrier_sync(world: int):
    import torch
    import torch.distributed as dist
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
        if torch.cuda.is_available():
            torch.cuda.synchronize()


def max_over_ranks(v: float, world: int) -> float:
    """The largest value over the ranks (every rank gets it): multi-GPU times are the slowest
    rank's.  NCCL reduces on the device; a gloo group (CPU tests) on the host."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=_collective_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args) -> dict | None:
    import torch
    from meanas_b200 import workloads
    from meanas_b200.operators import GridOperator
    from meanas_b200.solvers import generic

    rank, world, local = dist_setup(args.gpus)
    dev = torch.device('cuda', torch.cuda.current_device())
    p = workloads.BY_NAME[args.workload]()
    ncell = p.n_cells
    op = GridOperator(p.omega, p.dxes, p.epsilon, p.mu, p.pec, p.pmc, device=dev, fp32=True)
    J = torch.as_tensor(p.J, device=dev)
    stream = torch.cuda.current_stream()
    tuned = op.autotune(methods=tuple(args.methods.split(','))) if args.autotune else {}

    fields = {}  # the last timed field of each method

    def timed(method: str, steps: int, warmup: int, profile: bool):
        kw = dict(method=method, rtol=RTOL, criterion='true', profile=profile, maxiter=args.maxiter)
        for _ in range(warmup):
            op.solve(J, **kw)
        lat, infos = [], []
        barrier_sync(world)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            E, info = op.solve(J, **kw)
            b.record(stream)
            fields[method] = E
            infos.append(info)
            lat.append((a, b))
        t1.record(stream)
        barrier_sync(world)
        total_ms = t0.elapsed_time(t1)
        lats = [x.elapsed_time(y) for x, y in lat]
        return max_over_ranks(total_ms, world), lats, infos

    # Per-kernel CUDA-event timing inside the timed solves costs two event records per launch
    # and disables the iteration graphs (about 10 % at 160x160x128, far more on small grids),
    # so the timed solves run as they do in production (graph launches) and the kernel
    # durations of the roofline come from one profiled solve per method right after them.
    live = args.timed_profile == 'on'
    out = {}
    with Clocks(local) as clk:
        for method in args.methods.split(','):
            total_ms, lats, infos = timed(method, args.steps, args.warmup, profile=live)
            if args.maxiter is None:
                assert all(i.converged and i.residual <= RTOL for i in infos), infos
            prof_ms = total_ms
            if not live:
                prof_ms, _, pinfos = timed(method, 1, 0, profile=True)
            else:
                pinfos = infos
            kms = numpy.sum([i.kernel_ms for i in pinfos], axis=0)
            kcnt = numpy.sum([i.kernel_count for i in pinfos], axis=0)
            out[method] = dict(prof_ms=prof_ms,
                solves_per_s=world * args.steps / (total_ms / 1e3), ms_per_step=total_ms / args.steps,
                p50_ms=float(numpy.percentile(lats, 50)), p99_ms=float(numpy.percentile(lats, 99)),
                iterations=int(numpy.median([i.iterations for i in infos])),
                status=sorted({i.status for i in infos}),
                outer=int(numpy.median([i.outer_iterations for i in infos])),
                residual=max(i.residual for i in infos),
                launches=int(sum(i.kernel_launches for i in infos)),
                kernel_ms=kms.tolist(), kernel_count=kcnt.tolist())
    clocks = clk.summary()

    # end-to-end through the public API: host (pinned) inputs -> generic() -> host E
    e2e = None
    if args.e2e_steps > 0:
        Jh = torch.from_numpy(p.J).pin_memory()
        epsh = torch.from_numpy(p.epsilon).pin_memory()
        best = max(out, key=lambda m: out[m]['solves_per_s'])
        prec = 'mixed' if best == 'mixed' else 'fp64'
        extra = dict(mu=p.mu, pec=p.pec, pmc=p.pmc)
        generic(p.omega, p.dxes, Jh, epsh, precision=prec, criterion='true',
                matrix_solver_opts=dict(rtol=RTOL), device=dev, **extra)
        barrier_sync(world)
        t = time.perf_counter()
        for _ in range(args.e2e_steps):
            E = generic(p.omega, p.dxes, Jh, epsh, precision=prec, criterion='true',
                        matrix_solver_opts=dict(rtol=RTOL), device=dev, **extra)
        barrier_sync(world)
        el = max_over_ranks(time.perf_counter() - t, world)
        assert E.shape == (p.n_unknowns,)
        table_bytes = sum(16 * 2 * numpy.size(d) for g in p.dxes for d in g)
        opt_bytes = sum(8 * a.size for a in (p.mu, p.pec, p.pmc) if a is not None)
        from meanas_b200.solvers import last_solve_info
        e2e_info = last_solve_info()
        e2e = dict(value=world * args.e2e_steps / el, unit='solves/s', method=prec,
                   iterations=e2e_info.iterations, residual=e2e_info.residual,
                   tiling='a fresh plan per call, as generic() builds it, with the x-chunk tuned for this grid size',
                   h2d_bytes_per_step=int(Jh.numel() * 16 + epsh.numel() * 8 + table_bytes + opt_bytes),
                   d2h_bytes_per_step=int(p.n_unknowns * 16))

    if rank != 0:
        return None
    best = max(out, key=lambda m: out[m]['solves_per_s'])
    b = out[best]
    peak, peak_kind = peaks()
    # roofline of the dominant kernel of the reported method
    kinds = [0, 1] if best == 'cocg' else [2, 3]
    dom = max(kinds, key=lambda k: b['kernel_ms'][k])
    avg_ms = b['kernel_ms'][dom] / max(1, b['kernel_count'][dom])
    extra_bytes = 0  # mu^-1 (3 reals) and the mask byte read by the stencil passes
    if dom in (0, 2, 3):
        real = 8 if dom == 0 else 4
        extra_bytes = (3 * real if p.mu is not None else 0) + (1 if (p.pec is not None or p.pmc is not None) else 0)
    alg = (KERNEL_BYTES_PER_CELL[dom] + extra_bytes) * ncell
    achieved = alg / (avg_ms / 1e3) / 1e9
    traffic, traffic_source = profile_traffic(KERNEL_NAMES[dom], args.workload)
    share = b['kernel_ms'][dom] / b['prof_ms']
    steps_total = args.steps
    res = {
        'metric': METRIC, 'value': round(b['solves_per_s'], 4), 'unit': 'solves/s', 'n_gpus': world,
        'value_method': METHOD_NAMES.get(best, best),
        'steps': steps_total, 'warmup': args.warmup, 'ms_per_step': round(b['ms_per_step'], 3),
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'c64 inner + c128 refinement' if best == 'mixed' else 'c128',
        'data': 'synthetic (seeded)',
        'config': dict(workload_config(args.workload, p), method=best, parallelism=f'replicas x{world}'),
        'p50_ms': round(b['p50_ms'], 3), 'p99_ms': round(b['p99_ms'], 3),
        'mixed': ({k: v for k, v in out['mixed'].items() if k not in ('kernel_ms', 'kernel_count', 'prof_ms')}
                  if 'mixed' in out else None),
        'fp64': ({k: v for k, v in out['cocg'].items() if k not in ('kernel_ms', 'kernel_count', 'prof_ms')}
                 if 'cocg' in out else None),
        'mixed_over_fp64': (round(out['mixed']['solves_per_s'] / out['cocg']['solves_per_s'], 3)
                            if 'mixed' in out and 'cocg' in out else None),
        'roofline': {'bound': 'hbm', 'kernel': KERNEL_NAMES[dom], 'achieved': round(achieved, 1),
                     'peak': peak, 'unit': 'GB/s', 'frac': round(achieved / peak, 4),
                     'peak_kind': peak_kind, 'traffic': traffic, 'traffic_source': traffic_source,
                     'algorithmic_bytes_per_launch': alg, 'avg_launch_ms': round(avg_ms, 5),
                     'share_of_step': round(share, 3),
                     'timing': ('CUDA events around every launch of the timed solves' if live else
                                'CUDA events around every launch of one profiled solve after the '
                                'graph-launched timed solves')},
        'field_rel_err': field_errors(fields, args.workload),
        'gpu_launches': int(b['launches']),
        'tiling': {k: {'xchunk': v[0], 'us_per_iteration': round(v[1], 1)} for k, v in tuned.items()},
        'clocks': clocks,
        'e2e': e2e,
    }
    if world == 1 and args.cpu_sample_iters > 0:
        cb = cpu_baseline(p, args.cpu_sample_iters, out['cocg']['iterations'] if 'cocg' in out else b['iterations'],
                          fields=fields)
        # the timed fields checked on the host with the reference's CSR operator
        res['oracle_residual'] = cb.pop('oracle_residual', None)
        res['cpu_baseline'] = cb
    return res


# Krylov iterations of one full solve of each workload, for extrapolating the CPU sample:
# the reference's own QMR count where it was run (48^3: tests/golden/dipole48.npz), else
# the GPU complex128 COCG count measured on a B200 (QMR and COCG build the same Krylov
# space: 1189 vs 1192 iterations at 48^3); the masked case does not converge, so its cap.
REF_ITERS = {
    'dipole_core': (1189, 'the reference QMR count of this problem'),
    'aniso_blocks': (50591, 'the GPU complex128 COCG count of this problem (the reference QMR took 1189 '
                            'vs COCG 1192 on the 48^3 case)'),
    'masked_large': (150000, 'the iteration cap of the unconverged GPU run of this problem'),
}


def field_errors(fields: dict, workload: str) -> dict:
    """Relative field differences of the timed solves: the mixed-precision field against the
    FP64 one, and on the 48^3 case each against the reference's own QMR field
    (tests/golden/dipole48.npz, stored in complex64, so about 1e-7 is its floor)."""
    import torch
    out = {}
    try:
        if 'mixed' in fields and 'cocg' in fields:
            a, b = fields['mixed'], fields['cocg']
            out['mixed_vs_fp64'] = float((a - b).norm() / b.norm())
        if workload == 'dipole_core' and fields:
            ref = numpy.load(ROOT / 'tests' / 'golden' / 'dipole48.npz')['E'].astype(numpy.complex128)
            r = torch.as_tensor(ref, device=next(iter(fields.values())).device)
            for m, e in fields.items():
                out[('fp64' if m == 'cocg' else m) + '_vs_reference_qmr'] = float((e - r).norm() / r.norm())
    except Exception as exc:  # a report only: never a reason to lose the bench line
        out['error'] = repr(exc)
    return out


def host_cpu() -> dict:
    """The host's logical core count and CPU model (as /proc/cpuinfo names it)."""
    model = None
    try:
        for line in Path('/proc/cpuinfo').read_text().splitlines():
            if line.startswith('model name'):
                model = line.split(':', 1)[1].strip()
                break
    except OSError:
        pass
    return {'nproc': os.cpu_count(), 'model': model}


def reference_operator(p):
    """CSR A0 as the reference's e_full assembles it (mu, PEC and PMC included), built by the
    oracle port.  Returns (A0, assembly seconds)."""
    from oracle import fdfd_oracle as O
    t0 = time.perf_counter()
    A0 = O.e_full_csr(p.omega, p.dxes, p.epsilon, p.mu, p.pec, p.pmc)
    return A0, time.perf_counter() - t0


def reference_system(p, A0=None, t_a0: float = 0.0):
    """The system the reference's generic() hands to scipy's QMR: A0 symmetrised with
    Pl / Pr (oracle port).  Returns (A, b, assembly seconds)."""
    from scipy import sparse
    from oracle import fdfd_oracle as O
    if A0 is None:
        A0, t_a0 = reference_operator(p)
    t0 = time.perf_counter()
    pl = O.precond_pl(p.dxes)
    A = (sparse.diags_array(pl) @ A0 @ sparse.diags_array(1 / pl)).tocsr()
    b = pl * (-1j * p.omega * p.J)
    return A, b, t_a0 + time.perf_counter() - t0


def oracle_residuals(p, A0, fields: dict) -> dict:
    """||b0 - A0 E|| / ||b0|| of each timed GPU field with the host CSR operator of the
    reference's e_full (the test of meanas/test/test_fdfd.py:14-18), in FP64 on the CPU."""
    b0 = -1j * p.omega * p.J
    nb = numpy.linalg.norm(b0)
    out = {}
    for m, E in fields.items():
        e = E.detach().cpu().numpy()
        out['fp64' if m == 'cocg' else m] = float(numpy.linalg.norm(A0 @ e - b0) / nb)
    return out


def qmr_seconds_per_iteration(A, b, iters: int) -> float:
    """Wall seconds per scipy QMR iteration over one call of `iters` iterations from zero."""
    import scipy.sparse.linalg
    t = time.perf_counter()
    scipy.sparse.linalg.qmr(A, b, rtol=1e-30, atol=0.0, maxiter=iters)
    return (time.perf_counter() - t) / iters


def extrapolated(t_asm: float, t_iter: float, iters_full: int) -> float:
    """Seconds of one full reference solve: assembly + iters_full QMR iterations."""
    return t_asm + iters_full * t_iter


def cpu_baseline(p, sample_iters: int, iters_full: int, iters_source: str = '', fields: dict | None = None) -> dict:
    """Oracle port of the reference path timed on the host: assembly + `sample_iters`
    scipy QMR iterations, extrapolated to `iters_full` iterations per solve.  The assembled
    CSR operator also checks the timed GPU fields (`fields`): their true residuals go in
    the result's 'oracle_residual'."""
    A0, t_a0 = reference_operator(p)
    checked = oracle_residuals(p, A0, fields) if fields else None
    A, b, t_asm = reference_system(p, A0, t_a0)
    del A0
    t_iter = qmr_seconds_per_iteration(A, b, sample_iters)
    t_solve = extrapolated(t_asm, t_iter, iters_full)
    cpu = host_cpu()
    out = {'value': float(f'{1.0 / t_solve:.6g}'), 'unit': 'solves/s', 'cores': 1, 'kind': 'port',
           'host': cpu,
           'sample': f'CSR assembly ({t_asm:.1f} s) + {sample_iters} scipy QMR iterations '
                     f'({t_iter * 1e3:.0f} ms each; scipy\'s CSR product runs on one thread of the '
                     f'{cpu["nproc"]}-core host) on the full '
                     f'{"x".join(map(str, p.shape))} system, extrapolated to {iters_full} iterations '
                     f'({iters_source or "the GPU complex128 COCG count"})',
           'seconds_per_solve': round(t_solve, 1)}
    if checked is not None:
        out['oracle_residual'] = checked
    return out


def run_reference(args) -> dict | None:
    """Each step times `ref_step_iters` QMR iterations of the reference system (assembled
    once, timed once); the line reports the median step, extrapolated to a full solve."""
    rank = int(os.environ.get('RANK', 0))
    if rank != 0:
        return None
    from meanas_b200 import workloads
    p = workloads.BY_NAME[args.workload]()
    iters_full, source = REF_ITERS[args.workload]
    if args.ref_iters:
        iters_full, source = args.ref_iters, 'given on the command line'
    A, b, t_asm = reference_system(p)
    per_iter = [qmr_seconds_per_iteration(A, b, args.ref_step_iters)
                for _ in range(args.warmup + args.steps)][args.warmup:]
    t_iter = statistics.median(per_iter)
    v = float(f'{1.0 / extrapolated(t_asm, t_iter, iters_full):.6g}')
    cpu = host_cpu()
    sample = (f'CSR assembly ({t_asm:.1f} s, once) + {args.steps} timed steps of {args.ref_step_iters} '
              f'scipy QMR iterations each (median {t_iter * 1e3:.0f} ms per iteration, spread '
              f'{min(per_iter) * 1e3:.0f}-{max(per_iter) * 1e3:.0f} ms; scipy\'s CSR product runs on one '
              f'thread of the {cpu["nproc"]}-core host) on the full {"x".join(map(str, p.shape))} system, '
              f'extrapolated to {iters_full} iterations ({source})')
    # a step is the bounded sample (ms_per_step: its measured wall time); `value` is the
    # full solve it extrapolates to (extrapolated_ms_per_solve)
    return {'metric': METRIC, 'value': v, 'unit': 'solves/s', 'n_gpus': args.gpus, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': round(1e3 * t_iter * args.ref_step_iters, 3),
            'extrapolated_ms_per_solve': round(1e3 / v, 1), 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'c128', 'data': 'synthetic (seeded)', 'impl': 'reference',
            'config': dict(workload_config(args.workload, p), method='scipy qmr (reference generic() algorithm, CPU)'),
            'cpu_baseline': {'value': v, 'unit': 'solves/s', 'cores': 1, 'kind': 'port', 'host': cpu,
                             'sample': sample, 'seconds_per_iteration': round(t_iter, 4),
                             'iterations_extrapolated_to': iters_full},
            'e2e': {'value': v, 'unit': 'solves/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}


def kernel_mode(args) -> None:
    """A few iterations of each solver on one problem (for ncu captures): COCG (complex128),
    the mixed solver (complex64 BiCGSTAB passes + complex128 refinement) and the
    matrix-free products; prints per-kernel event timings."""
    import torch
    from meanas_b200 import workloads
    from meanas_b200.operators import GridOperator
    if args.workload == 'aniso_blocks':
        shape = tuple(args.shape) if args.shape else (160, 160, 128)
        p = workloads.aniso_blocks(shape=shape)
    else:
        p = workloads.BY_NAME[args.workload]()
    dev = torch.device('cuda', 0)
    blocks = set(args.kernel_blocks.split(','))
    extra_c128 = (24 if p.mu is not None else 0) + (1 if p.pec is not None or p.pmc is not None else 0)
    extra_c64 = (12 if p.mu is not None else 0) + (1 if p.pec is not None or p.pmc is not None else 0)
    x = torch.randn(p.n_unknowns, dtype=torch.complex128, device=dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if blocks & {'solvers', 'apply', 'fields'}:
        op = GridOperator(p.omega, p.dxes, p.epsilon, p.mu, p.pec, p.pmc, device=dev, fp32=True)
        if args.xchunk:
            op.set_xchunk('c128', args.xchunk)
        J = torch.as_tensor(p.J, device=dev)
    for method in (('cocg', 'mixed') if 'solvers' in blocks else ()):
        _, info = op.solve(J, method=method, rtol=1e-30, maxiter=args.kernel_iters, criterion='true',
                           profile=True, max_outer=1)
        for k in range(4):
            if info.kernel_count[k]:
                ms = info.kernel_ms[k] / info.kernel_count[k]
                extra = {0: extra_c128, 1: 0, 2: extra_c64, 3: extra_c64}[k]
                gbs = (KERNEL_BYTES_PER_CELL[k] + extra) * p.n_cells / (ms / 1e3) / 1e9
                print(f'{method:6s} {KERNEL_NAMES[k]:20s} {info.kernel_count[k]:5d} launches  '
                      f'{ms * 1e3:8.1f} us  {gbs:7.1f} GB/s algorithmic')
    for prec, xx in ((('c128', x), ('c64', x.to(torch.complex64))) if 'apply' in blocks else ()):
        for _ in range(3):
            op.apply(xx, precision=prec)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(10):
            op.apply(xx, precision=prec)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / 10
        per_cell = 6 * (16 if prec == 'c128' else 8) + 3 * (8 if prec == 'c128' else 4) + \
            (extra_c128 if prec == 'c128' else extra_c64)
        print(f'apply  A0_{prec:4s}               10 launches  {ms * 1e3:8.1f} us  '
              f'{per_cell * p.n_cells / (ms / 1e3) / 1e9:7.1f} GB/s algorithmic')
    # E -> (H, E x conj(H)) in one pass: read E, write H and S (3 x 48 B per cell; mu and the
    # mask byte when present)
    if 'fields' in blocks:
        for _ in range(3):
            op.poynting(x)
        a.record()
        for _ in range(10):
            op.poynting(x)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / 10
        per_cell = 3 * 48 + (24 if p.mu is not None else 0) + (1 if p.pmc is not None else 0)
        print(f'fields e2h+poynting c128         10 launches  {ms * 1e3:8.1f} us  '
              f'{per_cell * p.n_cells / (ms / 1e3) / 1e9:7.1f} GB/s algorithmic')
    # CSR product of the matrix_solver hook on a matrix shaped like the assembled operator:
    # 3N rows, 13 nonzeros per row at the curl-curl stencil's column offsets (synthetic
    # values); bytes = values + column indices + row pointers + x once + y
    if 'fdtd' in blocks:
        # FDTD: one H + one E half step of the plain Yee updates on float32 fields (E step: read
        # H, E, epsilon (float64), write E = 60 B/cell; H step: read E, H, write H = 36 B/cell)
        from meanas_b200 import fdtd
        rdx = [[numpy.abs(d).astype(float) for d in g] for g in p.dxes]
        eh2h, eh2e = fdtd.maxwell_h(0.3, rdx, device=dev), fdtd.maxwell_e(0.3, rdx, device=dev)
        ef = torch.randn((3, *p.shape), dtype=torch.float32, device=dev)
        hf = torch.randn_like(ef)
        epsf = torch.as_tensor(p.epsilon, device=dev)
        for _ in range(3):
            eh2h(ef, hf)
            eh2e(ef, hf, epsf)
        a.record()
        for _ in range(10):
            eh2h(ef, hf)
            eh2e(ef, hf, epsf)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / 10
        print(f'fdtd   H+E step f32                10 steps     {ms * 1e3:8.1f} us  '
              f'{96 * p.n_cells / (ms / 1e3) / 1e9:7.1f} GB/s algorithmic')
        del ef, hf
    if 'csr' not in blocks or p.n_unknowns > 12_000_000:
        return
    from scipy import sparse
    from meanas_b200.csr import CsrMatrix
    X, Y, Z = p.shape
    n = p.n_unknowns
    N = p.n_cells
    offs = numpy.array([0, 1, -1, Z, -Z, Y * Z, -Y * Z, N, -N, N + 1, N - Z, 2 * N, -2 * N + Y * Z])
    rows = numpy.repeat(numpy.arange(n, dtype=numpy.int64), offs.size)
    cols = (rows + numpy.tile(offs, n)) % n
    rng = numpy.random.default_rng(0)
    A = sparse.csr_array((rng.standard_normal(rows.size) + 1j, (rows, cols)), shape=(n, n))
    M = CsrMatrix(A, dev)
    del A, rows, cols
    for _ in range(3):
        M @ x
    a.record()
    for _ in range(10):
        M @ x
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / 10
    nnz = int(M.data.numel())
    csr_bytes = nnz * (16 + 4) + (n + 1) * 8 + 2 * 16 * n
    print(f'csr    spmv c128 ({nnz / n:.0f} nnz/row)   10 launches  {ms * 1e3:8.1f} us  '
          f'{csr_bytes / (ms / 1e3) / 1e9:7.1f} GB/s algorithmic')


def gradient_check(args) -> dict:
    """dL/d(eps) on the 96x96x64 adjoint problem (L = sum |E|^2 over the plane x=76) by
    torch.autograd (one forward + one adjoint GPU solve), checked two ways:

    * against the reference's own adjoint gradient (tests/golden/grad96.npz: the reference
      generic() forward solve and generic(adjoint=True) solve with scipy QMR, formed over the
      whole 40x40x8 design region);
    * against central finite differences of GPU FP64 solves (rtol `grad_rtol`) on `fd_cells`
      random design cells, Richardson-extrapolated from steps h and h/2
      ((4 D(h/2) - D(h)) / 3, truncation O(h^4)) so that a step large enough to keep the
      solves' residual noise (about rtol L / (2 h |g|)) small can be used.
    """
    import torch
    from meanas_b200 import workloads
    from meanas_b200.autograd import fdfd_solve
    p = workloads.adjoint_design()
    dev = torch.device('cuda', 0)
    mon = torch.as_tensor(p.extra['monitor'], device=dev)
    eps = torch.as_tensor(p.epsilon, device=dev).requires_grad_(True)
    kw = dict(rtol=args.grad_rtol, criterion='true', maxiter=args.grad_maxiter)

    def loss(e):
        E = fdfd_solve(e, p.J, p.omega, p.dxes, **kw)
        return (E.abs() ** 2)[mon].sum()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L = loss(eps)
    L.backward()
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t0
    g = eps.grad.cpu().numpy()
    n = p.n_cells
    dsl = p.extra['design_slices']
    g_design = g.reshape(3, *p.shape)[(slice(None), *dsl)]
    out = {'metric': 'adjoint gradient dL/deps vs the reference adjoint gradient and finite differences',
           'workload': 'adjoint_design 96x96x64, 10-cell SC-PML, omega=2pi/26, 40x40x8 design, L=sum|E|^2 at x=76',
           'gradient_seconds': round(t_grad, 3), 'loss': L.item(),
           'grad_norm_design': float(numpy.linalg.norm(g_design))}
    ref_file = ROOT / 'tests' / 'golden' / 'grad96.npz'
    if ref_file.exists():
        z = numpy.load(ref_file)
        if numpy.array_equal(z['eps_design'], p.epsilon.reshape(3, *p.shape)[(slice(None), *dsl)]):
            gr = z['grad_design']
            cell_gr, cell_g = gr.sum(axis=0), g_design.sum(axis=0)   # d/d(eps of a cell, all 3 components)
            sig = numpy.abs(cell_gr) >= 1e-3 * numpy.abs(cell_gr).max()
            out['vs_reference_adjoint'] = {
                'normwise_rel_err': float(numpy.linalg.norm(g_design - gr) / numpy.linalg.norm(gr)),
                'max_rel_err_significant_cells': float(numpy.max(numpy.abs(cell_g - cell_gr)[sig] /
                                                                 numpy.abs(cell_gr)[sig])),
                'significant_cells': int(sig.sum()), 'cells': int(sig.size),
                'reference_loss': float(z['loss']), 'loss_rel_err': abs(L.item() - float(z['loss'])) / float(z['loss']),
                'reference': f'reference generic() + generic(adjoint=True), scipy QMR rtol {float(z["rtol"]):g} '
                             f'(iterations {z["qmr_iterations"].tolist()}, residuals {float(z["residual"]):.1e} / '
                             f'{float(z["residual_adjoint"]):.1e})'}
        else:
            out['vs_reference_adjoint'] = {'error': 'grad96.npz was made for another design region'}
    cells = numpy.flatnonzero(p.extra['design_mask'].ravel())
    rng = numpy.random.default_rng(0)
    h = args.fd_h
    errs, errs_plain, errs_comp, fds, ads = [], [], [], [], []

    def central(idx, step):
        ep = eps.detach().clone()
        em = eps.detach().clone()
        ep[idx] += step
        em[idx] -= step
        return (loss(ep) - loss(em)).item() / (2 * step)
    with torch.no_grad():
        for cell in rng.choice(cells, args.fd_cells, replace=False):
            idx = [cell, n + cell, 2 * n + cell]
            d1, d2 = central(idx, h), central(idx, h / 2)
            fd = (4 * d2 - d1) / 3
            ad = float(g[idx].sum())
            errs.append(abs(fd - ad) / max(abs(fd), 1e-300))
            # the cell's derivative is a sum over its three components, which can cancel:
            # the same error relative to the components' magnitudes
            errs_comp.append(abs(fd - ad) / max(float(numpy.abs(g[idx]).sum()), 1e-300))
            errs_plain.append(abs(d2 - ad) / max(abs(d2), 1e-300))
            fds.append(fd)
            ads.append(ad)
    fds, ads = numpy.array(fds), numpy.array(ads)
    big = numpy.abs(fds) >= 1e-3 * numpy.abs(fds).max()
    out.update({'fd_cells': args.fd_cells, 'h': h, 'fd': 'Richardson (4 D(h/2) - D(h)) / 3 of central differences',
                'solve_rtol': args.grad_rtol, 'max_rel_err': max(errs), 'median_rel_err': float(numpy.median(errs)),
                'normwise_rel_err': float(numpy.linalg.norm(fds - ads) / numpy.linalg.norm(fds)),
                'max_rel_err_significant_cells': float(numpy.max(numpy.array(errs)[big])),
                'significant_cells': int(big.sum()),
                'max_err_over_component_magnitude': float(numpy.max(errs_comp)),
                'plain_central_h_over_2': {'max_rel_err_significant_cells':
                                           float(numpy.max(numpy.array(errs_plain)[big])),
                                           'median_rel_err': float(numpy.median(errs_plain))}})
    return out


def serving_run(args) -> dict:
    """The serving stream: seeded Poisson arrivals of requests (sizes uniform over 128^2..1024^2 x1 and
    32^3..128^3, lambda ~ U[16, 40] cells, random eps blocks, one dipole each), mixed precision
    to a true FP64 residual of 1e-8, served with continuous batching."""
    import torch
    from meanas_b200 import serving
    dev = torch.device('cuda', 0)
    stream = serving.poisson_stream(args.serving, rate=args.rate, seed=0)
    # warm each slot size (kernels, captured iteration graphs) with one request, untimed
    warm = {}
    for _, p in stream:
        warm.setdefault(p.shape, p)
    with serving.FDFDServer(dev, max_active=args.max_active, precision=args.serving_precision, rtol=RTOL,
                            maxiter=args.serving_maxiter) as srv:
        for p in warm.values():
            srv.submit(serving.Request(p.omega, p.dxes, p.J, p.epsilon)).result()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        results = serving.replay(srv, stream)
        t1 = time.perf_counter()
        stats = dict(srv.stats)
    lat = numpy.array([r.latency for r in results]) * 1e3
    ok = [r.info.converged and r.info.residual <= RTOL for r in results]
    by_size = {}
    for (_, p), r in zip(stream, results):
        by_size.setdefault('x'.join(map(str, p.shape)), []).append(r.latency * 1e3)
    return {'metric': 'FDFD serving solves/s and p50/p99 latency (continuous batching)',
            'value': round(len(results) / (t1 - t0), 3), 'unit': 'solves/s',
            'requests': len(results), 'arrival_rate_per_s': args.rate,
            'offered_seconds': round(stream[-1][0], 2), 'wall_seconds': round(t1 - t0, 2),
            'p50_ms': round(float(numpy.percentile(lat, 50)), 1),
            'p99_ms': round(float(numpy.percentile(lat, 99)), 1),
            'converged_to_1e-8': f'{sum(ok)}/{len(ok)}', 'maxiter': args.serving_maxiter,
            'max_active': args.max_active, 'slots': stats,
            'converged_by_size': {k: f"{sum(o for (_, p), o in zip(stream, ok) if 'x'.join(map(str, p.shape)) == k)}"
                                     f"/{len(v)}" for k, v in sorted(by_size.items())},
            'p50_ms_by_size': {k: round(float(numpy.median(v)), 1) for k, v in sorted(by_size.items())},
            'iterations_by_size': {k: int(numpy.median([r.info.iterations for (_, p), r in zip(stream, results)
                                                        if 'x'.join(map(str, p.shape)) == k]))
                                   for k in sorted(by_size)},
            'precision': args.serving_precision, 'data': 'synthetic (seeded)'}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', choices=['ours', 'reference'], default='ours')
    ap.add_argument('--e2e-steps', type=int, default=2)
    ap.add_argument('--cpu-sample-iters', type=int, default=12,
                    help='QMR iterations of the cpu_baseline sample')
    ap.add_argument('--ref-step-iters', type=int, default=4,
                    help='QMR iterations per step of the reference arm')
    ap.add_argument('--ref-iters', type=int, default=0,
                    help='QMR iterations per full solve used to extrapolate the reference arm '
                         '(0: the per-workload count in REF_ITERS)')
    ap.add_argument('--methods', default='mixed,cocg', help='GPU solvers to time (mixed, cocg)')
    ap.add_argument('--no-autotune', dest='autotune', action='store_false',
                    help='keep the default tiling instead of timing x-chunk candidates first')
    ap.add_argument('--workload', default='aniso_blocks', choices=sorted(WORKLOADS),
                    help='problem (default: the 160x160x128 headline case)')
    ap.add_argument('--kernel-iters', type=int, default=0,
                    help='profiling mode: run this many iterations of each solver (no convergence, no JSON)')
    ap.add_argument('--shape', type=int, nargs=3, default=None, help='profiling mode grid shape')
    ap.add_argument('--xchunk', type=int, default=0,
                    help='profiling mode: x planes per CTA of the complex128 passes (0: default tiling)')
    ap.add_argument('--kernel-blocks', default='solvers,apply,fields,fdtd,csr',
                    help='profiling mode: which kernel groups to run (comma list)')
    ap.add_argument('--timed-profile', choices=['on', 'off'], default='off',
                    help='per-launch CUDA events inside the timed solves (off: graph launches, kernel '
                         'durations from one profiled solve after them)')
    ap.add_argument('--maxiter', type=int, default=None,
                    help='cap the Krylov iterations of each timed solve (measurement runs; reports the status)')
    ap.add_argument('--gradient-check', action='store_true', help='adjoint gradient vs finite differences')
    ap.add_argument('--serving', type=int, default=0, help='serving mode: replay this many requests')
    ap.add_argument('--rate', type=float, default=50.0, help='serving: Poisson arrival rate (requests/s)')
    ap.add_argument('--max-active', type=int, default=8, help='serving: solves in flight at once')
    ap.add_argument('--serving-maxiter', type=int, default=50000, help='serving: Krylov iteration cap per request')
    ap.add_argument('--serving-precision', default='mixed', choices=['mixed', 'fp64'])
    ap.add_argument('--fd-cells', type=int, default=64)
    ap.add_argument('--fd-h', type=float, default=1e-2, help='finite-difference step (and h/2)')
    ap.add_argument('--grad-rtol', type=float, default=1e-12,
                    help='true FP64 residual of the gradient check solves (forward, adjoint and FD)')
    ap.add_argument('--grad-maxiter', type=int, default=400000, help='iteration cap of those solves')
    args = ap.parse_args()
    if args.kernel_iters > 0:
        return kernel_mode(args)
    if args.gradient_check:
        print(json.dumps(gradient_check(args)), flush=True)
        return None
    if args.serving > 0:
        print(json.dumps(serving_run(args)), flush=True)
        return None
    res = run_reference(args) if args.impl == 'reference' else run_ours(args)
    if res is not None:
        print(json.dumps(res), flush=True)
    if args.impl == 'ours' and int(os.environ.get('WORLD_SIZE', 1)) > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
