#!/usr/bin/env python
"""Benchmark: assembly + solve of the 72k-DoF penny crack on one B200.

Workload (the configuration the headline metric is quoted on): unit-disk
crack in z = 0, 4000 quadratic 6-node triangles (concentric rings, seeded
in-plane jitter <= 5 % of the ring spacing), N = 18 x 4000 = 72000 DoF,
G = 1, nu = 0.35, collocation offset 0.125, no fixed tip DoF, uniform
internal pressure 1 (sigma_zz = 1).  Synthetic seeded mesh (the reference has
no mesher).  One step = assemble the FP64 collocation matrix in HBM
(41.5 GB) + solve to a relative residual <= 1e-10 in one of three forms:

  --mode learned (default): the two-level preconditioner with the learned
        near-field blocks (a graph network over element adjacency,
        hfpx3d_b200/data/pc_gnn.bin) and flexible GMRES(50) on the operator,
        held by default in mixed precision (--operator mixed: FP32 entries,
        near-field blocks kept to ~2^-48 by FP32 low parts, products in FP64;
        --operator fp64: the FP64 matrix);
  --mode mixed: the FP32 LU of a copy with FP16 tcgen05 trailing updates and
        flexible GMRES on the FP64 operator preconditioned by it (--solver
        gmres, the default) or FP64 iterative refinement (--solver refine);
  --mode fp64: the plain FP64 GPU path (in-place FP64 LU).
After the timed loop the plain FP64 path is timed once (speed-up, opening
error against it; target rel err <= 1e-8), and the other fast form once.

Multi-GPU: the path has no exchange step; --gpus N runs N independent
replicas (one process per GPU, weak scaling); value = seconds per
assembly+solve, max over ranks.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

G, NU, BETA = 1.0, 0.35, 0.125
S_ZZ = np.array([0.0, 0.0, 1.0, 0.0, 0.0, 0.0])
METRIC = 'assembly+solve s at 72k DOF, mixed/learned vs plain FP64 GPU, rel err <=1e-8'
UNIT = 's'


def peaks():
    """(HBM GB/s, dense BF16/FP16 tensor TFLOP/s sustained, source)."""
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get('hbm_gbs', 6650.0), d.get('bf16_tflops_sustained', 1400.0), 'measured'
    return 6650.0, 1400.0, 'fallback'


# DRAM bytes per matrix entry written by the in-plane assembly kernel, from
# an ncu capture of one launch on the 1000-element penny (4.6305 GB for an
# 18 000 x 18 000 fill; traffic grows with the entries, so it scales by N^2)
ASM_DRAM_BYTES_PER_ENTRY = 4.630537e9 / 18000 ** 2
# DRAM bytes (read + write) per matrix entry of one FP64 operator product's
# resid_partial_kernel: 3.7327 GB read + 11.8 MB of partial sums written at
# N = 21 600 in an ncu capture of one launch (1200-element penny); the traffic
# grows with the entries, so N^2 times this is a launch at any N
RESID_DRAM_BYTES_PER_ENTRY = (3.732682e9 + 11.813888e6) / 21600.0 ** 2
# the same for the FP32 entries' product (resid_partial_f32_kernel, the
# mixed-precision operator's dense part): 1.8664 GB read + 9.5 MB written at
# N = 21 600 in the same capture
RESID32_DRAM_BYTES_PER_ENTRY = (1.8664e9 + 9.5e6) / 21600.0 ** 2
# DRAM bytes per matrix entry of the mixed-precision operator's fill (FP32
# entries + near-field low parts): 2.0153 GB written (2.8 MB read) for an
# 18 000 x 18 000 fill in an ncu capture of one launch on the 1000-element
# penny; scaled by N^2 like the FP64 fill's
ASM32_DRAM_BYTES_PER_ENTRY = (2.015346e9 + 2.779e6) / 18000 ** 2


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device):
        self.device, self.samples, self.proc = device, [], None

    def __enter__(self):
        q = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
             'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
             'clocks_event_reasons.sw_power_cap')
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.device), f'--query-gpu={q}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(',')])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        sm = [float(s[0]) for s in self.samples if s[0].replace('.', '').isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower() == 'active'})
        load = [x for x in sm if x > 0.5 * max(sm)] if sm else []
        return {'sm_mhz': statistics.median(load) if load else None, 'sm_max_mhz': max(mx) if mx else None,
                'reasons': reasons, 'samples': len(self.samples)}


def workload(n_el, seed=2026, mesh='penny'):
    """The timed crack: the C3 penny, or (mesh='wavy') a non-planar elliptical
    crack like the learned preconditioner's evaluation set (aspect 2, waviness
    0.12), whose pairs all take the off-plane (quadrature) path."""
    from hfpx3d_b200 import meshgen
    if mesh == 'wavy':
        return meshgen.wavy(n_el, aspect=2.0, amp=0.12, seed=seed)
    return meshgen.penny(n_el, seed=seed)


def replica_max(x, world, local_rank):
    """Max of x over the replicas: every rank's time, so the job's time is the
    slowest replica's (NCCL on the GPUs; gloo when the group runs on CPU)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = 'cpu' if dist.get_backend() == 'gloo' else f'cuda:{local_rank}'
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- engine arm
class Forms:
    """The three forms of one step on the device matrix A: FP64 assembly into
    A, then
      learned: the learned near-field preconditioner (made by
               hfpx_precond_create with the trained network on the first step,
               hfpx_precond_update in its storage on the next ones) and
               flexible GMRES(50) on the FP64
               operator (hfpx_gmres_precond_device);
      mixed:   the mixed LU (FP32 copy, FP16 tcgen05 updates) and flexible
               GMRES on the FP64 matrix preconditioned by it (hfpx_gmres_device);
      fp64:    the plain FP64 LU and its triangular solves.
    Four CUDA events per step on the engine's stream: before the assembly,
    after it, after the factorisation / preconditioner, after the solve."""

    def __init__(self, args, ctx, engine, L, torch, stream, dm, dof, n, A, d_rhs, d_x):
        self.args, self.ctx, self.engine, self.L, self.torch, self.stream = args, ctx, engine, L, torch, stream
        self.dm, self.dof, self.n, self.A, self.d_rhs, self.d_x = dm, dof, n, A, d_rhs, d_x
        self.info = engine.SolveInfo()
        self.net = None
        self.pcs = {}
        self.Am = None   # the mixed-precision operator (made on first use)
        self.host_ms = {}

    def operator(self, form):
        """The matrix a form works on: the learned form's operator is the
        mixed-precision one unless --operator fp64 ('learned64': always FP64)."""
        if form == 'learned' and self.args.operator == 'mixed':
            if self.Am is None:
                self.Am = self.engine.assemble_mixed(self.ctx, self.dm, self.dof, self.n, G, NU)
            return self.Am
        return self.A

    def _host(self, key, t0):
        self.host_ms[key] = self.host_ms.get(key, 0.0) + (time.perf_counter() - t0) * 1e3

    def step(self, form, ev=None):
        engine, L, ctx, A, torch = self.engine, self.L, self.ctx, self.A, self.torch
        rec = (lambda k: ev[k].record(self.stream)) if ev else (lambda k: None)
        A = self.operator(form)
        rec(0)
        engine.assemble_into(ctx, self.dm, self.dof, self.n, G, NU, A)
        rec(1)
        x = ctypes.c_void_p(self.d_x.data_ptr())
        if form in ('learned', 'learned64'):
            if self.net is None:
                self.net = engine.Gnn(ctx, path=engine.WEIGHTS_PATH)
            t0 = time.perf_counter()
            # blocks made again from this step's matrix, in the storage of
            # the first step's preconditioner (hfpx_precond_update)
            pc = self.pcs.get(form)
            if pc is None:
                kind = PC_KINDS[self.args.pc] | (engine.HFPX_PC_COARSE if self.args.coarse else 0)
                pc = self.pcs[form] = engine.Precond(ctx, self.dm, A, kind, net=self.net, shear_m=G)
            else:
                pc.update(A, net=self.net, shear_m=G)
            self._host('precond', t0)
            rec(2)
            with torch.cuda.stream(self.stream):
                self.d_x.copy_(self.d_rhs)
            t0 = time.perf_counter()
            rc = L.hfpx_gmres_precond_device(ctx.h, A.h, pc.h, x, self.args.tol, 50, 2000,
                                             ctypes.byref(self.info))
            self._host('gmres', t0)
            rec(3)
            ctx.check(rc)
            return
        mode = engine.HFPX_LU_MIXED if form == 'mixed' else engine.HFPX_LU_FP64
        info_ = ctypes.c_int64()
        ctx.check(L.hfpx_lu_factor(ctx.h, A.h, mode, ctypes.byref(info_)))
        rec(2)
        with torch.cuda.stream(self.stream):
            self.d_x.copy_(self.d_rhs)
        if form == 'mixed' and self.args.solver == 'gmres':
            ctx.check(L.hfpx_gmres_device(ctx.h, A.h, x, self.args.tol, 50, 200, ctypes.byref(self.info)))
        else:
            ctx.check(L.hfpx_lu_solve_device(ctx.h, A.h, x, 1, self.n, self.args.tol, 50, ctypes.byref(self.info)))
        rec(3)

    def timed(self, form, reps):
        """Best of `reps` steps after one warm-up: (phases ms, iterations, residual, x)."""
        torch = self.torch
        best = None
        for r in range(reps + 1):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            torch.cuda.synchronize()
            self.step(form, ev)
            torch.cuda.synchronize()
            t = [ev[0].elapsed_time(ev[k]) for k in (1, 2, 3)]
            if r > 0 and (best is None or t[2] < best[2]):
                best = t
        return best, self.info.iterations, self.info.residual, self.d_x.cpu().numpy()

    def close(self):
        for pc in self.pcs.values():
            pc.close()
        if self.net is not None:
            self.net.close()
        if self.Am is not None:
            self.Am.close()


def near_blocks(conn):
    """Blocks of the near-field pattern: every element with itself and with
    each element sharing a vertex with it."""
    v2e = {}
    for e in range(conn.shape[1]):
        for v in conn[:3, e]:
            v2e.setdefault(int(v), set()).add(e)
    return sum(len(set().union(*[v2e[int(v)] for v in conn[:3, e]])) for e in range(conn.shape[1]))


def opening(x):
    """Global z components of the nodal DD (no fixed DoF: 18 per element)."""
    return x[2::3]


def rel_opening_err(x, x64):
    return float(np.abs(opening(x) - opening(x64)).max() / np.abs(opening(x64)).max())


def run_engine(args, rank, world, local_rank):
    import torch
    from hfpx3d_b200 import build, engine
    if rank == 0:
        build.build()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.set_device(local_rank)
    ctx = engine.Context(local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f'cuda:{local_rank}')
    nods, conn = workload(args.n_el, mesh=args.mesh)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    rhs = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, S_ZZ)
    d_rhs = torch.empty(n, dtype=torch.float64, device=f'cuda:{local_rank}')
    d_x = torch.empty_like(d_rhs)
    d_rhs.copy_(torch.from_numpy(rhs))
    A = engine.assemble(ctx, dm, dof, n, G, NU)
    L = engine.lib()
    F = Forms(args, ctx, engine, L, torch, stream, dm, dof, n, A, d_rhs, d_x)

    for _ in range(args.warmup):
        F.step(args.mode)
    torch.cuda.synchronize()
    F.host_ms = {}
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    launches0 = L.hfpx_ctx_launch_count(ctx.h)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with Clocks(local_rank) as clk:
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        t_loop = time.perf_counter()
        for k in range(args.steps):
            t0 = time.perf_counter()
            F.step(args.mode, evs[k])
            F._host('step', t0)
        end.record(stream)
        F._host('loop', t_loop)
        torch.cuda.synchronize()
    launches = L.hfpx_ctx_launch_count(ctx.h) - launches0
    total_ms = start.elapsed_time(end)
    t_asm = [e[0].elapsed_time(e[1]) for e in evs]
    t_fac = [e[1].elapsed_time(e[2]) for e in evs]
    t_sol = [e[2].elapsed_time(e[3]) for e in evs]
    ms = total_ms / args.steps
    x_main = d_x.cpu().numpy()
    res_main, iters_main = F.info.residual, F.info.iterations
    ms = replica_max(ms, world, local_rank)

    # end to end through the C-ABI with host buffers (pinned), before the
    # seconds-long FP64 comparison heats the GPU
    e2e = None
    if rank == 0 and args.e2e_steps > 0:
        e2e = run_e2e(args, ctx, engine, L, nods, conn, dof, n, args.mode, stream, torch, F.operator(args.mode), F)

    # the plain FP64 GPU path, once, for the speed-up and the opening error
    other_s, rel_err, x64 = None, None, None
    if args.compare and rank == 0 and args.mode != 'fp64':
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        torch.cuda.synchronize()
        F.step('fp64', ev)
        torch.cuda.synchronize()
        other_s = ev[0].elapsed_time(ev[3]) / 1e3
        x64 = d_x.cpu().numpy()
        rel_err = rel_opening_err(x_main, x64)

    # the other fast forms (mixed LU, or learned; and the learned form on the
    # FP64 operator beside the mixed-precision one), best of 2 after a warm-up
    seconds = {}
    others = {'learned': ['mixed'] + (['learned64'] if args.operator == 'mixed' else []),
              'mixed': ['learned']}.get(args.mode, [])
    for second_form in (others if rank == 0 and args.second else []):
        t, it, res, xs = F.timed(second_form, 2)
        second = seconds[second_form] = {
            'value': t[2] / 1e3, 'unit': UNIT,
            'phases_ms': {'assembly': t[0], 'factor' if second_form == 'mixed' else 'preconditioner': t[1] - t[0],
                          'solve': t[2] - t[1]},
            'iterations': it, 'residual': res}
        if second_form == 'learned64':
            second['operator'] = 'FP64 matrix (41.5 GB), FP32 copy for products once the residual is small'
        if x64 is not None:
            second['opening_rel_err_vs_fp64'] = rel_opening_err(xs, x64)
            second['speedup_vs_plain_fp64'] = other_s / second['value']
        if second_form == 'mixed':
            flops_lu = 2.0 / 3.0 * float(n) ** 3
            fac_s = (t[1] - t[0]) / 1e3
            _, tensor_peak, peak_src = peaks()
            second['roofline'] = {'kernel': 'LU factorisation (panel_ll_kernel chain + tcgen05 FP16 updates)',
                                  'bound': 'tensor', 'achieved': flops_lu / fac_s / 1e12, 'peak': tensor_peak,
                                  'unit': 'TFLOP/s', 'frac': flops_lu / fac_s / 1e12 / tensor_peak, 'traffic': None,
                                  'peak_source': f'{peak_src} bf16_tflops_sustained'}

    # the dominant kernel of the learned form: the FP64 operator product
    # (resid_partial_kernel + resid_finish_kernel, one per GMRES step), timed
    # alone on the engine's stream: N^2 8 bytes of matrix per launch
    resid = None
    if rank == 0:
        Aop = F.operator(args.mode)
        engine.assemble_into(ctx, dm, dof, n, G, NU, Aop)  # the operator again (an FP64 step leaves factors)
        resid = time_residual(ctx, engine, L, torch, stream, Aop, d_rhs, d_x, n)

    # the 1025-element volume-control ellipse, measured on the engine as well
    c2 = run_c2(args, ctx, engine, L, torch, stream, local_rank) if rank == 0 and args.compare else None
    # one volume-control iteration with cohesion and friction on the same ellipse
    cf = run_cf(ctx, engine) if rank == 0 and args.cf else None
    # stresses at observation points (make_3dbem_stress_f_s) on the C1 penny
    stress = run_stress(ctx, engine, torch, stream) if rank == 0 and args.stress else None
    # the batched workload: 256 uneven meshes x 64 load cases in one graph
    c5 = run_c5(args, ctx, engine, torch, stream) if rank == 0 and args.batch else None
    F.close()

    if rank != 0:
        return None
    hbm, tensor_peak, peak_src = peaks()
    asm_ms = statistics.mean(t_asm)
    fac_ms = statistics.mean(t_fac)
    op_mixed = args.mode == 'learned' and args.operator == 'mixed'
    n_blocks = near_blocks(conn) if op_mixed else 0
    # algorithmic bytes of one assembly / one operator product: the matrix
    # entries once (FP64, or FP32 plus the near-field blocks' FP32 low parts)
    bytes_op = float(n) * n * 4 + 324.0 * 4 * n_blocks if op_mixed else float(n) * n * 8
    bytes_asm = bytes_op
    flops_lu = 2.0 / 3.0 * float(n) ** 3
    dtype = {'learned': ('f32 far field + near field to 2^-48 (f64 products) + bf16 network' if op_mixed
                         else 'f64 operator + bf16 network'), 'mixed': 'f64+f32+f16', 'fp64': 'f64'}[args.mode]
    line = {
        'metric': METRIC, 'value': ms / 1e3, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': False, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': dtype,
        'data': f'synthetic (seeded {args.n_el}-triangle {args.mesh} mesh, pressure 1)',
        'config': {'workload': f'{args.mesh} crack {args.n_el} el, N={n} DoF, assembly + '
                               f'{FORM_TEXT[args.mode].replace("OPERATOR", OPERATOR_TEXT[args.operator])} to rel '
                               f'residual {args.tol:g}', 'n_el': args.n_el, 'n_dof': n, 'form': args.mode,
                   'operator': args.operator if args.mode == 'learned' else 'fp64',
                   'preconditioner': ((args.pc + (' + coarse' if args.coarse else ''))
                                      if args.mode == 'learned' else None),
                   'parallelism': f'replicas x{world}',
                   'l2': ('inputs larger than L2 (the 20.7 GB mixed-precision operator rewritten each step)'
                          if op_mixed else 'inputs larger than L2 (41.5 GB matrix rewritten each step)')},
        'phases_ms': {'assembly': asm_ms, 'preconditioner' if args.mode == 'learned' else 'factor': fac_ms,
                      'solve': statistics.mean(t_sol)},
        'steps_ms': {'total': [round(a + b + c, 2) for a, b, c in zip(t_asm, t_fac, t_sol)],
                     'solve': [round(t, 2) for t in t_sol]},
        'solver': {'form': args.mode, 'iterations': iters_main, 'residual': res_main},
        'host_ms_per_step': {k: v / args.steps for k, v in F.host_ms.items()},
        'assemblies_per_s': 1e3 / asm_ms,
        'solves_per_s': 1e3 / ms,
        'roofline_assembly': {'kernel': ('assemble_kernel<in-plane> (mixed-precision operator fill: FP32 entries + '
                                         'near-field low parts)' if op_mixed else
                                         'assemble_kernel<in-plane> (FP64 matrix fill)'), 'bound': 'hbm',
                              'achieved': bytes_asm / (asm_ms / 1e3) / 1e9, 'peak': hbm, 'unit': 'GB/s',
                              'frac': bytes_asm / (asm_ms / 1e3) / 1e9 / hbm,
                              'traffic': (ASM32_DRAM_BYTES_PER_ENTRY * float(n) * n if op_mixed and
                                          ASM32_DRAM_BYTES_PER_ENTRY else
                                          None if op_mixed else ASM_DRAM_BYTES_PER_ENTRY * float(n) * n),
                              'peak_source': f'{peak_src} hbm_gbs', 'algorithmic_bytes': bytes_asm},
        'gpu_launches': int(launches),
        'clocks': clk.summary(),
        'e2e': e2e,
    }
    if args.mode == 'learned' and resid is not None:
        gbs = bytes_op / (resid['ms'] / 1e3) / 1e9
        line['roofline'] = {'kernel': ('resid_partial_f32_kernel + near_lo_kernel + resid_finish_kernel (the mixed-'
                                       'precision operator product, one per GMRES step)' if op_mixed else
                                       'resid_partial_kernel + resid_finish_kernel (FP64 operator product, one per '
                                       'GMRES step)'), 'bound': 'hbm', 'achieved': gbs, 'peak': hbm,
                            'unit': 'GB/s', 'frac': gbs / hbm,
                            'traffic': ((RESID32_DRAM_BYTES_PER_ENTRY if op_mixed else RESID_DRAM_BYTES_PER_ENTRY)
                                        * float(n) * n),
                            'peak_source': f'{peak_src} hbm_gbs', 'algorithmic_bytes': bytes_op,
                            'launch_ms': resid['ms']}
    else:
        line['roofline'] = {'kernel': 'LU factorisation (panel_ll_kernel chain + tcgen05 FP16 updates)',
                            'bound': 'tensor', 'achieved': flops_lu / (fac_ms / 1e3) / 1e12, 'peak': tensor_peak,
                            'unit': 'TFLOP/s', 'frac': flops_lu / (fac_ms / 1e3) / 1e12 / tensor_peak,
                            'traffic': None, 'peak_source': f'{peak_src} bf16_tflops_sustained',
                            'algorithmic_flops': flops_lu}
    if other_s is not None:
        line['plain_fp64_s'] = other_s
        line['speedup_vs_plain_fp64'] = other_s / (ms / 1e3)
        line['opening_rel_err_vs_fp64'] = rel_err
    for k, v in seconds.items():
        line['learned_fp64_operator' if k == 'learned64' else k] = v
    if args.cpu_baseline:
        cb = cpu_baseline(args)
        x_ref = cb.pop('_c2_x', None)
        line['cpu_baseline'] = cb
        if c2 is not None and cb['measured_c2']:
            c2['reference_cpu_s'] = cb['measured_c2']['value']
            c2['speedup_mixed_vs_reference_cpu'] = c2['reference_cpu_s'] / c2['engine_mixed_s']
            if x_ref is not None:
                for k in ('mixed', 'fp64'):
                    x = c2.pop('_x_' + k)
                    c2[f'rel_err_{k}_vs_reference'] = float(np.abs(x - x_ref).max() / np.abs(x_ref).max())
    if c2 is not None:
        for k in ('mixed', 'fp64'):
            c2.pop('_x_' + k, None)
        line['c2'] = c2
    if cf is not None:
        line['cf_iteration'] = cf
    if stress is not None:
        line['stress'] = stress
    if c5 is not None:
        cb = line.get('cpu_baseline') or {}
        fit = cb.get('fit')
        if fit:
            # the reference per mesh: assembly a Ne^2 + LU b N^3 (the fit of
            # the measured sizes), the 64 load cases' dgetrs neglected
            ref = sum(fit['a'] * ne ** 2 + fit['b'] * (18.0 * ne) ** 3 for ne in c5.pop('_n_el'))
            c5['reference_cpu_s'] = ref
            c5['reference_cpu_note'] = ('extrapolated per mesh from the fit of the measured CPU reference '
                                        '(a Ne^2 + b N^3, summed over the meshes)')
        c5.pop('_n_el', None)
        line['c5'] = c5
    return line


def run_stress(ctx, engine, torch, stream, reps=5):
    """Stress at observation points through the C-ABI with host buffers
    (hfpx_stress, make_3dbem_stress_f_s system_assembly.cpp:279-455; and
    hfpx_stress_batch for many load cases at once), on the seeded
    121-element penny: 100 seeded points in [-1.5, 1.5]^3 (the C1 set-up),
    one load case, and 64 load cases (pressures U[0.5, 2] and random in-situ
    stresses).  Best of `reps` host wall times of the call, and the device
    time between CUDA events on the engine's stream around it (copies and
    kernels, without the host-side wrapper)."""
    from hfpx3d_b200 import meshgen
    nods, conn = meshgen.penny(121, seed=4)
    ne = conn.shape[1]
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    A = engine.assemble(ctx, dm, dof, n, G, NU)
    rng = np.random.default_rng(64)
    S = np.zeros((6, 64))
    for kcase in range(64):
        if kcase % 2 == 0:
            S[2, kcase] = rng.uniform(0.5, 2.0)
        else:
            q, r = np.linalg.qr(rng.standard_normal((3, 3)))
            q = q * np.sign(np.diag(r))
            st = q @ np.diag(rng.uniform(-1.0, 0.0, 3)) @ q.T
            S[:, kcase] = [st[0, 0], st[1, 1], st[2, 2], st[0, 1], st[0, 2], st[1, 2]]
    rhs = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, S)
    X = engine.LU(ctx, A, engine.HFPX_LU_FP64).solve(rhs)
    dds = np.stack([engine.write_dd_vector_to_md(X[:, kcase], dof, ne) for kcase in range(64)])
    pts = meshgen.observation_points(100, seed=5, nods=nods, conn=conn)

    def best(fn):
        fn()
        ts, ds = [], []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e0.record(stream)
            fn()
            e1.record(stream)
            ts.append(time.perf_counter() - t0)
            torch.cuda.synchronize()
            ds.append(e0.elapsed_time(e1) / 1e3)
        return min(ts), min(ds)
    t1, d1 = best(lambda: engine.make_3dbem_stress_f_s(ctx, dm, G, NU, dds[0], pts, S[:, 0]))
    t64, d64 = best(lambda: engine.make_3dbem_stress_f_s_batch(ctx, dm, G, NU, dds, pts, S))
    A.close()
    dm.close()
    npts = pts.shape[1]
    return {'workload': f'penny {ne} el, {npts} seeded points in [-1.5, 1.5]^3; host buffers through the C-ABI',
            'one_case_s': t1, 'points_per_s': npts / t1, 'pair_evaluations_per_s': npts * ne / t1,
            'one_case_device_s': d1, 'cases_64_s': t64, 'cases_64_device_s': d64,
            'point_cases_per_s': 64 * npts / t64}


# near-field part of the learned form's preconditioner (hfpx_pc_kind)
PC_KINDS = {'learned': 3, 'neumann': 1, 'local': 2, 'jacobi': 0}
OPERATOR_TEXT = {'mixed': 'mixed-precision operator (FP32 entries, near-field blocks to 2^-48, FP64 products)',
                 'fp64': 'FP64 operator'}

FORM_TEXT = {'learned': 'two-level preconditioner (learned near-field blocks + coarse correction over element '
                        'aggregates) + GMRES(50) on the OPERATOR',
             'mixed': 'mixed LU (FP16 tcgen05 updates) + GMRES on the FP64 operator',
             'fp64': 'FP64 LU + triangular solves'}


def run_c5(args, ctx, engine, torch, stream, reps=3):
    """The batched workload: 256 seeded penny / 2:1
    ellipse meshes of 24-550 elements, 64 load cases each (pressures U[0.5, 2],
    random in-situ stresses), assembly + factorisation + solves of every mesh
    and load case in one CUDA-graph launch (hfpx_batch_run), best of `reps`
    replays after the capturing run; beside it the same meshes one by one
    through the per-mesh C-ABI (FP64 assembly, mixed LU, refined solves of
    the 64 load cases)."""
    from hfpx3d_b200 import meshgen
    meshes, S = meshgen.batch_workload(256, 64)
    n_el = [c.shape[1] for _, c in meshes]
    dms = [engine.DeviceMesh(ctx, engine.MeshGeom(nods, conn), BETA) for nods, conn in meshes]
    t0 = time.perf_counter()
    B = engine.Batch(ctx, dms, G, NU)
    B.set_loads(S)
    info = B.run(tol=args.tol)
    setup_s = time.perf_counter() - t0
    best = float('inf')
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        info = B.run(tol=args.tol)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        if t < best:
            best, phases = t, B.phases()
    flops = sum(2.0 / 3.0 * (18.0 * ne) ** 3 for ne in n_el)
    out = {'workload': '256 seeded penny / 2:1 ellipse meshes, 24-550 elements (meshgen.batch_workload), 64 load '
                       'cases each; one CUDA graph: assembly (mixed-precision operators) + FP32 tournament-pivoted '
                       'LU + solves of the 6 unit stress states + FP64 refinement + the 64 combinations',
           'n_mesh': len(meshes), 'elements': int(sum(n_el)), 'load_cases': int(S.shape[2]),
           'tiles': {'nb': B.nb, 'leaf_rows': B.leaf_rows}, 'graph_launches': B.launches,
           'batch_s': best, 'phases_ms': phases, 'meshes_per_s': len(meshes) / best,
           'load_case_solves_per_s': len(meshes) * S.shape[2] / best,
           'lu_tflops': flops / best / 1e12, 'residual': info.residual, 'converged': bool(info.converged),
           'refinement_steps': info.iterations,
           'first_run_s (capture + instantiate + run)': setup_s, '_n_el': n_el}
    B.close()
    # the same meshes one by one through the per-mesh C-ABI
    if args.c5_per_mesh:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for m, (nods, conn) in enumerate(meshes):
            mesh = engine.MeshGeom(nods, conn)
            dof, n = engine.make_dof_h_crack(mesh, 0)
            A = engine.assemble(ctx, dms[m], dof, n, G, NU)
            rhs = engine.add_s_inf_to_3dbem_rhs(ctx, dms[m], dof, n, S[m])
            engine.LU(ctx, A, engine.HFPX_LU_MIXED).solve(np.asfortranarray(rhs), tol=args.tol)
            A.close()
        e1.record(stream)
        torch.cuda.synchronize()
        out['per_mesh_path_s'] = e0.elapsed_time(e1) / 1e3
        out['speedup_vs_per_mesh_path'] = out['per_mesh_path_s'] / best
    for d in dms:
        d.close()
    return out


def time_residual(ctx, engine, L, torch, stream, A, d_b, d_x, n, reps=5):
    """CUDA-event time of one FP64 operator product r = b - A x (the GMRES
    step's pass over A), average of `reps` launches after one warm-up; the
    41.5 GB matrix is larger than L2, so every launch reads it from HBM."""
    d_r = torch.empty_like(d_x)
    args = (ctx.h, A.h, ctypes.c_void_p(d_x.data_ptr()), ctypes.c_void_p(d_b.data_ptr()),
            ctypes.c_void_p(d_r.data_ptr()))
    ctx.check(L.hfpx_residual_device(*args))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        ctx.check(L.hfpx_residual_device(*args))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    return {'ms': ms, 'gbs': float(n) * n * 8 / (ms / 1e3) / 1e9}


def run_c2(args, ctx, engine, L, torch, stream, local_rank, reps=3):
    """Assembly + LU + solve of the 1025-element VC ellipse on the engine,
    best of `reps`, in both precisions (CUDA events on the engine's stream)."""
    nods, conn, s_inf, vol = c2_case()
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    rhs = np.concatenate([engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, s_inf), [vol]])
    A = engine.assemble(ctx, dm, dof, n, G, NU, vc=True)
    d_rhs = torch.from_numpy(rhs).to(f'cuda:{local_rank}')
    d_x = torch.empty_like(d_rhs)
    info = engine.SolveInfo()
    out = {'workload': f'VC 2:1 ellipse {C2_NEL} el, N={n}+1, Haar in-situ stress, V=1'}
    for name, mode in (('mixed', engine.HFPX_LU_MIXED), ('fp64', engine.HFPX_LU_FP64)):
        best = float('inf')
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            engine.assemble_into(ctx, dm, dof, n, G, NU, A, vc=True)
            info_ = ctypes.c_int64()
            ctx.check(L.hfpx_lu_factor(ctx.h, A.h, mode, ctypes.byref(info_)))
            d_x.copy_(d_rhs)
            torch.cuda.synchronize()
            ctx.check(L.hfpx_lu_solve_device(ctx.h, A.h, ctypes.c_void_p(d_x.data_ptr()), 1, n + 1, 1e-12, 50,
                                             ctypes.byref(info)))
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        out[f'engine_{name}_s'] = best
        out['_x_' + name] = d_x.cpu().numpy()
    A.close()
    dm.close()
    return out


def run_e2e(args, ctx, engine, L, nods, conn, dof, n, form, stream, torch, A, F):
    """The same step through the C-ABI from pinned host buffers, the solution
    read back each step: hfpx_mesh_create -> hfpx_assemble_into ->
    hfpx_rhs_sinf -> (learned) hfpx_precond_create + hfpx_gmres_precond, or
    (mixed / fp64) hfpx_lu_factor + hfpx_gmres / hfpx_lu_solve.  The device
    matrix storage of the main loop and the loaded network are reused."""
    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a.reshape(-1, order='F'))).pin_memory()
        return t, t.numpy()
    tn, hn = pinned(nods)
    tc, hc = pinned(conn)
    td, hd = pinned(dof)
    tr, hr = pinned(np.zeros(n))
    s = np.ascontiguousarray(S_ZZ)
    if form == 'learned' and F.net is None:
        F.net = engine.Gnn(ctx, path=engine.WEIGHTS_PATH)
    times = []
    host = {}

    def tick(key, t0):
        if k >= args.e2e_warmup:
            host[key] = host.get(key, 0.0) + (time.perf_counter() - t0) * 1e3
        return time.perf_counter()
    for k in range(args.e2e_warmup + args.e2e_steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        t0 = time.perf_counter()
        mh = ctypes.c_void_p()
        ctx.check(L.hfpx_mesh_create(ctx.h, engine._dp(hn), nods.shape[0], nods.shape[1], engine._lp(hc),
                                     conn.shape[0], conn.shape[1], BETA, ctypes.byref(mh)))
        t0 = tick('mesh_create', t0)
        ctx.check(L.hfpx_assemble_into(ctx.h, mh, engine._lp(hd), n, G, NU, 0, 0, A.h))
        hr[:] = 0.0
        ctx.check(L.hfpx_rhs_sinf(ctx.h, mh, engine._lp(hd), n, engine._dp(s), 1, engine._dp(hr), n))
        t0 = tick('assemble_rhs', t0)
        si = engine.SolveInfo()
        if form == 'learned':
            pc = ctypes.c_void_p()
            kind = PC_KINDS[args.pc] | (engine.HFPX_PC_COARSE if args.coarse else 0)
            ctx.check(L.hfpx_precond_create(ctx.h, mh, A.h, kind, F.net.h, G, ctypes.byref(pc)))
            t0 = tick('precond_create', t0)
            rc = L.hfpx_gmres_precond(ctx.h, A.h, pc, engine._dp(hr), args.tol, 50, 2000, ctypes.byref(si))
            t0 = tick('gmres', t0)
            L.hfpx_precond_destroy(pc)
            t0 = tick('precond_destroy', t0)
            ctx.check(rc)
        else:
            info_ = ctypes.c_int64()
            mode = engine.HFPX_LU_MIXED if form == 'mixed' else engine.HFPX_LU_FP64
            ctx.check(L.hfpx_lu_factor(ctx.h, A.h, mode, ctypes.byref(info_)))
            if args.solver == 'gmres' and form == 'mixed':
                ctx.check(L.hfpx_gmres(ctx.h, A.h, engine._dp(hr), args.tol, 50, 200, ctypes.byref(si)))
            else:
                ctx.check(L.hfpx_lu_solve(ctx.h, A.h, engine._dp(hr), 1, n, args.tol, 50, ctypes.byref(si)))
        e1.record(stream)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.hfpx_mesh_destroy(mh)
        tick('mesh_destroy (after the timed region)', t0)
        if k >= args.e2e_warmup:
            times.append(e0.elapsed_time(e1))
    h2d = hn.nbytes + hc.nbytes + 2 * hd.nbytes + hr.nbytes + s.nbytes  # dof_h goes up twice
    return {'value': statistics.mean(times) / 1e3, 'unit': UNIT, 'h2d_bytes_per_step': int(h2d),
            'd2h_bytes_per_step': int(hr.nbytes), 'steps': len(times), 'steps_ms': [round(t, 2) for t in times],
            'host_ms_per_step': {key: round(v / max(1, len(times)), 2) for key, v in host.items()}}


# ------------------------------------------------------------- CPU reference
# The reference's own CPU path (oracle/_ref/libhfpx_ref_cpu.so: its sources
# compiled with OpenMP, il::LU on multithreaded OpenBLAS; run and timed as
# its main.cpp does, "Assembly" and "Solution"), or, where that library was
# not built, the CPU oracle port with numpy's LAPACK.  Measured on penny
# meshes of the same family at FIT_SIZES elements, and at the 1025-element
# volume-control ellipse for real; the 4000-element value is fitted from the
# measured sizes (t_asm = a Ne^p, t_lu = b N^q by least squares in log-log)
# and labelled extrapolated.
FIT_SIZES = (600, 900, 1200)
C2_NEL, C2_SEED = 1025, 1025


def run_cf(ctx, engine, steps=3):
    """Steps of the volume-control iteration with cohesion and friction
    (hfpx_vc_cf_iteration) on the 1025-element ellipse's bordered matrix (DD
    in local coordinates): opened within rho < 0.5 of the ellipse's scaled
    radius (fully within 0.3), earlier slip in 0.5 < rho < `ring`, pressure 1
    where opened, two materials; 10 % more volume each step.  Host arrays in
    and out through the C-ABI; wall time per step (each call synchronises).
    Once with the mixed factors of the full system (few intact points: the
    capacitance solve), once with many intact points (the truncated system
    factored)."""
    nods, conn, s_inf, _ = c2_case()
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 1)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    A = engine.assemble(ctx, dm, dof, n, G, NU, is_dd_local=True, vc=True)
    vrow = A.block(n, 0, 1, n + 1)[0]
    lu = engine.LU(ctx, A, engine.HFPX_LU_MIXED)
    ne = conn.shape[1]
    pos = np.zeros((6 * ne, 2))
    for a in range(3):
        pos[a::6] = nods[:2, conn[a]].T
        pos[3 + a::6] = 0.5 * (nods[:2, conn[(a + 1) % 3]] + nods[:2, conn[(a + 2) % 3]]).T
    ax = np.abs(nods[:2]).max(axis=1)
    rho = np.hypot(pos[:, 0] / ax[0], pos[:, 1] / ax[1])
    rng = np.random.default_rng(9)
    mats = [dict(cr_open=0.02, peak_ts=0.8, cr_slip=0.02, peak_sc=0.2, peak_sf=0.6, res_sf=0.3, cohesion_model=1,
                 friction_model=1),
            dict(cr_open=0.03, peak_ts=1.2, cr_slip=0.03, peak_sc=0.1, peak_sf=0.5, res_sf=0.5, cohesion_model=0,
                 friction_model=0)]
    out = {'workload': f'VC 2:1 ellipse {C2_NEL} el, N={n}+1, DD local, tip vertices fixed; {steps} steps, '
                       'all traction components, releasing sign',
           'runs': []}
    for ring in (0.995, 0.8):
        dd = np.zeros((6 * ne, 3))
        dd[:, 2] = 0.02 * np.sqrt(np.clip(1 - (rho / 0.5) ** 2, 0, None))
        st = engine.CfState(ne, dd=dd, pp=np.where(rho < 0.5, 1.0, 0.0),
                            mr_open=np.where(rho < 0.3, 1.0, np.where(rho < 0.5, 0.5, 0.0)),
                            mr_slip=np.where((rho > 0.5) & (rho < ring), 0.3, 0.0),
                            mat_id=(rng.random(6 * ne) < 0.3).astype(np.int32))
        x = np.zeros(n + 1)
        for l in range(18):
            kept = dof[:, l] >= 0
            x[dof[kept, l]] = st.dd[6 * np.arange(ne)[kept] + l // 3, l % 3]
        vol = float(vrow @ x)
        run = {'slip_ring': ring, 'steps_s': [], 'n_fixed': [], 'solver': [], 'residual': []}
        for k in range(steps + 1):   # step 0 warms up
            t0 = time.perf_counter()
            info = engine.vc_cf_iteration(ctx, dm, A, dof, n, mats, st, s_inf, int(np.argmin(rho)), 1.1 * vol,
                                          is_dd_local=True, all_components=True, release_sign=True)
            dt = time.perf_counter() - t0
            if k == 0:
                continue
            run['steps_s'].append(round(dt, 5))
            run['n_fixed'].append(int(info.n_fixed))
            run['solver'].append('full factors + capacitance' if info.solver == 0 else 'truncated system factored')
            run['residual'].append(float(info.residual))
        out['runs'].append(run)
    del lu
    A.close()
    dm.close()
    return out


def c2_case():
    """The 1025-element 2:1 volume-control ellipse: mesh, Haar in-situ stress, V = 1."""
    from hfpx3d_b200 import meshgen
    nods, conn = meshgen.ellipse(C2_NEL, seed=C2_SEED)
    rng = np.random.default_rng(C2_SEED)
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    st = q @ np.diag(rng.uniform(-1.0, 0.0, 3)) @ q.T
    s_inf = np.array([st[0, 0], st[1, 1], st[2, 2], st[0, 1], st[0, 2], st[1, 2]])
    return np.asfortranarray(nods), np.asfortranarray(conn, dtype=np.int64), s_inf, 1.0


class RefCPU:
    def __init__(self):
        sys.path.insert(0, os.path.join(ROOT, 'tests'))
        import oracle_lib
        self.ol = oracle_lib
        path = os.path.join(ROOT, 'oracle', '_ref', 'libhfpx_ref_cpu.so')
        self.lib = None
        if os.path.exists(path):
            D, L = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)
            lib = ctypes.CDLL(path)
            lib.ref_cpu_path.restype = ctypes.c_int
            lib.ref_cpu_path.argtypes = [D, ctypes.c_int64, ctypes.c_int64, L, ctypes.c_int64, ctypes.c_int64,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, D,
                                         ctypes.c_double, D, D, D, L]
            self.lib = lib
        self.kind = 'reference' if self.lib else 'port'

    def run(self, nods, conn, s_inf, vc=False, volume=0.0):
        """(t_assembly, t_solution, x) of one assembly + solve."""
        ol = self.ol
        ne = conn.shape[1]
        s = np.ascontiguousarray(s_inf, dtype=np.float64)
        if self.lib:
            x = np.zeros(18 * ne + 1)
            ta, ts, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
            rc = self.lib.ref_cpu_path(ol.dp(nods), nods.shape[0], nods.shape[1], ol.lp(conn), conn.shape[0], ne,
                                       G, NU, BETA, int(vc), ol.dp(s), volume, ctypes.byref(ta), ctypes.byref(ts),
                                       ol.dp(x), ctypes.byref(n))
            if rc != 0:
                raise RuntimeError(f'reference LU reports a singular matrix (rc {rc})')
            return ta.value, ts.value, x[:n.value]
        o = ol.Oracle()
        t0 = time.perf_counter()
        dof, n = o.dof_handle(nods, conn, 0)
        A = o.assemble(nods, conn, dof, n, vc=int(vc))
        b = o.rhs(nods, conn, dof, n, s)
        if vc:
            b = np.concatenate([b, [volume]])
        t_asm = time.perf_counter() - t0
        t0 = time.perf_counter()
        x = np.linalg.solve(A, b)
        return t_asm, time.perf_counter() - t0, x


def fit_power(sizes, times):
    """Least-squares t = c size^p in log-log: (c, p, max relative residual)."""
    ls, lt = np.log(np.asarray(sizes, float)), np.log(np.asarray(times, float))
    p, lc = np.polyfit(ls, lt, 1)
    resid = float(np.max(np.abs(np.exp(lc + p * ls) / np.exp(lt) - 1.0)))
    return float(np.exp(lc)), float(p), resid


def cpu_measurement(passes, warmup, n_el_target, sizes=FIT_SIZES, with_c2=True):
    """Best-of-`passes` times of the CPU path at `sizes` (penny elements) and
    at the C2 ellipse, and the fitted value at n_el_target elements."""
    from hfpx3d_b200 import meshgen
    R = RefCPU()
    sizes = tuple(sorted(sizes))
    meshes = {ne: tuple(np.asfortranarray(a) for a in meshgen.penny(ne, seed=7)) for ne in sizes}
    meshes = {ne: (m[0], m[1].astype(np.int64)) for ne, m in meshes.items()}
    for _ in range(warmup):                      # warm-up: the smallest sample
        R.run(*meshes[sizes[0]], S_ZZ)
    best = {ne: [np.inf, np.inf] for ne in sizes}
    c2_best = [np.inf, np.inf]
    c2_x = None
    if with_c2:
        c2_nods, c2_conn, c2_s, c2_v = c2_case()
    for _ in range(passes):
        for ne in sizes:
            ta, ts, _ = R.run(*meshes[ne], S_ZZ)
            best[ne] = [min(best[ne][0], ta), min(best[ne][1], ts)]
        if with_c2:
            ta, ts, c2_x = R.run(c2_nods, c2_conn, c2_s, vc=True, volume=c2_v)
            c2_best = [min(c2_best[0], ta), min(c2_best[1], ts)]
    # Extrapolation with the work's own exponents: the assembly evaluates
    # every (collocation point, element) pair, Ne^2 at a fixed cost per pair
    # (coefficient: the median over the sizes, robust to one noisy sample);
    # the LU does 2/3 N^3 flops, at the efficiency of the largest sample held
    # constant (OpenBLAS dgetrf is near its peak there, so efficiency does
    # not keep rising).  Free log-log fits are reported beside it.
    _, pa, ra = fit_power(sizes, [best[ne][0] for ne in sizes])
    _, pl, rl = fit_power([18 * ne for ne in sizes], [best[ne][1] for ne in sizes])
    FIT = sizes
    ca = float(np.median([best[ne][0] / float(ne) ** 2 for ne in sizes]))
    cl = best[sizes[-1]][1] / float(18 * sizes[-1]) ** 3
    t_asm = ca * float(n_el_target) ** 2
    t_lu = cl * float(18 * n_el_target) ** 3
    threads = len(os.sched_getaffinity(0))
    return {
        'value': t_asm + t_lu, 'unit': UNIT, 'cores': threads, 'kind': R.kind, 'extrapolated': True,
        'sample': (f'{"the reference (OpenMP assembly, il::LU on OpenBLAS)" if R.kind == "reference" else "the CPU oracle port + numpy LAPACK"} '
                   f'on {threads} host threads, best of {passes}, measured on seeded pennies of '
                   f'{"/".join(str(s) for s in FIT)} elements; {n_el_target} elements extrapolated as '
                   f'a Ne^2 (assembly, median coefficient) + b N^3 (LU, at the {FIT[-1]}-element '
                   f'efficiency); free log-log fits give exponents {pa:.2f} / {pl:.2f}, residuals '
                   f'{ra:.1%} / {rl:.1%}'),
        'assembly_s': t_asm, 'solve_s': t_lu,
        'fit': {'sizes_el': list(FIT), 'assembly_s': [round(best[ne][0], 4) for ne in FIT],
                'solution_s': [round(best[ne][1], 4) for ne in FIT], 'model': 'a Ne^2 + b N^3',
                'a': ca, 'b': cl, 'free_fit_assembly_exponent': pa, 'free_fit_lu_exponent': pl,
                'free_fit_assembly_residual': ra, 'free_fit_lu_residual': rl},
        'measured_c2': ({'workload': f'VC 2:1 ellipse {C2_NEL} el, N={18 * C2_NEL}+1, Haar in-situ stress, V=1',
                         'assembly_s': c2_best[0], 'solution_s': c2_best[1], 'value': c2_best[0] + c2_best[1]}
                        if with_c2 else None),
        '_c2_x': c2_x,
    }


def fit_sizes(args):
    return tuple(int(x) for x in args.fit_sizes.split(','))


def cpu_baseline(args):
    return cpu_measurement(passes=3, warmup=0, n_el_target=args.n_el, sizes=fit_sizes(args),
                           with_c2=args.c2_ref)


def run_reference(args, rank):
    if rank != 0:
        return None
    # each step is one pass over the measured sizes and the C2 ellipse; the
    # warm-up steps run the smallest sample only
    m = cpu_measurement(passes=max(1, args.steps), warmup=args.warmup, n_el_target=args.n_el,
                        sizes=fit_sizes(args), with_c2=args.c2_ref)
    m.pop('_c2_x', None)
    v = m['value']
    return {'metric': METRIC, 'value': v, 'unit': UNIT, 'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': v * 1e3, 'higher_is_better': False, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f64', 'data': 'synthetic (seeded penny and ellipse meshes)', 'impl': 'reference',
            'extrapolated': True,
            'config': {'workload': f'penny crack {args.n_el} el, N={18 * args.n_el} DoF, assembly + LU solve',
                       'n_el': args.n_el, 'mode': 'fp64'},
            'measured_c2': m['measured_c2'], 'fit': m['fit'],
            'cpu_baseline': {k: m[k] for k in ('value', 'unit', 'cores', 'kind', 'sample', 'extrapolated')},
            'e2e': {'value': v, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='engine', choices=['engine', 'reference'])
    ap.add_argument('--mode', default='learned', choices=['learned', 'mixed', 'fp64'],
                    help='the form of the timed step (the other fast form is timed once beside it)')
    ap.add_argument('--n-el', type=int, default=4000)
    ap.add_argument('--mesh', choices=['penny', 'wavy'], default='penny',
                    help='penny: the C3 crack (timed by default); wavy: a non-planar crack (off-plane pairs)')
    ap.add_argument('--tol', type=float, default=1e-10)
    ap.add_argument('--operator', choices=['mixed', 'fp64'], default='mixed',
                    help='learned form: the operator in mixed precision (FP32 far field, near-field blocks to '
                         '2^-48) or the FP64 matrix')
    ap.add_argument('--coarse', dest='coarse', action='store_true', default=True,
                    help='learned form: two-level preconditioner (coarse correction over element aggregates)')
    ap.add_argument('--no-coarse', dest='coarse', action='store_false')
    ap.add_argument('--pc', choices=sorted(PC_KINDS), default='learned',
                    help='learned form: the near-field part of the preconditioner (the network by default)')
    ap.add_argument('--solver', default='gmres', choices=['refine', 'gmres'],
                    help='mixed mode: FP64 iterative refinement or flexible GMRES, both preconditioned by the '
                         'FP32 factors')
    ap.add_argument('--no-compare', dest='compare', action='store_false')
    ap.add_argument('--no-stress', dest='stress', action='store_false',
                    help='skip the stress-at-points timing (121-element penny, 100 points, 1 and 64 load cases)')
    ap.add_argument('--no-second', dest='second', action='store_false',
                    help='skip the timing of the other fast form (mixed beside learned, or learned beside mixed)')
    ap.add_argument('--no-cpu-baseline', dest='cpu_baseline', action='store_false')
    ap.add_argument('--fit-sizes', default=','.join(str(x) for x in FIT_SIZES),
                    help='penny sizes (elements) the CPU reference is measured at and fitted from')
    ap.add_argument('--no-c2-ref', dest='c2_ref', action='store_false',
                    help='skip the CPU reference run of the 1025-element VC ellipse')
    ap.add_argument('--no-cf', dest='cf', action='store_false',
                    help='skip the cohesion/friction iteration steps on the ellipse')
    ap.add_argument('--no-batch', dest='batch', action='store_false',
                    help='skip the batched workload (256 uneven meshes x 64 load cases in one graph)')
    ap.add_argument('--no-c5-per-mesh', dest='c5_per_mesh', action='store_false',
                    help='skip the per-mesh C-ABI timing of the batched workload')
    ap.add_argument('--e2e-steps', type=int, default=3)
    ap.add_argument('--e2e-warmup', type=int, default=3)
    args = ap.parse_args()
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        line = run_reference(args, rank)
        if line:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
    if rank != 0 or world > 1:
        args.cpu_baseline = args.cpu_baseline and rank == 0 and world == 1
    line = run_engine(args, rank, world, local_rank)
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)


if __name__ == '__main__':
    main()
