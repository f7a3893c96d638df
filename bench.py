"""Throughput of the p=619 production lease on B200 (focused candidate positions per second).

Workload: 256-batch leases (1.6384e12 canonical v each, 16,384 subtiles of 1e8) of
Config(619, 10^27, 3*10^27, A619, B619), starting at the seeded batch index
random.Random(619003).randrange(0, 108298516 - 256 + 1); step k is the k-th consecutive lease
after the warm-up leases.  One step = windows of both focuses from the resident wheel tables,
per-v bounds, the fused bitset/128-bit kernel over every subtile, and the counters and outputs
back on the host.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own leases (replicas, no data exchange); rank 0 prints one
JSON line.  ``--impl reference`` times the CPU restatement of the reference path (oracle/, with
every host thread) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import random
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = 'focused candidate positions/s (p=619 production lease)'
UNIT = 'positions/s'
BATCHES_TOTAL = 108298517
LEASE_BATCHES = 256
OPS_PER_POSITION = 0.53071   # algorithmic 32-bit lane-ops per focused position (3W + 18S1 + 12T + 24Nv)
# DRAM bytes per focused position of k_match from one ncu capture of a full lease (first seeded
# lease; dram__bytes_read.sum + dram__bytes_write.sum of the k_match launch: 716,375,552 + 29,217,280
# bytes over 274,244,194,629 positions; profiles/)
DRAM_BYTES_PER_POSITION = (716_375_552 + 29_217_280) / 274244194629


def seeded_first_batch() -> int:
    return random.Random(619003).randrange(0, BATCHES_TOTAL - 1 - LEASE_BATCHES + 1)


def lease_bounds(index: int, batches: int = LEASE_BATCHES) -> tuple[int, int]:
    from psuedocubes_b200.focus import B619
    from psuedocubes_b200.optimized import BATCH_WIDTH
    width = batches * BATCH_WIDTH
    first = (seeded_first_batch() * BATCH_WIDTH + index * width) % (B619 - width)
    first -= first % BATCH_WIDTH
    return first, first + width


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device: int) -> None:
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self) -> 'ClockSampler':
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.device}', f'--query-gpu={self.QUERY}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            deadline = time.monotonic() + 5.0                 # sampling is running before the timed region
            while not self.rows and time.monotonic() < deadline:
                time.sleep(0.02)
        except OSError:
            self.proc = None
        return self

    def _read(self) -> None:
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(',')])

    def __exit__(self, *exc) -> None:
        if self.proc:
            seen, deadline = len(self.rows), time.monotonic() + 1.0   # one sample after the timed region
            while len(self.rows) == seen and time.monotonic() < deadline:
                time.sleep(0.02)
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        if not self.rows:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=['unsampled'])
        sm = [float(r[1]) for r in self.rows if r[1].replace('.', '').isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace('.', '').isdigit()]
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v.lower() == 'active'})
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                    reasons=reasons, samples=len(self.rows))


def dist_setup(n_gpus: int):
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
        return rank, world, local, dist
    return 0, 1, 0, None


def max_over_ranks(dist, value: float, local: int) -> float:
    if dist is None:
        return value
    import torch
    device = 'cpu' if dist.get_backend() == 'gloo' else f'cuda:{local}'
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def cpu_sample(steps: int, warmup: int, batches: int = 16) -> dict:
    """The oracle over `batches` batches of the first timed lease, every host thread."""
    from oracle import pcube_oracle as O
    g = O.Geometry(619, 10**27, 3 * 10**27, O.A619, O.B619)
    fa, fb = O.OracleFocus(g, 'A'), O.OracleFocus(g, 'B')
    # stage 1 through the reference's own CPU window producer (review/focus_window_cpu.cpp,
    # compiled into oracle/_ref) where it was built; stages 2 and 3 are the C restatement
    stage1 = 'reference' if O.reference_producer() is not None else 'port'
    fa.producer = fb.producer = stage1
    first, _ = lease_bounds(warmup)
    cores = os.cpu_count() or 1
    positions, elapsed = 0, 0.0
    for k in range(max(1, steps)):
        start = first + k * batches * O.BATCH_WIDTH
        t0 = time.perf_counter()
        r = O.lease(g, fa, fb, start, start + batches * O.BATCH_WIDTH, workers=cores, threads_per_batch=1)
        elapsed += time.perf_counter() - t0
        positions += r['valid_focused_candidates']
    return dict(value=positions / elapsed, unit=UNIT, cores=cores, kind='port',
                sample=f'{batches} consecutive p=619 batches ({batches * 64} subtiles) per step, {max(1, steps)} steps; '
                       + ('stage 1 by the reference\'s focus_window_cpu.cpp' if stage1 == 'reference'
                          else 'stage 1 by the C restatement of the window producer')
                       + f', the masked matcher by the C restatement; {cores} threads',
                seconds=elapsed, positions=positions)


def run_reference(args) -> None:
    rank, world, local, dist = dist_setup(args.gpus)
    if rank != 0:
        return
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_sample(1, 0, batches=4)
    sample = cpu_sample(args.steps, args.warmup, batches=32)
    line = dict(metric=METRIC, value=sample['value'], unit=UNIT, n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=1000 * sample['seconds'] / max(1, args.steps),
                higher_is_better=True, scaling='weak', vs_baseline=None, dtype='u64', data='synthetic',
                impl='reference',
                config=dict(workload='p=619 production lease, 256 batches x 64 subtiles x 1e8 v (bounded CPU sample)',
                            p=619, lease_batches=LEASE_BATCHES, first_batch=seeded_first_batch()),
                cpu_baseline=dict(value=sample['value'], unit=UNIT, cores=sample['cores'], kind=sample['kind'],
                                  sample=sample['sample']),
                e2e=dict(value=sample['value'], unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import numpy as np
    from psuedocubes_b200 import _native as N
    from psuedocubes_b200.batch_experiment import MaskedMatcher
    from psuedocubes_b200.focus import A619, B619, Config
    from psuedocubes_b200.gpu import GPUFocus, MASK, Runtime
    from psuedocubes_b200.optimized import PROFILE, compute_leases

    rank, world, local, dist = dist_setup(args.gpus)
    runtime = Runtime(time.monotonic() + 7200, 16 * 1024**3, 0.5, device=local)
    config = Config(619, 10**27, 3 * 10**27, A619, B619)
    af, bf = (GPUFocus(runtime, f) for f in config.focuses())
    tuning = {k: v for k, v in (('bitset_filters', args.bitset_filters), ('block_words', args.block_words),
                                ('threads', args.threads)) if v}
    matcher = MaskedMatcher(runtime, config, tuning)
    width = PROFILE['tile_width']
    nt = args.lease_batches * 64
    ng = len(matcher.filter_groups)
    counts = N.pinned(nt * (ng + 3))                   # page-locked result buffers (pc_host_alloc)
    geometry = N.pinned(2 * nt)
    cap = 1 << 16
    records = N.pinned(2 * cap)
    n_out = ctypes.c_uint64()
    stats = N.Stats()
    lib, ctx = runtime.lib, runtime.ctx
    c = config

    effective: dict = {}

    def step(index: int) -> tuple[int, dict]:
        first, end = lease_bounds(index * world + rank, args.lease_batches)
        runtime.call(lib.pc_run_lease(ctx, af.handle, bf.handle, matcher.filters.handle, ctypes.byref(matcher.tuning),
                                      first, end, width, c.lo & MASK, c.lo >> 64, c.hi & MASK, c.hi >> 64, counts,
                                      geometry, records, cap, ctypes.byref(n_out), ctypes.byref(stats)))
        info = stats.as_dict()
        effective.update({k: info[k] for k in ('bitset_filters', 'block_words', 'threads')})
        return int(counts.reshape(nt, ng + 3)[:, 0].sum()), info

    for k in range(args.warmup):
        step(k)
    barrier(dist)
    runtime.synchronize()
    positions, kernel_ms, launches, outputs, h2d, d2h_lib = 0, 0.0, 0, 0, 0, 0
    stage_ms = dict(window_ms=0.0, bounds_ms=0.0, kernel_ms=0.0)
    with ClockSampler(local) as clocks:
        runtime.call(lib.pc_mark(ctx, 0))
        for k in range(args.steps):
            p, st = step(args.warmup + k)
            positions += p
            kernel_ms += st['kernel_ms']
            launches += st['launches']
            outputs += st['outputs']
            h2d += st['h2d_bytes']
            d2h_lib += st['d2h_bytes']
            for key in stage_ms:
                stage_ms[key] += st[key] / args.steps
        runtime.call(lib.pc_mark(ctx, 1))
        elapsed = ctypes.c_double()
        runtime.call(lib.pc_elapsed(ctx, 0, 1, ctypes.byref(elapsed)))
    seconds = max_over_ranks(dist, elapsed.value / 1000, local)
    total_positions = positions * world   # every rank runs the same number of equal-size leases
    # end to end through the public API: compute_leases over consecutive leases (the device runs
    # them back to back in the library's lease loop; host assembly, verification and transcript of
    # each lease overlap the device work of the next)
    e2e_steps = args.e2e_steps
    e2e_positions = 0
    leases = [lease_bounds((args.warmup + args.steps + k) * world + rank, args.lease_batches) for k in range(e2e_steps)]
    if e2e_steps:                                     # warm the API's reusable page-locked buffers
        for _ in compute_leases(matcher, af, bf, leases[:1]):
            pass
    barrier(dist)
    t0 = time.perf_counter()
    for result in compute_leases(matcher, af, bf, leases):
        e2e_positions += result['valid_focused_candidates']
    e2e_seconds = max_over_ranks(dist, time.perf_counter() - t0, local) if e2e_steps else 0.0
    # the library's own count of the bytes one lease call copies (window and segment descriptors,
    # subtile map up; counters, envelope sizes, records and scalars down), as in compute_leases
    h2d_step, d2h_step = h2d // max(1, args.steps), d2h_lib // max(1, args.steps)
    if rank == 0:
        clock = clocks.summary()
        sm_mhz = clock['sm_max_mhz'] or 1965.0
        peak = runtime.sm_count * 4 * 32 * sm_mhz * 1e6 / 1e12    # Tlane-op/s integer issue
        achieved = OPS_PER_POSITION * positions / (kernel_ms / 1000) / 1e12 if kernel_ms else None
        line = dict(metric=METRIC, value=total_positions / seconds, unit=UNIT, n_gpus=world, steps=args.steps,
                    warmup=args.warmup, ms_per_step=1000 * seconds / args.steps, higher_is_better=True,
                    scaling='weak', vs_baseline=None, dtype='u64', data='synthetic',
                    config=dict(workload='p=619 production lease: 256 batches x 64 subtiles x 1e8 canonical v, '
                                         'Config(619, 10^27, 3*10^27, A619, B619)',
                                first_batch=seeded_first_batch(), lease_batches=args.lease_batches, parallelism=f'replicas{world}',
                                l2='inputs larger than L2 (resident wheel tables 208 MB, per-lease lists and bounds ~0.7 GB)'),
                    roofline=dict(bound='int_alu', achieved=achieved, peak=peak, unit='Tlaneop/s',
                                  frac=achieved / peak if achieved else None,
                                  traffic=DRAM_BYTES_PER_POSITION * positions / args.steps,
                                  traffic_unit='bytes per launch (ncu capture of a full lease, scaled by positions)',
                                  kernel='k_match (fused bitset + 128-bit filters)',
                                  ops_per_position=OPS_PER_POSITION,
                                  peak_basis=f'{runtime.sm_count} SMs x 4 SMSP x 32 lanes x {sm_mhz:.0f} MHz'),
                    e2e=dict(value=e2e_positions * world / e2e_seconds if e2e_seconds else None, unit=UNIT,
                             h2d_bytes_per_step=int(h2d_step), d2h_bytes_per_step=int(d2h_step),
                             api='psuedocubes_b200.optimized.compute_leases',
                             inputs='per lease: window, segment and subtile descriptors; the focus lists are '
                                    'generated on the device from the resident wheel tables'),
                    gpu_launches=launches, clocks=clock, tuning=effective,
                    kernel_ms_per_step=kernel_ms / args.steps, stage_ms_per_step=stage_ms)
        if kernel_ms and effective.get('bitset_filters'):
            # the resource k_match actually saturates: shared-memory bandwidth of the bitset tier,
            # which reads one 16-byte row unit per bitset filter per 128 positions
            smem_bytes = effective['bitset_filters'] * 16 / 128 * positions
            smem_peak = runtime.sm_count * 128 * sm_mhz * 1e6 / 1e12          # TB/s, 128 B per clock per SM
            smem_achieved = smem_bytes / (kernel_ms / 1000) / 1e12
            line['roofline']['shared_memory'] = dict(
                bound='smem', achieved=smem_achieved, peak=smem_peak, unit='TB/s', frac=smem_achieved / smem_peak,
                bytes_per_position=effective['bitset_filters'] * 16 / 128,
                basis='bitset-tier row reads only (survivor recompute, row build and cheap tier add to them)')
        if world == 1 and not args.no_cpu:
            line['cpu_baseline'] = {k: v for k, v in cpu_sample(1, args.warmup, batches=64).items()
                                    if k in ('value', 'unit', 'cores', 'kind', 'sample')}
        print(json.dumps(line), flush=True)
    del af, bf, matcher
    runtime.close()
    if dist is not None:
        dist.destroy_process_group()


WINDOWS_METRIC = 'focused candidate positions/s (512 uneven windows, p in [499, 619], CUDA-graph replay)'


def run_windows(args) -> None:
    """Batched uneven windows: 512 seeded windows (span floor(10^U(6,10)) v, first uniform in
    [0, B - span), p uniform over the primes in [499, 619] with p = 1 mod 3) in one launch
    sequence replayed as a CUDA graph; beside it the plain per-window tile loop of the same build
    on a sample of the windows, checked window by window."""
    from psuedocubes_b200.batched import Autotuner, BatchedEngine, DEFAULT_SETTINGS, seeded_windows, workload_digest
    from psuedocubes_b200.gpu import Matcher, Runtime
    from psuedocubes_b200.run_production import compute_batch

    rank, world, local, dist = dist_setup(args.gpus)
    runtime = Runtime(time.monotonic() + 7200, 16 * 1024**3, 0.5, device=local)
    engine = BatchedEngine(runtime)
    windows = seeded_windows(512, 619003 + rank)
    tuner = Autotuner(engine)
    settings = dict(DEFAULT_SETTINGS)
    tuned = 'defaults'
    if args.tune:
        settings, tuned = tuner.tune(windows, reuse=False).settings, 'tuned in this run'
    elif tuner.load(windows):
        settings, tuned = tuner.load(windows), 'persisted tuning'
    tuning = {k: v for k, v in settings.items() if k != 'width'}
    batch = engine.plan(windows, settings['width'], tuning, output_cap=1 << 16)
    eager = batch.run()
    for _ in range(max(1, args.warmup)):
        batch.run(graph=True)
    positions = batch.positions()
    lib, ctx = runtime.lib, runtime.ctx
    barrier(dist)
    graph_ms = []
    with ClockSampler(local) as clocks:
        runtime.call(lib.pc_mark(ctx, 0))
        for _ in range(args.steps):
            graph_ms.append(batch.run(graph=True)['kernel_ms'])
        runtime.call(lib.pc_mark(ctx, 1))
        elapsed = ctypes.c_double()
        runtime.call(lib.pc_elapsed(ctx, 0, 1, ctypes.byref(elapsed)))
    seconds = max_over_ranks(dist, elapsed.value / 1000, local)
    counts, geometry, records = batch.raw()
    launches = int(batch.last_stats.get('launches', 0))
    layout = dict(batch.layout)
    batch.close()
    # end to end through the public API: plan (descriptors to the device), eager run, results with
    # host verification of every window
    e2e_times, phases = [], []
    rows = None
    c0 = runtime.copies()
    for _ in range(max(1, args.e2e_steps)):
        t0 = time.perf_counter()
        b = engine.plan(windows, settings['width'], tuning, output_cap=1 << 16)
        t1 = time.perf_counter()
        b.run()
        t2 = time.perf_counter()
        rows = b.results()
        b.close()
        t3 = time.perf_counter()
        e2e_times.append(t3 - t0)
        phases.append((t1 - t0, t2 - t1, t3 - t2))
    c1 = runtime.copies()
    e2e_steps = max(1, args.e2e_steps)
    e2e_h2d, e2e_d2h = (c1[0] - c0[0]) // e2e_steps, (c1[1] - c0[1]) // e2e_steps
    # the same sets through the pipelined stream: set k + 1 on the device while set k is assembled
    c2 = runtime.copies()
    t0 = time.perf_counter()
    for got in engine.stream([windows] * e2e_steps, settings['width'], tuning, output_cap=1 << 16):
        rows = got
    stream_seconds = (time.perf_counter() - t0) / e2e_steps
    c3 = runtime.copies()
    stream_h2d, stream_d2h = (c3[0] - c2[0]) // e2e_steps, (c3[1] - c2[1]) // e2e_steps
    # the recorded graph replayed on its resident windows, with the results on the host each step
    replay = engine.plan(windows, settings['width'], tuning, output_cap=1 << 16)
    replay.run(graph=True)
    replay_times = []
    for _ in range(max(1, args.e2e_steps)):
        t0 = time.perf_counter()
        replay.run(graph=True)
        replay.results()
        replay_times.append(time.perf_counter() - t0)
    replay.close()
    # the plain per-window tile loop (Matcher.tile over 1e8-v tiles) on a sample, checked per window
    sample = windows[:args.plain_windows]
    mismatches, plain_positions = 0, 0
    t0 = time.perf_counter()
    for w, row in zip(sample, rows):
        c = w.config()
        af, bf = c.focuses()
        want = compute_batch(Matcher(runtime, c), engine.focus(af), engine.focus(bf), w.first, w.end, 100_000_000)
        plain_positions += want['valid_focused_candidates']
        same = all(row[k] == want[k] for k in ('valid_focused_candidates', 'group_survivors', 'local_survivors',
                                                'genuine_cubes', 'filter_groups'))
        same = same and sorted(map(int, row['all_values'])) == sorted(map(int, want['all_values']))
        mismatches += 0 if same else 1
    plain_seconds = time.perf_counter() - t0
    if rank == 0:
        clock = clocks.summary()
        sm_mhz = clock['sm_max_mhz'] or 1965.0
        peak = runtime.sm_count * 4 * 32 * sm_mhz * 1e6 / 1e12
        mean_graph_ms = sum(graph_ms) / len(graph_ms)
        achieved = OPS_PER_POSITION * positions / (mean_graph_ms / 1000) / 1e12
        plan_s, run_s, results_s = (statistics.median(p[k] for p in phases) for k in range(3))
        line = dict(metric=WINDOWS_METRIC, value=positions * world * args.steps / seconds, unit=UNIT, n_gpus=world,
                    steps=args.steps, warmup=args.warmup, ms_per_step=1000 * seconds / args.steps,
                    higher_is_better=True, scaling='weak', vs_baseline=None, dtype='u64', data='synthetic',
                    config=dict(workload='512 windows, span floor(10^U(6,10)) v, first U[0, B619 - span), '
                                         'p U{499..619, p = 1 mod 3}, Config(p, 10^27, 3*10^27, A619, B619)',
                                seed=619003, windows_sha256=workload_digest(windows),
                                span_total=sum(w.end - w.first for w in windows), positions=positions,
                                settings=settings, settings_source=tuned, layout=layout,
                                l2='inputs larger than L2 (wheel tables 208 MB; lists and per-v records of all windows)'),
                    roofline=dict(bound='int_alu', achieved=achieved, peak=peak, unit='Tlaneop/s', frac=achieved / peak,
                                  traffic=DRAM_BYTES_PER_POSITION * positions,
                                  traffic_unit='bytes per replay (lease ncu capture, scaled by positions)',
                                  kernel='whole graph (windows, bounds, k_match, k_deep): a lower bound for k_match',
                                  ops_per_position=OPS_PER_POSITION),
                    e2e=dict(value=positions * world / stream_seconds, unit=UNIT,
                             h2d_bytes_per_step=int(stream_h2d), d2h_bytes_per_step=int(stream_d2h),
                             api='BatchedEngine.stream: plan, eager run and copies of set k + 1 on the device '
                                 'thread while the host assembles and verifies the results of set k'),
                    serial_e2e=dict(value=positions * world / statistics.median(e2e_times), unit=UNIT,
                                    h2d_bytes_per_step=int(e2e_h2d), d2h_bytes_per_step=int(e2e_d2h),
                                    api='BatchedEngine.plan + WindowBatch.run + results, one after another',
                                    ms=dict(plan=1000 * plan_s, run=1000 * run_s, results=1000 * results_s)),
                    replay_e2e=dict(value=positions * world / statistics.median(replay_times), unit=UNIT,
                                    api='WindowBatch.run(graph=True) + results on a planned batch'),
                    eager=dict(ms=eager['total_ms'], kernel_ms=eager['kernel_ms'], window_ms=eager['window_ms']),
                    plain_path=dict(value=plain_positions / plain_seconds, unit=UNIT, windows=len(sample),
                                    seconds=plain_seconds, mismatches=mismatches,
                                    api='run_production.compute_batch(Matcher) per window, 1e8-v tiles'),
                    gpu_launches=launches, clocks=clock)
        print(json.dumps(line), flush=True)
    del batch, engine
    runtime.close()
    if dist is not None:
        dist.destroy_process_group()


SERVED_METRIC = 'served focused positions/s and p50/p99 latency (Poisson 20 req/s range certification)'


def run_served(args) -> None:
    """Served range certification: Poisson arrivals at 20 requests/s of (p, x_lo, x_hi), p uniform
    over the accepted primes in [499, 619], x_lo = 10^U(20, log10 3e27), span = 10^U(15, 22),
    admitted by device memory under an 8 GiB cap, continuous batching; beside it the sequential
    plain per-request loop on the same arrival stream, under a time limit.  Two more runs make the
    comparison uncensored: the same distribution at a rate the device sustains (``--sustained-rate``),
    and a sub-stream of the stream's small-span requests that both loops finish."""
    from psuedocubes_b200.gpu import Runtime
    from psuedocubes_b200.served import ServedLoop, latency_summary, plain_loop, poisson_requests, rescaled

    rank, world, local, dist = dist_setup(args.gpus)
    runtime = Runtime(time.monotonic() + 7200, 8 * 1024**3, 0.5, device=local)
    requests = poisson_requests(args.requests, rate=20.0, seed=619003 + rank)
    warm = [r for r in poisson_requests(40, rate=20.0, seed=7) if r.hi - r.lo <= 10**17][:3]
    ServedLoop(runtime).run(warm, realtime=False)
    barrier(dist)
    keys = ('valid_focused_candidates', 'group_survivors', 'local_survivors', 'genuine_cubes', 'output_sha256')

    def compare(a: dict, b: dict) -> tuple[int, int]:
        compared = mismatches = 0
        for rid, want in b['results'].items():
            got = a['results'].get(rid)
            if got is not None:
                compared += 1
                mismatches += any(got[k] != want[k] for k in keys)
        return compared, mismatches

    loop = ServedLoop(runtime)
    with ClockSampler(local) as clocks:
        served = loop.run(requests, realtime=True, time_limit=args.served_limit)
    served_summary = latency_summary(served, requests)
    print(json.dumps(dict(served=served_summary, seconds=served['seconds'])), file=sys.stderr, flush=True)
    plain = plain_loop(runtime, requests, time_limit=args.plain_limit)
    plain_summary = latency_summary(plain, requests)
    compared, mismatches = compare(served, plain)
    kernel_ms = sum(s['kernel_ms'] for s in loop.steps)
    breakdown = {k: sum(s[k] for s in loop.steps) for k in ('window_ms', 'bounds_ms', 'kernel_ms', 'total_ms',
                                                             'u_entries', 'v_entries', 'positions', 'windows')}
    # the same distribution at a load the device sustains: p50/p99 of the engine, not of a backlog
    sustained_requests = poisson_requests(args.requests, rate=args.sustained_rate, seed=619003 + rank)
    sustained_loop = ServedLoop(runtime)
    sustained = sustained_loop.run(sustained_requests, realtime=True, time_limit=args.served_limit)
    sustained_summary = latency_summary(sustained, sustained_requests)
    sustained_ms = sum(s['kernel_ms'] for s in sustained_loop.steps)
    # the stream's small-span requests, which the plain loop also finishes: both loops uncensored
    small = rescaled([r for r in requests if r.hi - r.lo <= args.small_span][:args.small_requests], args.small_rate)
    small_served = ServedLoop(runtime).run(small, realtime=True)
    small_plain = plain_loop(runtime, small)
    small_compared, small_mismatches = compare(small_served, small_plain)
    steps = loop.steps + sustained_loop.steps
    if rank == 0:
        line = dict(metric=SERVED_METRIC, value=served_summary['positions_per_second'], unit=UNIT, n_gpus=world,
                    steps=len(loop.steps), warmup=len(warm), ms_per_step=1000 * served['seconds'] / max(1, len(loop.steps)),
                    higher_is_better=True, scaling='weak', vs_baseline=None, dtype='u64', data='synthetic',
                    config=dict(workload='Poisson 20 req/s; p U{499..619, p = 1 mod 3}; x_lo = 10^U(20, log10 3e27); '
                                         'span = 10^U(15, 22); per-request focus split; 8 GiB admission cap',
                                requests=len(requests), seed=619003, arrival_span_s=requests[-1].arrival,
                                served_time_limit_s=args.served_limit, plain_time_limit_s=args.plain_limit),
                    served=dict(served_summary, seconds=served['seconds'], positions=served['positions'],
                                device_ms=kernel_ms, device_busy=kernel_ms / 1000 / served['seconds'],
                                breakdown=breakdown),
                    plain_path=dict(plain_summary, seconds=plain['seconds'], positions=plain['positions'],
                                    api='sequential plain per-request loop (Matcher.tile over the same windows)',
                                    note='censored: requests unfinished at the time limit count with the limit as '
                                         'their latency, so p50/p99 are lower bounds' if plain_summary['censored'] else ''),
                    compared_requests=compared, mismatches=mismatches,
                    sustained=dict(sustained_summary, rate=args.sustained_rate, seconds=sustained['seconds'],
                                   positions=sustained['positions'], device_ms=sustained_ms,
                                   device_busy=sustained_ms / 1000 / sustained['seconds']),
                    small_spans=dict(requests=len(small), rate=args.small_rate, max_span=args.small_span,
                                     served=latency_summary(small_served, small), plain=latency_summary(small_plain, small),
                                     compared_requests=small_compared, mismatches=small_mismatches),
                    e2e=dict(value=served_summary['positions_per_second'], unit=UNIT,
                             h2d_bytes_per_step=int(sum(s.get('h2d_bytes', 0) for s in loop.steps) / max(1, len(loop.steps))),
                             d2h_bytes_per_step=int(sum(s.get('d2h_bytes', 0) for s in loop.steps) / max(1, len(loop.steps))),
                             api='ServedLoop.run (requests in, verified results out)'),
                    gpu_launches=int(sum(s.get('launches', 0) for s in steps)), clocks=clocks.summary())
        print(json.dumps(line), flush=True)
    runtime.close()
    if dist is not None:
        dist.destroy_process_group()


CUBE_ROOTS = (1000000001, 1442249570, 619)   # cube roots of (10^27, 3*10^27], tools/check_cpu.py:24-29
CUBE_METRIC = 'cube roots checked/s (genuine-cube control, p=619, roots of (1e27, 3e27])'


def cube_groups(p: int) -> int:
    """Prime groups of the device sieve (products <= 2^16), as pc_cube_roots forms them."""
    primes = [q for q in range(2, p + 1) if all(q % d for d in range(2, int(q ** 0.5) + 1))]
    groups, product = 0, None
    for q in primes:
        if product is None or product * q > 1 << 16:
            groups, product = groups + 1, q
        else:
            product *= q
    return groups


def reference_cube_count(first: int, last: int, p: int) -> tuple[int, float]:
    """The reference's own checker (review/cube_count.c, built into oracle/_ref), one host thread."""
    exe = ROOT / 'oracle' / '_ref' / 'cube_count'
    t0 = time.perf_counter()
    row = json.loads(subprocess.check_output([str(exe), str(first), str(last), str(p)], text=True))
    return int(row['count']), time.perf_counter() - t0


def run_cubes(args) -> None:
    """The genuine-cube control over the whole p=619 interval: 442,249,570 roots per step."""
    from psuedocubes_b200 import cubes
    from psuedocubes_b200.gpu import Runtime
    rank, world, local, dist = dist_setup(args.gpus)
    runtime = Runtime(time.monotonic() + 3600, 1 << 30, 0.5, device=local)
    lib, ctx = runtime.lib, runtime.ctx
    first, last, p = CUBE_ROOTS
    n = last - first + 1
    count, kms = ctypes.c_uint64(), ctypes.c_double()

    def step() -> float:
        runtime.call(lib.pc_cube_roots(ctx, first, last, p, None, 0, ctypes.byref(count), ctypes.byref(kms)))
        if count.value != 38322775:
            raise ArithmeticError(f'genuine-cube control counted {count.value}, want 38322775')
        return kms.value

    for _ in range(args.warmup):
        step()
    barrier(dist)
    runtime.synchronize()
    kernel_ms = []
    with ClockSampler(local) as clocks:
        runtime.call(lib.pc_mark(ctx, 0))
        for _ in range(args.steps):
            kernel_ms.append(step())
        runtime.call(lib.pc_mark(ctx, 1))
        elapsed = ctypes.c_double()
        runtime.call(lib.pc_elapsed(ctx, 0, 1, ctypes.byref(elapsed)))
    seconds = max_over_ranks(dist, elapsed.value / 1000, local)
    t0 = time.perf_counter()
    e2e_steps = max(1, args.e2e_steps)
    for _ in range(e2e_steps):
        assert cubes.count_roots(runtime, first, last, p) == 38322775
    e2e_seconds = max_over_ranks(dist, time.perf_counter() - t0, local)
    if rank == 0:
        clock = clocks.summary()
        sm_mhz = clock['sm_max_mhz'] or 1965.0
        peak = runtime.sm_count * 4 * 32 * sm_mhz * 1e6 / 1e12
        groups = cube_groups(p)
        ops_per_root = 3 * groups / 32     # per (prime group, 32-root word): pattern load, funnel shift, OR
        mean_ms = statistics.mean(kernel_ms)
        achieved = ops_per_root * n / (mean_ms / 1000) / 1e12
        line = dict(metric=CUBE_METRIC, value=n * args.steps * world / seconds, unit='roots/s', n_gpus=world,
                    steps=args.steps, warmup=args.warmup, ms_per_step=1000 * seconds / args.steps,
                    higher_is_better=True, scaling='weak', vs_baseline=None, dtype='u32', data='synthetic',
                    config=dict(workload='genuine-cube control: roots [1000000001, 1442249570] coprime to every '
                                         'prime <= 619 (tools/check_cpu.py --full-cube-count)',
                                first=first, last=last, p=p, count=38322775, parallelism=f'replicas{world}',
                                l2='no input beyond 85 KB of prime patterns per CTA, staged in shared memory (compute bound)'),
                    roofline=dict(bound='int_alu', achieved=achieved, peak=peak, unit='Tlaneop/s', frac=achieved / peak,
                                  traffic=None, kernel='k_roots (count)', ops_per_root=ops_per_root, prime_groups=groups,
                                  kernel_ms=mean_ms,
                                  peak_basis=f'{runtime.sm_count} SMs x 4 SMSP x 32 lanes x {sm_mhz:.0f} MHz'),
                    e2e=dict(value=n * e2e_steps * world / e2e_seconds, unit='roots/s', h2d_bytes_per_step=0,
                             d2h_bytes_per_step=8, api='psuedocubes_b200.cubes.count_roots'),
                    gpu_launches=args.steps, clocks=clock)
        if world == 1 and not args.no_cpu:
            ref_count, ref_seconds = reference_cube_count(first, last, p)
            assert ref_count == 38322775
            line['cpu_baseline'] = dict(value=n / ref_seconds, unit='roots/s', cores=1, kind='reference',
                                        sample='the whole interval, 442,249,570 roots, review/cube_count.c '
                                               '(built from the reference sources into oracle/_ref)')
        print(json.dumps(line), flush=True)
    runtime.close()
    if dist is not None:
        dist.destroy_process_group()


def run_reference_cubes(args) -> None:
    rank, world, local, dist = dist_setup(args.gpus)
    if rank != 0:
        return
    first, last, p = CUBE_ROOTS
    n = last - first + 1
    for _ in range(max(0, min(args.warmup, 1))):
        reference_cube_count(first, first + 10**7, p)
    seconds = 0.0
    for _ in range(args.steps):
        count, t = reference_cube_count(first, last, p)
        assert count == 38322775
        seconds += t
    value = n * args.steps / seconds
    line = dict(metric=CUBE_METRIC, value=value, unit='roots/s', n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=1000 * seconds / args.steps, higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype='u32', data='synthetic', impl='reference',
                config=dict(workload='genuine-cube control: roots [1000000001, 1442249570] coprime to every prime <= 619',
                            first=first, last=last, p=p, count=38322775),
                cpu_baseline=dict(value=value, unit='roots/s', cores=1, kind='reference',
                                  sample='the whole interval per step, review/cube_count.c (oracle/_ref)'),
                e2e=dict(value=value, unit='roots/s', h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument('--gpus', type=int, default=1)
    parser.add_argument('--steps', type=int, default=5)
    parser.add_argument('--warmup', type=int, default=3)
    parser.add_argument('--impl', choices=('ours', 'reference'), default='ours')
    parser.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline sample')
    parser.add_argument('--lease-batches', type=int, default=LEASE_BATCHES,
                        help='batches per step (256 = a full lease; smaller only for profiling)')
    parser.add_argument('--e2e-steps', type=int, default=16)
    parser.add_argument('--bitset-filters', type=int, default=0, help='tuning override (0 = library default)')
    parser.add_argument('--block-words', type=int, default=0, help='tuning override (0 = library default)')
    parser.add_argument('--threads', type=int, default=0, help='tuning override (0 = library default)')
    parser.add_argument('--workload', choices=('lease', 'windows', 'served', 'cubes'), default='lease',
                        help='lease: the p=619 production lease (headline); windows: 512 uneven windows; '
                             'served: Poisson range-certification requests; cubes: the genuine-cube control '
                             'over the whole p=619 interval')
    parser.add_argument('--requests', type=int, default=100, help='served: requests in the arrival stream')
    parser.add_argument('--served-limit', type=float, default=240.0, help='served: seconds before the loop stops')
    parser.add_argument('--plain-limit', type=float, default=60.0, help='served: seconds for the plain loop')
    parser.add_argument('--sustained-rate', type=float, default=2.0,
                        help='served: arrival rate of the second run, one the device sustains')
    parser.add_argument('--small-span', type=int, default=10**16,
                        help='served: largest span of the small-span sub-stream both loops finish')
    parser.add_argument('--small-requests', type=int, default=12, help='served: requests in the small-span sub-stream')
    parser.add_argument('--small-rate', type=float, default=1.0, help='served: arrival rate of the small-span sub-stream')
    parser.add_argument('--tune', action='store_true', help='windows: run the autotuner first')
    parser.add_argument('--plain-windows', type=int, default=64,
                        help='windows: how many windows the plain per-window loop is timed and checked on')
    args = parser.parse_args()
    if args.impl == 'reference' and args.workload == 'cubes':
        run_reference_cubes(args)
    elif args.impl == 'reference':
        run_reference(args)
    elif args.workload == 'cubes':
        run_cubes(args)
    elif args.workload == 'windows':
        run_windows(args)
    elif args.workload == 'served':
        run_served(args)
    else:
        run_ours(args)


if __name__ == '__main__':
    main()
