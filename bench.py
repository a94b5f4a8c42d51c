"""Benchmark: body-steps/s of the omi_physics step on B200.

Default workload (N=1): the batched serving mix — 1024 independent debris
worlds, body counts log-uniform in [16, 2048], all resident in HBM and
advanced as concurrently stepped groups (the autotuner's cached group count
for this GPU and workload, else 4; one context, stream and CUDA graph per
group; one "step" = every world advances one dt). Reported beside it:
  * e2e: the same steps through the C ABI with every world's mutable state
    uploaded from pinned host memory and downloaded back every step (each
    group round-trips independently, so copies overlap other groups' kernels);
  * plain: the drop-in per-world path (one context per world, one graph
    launch + sync per world per step) on a sample of the mix;
  * roofline of the dominant stage from per-stage CUDA events;
  * cpu_baseline: the reference's own CPU step (oracle/_ref, NumPy + its
    Cython accelerators) on a bounded sample, all host cores;
  * capsule_triangles: the capsule-against-triangles query (65536 capsules x
    256 candidate triangles by default) device-resident, through host
    buffers, against the reference's compiled routine on all host cores, with
    its own roofline.

``--impl reference`` times the reference CPU implementation on the same
workload and prints its JSON line (rank 0 only under torchrun).
Multi-GPU (torchrun): each rank steps its own seeded copy of the mix (weak
scaling, the default) or its bin-packed share of one mix (``--scaling
strong``) — worlds are independent, so there is no collective on the data
path; the barrier and the max-over-ranks time use torch.distributed.
``--workload`` times one of the other benchmark configurations over its whole
run instead.
"""
import argparse
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

from omi_physics_b200.shard import (ShardedWorlds, barrier, max_over_ranks, merge_ticks,  # noqa: E402
                                    shard_requests, sum_over_ranks)

MEASURED = os.path.join(ROOT, 'MEASURED_PEAKS.json')
FALLBACK_HBM = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=30)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--worlds', type=int, default=1024)
    ap.add_argument('--plain-sample', type=int, default=48)
    ap.add_argument('--cpu-sample-s', type=float, default=15.0)
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--preroll', type=int, default=240,
                    help='steps every world is advanced before timing (settled piles)')
    ap.add_argument('--no-extras', action='store_true')
    ap.add_argument('--serve-requests', type=int, default=None,
                    help='requests in the serving run (default: --worlds; 0 skips it)')
    ap.add_argument('--serve-slots', type=int, default=96, help='slots per size class')
    ap.add_argument('--capsule-blocks', type=int, default=64,
                    help='capsule-triangle workload: blocks of 1024 capsules x 256 triangles (0 skips it)')
    ap.add_argument('--capsule-only', action='store_true',
                    help='run only the capsule-triangle measurement (device part) and print it')
    ap.add_argument('--groups', type=int, default=None,
                    help='worlds are stepped as this many concurrent groups (one context + stream each); '
                         'default: the autotuner\'s cached choice for this GPU and workload, else 4')
    ap.add_argument('--tune', action='store_true',
                    help='run the autotuner on the workload first (and cache its choice)')
    ap.add_argument('--workload', default='serving-mix',
                    choices=['serving-mix', 'pyramid', 'debris4096', 'convex32768', 'joints512'],
                    help='serving-mix (default): the batched headline; the others time one benchmark '
                         'configuration over its whole run from its initial state')
    ap.add_argument('--scaling', default='weak', choices=['weak', 'strong'],
                    help='serving mix under torchrun: weak = every rank steps its own seeded mix; '
                         'strong = one mix split across the ranks by body-count bin-packing')
    ap.add_argument('--config-steps', type=int, default=None,
                    help='steps of a configuration run (default: the configuration\'s own count)')
    ap.add_argument('--just-step', type=int, default=0,
                    help='only build the workload (--workload, --worlds, --seed) as one batch, step it '
                         'this many times and exit: the program a profiler captures')
    return ap.parse_args()


def just_step(args):
    """Build the workload as one WorldBatch on cuda:0 and step it; no timing."""
    import torch
    from omi_physics_b200 import WorldBatch, scenes
    if args.workload == 'serving-mix':
        _, worlds = build_mix(args.worlds, args.seed)
        dts = [w.fixed_dt for w in worlds]
    else:
        worlds, dts = scenes.CONFIGS[args.workload][0]()
    b = WorldBatch(worlds, dts=dts)
    # one step per call: a step that overflows its buffers is re-run at once,
    # so the k-th launch of a kernel belongs to step k (plus one per overflow)
    # and not to a batch of steps made no-ops behind an overflow
    for _ in range(args.just_step):
        b.step(1)
    torch.cuda.synchronize()
    print(json.dumps({'workload': args.workload, 'worlds': len(worlds), 'steps': args.just_step,
                      'contacts': int(b.counts()[1].sum())}))


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_init(n):
    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device('cuda', local))
    return rank, world, local


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock, its maximum and the slowdown reasons, sampled during the timed
    region: NVML read in-process every 5 ms (the first sample is taken before
    the region opens), else ``nvidia-smi -lms 100``. Read-only queries."""
    FIELDS = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
              'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
              'clocks_event_reasons.sw_power_cap')
    PERIOD_S = 0.005

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.nvml = None
        self.lines = []
        self._stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            p = torch.cuda.get_device_properties(self.device)
            bus = '%08X:%02X:%02X.0' % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _nvml_sample(self):
        nv, h = self.nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        flags = ['Active' if r & b else 'Not Active' for b in bits]
        self.lines.append(', '.join([str(sm), str(mx), ''] + flags))

    def _poll(self):
        while not self._stop.is_set():
            try:
                self._nvml_sample()
            except Exception:
                return
            self._stop.wait(self.PERIOD_S)

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            self._nvml_sample()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.device), '--query-gpu=' + self.FIELDS,
                 '--format=csv,noheader,nounits', '-lms', '100'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.nvml is not None:
            self._stop.set()
            self.t.join(timeout=5)
            try:
                self._nvml_sample()
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        for line in self.lines:
            parts = [p.strip() for p in line.split(',')]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, val in zip(names, parts[3:7]):
                if val.lower() == 'active':
                    reasons.add(name)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': max(mx), 'reasons': sorted(reasons),
                'samples': len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def build_mix(n_worlds, seed):
    from omi_physics_b200 import scenes
    reqs = scenes.serving_requests(n_worlds, seed=seed)
    worlds = [scenes.serving_world(r)[0] for r in reqs]
    return reqs, worlds


def dynamic_bodies(worlds):
    return int(sum(int(np.count_nonzero(w.motion_type == 2)) for w in worlds))


def algorithmic_bytes(stage, N, P, K):
    """Compulsory fp64 bytes per step of each stage (N bodies, P candidate pairs, K contacts)."""
    return {
        'refit+integrate_forces': 269 * N,
        'broadphase': 48 * N + 256 * N + 8 * P,
        'narrowphase': 160 * P + 64 * K,
        'solve': 160 * K + 168 * N,
        'integrate_positions_sleep': 170 * N,
    }[stage]


STAGE_GROUPS = {
    'refit+integrate_forces': ('refit', 'integrate_forces'),
    'broadphase': ('sort', 'pair_count', 'pair_scan', 'pair_emit'),
    'narrowphase': ('narrow', 'gjk_epa', 'contact_scan', 'contact_compact'),
    'solve': ('wake', 'prep', 'levels', 'solve', 'triggers', 'cache_store'),
    'integrate_positions_sleep': ('integrate_positions_sleep',),
}


def run_ours(args, rank, world, local):
    import torch
    from omi_physics_b200.groups import WorldGroups
    from omi_physics_b200._lib import D, U8, OmiError, ptr
    torch.cuda.set_device(local)
    t0 = time.time()
    if args.scaling == 'strong':
        # one mix for the whole job, split across ranks (each builds only its worlds)
        from omi_physics_b200 import scenes
        reqs = scenes.serving_requests(args.worlds, seed=args.seed)
        sw = ShardedWorlds([r['bodies'] + 1 for r in reqs],
                           lambda i: (lambda r: (r[0], r[1]['dt']))(scenes.serving_world(reqs[i])),
                           rank, world, groups=args.groups, device=local)
        worlds, grp = sw.worlds, sw.groups
        reqs = [reqs[i] for i in sw.indices]
    else:
        reqs, worlds = build_mix(args.worlds, args.seed + 1000 * rank)
        if args.tune:
            from omi_physics_b200 import tune
            tune.autotune(worlds, device=local, preroll=args.preroll)
        grp = WorldGroups(worlds, groups=args.groups, device=local)
    grp.step(args.preroll)
    setup_s = time.time() - t0
    N = dynamic_bodies(worlds)
    NB = sum(b.packed.n_bodies for b in grp.batches)
    # one torch stream per group, shared with the library, and a main stream
    # whose events bracket every group's work
    streams = [torch.cuda.Stream(device=local) for _ in range(len(grp))]
    grp.set_streams([s.cuda_stream for s in streams])
    main = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(main)

    def timed_steps(n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for s in streams:
            s.wait_event(e0)
        grp.step_async(n)
        for s in streams:
            ev = torch.cuda.Event()
            ev.record(s)
            main.wait_event(ev)
        e1.record(main)
        return e0, e1

    # ---- device-resident batched steps (the headline) ----
    grp.step(args.warmup)
    torch.cuda.synchronize()
    barrier(world)
    for attempt in range(4):
        launches0 = grp.launches()
        with ClockSampler(local) as clk:
            torch.cuda.synchronize()
            barrier(world)
            ev0, ev1 = timed_steps(args.steps)
            torch.cuda.synchronize()
            barrier(world)
        try:
            grp.sync()            # raises if a step overflowed its buffers (then it did nothing)
            ok = 1.0
        except OmiError:
            ok = 0.0
        if max_over_ranks(1.0 - ok, world) == 0.0:
            break
        grp.step(1)               # synchronous steps regrow the buffers; time again
    ms = ev0.elapsed_time(ev1)
    launches = grp.launches() - launches0
    ms_max = max_over_ranks(ms, world)
    total_N = sum_over_ranks(N, world)
    value = total_N * args.steps / (ms_max / 1e3)
    pairs, contacts = grp.counts()
    P, K = int(pairs.sum()), int(contacts.sum())

    # per-step tick latency distribution (every world one step, synchronised per tick)
    ticks = []
    for _ in range(max(10, min(args.steps, 50))):
        barrier(world)
        a, b = timed_steps(1)
        b.synchronize()
        ticks.append(a.elapsed_time(b))
    grp.sync()
    ticks = merge_ticks(ticks, world)          # a tick ends when its slowest rank's does

    # ---- roofline: per-stage device time of eagerly launched steps (groups one
    # after another, so the sums are the stage times of the whole mix) ----
    prof = {}
    n_prof = 5
    for _ in range(n_prof):
        for bt in grp.batches:
            for k, v in bt.profile().items():
                prof[k] = prof.get(k, 0.0) + v / n_prof
    groups = {g: sum(prof.get(k, 0.0) for k in ks) for g, ks in STAGE_GROUPS.items()}
    dominant = max(groups, key=groups.get)
    dom_ms = groups[dominant]
    alg = algorithmic_bytes(dominant, NB, P, K)
    peaks = {}
    if os.path.exists(MEASURED):
        peaks = json.load(open(MEASURED))
    peak = float(peaks.get('hbm_gbs', FALLBACK_HBM))
    achieved = alg / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    traffic = None
    tpath = os.path.join(ROOT, 'profiles', 'traffic.json')
    if os.path.exists(tpath):
        tr = json.load(open(tpath)).get(dominant)
        if tr is not None:
            traffic = tr.get('bytes_per_body', 0.0) * NB + tr.get('bytes_per_contact', 0.0) * K
    n_groups = len(grp.batches)
    roofline = {'bound': 'hbm', 'kernel': dominant, 'achieved': round(achieved, 3), 'peak': peak,
                'unit': 'GB/s', 'frac': achieved / peak, 'traffic': traffic,
                'algorithmic_bytes': alg, 'kernel_ms': dom_ms,
                'basis': ('the stage\'s CUDA-event time summed over the %d groups, each group\'s steps '
                          'launched eagerly one group after another (in the timed step the groups run '
                          'concurrently, so kernel_ms may exceed ms_per_step); bytes and time both sum '
                          'over the groups' % n_groups),
                'launches_per_step': n_groups,
                'kernel_ms_per_launch': dom_ms / max(n_groups, 1),
                'step_frac': (sum(algorithmic_bytes(g, NB, P, K) for g in STAGE_GROUPS)
                              / (ms / args.steps / 1e3) / 1e9 / peak),
                'peak_source': 'measured' if 'hbm_gbs' in peaks else 'fallback',
                'stage_ms': {k: round(v, 4) for k, v in groups.items()},
                'kernel_group_ms': {k: round(v, 4) for k, v in prof.items()}}

    # ---- e2e: every group's state through pinned host buffers every step ----
    def pinned(shape, dtype=np.float64):
        return torch.empty(shape, dtype=torch.float64 if dtype == np.float64 else torch.uint8,
                           pin_memory=True).numpy()
    bufs = grp.host_buffers(alloc=pinned)
    for bt, h in zip(grp.batches, bufs):
        nb = bt.packed.n_bodies
        bt.ctx.call('download_state', 0, nb, ptr(h['pos'], D), ptr(h['q'], D), ptr(h['v'], D),
                    ptr(h['w'], D), ptr(h['awake'], U8), ptr(h['timer'], D), None, None)
    h2d = sum(a.nbytes for h in bufs for a in h.values())
    e2e_steps = max(3, min(args.steps, 20))
    grp.step_from_host(bufs, 1)
    barrier(world)
    t = time.perf_counter()
    grp.step_from_host(bufs, 1, rounds=e2e_steps)      # every step a host round trip per group
    e2e_s = max_over_ranks(time.perf_counter() - t, world)
    e2e = {'value': total_N * e2e_steps / e2e_s, 'unit': 'body-steps/s', 'h2d_bytes_per_step': h2d,
           'd2h_bytes_per_step': h2d,
           'path': 'every step, per group: omi_upload_state + omi_step + omi_download_state from pinned '
                   'memory; groups run concurrently without a barrier between steps'}
    stream = main

    extras = {}
    n_serve = args.worlds if args.serve_requests is None else args.serve_requests
    if not args.no_extras and n_serve > 0:
        if args.scaling == 'strong':
            extras['serving'] = serving_run(n_serve, args.seed, args.serve_slots, stream,
                                            shard=(rank, world))
        else:
            extras['serving'] = serving_run(n_serve, args.seed + 1000 * rank, args.serve_slots, stream)
        barrier(world)
    if not args.no_extras and rank == 0:
        extras['plain'] = plain_per_world(worlds, reqs, args.plain_sample, local, args.preroll)
    note = _tuning_note(grp)
    grp.close()
    return dict(value=value, ms=ms_max, N=total_N, P=P, K=K, launches=launches, setup_s=setup_s,
                ticks=ticks, roofline=roofline, e2e=e2e, clocks=clk.summary(), extras=extras,
                NB=NB, tuning=note)


def _tuning_note(grp):
    """Which launch configuration and group count ran, and where they came from."""
    launch = grp.batches[0].ctx.tuning() if grp.batches else {}
    return {'groups': len(grp.batches), 'launch': launch,
            'source': 'autotuner cache' if grp.tuned is not None else 'library defaults'}


SERVE_BUDGET = 120 * 10 ** 9


def serving_run(n_requests, seed, per_class, stream, shard=None):
    """The request loop: Poisson arrivals (200/s), each world admitted into a
    free slot of its size class under the HBM budget, stepped with every other
    resident world once per tick until its 60-600 steps are done. ``shard``
    (rank, ranks): this rank serves only its share of one request stream."""
    from omi_physics_b200 import scenes
    from omi_physics_b200.serving import Server, size_classes
    reqs = scenes.serving_requests(n_requests, seed=seed)
    if shard is not None:
        reqs = [reqs[i] for i in shard_requests(reqs, shard[0], shard[1])]
    srv = Server(size_classes(2048, per_class=per_class), budget_bytes=SERVE_BUDGET,
                 stream=stream.cuda_stream)
    for r in reqs:
        w, meta = scenes.serving_world(r)
        srv.submit(w, r['steps'], dt=meta['dt'], arrival=r['arrival'])
    srv.ctx.call('step', 1)         # capture the step graph while every slot is empty
    st = srv.run(clock='wall').summary()
    srv.close()
    st.update(requests=n_requests, arrival_rate_per_s=200.0, slots=srv.W,
              slot_classes='bodies 33..2049 (powers of two + ground), %d each' % per_class,
              budget_bytes=SERVE_BUDGET,
              note='wall-clock ticks: admit (omi_load_world) + one omi_step of all resident '
                   'worlds + retire (state download); body-steps/s is bounded by the arrival rate')
    return st


def plain_per_world(worlds, reqs, sample, device, preroll):
    """The drop-in path: one context per world, one step launch + sync each."""
    from omi_physics_b200 import WorldBatch, scenes
    rng = np.random.default_rng(7)
    idx = sorted(rng.choice(len(reqs), size=min(sample, len(reqs)), replace=False))
    sub = [scenes.serving_world(reqs[i])[0] for i in idx]
    batches = [WorldBatch([w], device=device) for w in sub]
    for b in batches:
        b.step(preroll)
    steps = 5
    t = time.perf_counter()
    for _ in range(steps):
        for b in batches:
            b.ctx.call('step', 1)
    dt = time.perf_counter() - t
    n = sum(int(np.count_nonzero(w.motion_type == 2)) for w in sub)
    rate = n * steps / dt
    for b in batches:
        b.ctx.close()
    return {'value': rate, 'unit': 'body-steps/s', 'worlds_sampled': len(sub),
            'method': 'sequential per-world omi_step (graph launch + sync) over a sample of the mix'}


# ---------------------------------------------------------------------------
# capsule against triangles (the character controller's query, batched)
# ---------------------------------------------------------------------------
CAPS_PER_BLOCK, TRIS_PER_CAPSULE = 1024, 256
CT_BYTES = 72 + 57          # per triangle: vertices in; hit, point, normal, depth out


def capsule_block(seed, b):
    """Block ``b``: 1024 capsules (random pose, half height [0, 0.9), radius
    [0.2, 0.8)), each with 256 candidate triangles scattered around it."""
    rng = np.random.default_rng([seed, b])
    q, k = CAPS_PER_BLOCK, TRIS_PER_CAPSULE
    centres = rng.uniform(-50, 50, size=(q, 3))
    axes = rng.normal(size=(q, 3))
    axes /= np.linalg.norm(axes, axis=1, keepdims=True)
    half = rng.uniform(0.0, 0.9, size=q)
    caps = np.concatenate([centres - axes * half[:, None], centres + axes * half[:, None],
                           rng.uniform(0.2, 0.8, size=(q, 1))], axis=1)
    verts = np.repeat(centres, k, axis=0)[:, None, :] + rng.normal(scale=1.0, size=(q * k, 3, 3))
    return caps, verts


def _capsule_ref_worker(payload):
    seed, blocks = payload
    sys.path.insert(0, os.path.join(ROOT, 'oracle', '_ref'))
    from omi_physics import collide
    nat = collide._native
    k = TRIS_PER_CAPSULE
    hit = np.zeros(k, np.uint8)
    pts, nrm, dep = np.zeros((k, 3)), np.zeros((k, 3)), np.zeros(k)
    done, spent = 0, 0.0
    for b in blocks:
        caps, verts = capsule_block(seed, b)
        t = time.perf_counter()
        for c in range(len(caps)):
            nat.capsule_triangles(caps[c, :3], caps[c, 3:6], float(caps[c, 6]), verts[c * k:(c + 1) * k],
                                  hit, pts, nrm, dep)
        spent += time.perf_counter() - t
        done += len(verts)
    return done, spent


def capsule_cpu_reference(seed, blocks, cores=None):
    """The reference's compiled capsule_triangles (oracle/_ref) over the same
    capsules, one call per capsule with reused output arrays, blocks spread
    over a process pool."""
    import multiprocessing as mp
    if not os.path.isdir(os.path.join(ROOT, 'oracle', '_ref', 'omi_physics')):
        return None
    cores = min(cores or os.cpu_count() or 1, blocks)
    chunks = [list(range(i, blocks, cores)) for i in range(cores)]
    t = time.perf_counter()
    with mp.get_context('spawn').Pool(cores) as pool:
        res = pool.map(_capsule_ref_worker, [(seed, c) for c in chunks])
    wall = time.perf_counter() - t
    tris = sum(r[0] for r in res)
    slowest = max(r[1] for r in res)
    per_core = tris / sum(r[1] for r in res)
    return {'value': tris / slowest, 'unit': 'triangles/s', 'cores': cores, 'kind': 'reference',
            'sample': '%d triangles (%d capsules x %d), _native.capsule_triangles per capsule with '
                      'reused outputs, %d processes, %.1f s wall' % (tris, tris // TRIS_PER_CAPSULE,
                                                                     TRIS_PER_CAPSULE, cores, wall),
            'per_core': per_core}


def capsule_triangles_run(seed, blocks, local, steps, warmup, device_only=False):
    """Device-resident throughput of k_capsule_triangles (CUDA events on the
    launching stream), the same through host buffers (omi_capsule_triangles_batch
    from pinned memory, copies inside the timed region), and the reference's
    compiled routine on the host cores."""
    import torch
    from omi_physics_b200 import collide as oc
    parts = [capsule_block(seed, b) for b in range(blocks)]
    caps = np.concatenate([p[0] for p in parts])
    verts = np.concatenate([p[1] for p in parts])
    del parts
    q, n = len(caps), len(verts)
    off = np.arange(0, n + 1, TRIS_PER_CAPSULE, dtype=np.int64)
    dev = torch.device('cuda', local)
    tc, to = torch.from_numpy(caps).to(dev), torch.from_numpy(off).to(dev)
    tv = torch.from_numpy(verts).to(dev)
    th = torch.empty(n, dtype=torch.uint8, device=dev)
    tp = torch.empty((n, 3), dtype=torch.float64, device=dev)
    tn = torch.empty((n, 3), dtype=torch.float64, device=dev)
    td = torch.empty(n, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    ctx, lock = oc.context(local)
    with lock:
        ctx.call('set_stream', stream.cuda_stream)
        args = (ctx, q, tc.data_ptr(), to.data_ptr(), tv.data_ptr(), n, th.data_ptr(), tp.data_ptr(),
                tn.data_ptr(), td.data_ptr())
        for _ in range(max(3, warmup)):
            oc.capsule_triangles_device(*args)
        torch.cuda.synchronize(dev)
        launches0 = ctx.launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(steps, 10 * steps)       # long enough for the clock sampler to see it
        with ClockSampler(local) as clk:
            e0.record(stream)
            for _ in range(reps):
                oc.capsule_triangles_device(*args)
            e1.record(stream)
            torch.cuda.synchronize(dev)
        launches = ctx.launches() - launches0
        ms = e0.elapsed_time(e1) / reps
        ctx.call('set_stream', None)
    hits = int(th.sum().item())
    value = n / (ms / 1e3)
    peaks = json.load(open(MEASURED)) if os.path.exists(MEASURED) else {}
    peak = float(peaks.get('hbm_gbs', FALLBACK_HBM))
    achieved = CT_BYTES * n / (ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, 'profiles', 'traffic.json')
    if os.path.exists(tpath):
        tr = json.load(open(tpath)).get('capsule_triangles')
        if tr is not None:
            traffic = tr.get('bytes_per_triangle', 0.0) * n
    del tv, th, tp, tn, td
    torch.cuda.empty_cache()
    if device_only:
        return {'workload': '%d capsules x %d triangles' % (q, TRIS_PER_CAPSULE), 'value': value,
                'unit': 'triangles/s', 'ms_per_launch': ms, 'achieved_gbs': achieved, 'peak_gbs': peak,
                'frac': achieved / peak, 'gpu_launches': launches, 'clocks': clk.summary()}

    # host buffers: pinned, copies in the timed region
    def pinned(shape, dt):
        return torch.empty(shape, dtype=dt, pin_memory=True).numpy()
    hv = pinned((n, 3, 3), torch.float64)
    hv[:] = verts
    del verts
    out = (pinned(n, torch.uint8), pinned((n, 3), torch.float64), pinned((n, 3), torch.float64),
           pinned(n, torch.float64))
    oc.capsule_triangles_many(caps, off, hv, device=local, out=out)
    e2e_calls = 3
    t = time.perf_counter()
    for _ in range(e2e_calls):
        oc.capsule_triangles_many(caps, off, hv, device=local, out=out)
    e2e_s = (time.perf_counter() - t) / e2e_calls
    cb = capsule_cpu_reference(seed, blocks)
    line = {'workload': '%d capsules x %d triangles (%d triangles, %.2f GB in + out)'
                        % (q, TRIS_PER_CAPSULE, n, CT_BYTES * n / 1e9),
            'metric': 'triangles/s', 'value': value, 'ms_per_launch': ms, 'hit_fraction': hits / n,
            'gpu_launches': launches, 'dtype': 'f64', 'clocks': clk.summary(),
            'l2': 'inputs larger than L2 (%.1f GB of vertices)' % (72 * n / 1e9),
            'roofline': {'bound': 'hbm', 'kernel': 'k_capsule_triangles', 'achieved': round(achieved, 3),
                         'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak, 'traffic': traffic,
                         'algorithmic_bytes': CT_BYTES * n,
                         'peak_source': 'measured' if 'hbm_gbs' in peaks else 'fallback'},
            'e2e': {'value': n / e2e_s, 'unit': 'triangles/s', 'h2d_bytes_per_step': 72 * n + caps.nbytes +
                    off.nbytes, 'd2h_bytes_per_step': 57 * n,
                    'path': 'omi_capsule_triangles_batch from pinned host arrays (2 streams, 2M-triangle '
                            'chunks)'}}
    if cb is not None:
        line['cpu_baseline'] = {k: cb[k] for k in ('value', 'unit', 'cores', 'kind', 'sample', 'per_core')}
        line['e2e_over_cpu'] = line['e2e']['value'] / cb['value']
    return line


# ---------------------------------------------------------------------------
# CPU reference (oracle/_ref: the reference built from its own sources)
# ---------------------------------------------------------------------------
def _ref_worker(payload):
    idx, seed, n_worlds, budget_s, preroll = payload
    sys.path.insert(0, os.path.join(ROOT, 'oracle', '_ref'))
    from types import SimpleNamespace
    import omi_physics as ref
    from omi_physics import joints as rj, model as rm
    from omi_physics_b200 import scenes
    api = SimpleNamespace(PhysicsWorld=ref.PhysicsWorld, model=rm, joints=rj)
    reqs = scenes.serving_requests(n_worlds, seed=seed)
    done = 0
    t_total = 0.0
    start = time.perf_counter()
    for i in idx:
        w, meta = scenes.serving_world(reqs[i], api=api)
        n = int(np.count_nonzero(w.motion_type == 2))
        for _ in range(preroll):                 # same settled state as the GPU arm
            w.step(meta['dt'])
        t = time.perf_counter()
        for _ in range(2):
            w.step(meta['dt'])
        t_total += time.perf_counter() - t
        done += 2 * n
        if time.perf_counter() - start > budget_s:
            break
    return done, t_total


def cpu_reference(n_worlds, seed, budget_s, preroll, cores=None):
    import multiprocessing as mp
    cores = cores or os.cpu_count() or 1
    ref_dir = os.path.join(ROOT, 'oracle', '_ref', 'omi_physics')
    if not os.path.isdir(ref_dir):
        return None
    rng = np.random.default_rng(11)
    order = list(rng.permutation(n_worlds))
    chunks = [order[i::cores] for i in range(cores)]
    ctx = mp.get_context('spawn')
    t = time.perf_counter()
    with ctx.Pool(cores) as pool:
        res = pool.map(_ref_worker, [(c, seed, n_worlds, budget_s, preroll) for c in chunks])
    wall = time.perf_counter() - t
    body_steps = sum(r[0] for r in res)
    step_time = sum(r[1] for r in res)
    # each process advanced its worlds one step each; throughput with all cores
    per_core = body_steps / step_time if step_time > 0 else 0.0
    return {'value': per_core * cores, 'unit': 'body-steps/s', 'cores': cores, 'kind': 'reference',
            'sample': '%d body-steps: worlds of the serving mix pre-rolled %d steps, then 2 timed '
                      'steps each; %d processes, %.1f s wall' % (body_steps, preroll, cores, wall),
            'per_core': per_core}


# ---------------------------------------------------------------------------
# the other benchmark configurations, each timed over its whole run
# ---------------------------------------------------------------------------
CONFIG_META = {
    'pyramid': dict(desc='10-level pyramid of 55 unit boxes on a 20x1x20 m ground box', dt='1/60 s',
                    iterations=10, cpu_budget_s=20.0),
    'debris4096': dict(desc='4096 bodies, 70% boxes [0.5,1.5] m / 30% spheres r [0.25,0.75] m, '
                            'density 1000, above a 60x1x60 m ground box', dt='1/120 s', iterations=8,
                       cpu_budget_s=40.0),
    'convex32768': dict(desc='32768 bodies, 50% boxes / 25% spheres / 25% convex hulls (12-32 points on '
                             'ellipsoids, GJK/EPA) in a walled 100x100 m arena, sleeping on',
                        dt='1/120 s', iterations=8, cpu_budget_s=60.0),
    'joints512': dict(desc='512 worlds: chains of 16-128 links (point joints, 10% motored) under 64-512 '
                           'loose boxes', dt='1/240 s', iterations=12, cpu_budget_s=40.0),
}


def _cfg_ref_worker(payload):
    """Reference CPU step (oracle/_ref) on worlds ``idx`` of a configuration:
    each world from its initial state for up to ``max_steps`` steps, within
    ``budget_s``. Returns (body-steps, seconds stepping, per-step seconds of
    the first world, steps done)."""
    name, idx, max_steps, budget_s = payload
    sys.path.insert(0, os.path.join(ROOT, 'oracle', '_ref'))
    from types import SimpleNamespace
    import omi_physics as ref
    from omi_physics import gravity as rg, joints as rj, model as rm
    from omi_physics_b200 import scenes
    api = SimpleNamespace(PhysicsWorld=ref.PhysicsWorld, model=rm, joints=rj, gravity=rg)
    builder, _ = scenes.CONFIGS[name]
    if name == 'joints512':
        worlds, dts = scenes.joint_chains(512, 21, api, which=idx)
    else:
        worlds, dts = builder(api)
    start = time.perf_counter()
    done = spent = 0.0
    per_step = []
    steps_done = 0
    for s in range(max_steps):
        for w, dt in zip(worlds, dts):
            n = int(np.count_nonzero(w.motion_type == 2))
            t = time.perf_counter()
            w.step(dt)
            el = time.perf_counter() - t
            spent += el
            done += n
            if w is worlds[0]:
                per_step.append(el)
        steps_done = s + 1
        if time.perf_counter() - start > budget_s:
            break
    return done, spent, per_step, steps_done


def config_cpu_reference(name, max_steps, budget_s, cores=None):
    """The reference's CPU step on a bounded sample of a configuration run
    (its first steps from the initial state): one process for a one-world
    configuration (the reference is single-threaded), all host cores through
    a spawn pool for the multi-world one."""
    import multiprocessing as mp
    if not os.path.isdir(os.path.join(ROOT, 'oracle', '_ref', 'omi_physics')):
        return None
    ctx = mp.get_context('spawn')
    t = time.perf_counter()
    if name == 'joints512':
        cores = cores or os.cpu_count() or 1
        chunks = [list(range(i, 512, cores)) for i in range(cores)]
        with ctx.Pool(cores) as pool:
            res = pool.map(_cfg_ref_worker, [(name, c, max_steps, budget_s) for c in chunks])
        wall = time.perf_counter() - t
        body_steps = sum(r[0] for r in res)
        slowest = max(r[1] for r in res)
        steps = min(r[3] for r in res)
        return {'value': body_steps / slowest, 'unit': 'body-steps/s', 'cores': cores, 'kind': 'reference',
                'per_core': body_steps / sum(r[1] for r in res), 'steps': steps,
                'sample': '%d body-steps: every world from its initial state for its first %d+ steps, '
                          '%d processes, %.1f s wall' % (body_steps, steps, cores, wall)}
    with ctx.Pool(1) as pool:
        done, spent, per_step, steps = pool.map(_cfg_ref_worker, [(name, [0], max_steps, budget_s)])[0]
    wall = time.perf_counter() - t
    return {'value': done / spent, 'unit': 'body-steps/s', 'cores': 1, 'kind': 'reference',
            'per_core': done / spent, 'steps': steps, 'ms_per_step': [1e3 * x for x in per_step],
            'sample': 'the first %d steps of the run from the initial state, one process (%.1f s wall '
                      'with the world build)' % (steps, wall)}


def run_config(args, rank, world_size, local):
    """One benchmark configuration over its whole run: the initial state, every
    step of the run timed on the device (CUDA events around each step, L2
    flushed between steps), after an untimed warm-up run of the same steps
    that sizes the pair and contact buffers."""
    import torch
    from omi_physics_b200 import scenes
    from omi_physics_b200._lib import D, U8, ptr
    from omi_physics_b200.groups import WorldGroups
    torch.cuda.set_device(local)
    builder, cfg_steps = scenes.CONFIGS[args.workload]
    steps = args.config_steps or cfg_steps
    t0 = time.time()
    worlds, dts = builder()
    N = dynamic_bodies(worlds)
    if args.tune:
        from omi_physics_b200 import tune
        tune.autotune(worlds, dts, device=local)
    grp = WorldGroups(worlds, dts=dts, groups=args.groups if len(worlds) > 1 else 1, device=local)
    snaps = [[b.snapshot(j) for j in range(len(b.worlds))] for b in grp.batches]

    def restore():
        for b, ss in zip(grp.batches, snaps):
            for j, sn in enumerate(ss):
                b.restore(j, sn)
        torch.cuda.synchronize()

    streams = [torch.cuda.Stream(device=local) for _ in range(len(grp))]
    grp.set_streams([s.cuda_stream for s in streams])
    grp.step(steps)                       # warm-up: the whole run once (buffers grow to what it needs)
    restore()
    setup_s = time.time() - t0
    main = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(main)
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device='cuda:%d' % local)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    launches0 = grp.launches()
    barrier(world_size)
    with ClockSampler(local) as clk:
        for e0, e1 in evs:
            flush.zero_()                 # L2 flushed between timed steps (outside the events)
            e0.record(main)
            for s in streams:
                s.wait_event(e0)
            grp.step_async(1)
            for s in streams:
                ev = torch.cuda.Event()
                ev.record(s)
                main.wait_event(ev)
            e1.record(main)
        torch.cuda.synchronize()
    grp.sync()                            # raises if a step overflowed (it cannot: same run as the warm-up)
    launches = grp.launches() - launches0
    step_ms = np.array([a.elapsed_time(b) for a, b in evs])
    total_ms = max_over_ranks(float(step_ms.sum()), world_size)
    value = sum_over_ranks(N, world_size) * steps / (total_ms / 1e3)
    pairs, contacts = grp.counts()
    P, K = int(pairs.sum()), int(contacts.sum())
    NB = sum(b.packed.n_bodies for b in grp.batches)
    # roofline of the dominant stage at the end of the run (eager per-stage events, one group after another)
    prof = {}
    for _ in range(3):
        for bt in grp.batches:
            for k, v in bt.profile().items():
                prof[k] = prof.get(k, 0.0) + v / 3
    stage = {g: sum(prof.get(k, 0.0) for k in ks) for g, ks in STAGE_GROUPS.items()}
    dominant = max(stage, key=stage.get)
    peaks = json.load(open(MEASURED)) if os.path.exists(MEASURED) else {}
    peak = float(peaks.get('hbm_gbs', FALLBACK_HBM))
    alg = algorithmic_bytes(dominant, NB, P, K)
    achieved = alg / (stage[dominant] / 1e3) / 1e9 if stage[dominant] > 0 else 0.0
    step_bytes = sum(algorithmic_bytes(g, NB, P, K) for g in STAGE_GROUPS)
    roofline = {'bound': 'hbm', 'kernel': dominant, 'achieved': round(achieved, 3), 'peak': peak,
                'unit': 'GB/s', 'frac': achieved / peak, 'traffic': None, 'algorithmic_bytes': alg,
                'kernel_ms': stage[dominant], 'peak_source': 'measured' if 'hbm_gbs' in peaks else 'fallback',
                'basis': 'per-stage CUDA events of 3 eagerly launched steps at the end of the run',
                'stage_ms': {k: round(v, 4) for k, v in stage.items()},
                'kernel_group_ms': {k: round(v, 4) for k, v in prof.items()},
                'step_algorithmic_bytes': step_bytes,
                'step_frac': step_bytes / (float(np.mean(step_ms[-20:])) / 1e3) / 1e9 / peak}
    # e2e: the same run through the C ABI with host buffers every step
    restore()

    def pinned(shape, dtype=np.float64):
        return torch.empty(shape, dtype=torch.float64 if dtype == np.float64 else torch.uint8,
                           pin_memory=True).numpy()
    bufs = grp.host_buffers(alloc=pinned)
    for bt, h in zip(grp.batches, bufs):
        nb = bt.packed.n_bodies
        bt.ctx.call('download_state', 0, nb, ptr(h['pos'], D), ptr(h['q'], D), ptr(h['v'], D),
                    ptr(h['w'], D), ptr(h['awake'], U8), ptr(h['timer'], D), None, None)
    h2d = sum(a.nbytes for h in bufs for a in h.values())
    torch.cuda.synchronize()
    t = time.perf_counter()
    grp.step_from_host(bufs, 1, rounds=steps)
    e2e_s = max_over_ranks(time.perf_counter() - t, world_size)
    e2e = {'value': sum_over_ranks(N, world_size) * steps / e2e_s, 'unit': 'body-steps/s',
           'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': h2d,
           'path': 'the whole run from the initial state, every step: omi_upload_state + omi_step + '
                   'omi_download_state from pinned memory (per group, groups concurrent)'}
    note = _tuning_note(grp)
    grp.close()
    return dict(value=value, steps=steps, step_ms=step_ms, N=N, NB=NB, P=P, K=K, launches=launches,
                roofline=roofline, e2e=e2e, clocks=clk.summary(), setup_s=setup_s,
                worlds=len(worlds), tuning=note)


def main_config(args, rank, world_size, local):
    name = args.workload
    meta = CONFIG_META[name]
    metric = 'body-steps/s (%s configuration, whole run)' % name
    config = {'workload': name, 'scene': meta['desc'], 'dt': meta['dt'], 'iterations': meta['iterations'],
              'steps': args.config_steps or None, 'l2': 'flushed between timed steps (256 MB write)',
              'parallelism': 'one GPU' if world_size == 1 else 'replicas x%d' % world_size}
    from omi_physics_b200 import scenes
    cfg_steps = args.config_steps or scenes.CONFIGS[name][1]
    config['steps'] = cfg_steps
    if args.impl == 'reference':
        if rank == 0:
            r = config_cpu_reference(name, cfg_steps, max(5.0, meta['cpu_budget_s']))
            if r is None:
                print(json.dumps({'impl': 'reference', 'unavailable':
                                  'oracle/_ref (the reference built from its sources) is missing'}))
            else:
                print(json.dumps({'impl': 'reference', 'metric': metric, 'value': r['value'],
                                  'unit': 'body-steps/s', 'n_gpus': args.gpus, 'steps': r['steps'],
                                  'warmup': 0, 'higher_is_better': True, 'scaling': 'weak', 'dtype': 'f64',
                                  'data': 'synthetic', 'config': config,
                                  'cpu_baseline': {k: r[k] for k in ('value', 'unit', 'cores', 'kind',
                                                                     'sample', 'per_core')},
                                  'e2e': {'value': r['value'], 'unit': 'body-steps/s',
                                          'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}))
        return
    res = run_config(args, rank, world_size, local)
    if rank != 0:
        return
    sm = res['step_ms']
    line = {'metric': metric, 'value': res['value'], 'unit': 'body-steps/s', 'n_gpus': world_size,
            'steps': res['steps'], 'warmup': res['steps'], 'ms_per_step': float(sm.mean()),
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic (seeded %s scene)' % name, 'config': config, 'e2e': res['e2e'],
            'roofline': res['roofline'], 'clocks': res['clocks'], 'gpu_launches': res['launches'],
            'step_latency_ms': {'p50': float(np.percentile(sm, 50)), 'p99': float(np.percentile(sm, 99)),
                                'max': float(sm.max()), 'first': float(sm[0])},
            'dynamic_bodies': res['N'], 'worlds': res['worlds'], 'final_pairs': res['P'],
            'final_contacts': res['K'], 'tuning': res['tuning']}
    if not args.no_extras:
        cb = config_cpu_reference(name, res['steps'], CONFIG_META[name]['cpu_budget_s'])
        if cb is not None:
            line['cpu_baseline'] = {k: cb[k] for k in ('value', 'unit', 'cores', 'kind', 'sample', 'per_core')}
            k = cb['steps']
            win = float(sm[:k].sum())
            line['gpu_same_window'] = {'steps': k, 'value': res['N'] * k / (win / 1e3), 'unit': 'body-steps/s',
                                       'note': 'device time of the same first steps the CPU sample ran'}
            line['same_window_over_cpu'] = line['gpu_same_window']['value'] / cb['value']
    print(json.dumps(line))


def main():
    args = parse()
    if args.just_step:
        return just_step(args)
    rank, world, local = dist_init(args.gpus)
    if args.workload != 'serving-mix':
        main_config(args, rank, world, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    metric = 'body-steps/s (batched serving mix, 1 B200 per rank)'
    config = {'workload': 'serving-mix',
              ('worlds' if args.scaling == 'strong' else 'worlds_per_gpu'): args.worlds,
              'bodies': 'log-uniform [16,2048] per world, debris contents', 'dt': '1/120 s',
              'iterations': 8, 'l2': 'inputs larger than L2 (arena state > 126 MB)',
              'parallelism': ('one mix split across %d GPUs by body-count bin-packing' % world
                              if args.scaling == 'strong' else
                              'world-sharded x%d (no data-path collective)' % world),
              'groups_per_gpu': args.groups or 'autotuned (else 4)'}
    if args.impl == 'reference':
        if rank == 0:
            budget = max(5.0, args.cpu_sample_s)
            r = cpu_reference(args.worlds, args.seed, budget, args.preroll)
            if r is None:
                print(json.dumps({'impl': 'reference', 'unavailable':
                                  'oracle/_ref (the reference built from its sources) is missing'}))
            else:
                line = {'impl': 'reference', 'metric': metric, 'value': r['value'],
                        'unit': 'body-steps/s', 'n_gpus': args.gpus, 'steps': args.steps,
                        'warmup': args.warmup, 'higher_is_better': True, 'scaling': args.scaling,
                        'dtype': 'f64', 'data': 'synthetic', 'config': config,
                        'cpu_baseline': {k: r[k] for k in ('value', 'unit', 'cores', 'kind', 'sample', 'per_core')},
                        'e2e': {'value': r['value'], 'unit': 'body-steps/s',
                                'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
                print(json.dumps(line))
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.capsule_only:
        if rank == 0:
            print(json.dumps(capsule_triangles_run(args.seed, args.capsule_blocks, local, args.steps,
                                                   args.warmup, device_only=True)))
        return
    res = run_ours(args, rank, world, local)
    if rank == 0:
        ticks = sorted(res['ticks'])
        line = {
            'metric': metric, 'value': res['value'], 'unit': 'body-steps/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': res['ms'] / args.steps,
            'higher_is_better': True, 'scaling': args.scaling, 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic (seeded serving-mix scenes)', 'config': config,
            'e2e': res['e2e'], 'roofline': res['roofline'], 'clocks': res['clocks'],
            'gpu_launches': res['launches'],
            'tick_latency_ms': {'p50': float(np.percentile(ticks, 50)),
                                'p99': float(np.percentile(ticks, 99))},
            'dynamic_bodies': res['N'], 'rows': res['NB'], 'pairs': res['P'], 'contacts': res['K'],
            'tuning': res['tuning'],
        }
        ex = res['extras']
        if 'serving' in ex:
            line['serving'] = ex['serving']
        if 'plain' in ex:
            line['plain_per_world'] = ex['plain']
            line['batched_over_plain'] = res['value'] / world / ex['plain']['value']
        if not args.no_extras:
            cb = cpu_reference(args.worlds, args.seed, args.cpu_sample_s, args.preroll)
            if cb is not None:
                line['cpu_baseline'] = {k: cb[k] for k in ('value', 'unit', 'cores', 'kind', 'sample', 'per_core')}
            if args.capsule_blocks > 0:
                line['capsule_triangles'] = capsule_triangles_run(args.seed, args.capsule_blocks, local,
                                                                  args.steps, args.warmup)
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
