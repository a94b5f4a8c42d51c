"""Benchmark: body-steps/s of the omi_physics step on B200.

Default workload (N=1): the batched serving mix — 1024 independent debris
worlds, body counts log-uniform in [16, 2048], all resident in HBM and
advanced as 4 concurrently stepped groups (one context, stream and CUDA graph
per group; one "step" = every world advances one dt). Reported beside it:
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
Multi-GPU (torchrun): each rank steps its own seeded copy of the mix — worlds
are independent, so there is no collective on the data path (weak scaling);
the barrier and the max-over-ranks time use torch.distributed.
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

from omi_physics_b200.shard import barrier, max_over_ranks, sum_over_ranks  # noqa: E402

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
    ap.add_argument('--groups', type=int, default=4,
                    help='worlds are stepped as this many concurrent groups (one context + stream each)')
    return ap.parse_args()


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
    reqs, worlds = build_mix(args.worlds, args.seed + 1000 * rank)
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
        a, b = timed_steps(1)
        b.synchronize()
        ticks.append(a.elapsed_time(b))
    grp.sync()

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
    roofline = {'bound': 'hbm', 'kernel': dominant, 'achieved': round(achieved, 3), 'peak': peak,
                'unit': 'GB/s', 'frac': achieved / peak, 'traffic': traffic,
                'algorithmic_bytes': alg, 'kernel_ms': dom_ms,
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
        extras['serving'] = serving_run(n_serve, args.seed + 1000 * rank, args.serve_slots, stream)
        barrier(world)
    if not args.no_extras and rank == 0:
        extras['plain'] = plain_per_world(worlds, reqs, args.plain_sample, local, args.preroll)
    grp.close()
    return dict(value=value, ms=ms_max, N=total_N, P=P, K=K, launches=launches, setup_s=setup_s,
                ticks=ticks, roofline=roofline, e2e=e2e, clocks=clk.summary(), extras=extras,
                NB=NB)


SERVE_BUDGET = 120 * 10 ** 9


def serving_run(n_requests, seed, per_class, stream):
    """The request loop: Poisson arrivals (200/s), each world admitted into a
    free slot of its size class under the HBM budget, stepped with every other
    resident world once per tick until its 60-600 steps are done."""
    from omi_physics_b200 import scenes
    from omi_physics_b200.serving import Server, size_classes
    reqs = scenes.serving_requests(n_requests, seed=seed)
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


def main():
    args = parse()
    rank, world, local = dist_init(args.gpus)
    metric = 'body-steps/s (batched serving mix, 1 B200 per rank)'
    config = {'workload': 'serving-mix', 'worlds_per_gpu': args.worlds,
              'bodies': 'log-uniform [16,2048] per world, debris contents', 'dt': '1/120 s',
              'iterations': 8, 'l2': 'inputs larger than L2 (arena state > 126 MB)',
              'parallelism': 'world-sharded x%d (no data-path collective)' % world,
              'groups_per_gpu': args.groups}
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
                        'warmup': args.warmup, 'higher_is_better': True, 'scaling': 'weak',
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
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic (seeded serving-mix scenes)', 'config': config,
            'e2e': res['e2e'], 'roofline': res['roofline'], 'clocks': res['clocks'],
            'gpu_launches': res['launches'],
            'tick_latency_ms': {'p50': float(np.percentile(ticks, 50)),
                                'p99': float(np.percentile(ticks, 99))},
            'dynamic_bodies': res['N'], 'rows': res['NB'], 'pairs': res['P'], 'contacts': res['K'],
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
