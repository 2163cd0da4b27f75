"""Benchmark: bit-exact 4K 10-bit AV1 reconstruction on one B200.

Headline workload (`value`, `e2e`): the single-stream configuration - coded
2880x2160 10-bit 4:2:0, superres to 3840x2160, 128x128 superblocks, every tool
(64-point transforms, all transform types, CFL, palette, filter intra,
compound with wedge / difference-weighted masks, OBMC, global warp,
deblocking, CDEF, loop restoration after superres, film grain) and an NV12
output at pitch 4096. Synthetic FrameSyntax from a seed (the workload
generator, libav1synth.so); no bitstream is involved.

A step is one group of pictures: one key frame and 29 inter frames (the
configuration's key interval), each decoded into a reference slot and packed
to NV12.

  bitexact  before anything is timed, the step runs once with every frame's
            output planes and NV12 read back, and each frame's hashes are
            compared with the oracle's (tests/golden/workloads.json, made by
            the reference's CPU backend from the same seed). A mismatch
            prints "bitexact": false and exits 1.
  value     frames/s with every frame's syntax already planned and resident in
            HBM (av1b_plan_frame before the timed region), device work only:
            reconstruction, filters, reference store, grain, NV12 into device
            memory. Per-frame inputs (~40-75 MB) and pictures exceed the 126 MB
            L2 over a step, so no flush is needed between steps.
  e2e       frames/s through the public API with host buffers: every frame's
            serialized syntax is read from pinned host memory, planned,
            uploaded, decoded, and its NV12 read back to the host. The API's
            plan / decode split is used as intended: planner threads plan
            frames k + 1 .. k + 6 (av1b_plan_frame) while frame k decodes, and
            frame k - 1's NV12 (packed on the device) is read back meanwhile.
  stages    per kernel stage: ms per frame (CUDA events around every launch on
            the decoder's stream), its algorithmic bytes against the measured
            HBM bandwidth and its counted integer operations against the
            measured integer-ALU peak (av1b_int_peak), from the work counts of
            the planned frames (av1b_plan_stats); `roofline` is the dominant
            stage, bound by whichever fraction is larger.

Multi-GPU (torchrun): replicas only - each rank decodes its own stream; the
timing is the max over ranks and `value` sums all ranks' frames.

`--impl reference` times the reference's own CPU backend (oracle/_ref, built
from the reference sources) on all host cores through its public API
(decode_reference + to_nv12), on the same GOP: each timed step decodes the 30
frames, one key and 29 inter, from files a separate process wrote, so the
timing process maps only the reference's library.
"""
import argparse
import datetime
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from concurrent.futures import ThreadPoolExecutor

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'bit-exact 4K 10-bit fps (3840x2160 superres 2880->3840, all tools, NV12 pitch 4096)'
UNIT = 'frames/s'
PITCH = 4096
GOP = 30
SEED = 20261203
CONFIG = 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--scale', type=int, default=1, help='divide the picture size (tests only)')
    ap.add_argument('--frames', type=int, default=GOP, help='frames per step')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true', help='skip the end-to-end leg (profiling runs)')
    ap.add_argument('--no-verify', action='store_true', help='skip the bit-exact check (profiling runs)')
    ap.add_argument('--no-batched', action='store_true', help='skip the batched leg')
    ap.add_argument('--batch-frames', type=int, default=120, help='frames per stream, batched leg')
    ap.add_argument('--no-serve', action='store_true', help='skip the served leg')
    ap.add_argument('--only-batched', action='store_true',
                    help='the batched leg alone, without the plain comparison or autotuning '
                         '(a short run to profile the batched kernels)')
    ap.add_argument('--serve-seconds', type=float, default=1.5, help='arrival window per load point')
    return ap.parse_args()


def rank_info():
    return (int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1')),
            int(os.environ.get('LOCAL_RANK', '0')))


def slowest_rank(x, dist, device):
    """The largest of every rank's `x` (a time), the same on every rank; `x`
    itself without a process group. Every rank must call it, in the same
    order."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, world, seconds):
    """Whole-job throughput of `world` replicas that each processed
    `units_per_rank` units: all ranks' units over the slowest rank's time."""
    return units_per_rank * world / seconds


def config_dict(w, h, cw, frames, world):
    """The `config` of both arms' lines (identical for the same workload)."""
    return {'workload': 'config3: %dx%d (coded %d) 10-bit 4:2:0 superres, 128x128 SB, all tools, '
                        'film grain, NV12 pitch %d' % (w, h, cw, PITCH),
            'seed': SEED, 'frames_per_step': frames, 'gop': '1 key + %d inter' % (frames - 1),
            'l2': 'inputs larger than L2 (per-step syntax + pictures > 126 MB)',
            'parallelism': 'replicas x%d' % world}


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons every 100 ms. Started
    before the warm-up (nvidia-smi takes a moment to begin), it keeps only the
    samples whose own timestamps lie between begin() and stop(): the timed
    region (nvidia-smi's output to a pipe may arrive in bursts, so the time a
    line is read says nothing about when it was sampled)."""
    FIELDS = ('timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.t = None
        self.lines = []
        self.t0 = None

    def start(self):
        cmd = ['nvidia-smi', '-i', str(self.device), '--query-gpu=' + self.FIELDS,
               '--format=csv,noheader,nounits', '-lms', '100']
        if shutil.which('stdbuf'):
            cmd = ['stdbuf', '-oL'] + cmd   # a line at a time, not in blocks
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def begin(self):
        self.t0 = time.time()

    @staticmethod
    def sample_time(field):
        """nvidia-smi's timestamp (local time, 'YYYY/MM/DD HH:MM:SS.fff') as
        seconds since the epoch, or None."""
        try:
            return datetime.datetime.strptime(field, '%Y/%m/%d %H:%M:%S.%f').timestamp()
        except ValueError:
            return None

    def stop(self):
        t1 = time.time()
        if not self.proc:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t is not None:
            self.t.join(timeout=2)
        return self.summarize(self.lines, self.t0 if self.t0 is not None else 0.0, t1)

    @classmethod
    def summarize(cls, lines, t0, t1):
        sm, smax, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in lines:
            f = [x.strip() for x in ln.split(',')]
            if len(f) < 10:
                continue
            ts = cls.sample_time(f[0])
            if ts is None or ts < t0 or ts > t1:
                continue
            try:
                sm.append(float(f[2]))
                smax.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[6:10]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        return {'sm_mhz': statistics.median(sm) if sm else None,
                'sm_max_mhz': max(smax) if smax else None, 'reasons': sorted(reasons),
                'samples': len(sm)}


# ---- the reference arm ---------------------------------------------------------------------
def reference_frames(scale, frames, seed):
    """The GOP's frames as bytes, written by a separate process (the generator
    library is not mapped into this one), and the geometry."""
    with tempfile.TemporaryDirectory() as tmp:
        r = subprocess.run([sys.executable, '-m', 'av1ongpu_b200.workload', '--config', str(CONFIG),
                            '--scale', str(scale), '--seed', str(seed), '--frames', str(frames),
                            '--out', tmp], capture_output=True, text=True, cwd=ROOT)
        if r.returncode:
            raise RuntimeError('workload writer failed: ' + r.stderr[-500:])
        header = [int(v) for v in r.stdout.split()]
        data = []
        for k in range(frames):
            with open(os.path.join(tmp, 'frame_%04d.av1s' % k), 'rb') as f:
                data.append(f.read())
    return header, data


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import refdec
    if not refdec.available():
        print(json.dumps({'impl': 'reference', 'unavailable': 'oracle/_ref/libav1ref.so not built'}))
        return 0
    (w, cw, h, _bd, _sx, _sy), data = reference_frames(args.scale, args.frames, SEED)
    cw = cw or w
    lib = refdec.ref_lib()
    lib.av1ref_set_threads(os.cpu_count() or 1)
    cores = lib.av1ref_max_threads()
    ref = refdec.RefDecoder()

    def gop(n_frames):
        """Decodes the GOP's first n_frames frames (key frame first) with the
        reference's decode_reference + to_nv12, slots released as the stream
        advances; returns the seconds it took."""
        stream = refdec.Stream(ref)
        blobs = [refdec.RefBlob(b) for b in data[:n_frames]]
        t0 = time.perf_counter()
        for k, b in enumerate(blobs):
            slot, _ = stream.decode(k, b, read_back=True)
            ref.to_nv12(slot, PITCH, w, h)
        dt = time.perf_counter() - t0
        for s in list(stream.slots.values()):
            ref.release_reference(s)
        return dt

    # warm-up steps: the GOP's key frame and first inter frame each (the CPU
    # path's thread pool and page faults; a full GOP per warm-up step would
    # only lengthen the run)
    for _ in range(args.warmup):
        gop(min(2, args.frames))
    times = [gop(args.frames) for _ in range(args.steps)]
    fps = args.frames * len(times) / sum(times)
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': fps, 'unit': UNIT, 'n_gpus': args.gpus,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * sum(times) / len(times),
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'int32',
        'data': 'synthetic FrameSyntax (seeded generator), written by a separate process',
        'config': config_dict(w, h, cw, args.frames, 1),
        'cpu_baseline': {'value': fps, 'unit': UNIT, 'cores': cores, 'kind': 'reference',
                         'sample': 'each step the whole GOP (1 key + %d inter) of the %dx%d workload, '
                                   'decode_reference + to_nv12; warm-up steps the key frame and the '
                                   'first inter frame' % (args.frames - 1, w, h)},
        'e2e': {'value': fps, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line))
    return 0


# ---- stage rooflines ------------------------------------------------------------------------
# Counted integer operations per unit of work, one per add, subtract, shift,
# logic op, compare, min / max and multiply-add (the hardware issues a
# multiply-add as one instruction), from the stage's arithmetic (the
# reference's loops, av1gpu_kernels.h): each figure is the sum of the
# operations one unit of the stage's loop body performs. Units: `ref` a
# predicted sample per reference,
# `tx` a transform sample, `unit` a phase B sample, `coded` / `display` a
# picture sample, `nv12` a display sample.
OPS = {
    'inter': ('inter_ref', 31), 'itx': ('tx', 25), 'units': ('unit', 15),
    'deblock_v': ('coded', 10), 'deblock_h': ('coded', 10), 'cdef': ('coded', 100),
    'upscale': ('display', 12), 'lr': ('display', 50), 'grain_blend': ('display', 20),
    'nv12': ('display', 2), 'grain_template': ('grain', 30),
}
# film grain templates: 82x73 luma and two chroma templates (44x38 at 4:2:0)
GRAIN_TEMPLATE_SAMPLES = 82 * 73 + 2 * 44 * 38


def frame_counts(info, nv12_bytes):
    """Per-frame work of one planned frame, by unit (samples)."""
    w, h, cw = info['width'], info['height'], info['coded_width'] or info['width']
    coded = cw * h + 2 * ((cw + 1) // 2) * ((h + 1) // 2)
    display = w * h + 2 * ((w + 1) // 2) * ((h + 1) // 2)
    return {'coded': coded, 'display': display, 'nv12_bytes': nv12_bytes,
            'unit': info['phase_b_samples'], 'inter': info['inter_samples'],
            'inter_ref': info['inter_ref_samples'], 'tx': info['tx_samples'],
            'coef': info['coef_samples'], 'upscaled': info['upscaled'],
            'restored': info['restored'], 'grain': GRAIN_TEMPLATE_SAMPLES if info['grain'] else 0,
            'depth': info['depth']}


def stage_bytes(c, stage):
    """Algorithmic bytes of one frame's `stage` (samples are 2 bytes)."""
    return {
        'deblock_v': 4 * c['coded'], 'deblock_h': 4 * c['coded'],  # read + write each coded sample
        'cdef': 4 * c['coded'],                                    # snapshot read + picture write
        'upscale': (2 * c['coded'] + 2 * c['display']) if c['upscaled'] else 0,
        'lr': 4 * c['display'] if c['restored'] else 0,            # CDEF output read + write
        'grain_blend': 4 * c['display'] if c['grain'] else 0,      # picture read + display write
        'nv12': 2 * c['display'] + c['nv12_bytes'],                # picture read + NV12 write
        'inter': 2 * c['inter'] + 2 * c['inter_ref'],              # write + each reference read once
        'units': 6 * c['unit'],                                    # residual (4 B) + picture write
        'itx': 4 * c['coef'] + 4 * c['tx'],                        # coefficients + picture read/write
        'grain_template': 2 * c['grain'],                          # the templates written
    }.get(stage, 0)


def stage_ops(c, stage):
    unit, per = OPS.get(stage, (None, 0))
    return per * c.get(unit, 0) if unit else 0


def read_traffic():
    """DRAM traffic per launch of each stage, from the committed ncu summary."""
    path = os.path.join(ROOT, 'profiles', 'traffic.json')
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def peaks(local):
    import av1ongpu_b200 as av1b
    p = {}
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
    except (OSError, ValueError):
        pass
    hbm = p.get('hbm_gbs')
    out = {'hbm_gbs': hbm or 6650.0, 'hbm_source': 'measured (MEASURED_PEAKS.json)' if hbm else
           'fallback (6.65 TB/s, earlier measurement on this pool)'}
    out['int_add_ops'] = av1b.int_peak(local, 0)
    out['int_mad_ops'] = av1b.int_peak(local, 1)
    out['int_source'] = 'measured live (av1b_int_peak: 32-bit add rings on every SM)'
    try:
        out['handoff_ns'] = av1b.handoff_peak(local)
    except av1b.Av1bError:
        out['handoff_ns'] = None
    return out


def dependency_roof(prof, counts, pk):
    """The dependency-scheduled phase against its own floor: each launch
    walks its frame's critical path (`depth` blocks, each published on one SM
    and waited for on another), and no step can take less than one flag
    handoff between SMs (av1b_handoff_peak)."""
    ms, n = prof['units']
    steps = sum(c['depth'] for c in counts) / max(1, n)
    floor_us = pk['handoff_ns'] / 1e3 if pk.get('handoff_ns') else None
    achieved_us = ms / max(1, n) * 1e3 / max(1.0, steps)
    return {'bound': 'latency', 'steps_per_launch': round(steps, 1),
            'achieved_us_per_step': round(achieved_us, 3),
            'floor_us_per_step': round(floor_us, 3) if floor_us else None,
            'frac': round(floor_us / achieved_us, 4) if floor_us else None,
            'peak_source': 'measured live (av1b_handoff_peak: release store / acquire polls '
                           'between warps on two SMs, median of 16 SM pairs x 8 flag places)'}


def stage_report(prof, counts, frames, pk):
    """{stage: ms per frame, GB/s and fraction of HBM, int-op/s and fraction of
    the integer peak, bound} from the profiled pass and the frames' counts."""
    out = {}
    traffic = read_traffic()
    for st, (ms, n) in prof.items():
        if n <= 0 or st.endswith('_host') or st == 'copy':
            out[st] = {'ms_per_frame': round(ms / frames, 4), 'launches': n}
            continue
        b = sum(stage_bytes(c, st) for c in counts)
        ops = sum(stage_ops(c, st) for c in counts)
        sec = ms / 1e3
        gbs = b / sec / 1e9 if b else 0.0
        iops = ops / sec if ops else 0.0
        fh = gbs / pk['hbm_gbs']
        fi = iops / pk['int_add_ops']
        out[st] = {'ms_per_frame': round(ms / frames, 4), 'launches': n,
                   'bytes_per_frame': b // frames, 'ops_per_frame': ops // frames,
                   'gbs': round(gbs, 1), 'hbm_frac': round(fh, 4),
                   'int_tops': round(iops / 1e12, 3), 'int_frac': round(fi, 4),
                   'bound': 'hbm' if fh >= fi else 'int-alu',
                   'traffic_per_launch': traffic.get(st)}
    return out


# ---- our arm ------------------------------------------------------------------------------------
def verify(av1b, dec, plans, ring, geo, frames):
    """Runs the step once, untimed, reading back every frame's planes and NV12,
    and compares their hashes with the oracle's (tests/golden/workloads.json).
    Returns (ok, frames compared, first mismatch or None)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, 'tests'))
    import golden_util
    want = golden_util.load_workloads()['bench_config3']
    shapes = av1b.plane_shapes(geo['w'], geo['h'], 1, 1)
    for k, pl in enumerate(plans):
        planes = [np.empty(s, dtype=np.uint16) for s in shapes]
        dec.decode_planned(pl, slot=ring[k % 4], keep=True, wait=True, planes=planes)
        nv12 = dec.to_nv12(ring[k % 4], PITCH, geo['w'], geo['h'])
        got = [golden_util.digest(planes), golden_util.digest([nv12])]
        if got != want['frames'][k]:
            return False, k + 1, 'frame %d: %s, oracle %s' % (k, got, want['frames'][k])
    return True, frames, None


def run_only_batched(args):
    """A short batched run for profilers: plans, then every frame-set once."""
    import torch
    import av1ongpu_b200 as av1b
    local = rank_info()[2]
    torch.cuda.set_device(local)
    streams = BATCH_STREAMS
    F = args.batch_frames
    decs = [av1b.Decoder(local, planners=1, planner_threads=2) for _ in streams]
    rings = [[d.reserve_reference() for _ in range(4)] for d in decs]
    plans = plan_streams(av1b, decs, rings, streams, F, 4000)
    nv = []
    for (w, h, _bd, _r) in streams:
        pitch = (w + 63) // 64 * 64
        n = av1b.nv12_size(w, h, 1, 1, pitch)
        nv.append((torch.empty(n, dtype=torch.uint8, device='cuda:%d' % local), pitch, n))
    batch = av1b.Batch(local)
    for k in range(F):
        batch.decode(decs, [plans[i][k] for i in range(len(streams))], slots=[r[k % 4] for r in rings],
                     nv12=[(t.data_ptr(), p, n) for t, p, n in nv])
    batch.sync()
    print(json.dumps({'only_batched': True, 'frame_sets': F, 'streams': len(streams)}))
    return 0


def run_ours(args):
    import ctypes
    import torch
    import av1ongpu_b200 as av1b
    if args.only_batched:
        return run_only_batched(args)

    rank, world, local = rank_info()
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    seed = SEED + 7919 * rank
    F = args.frames

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        blobs = list(ex.map(lambda k: av1b.synth_frame(CONFIG, args.scale, seed, k), range(F)))
    w, cw, h, _bd, sx, sy = blobs[0].header
    geo = {'w': w, 'h': h, 'coded_w': cw or w, 'nv12': av1b.nv12_size(w, h, sx, sy, PITCH)}
    dec = av1b.Decoder(local)
    stream = torch.cuda.ExternalStream(dec.stream(), device=local)

    # ---- planned frames resident in HBM --------------------------------------------------------
    ring = [dec.reserve_reference() for _ in range(4)]
    plans = []
    for k, b in enumerate(blobs):
        dists = b.get_refs()
        b.set_refs([ring[(k - d) % 4] for d in dists])
        plans.append(dec.plan(b))
        b.set_refs(dists)
    counts = [frame_counts(dec.plan_stats(pl), geo['nv12']) for pl in plans]

    # ---- bit exactness of the frames the step times ----------------------------------------
    bitexact, checked, mismatch = None, 0, None
    exact_workload = args.scale == 1 and F == GOP and seed == SEED
    if not args.no_verify and exact_workload:
        bitexact, checked, mismatch = verify(av1b, dec, plans, ring, geo, F)
        if not bitexact and rank == 0:
            print(json.dumps({'metric': METRIC, 'bitexact': False, 'mismatch': mismatch}))
            return 1

    nv12_dev = torch.empty(geo['nv12'], dtype=torch.uint8, device='cuda:%d' % local)

    def device_step(launch_counts=None):
        for k, pl in enumerate(plans):
            s = ring[k % 4]
            dec.decode_planned(pl, slot=s, keep=True, wait=False)
            if launch_counts is not None:
                # the frame's kernels (the decoder counts each launch) and the NV12 pack
                launch_counts.append(dec.stats().kernel_launches + 1)
            dec.to_nv12_device(s, PITCH, nv12_dev.data_ptr(), geo['nv12'])

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        device_step()
    dec.sync()

    def barrier():
        if dist is not None:
            dist.barrier()

    barrier()
    torch.cuda.synchronize()
    clocks.begin()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        device_step()
    e1.record(stream)
    dec.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = slowest_rank(e0.elapsed_time(e1), dist, 'cuda:%d' % local)
    barrier()
    value = replica_rate(F * args.steps, world, ms / 1e3)

    # ---- per-stage device times (a separate profiled pass over the same step) ----------
    dec.set_profiling(True)
    step_launches = []
    device_step(step_launches)
    dec.sync()
    prof = dec.profile()
    dec.set_profiling(False)
    pk = peaks(local)
    stages = stage_report(prof, counts, F, pk)
    # the dominant stage: the most device time per frame (the grain templates
    # included, although they overlap reconstruction on a side stream)
    timed = {k: v for k, v in stages.items() if 'bound' in v}
    dom = max(timed, key=lambda k: timed[k]['ms_per_frame']) if timed else None
    roofline = None
    if dom:
        s = timed[dom]
        avg_ms = prof[dom][0] / prof[dom][1]
        per_launch_bytes = s['bytes_per_frame'] * F / prof[dom][1]
        per_launch_ops = s['ops_per_frame'] * F / prof[dom][1]
        hbm = {'achieved': s['gbs'], 'peak': pk['hbm_gbs'], 'unit': 'GB/s', 'frac': s['hbm_frac'],
               'peak_source': pk['hbm_source'], 'algorithmic_bytes_per_launch': per_launch_bytes}
        alu = {'achieved': s['int_tops'], 'peak': round(pk['int_add_ops'] / 1e12, 3),
               'unit': 'T int-op/s', 'frac': s['int_frac'], 'peak_source': pk['int_source'],
               'counted_ops_per_launch': per_launch_ops}
        main = hbm if s['bound'] == 'hbm' else alu
        roofline = {'bound': s['bound'], 'kernel': dom, 'achieved': main['achieved'],
                    'peak': main['peak'], 'unit': main['unit'], 'frac': main['frac'],
                    'traffic': s['traffic_per_launch'], 'avg_launch_ms': avg_ms,
                    'hbm': hbm, 'int_alu': alu,
                    'note': 'frac of measured peaks; traffic = ncu dram bytes per launch '
                            '(profiles/traffic.json)'}
        if dom == 'units':
            roofline['dependency'] = dependency_roof(prof, counts, pk)

    # ---- e2e: public API with host buffers ------------------------------------------------
    pinned = []
    for b in blobs:
        t = torch.empty(b.size + 64, dtype=torch.uint8, pin_memory=True)
        off = (-t.data_ptr()) % 64
        ctypes.memmove(t.data_ptr() + off, b.ptr, b.size)
        pb = av1b.Blob(t.data_ptr() + off, b.size, False)
        pb._keep = t
        pinned.append(pb)
    h2d = sum(b.size for b in pinned)
    e2e_dec = av1b.Decoder(local)
    e2e_ring = [e2e_dec.reserve_reference() for _ in range(4)]

    def e2e_run(steps):
        """`steps` steps through the public plan / decode API, pipelined the way
        the API is meant for and the way a stream runs, without a drain between
        steps: three planner threads plan frames k + 1 .. k + 6 (validation,
        records, upload from the pinned host blob) while the device decodes
        frame k; its NV12 goes out through the split pack (av1b_nv12_pack_begin
        / wait / release: packed on the device, read back into the library's
        page-locked memory on its copy stream while frame k + 1 decodes).
        Frames decode in order; the host holds frame k - 1's NV12 once frame k
        is queued. Step s decodes the GOP's frames again as frames
        s * F .. s * F + F - 1 of the stream."""
        ahead = 6
        n = steps * len(pinned)

        def plan(k):
            b = pinned[k % len(pinned)]
            dists = b.get_refs()
            b.set_refs([e2e_ring[(k - d) % 4] for d in dists])
            view = ctypes.create_string_buffer(4096)
            av1b.lib().av1b_syntax_view(b.ptr, b.size, view)
            hh = ctypes.c_void_p()
            rc = av1b.lib().av1b_plan_frame(e2e_dec.h, view, ctypes.byref(hh))
            b.set_refs(dists)
            if rc:
                raise av1b.Av1bError(rc, 'plan_frame')
            return hh

        packs = []
        with ThreadPoolExecutor(max_workers=3) as ex:
            futs = {k: ex.submit(plan, k) for k in range(min(ahead, n))}
            for k in range(n):
                hh = futs.pop(k).result()
                if k + ahead < n:
                    futs[k + ahead] = ex.submit(plan, k + ahead)
                got = ctypes.c_int(-1)
                rc = av1b.lib().av1b_decode_planned(e2e_dec.h, hh, e2e_ring[k % 4], 1, None,
                                                     ctypes.byref(got), 0)
                if rc:
                    raise av1b.Av1bError(rc, 'decode_planned')
                av1b.lib().av1b_plan_free(e2e_dec.h, hh)
                packs.append(e2e_dec.nv12_pack_begin(e2e_ring[k % 4], PITCH))
                if len(packs) > 1:
                    hd = packs.pop(0)
                    e2e_dec.nv12_pack_wait(hd)  # frame k - 1's NV12 is on the host
                    e2e_dec.nv12_pack_release(hd)
            e2e_dec.sync()
            for hd in packs:
                e2e_dec.nv12_pack_wait(hd)
                e2e_dec.nv12_pack_release(hd)

    e2e_s = float('inf')
    # the timed stream starts cold (its key frame's plan before the first
    # decode) and runs at least the workload's 120 frames (4 GOPs)
    e2e_steps = max(args.steps, 4)
    if not args.no_e2e:
        e2e_run(args.warmup)  # the planners' lists and plans reach their sizes
        barrier()
        t0 = time.perf_counter()
        e2e_run(e2e_steps)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
    e2e_s = slowest_rank(e2e_s, dist, 'cuda:%d' % local)
    e2e = {'value': replica_rate(F * e2e_steps, world, e2e_s), 'unit': UNIT, 'h2d_bytes_per_step': h2d,
           'd2h_bytes_per_step': geo['nv12'] * F, 'frames_timed': F * e2e_steps}

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(blobs, geo)
    batched = None
    if not args.no_batched:
        batched = run_batched_leg(args, av1b, torch, local)
    serving = None
    if not args.no_serve and world == 1:
        serving = run_serving_leg(args, av1b, local)

    for pl in plans:
        dec.free_plan(pl)
    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'int32',
            'data': 'synthetic FrameSyntax (seeded generator), device-resident plans',
            'config': config_dict(geo['w'], geo['h'], geo['coded_w'], F, world),
            'bitexact': bitexact, 'bitexact_frames': checked,
            'bitexact_ref': 'per-frame hashes of the output planes and NV12 against the oracle '
                            '(tests/golden/workloads.json)' if bitexact is not None else
                            'not checked (not the exact workload, or --no-verify)',
            'e2e': e2e, 'roofline': roofline, 'cpu_baseline': base,
            'clocks': clk, 'gpu_launches': sum(step_launches) * args.steps,
            'peaks': {k: v for k, v in pk.items()},
            'stages': stages,
            'batched': batched,
            'serving': serving,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---- batched form (config 4) ---------------------------------------------------------------
# 16 streams: (width, height, bit depth, reference slots an inter frame draws from)
BATCH_STREAMS = ([(640, 360, 8, 2)] * 4 + [(1280, 720, 8, 2)] * 6 + [(1920, 1080, 10, 3)] * 4 +
                 [(3840, 2160, 10, 3)] * 2)
BATCH_KEY = 60


def plan_streams(av1b, decs, rings, streams, frames, seed0):
    """Every stream's frames planned into device memory (generated and
    planned on all host cores; a frame's blob is dropped once planned)."""
    plans = [[None] * frames for _ in streams]

    def one(job):
        i, k = job
        w, h, bd, refs = streams[i]
        b = av1b.synth_frame_ex(w, h, 0, bd, 64, av1b.TOOLS_ALL, seed0 + 1000 * i, k, BATCH_KEY,
                                max_refs=refs)
        d = b.get_refs()
        b.set_refs([rings[i][(k - x) % 4] for x in d])
        plans[i][k] = decs[i].plan(b)

    jobs = [(i, k) for k in range(frames) for i in range(len(streams))]
    with ThreadPoolExecutor(max_workers=max(2, (os.cpu_count() or 2) // 2)) as ex:
        list(ex.map(one, jobs))
    return plans


def run_batched_leg(args, av1b, torch, local):
    """Aggregate megapixels/s of the 16 mixed streams: one at a time through
    the plain path, and together through the batched form (autotuned, one
    CUDA graph replay a frame-set), device-resident plans in both."""
    streams = BATCH_STREAMS
    F = args.batch_frames
    decs = [av1b.Decoder(local, planners=1, planner_threads=2) for _ in streams]
    rings = [[d.reserve_reference() for _ in range(4)] for d in decs]
    t0 = time.perf_counter()
    plans = plan_streams(av1b, decs, rings, streams, F, 4000)
    plan_s = time.perf_counter() - t0
    nv = []
    for (w, h, bd, _r) in streams:
        pitch = (w + 63) // 64 * 64
        n = av1b.nv12_size(w, h, 1, 1, pitch)
        nv.append((torch.empty(n, dtype=torch.uint8, device='cuda:%d' % local), pitch, n))
    mpx = sum(w * h for (w, h, _b, _r) in streams) * F / 1e6

    def plain(frames):
        for i, d in enumerate(decs):
            for k in frames:
                s = rings[i][k % 4]
                d.decode_planned(plans[i][k], slot=s, keep=True, wait=False)
                d.to_nv12_device(s, nv[i][1], nv[i][0].data_ptr(), nv[i][2])
            d.sync()

    batch = av1b.Batch(local)
    bstream = torch.cuda.ExternalStream(batch.stream(), device=local)

    def batched(frames):
        for k in frames:
            batch.decode(decs, [plans[i][k] for i in range(len(streams))],
                         slots=[r[k % 4] for r in rings],
                         nv12=[(t.data_ptr(), p, n) for t, p, n in nv])
        batch.sync()

    # bit exactness: the first two frame-sets (key frames, then inter frames)
    # batched against plain, every stream's NV12 byte for byte
    exact = True
    for k in range(min(2, F)):
        plain([k])
        want = [t.clone() for t, _p, _n in nv]
        for t, _p, _n in nv:
            t.zero_()
        batched([k])
        exact = exact and all(torch.equal(a, t) for a, (t, _p, _n) in zip(want, nv))
    # the autotuner, on the inter frame-set 1 (its references are frame 0's)
    tuned, tune_ms = None, None
    default_ms = None
    if F >= 2:
        cache = os.environ.get('AV1B_TUNE_CACHE') or os.path.join(tempfile.gettempdir(),
                                                                 'av1b_batch_tuning.txt')
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(bstream)
        for _ in range(3):
            batched([1])
        e1.record(bstream)
        torch.cuda.synchronize()
        default_ms = e0.elapsed_time(e1) / 3
        tuned, tune_ms = batch.autotune(decs, [plans[i][1] for i in range(len(streams))],
                                        slots=[r[1] for r in rings],
                                        nv12=[(t.data_ptr(), p, n) for t, p, n in nv],
                                        cache_path=cache, reps=3)
    frames = list(range(F))
    plain(frames[:2])  # warm-up
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in decs]
    torch.cuda.synchronize()
    for i, d in enumerate(decs):
        st = torch.cuda.ExternalStream(d.stream(), device=local)
        ev[i][0].record(st)
        for k in frames:
            s = rings[i][k % 4]
            d.decode_planned(plans[i][k], slot=s, keep=True, wait=False)
            d.to_nv12_device(s, nv[i][1], nv[i][0].data_ptr(), nv[i][2])
        ev[i][1].record(st)
        d.sync()
    plain_ms = sum(a.elapsed_time(b) for a, b in ev)
    batched(frames[:2])  # warm-up (graph captured)
    b0 = torch.cuda.Event(enable_timing=True)
    b1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    b0.record(bstream)
    batched(frames)
    b1.record(bstream)
    torch.cuda.synchronize()
    batch_ms = b0.elapsed_time(b1)
    # per-stage device time of the batched step (ungraphed, events between
    # stages): the key frame-set alone, then the inter frame-sets
    stage_ms = {}
    for name, fr in (('key', frames[:1]), ('inter', frames[1:min(F, 31)])):
        if not fr:
            continue
        batch.set_profiling(True)
        batched(fr)
        prof, n = batch.profile()
        batch.set_profiling(False)
        stage_ms[name] = {k: round(v / max(1, n), 4) for k, v in prof.items() if v > 0}
        stage_ms[name]['frame_sets'] = n
    for i, d in enumerate(decs):
        for pl in plans[i]:
            d.free_plan(pl)
        d.close()
    batch.close()
    return {
        'metric': 'batched Mpx/s vs plain path (16 mixed streams)', 'unit': 'Mpx/s',
        'value': mpx / (batch_ms / 1e3), 'plain_value': mpx / (plain_ms / 1e3),
        'speedup': plain_ms / batch_ms, 'bitexact_vs_plain': exact,
        'bitexact_frames': '%d streams x %d frame-sets' % (len(streams), min(2, F)),
        'frames_per_stream': F, 'key_interval': BATCH_KEY, 'mpx': mpx,
        'batched_ms': batch_ms, 'plain_ms': plain_ms,
        'ms_per_frame_set': batch_ms / F, 'plain_ms_per_frame_set': plain_ms / F,
        'streams': '4x 640x360 8-bit, 6x 1280x720 8-bit, 4x 1920x1080 10-bit, 2x 3840x2160 10-bit; '
                   'all tools, 64x64 SB, 2 (8-bit) / 3 (10-bit) reference slots, NV12 out',
        'plan_s': plan_s, 'autotune': {'config': tuned, 'best_step_ms': tune_ms,
                                       'default_step_ms': default_ms},
        'stage_ms_per_frame_set': stage_ms,
        'timing': 'device (CUDA events): plain = sum over streams decoded one at a time, each on '
                  'its decoder stream; batched = one graph replay a frame-set on the batch stream',
    }


# ---- served form (config 5) -----------------------------------------------------------------
# 64 streams: (width, height, bit depth, reference slots), how many
SERVE_CLASSES = [((640, 360, 8, 2), 19), ((1280, 720, 8, 2), 22), ((1920, 1080, 10, 3), 16),
                 ((3840, 2160, 10, 3), 7)]
SERVE_GOP = 30          # each stream cycles through a 30-frame group (key frame first)
SERVE_LOADS = (0.25, 0.5, 0.75, 1.0, 1.2)


def percentile(v, q):
    if not v:
        return None
    v = sorted(v)
    return v[min(len(v) - 1, int(round(q / 100.0 * (len(v) - 1))))]


def run_serving_leg(args, av1b, local):
    """The request loop over 64 streams: Poisson arrivals at 30 or 60 frames/s
    a stream, scaled so that the offered load sweeps 25 %..120 % of the
    served capacity (a saturation run first); p50 / p99 of each frame's
    latency (arrival to device completion) and the delivered Mpx/s."""
    import random
    streams = []
    for (geo, count) in SERVE_CLASSES:
        streams += [geo] * count
    classes = sorted(set(streams))
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        pools = {}
        for c, (w, h, bd, refs) in enumerate(classes):
            pools[(w, h, bd, refs)] = list(ex.map(
                lambda k: av1b.synth_frame_ex(w, h, 0, bd, 64, av1b.TOOLS_ALL, 5000 + c, k, SERVE_GOP,
                                              max_refs=refs), range(SERVE_GOP)))
    # the requests in page-locked memory, as a server receives them: a plan's
    # upload of the frame's coefficients then runs at the copy engines' rate
    import ctypes
    import torch
    for key, blobs in pools.items():
        pinned = []
        for b in blobs:
            t = torch.empty(b.size + 64, dtype=torch.uint8, pin_memory=True)
            off = (-t.data_ptr()) % 64
            ctypes.memmove(t.data_ptr() + off, b.ptr, b.size)
            pb = av1b.Blob(t.data_ptr() + off, b.size, False)
            pb._keep = t
            pinned.append(pb)
        pools[key] = pinned
    srv = av1b.Server(local, max_inflight=2, planner_threads=max(2, (os.cpu_count() or 4) // 2))
    sids = []
    for (w, h, bd, refs) in streams:
        sid, _ = srv.open(w, h, bd, max_refs=refs, nv12_pitch=(w + 63) // 64 * 64)
        sids.append(sid)
    fps = [30 if j % 2 == 0 else 60 for j in range(len(streams))]
    px = [w * h for (w, h, _b, _r) in streams]
    natural = sum(f * p for f, p in zip(fps, px)) / 1e6
    index = [0] * len(streams)
    cls_name = {(640, 360, 8, 2): '360p', (1280, 720, 8, 2): '720p', (1920, 1080, 10, 3): '1080p',
                (3840, 2160, 10, 3): '2160p'}

    def run(events):
        """Submits (time s, stream) events at their times; returns the results."""
        out = []
        tags = {}
        t0 = time.perf_counter()
        for t, j in events:
            while True:
                dt = t0 + t - time.perf_counter()
                if dt <= 0:
                    break
                time.sleep(dt if dt > 0.0005 else 0)
            k = index[j]
            index[j] += 1
            tag = len(tags)
            tags[tag] = j
            srv.submit(sids[j], pools[streams[j]][k % SERVE_GOP], tag=tag)
            if tag % 64 == 0:
                out += srv.poll(4096)
        srv.drain(120000)
        out += srv.poll(1 << 16)
        while True:
            more = srv.poll(1 << 16)
            if not more:
                break
            out += more
        return out, tags

    def summarize(res, tags, offered):
        lat = [r.latency_ms for r in res if r.status == 0]
        first = min(r.arrival_ms for r in res)
        last = max(r.done_ms for r in res)
        mpx = sum(px[tags[r.tag]] for r in res if r.status == 0) / 1e6
        by = {}
        plan_wait = {}
        for r in res:
            c = cls_name[streams[tags[r.tag]]]
            by.setdefault(c, []).append(r.latency_ms)
            plan_wait.setdefault(c, []).append(r.planned_ms - r.arrival_ms)
        return {'offered_mpx_s': offered, 'delivered_mpx_s': mpx / ((last - first) / 1e3),
                'frames': len(res), 'failed': sum(1 for r in res if r.status != 0),
                'p50_ms': percentile(lat, 50), 'p99_ms': percentile(lat, 99),
                'arrival_to_planned_p50_ms': {c: percentile(v, 50) for c, v in sorted(plan_wait.items())},
                'mean_batch': sum(r.batch_size for r in res) / max(1, len(res)),
                'by_class': {c: {'p50_ms': percentile(v, 50), 'p99_ms': percentile(v, 99),
                                 'frames': len(v)} for c, v in sorted(by.items())}}

    # bring every stream to steady state: its key frame, and enough frames at
    # once that its decoder's plan pool and buffers reach their sizes
    run([(0.0, j) for _ in range(8) for j in range(len(streams))])
    # capacity: every stream's next 30 frames at once, as fast as they can go
    burst = [(0.0, j) for _ in range(SERVE_GOP) for j in range(len(streams))]
    res, tags = run(burst)
    cap = summarize(res, tags, None)
    capacity = cap['delivered_mpx_s']
    sweep = []
    rng = random.Random(11)
    duration = args.serve_seconds
    for load in SERVE_LOADS:
        alpha = load * capacity / natural
        events = []
        for j in range(len(streams)):
            t = rng.expovariate(alpha * fps[j])
            while t < duration:
                events.append((t, j))
                t += rng.expovariate(alpha * fps[j])
        events.sort()
        res, tags = run(events)
        row = summarize(res, tags, load * capacity)
        row['load'] = load
        sweep.append(row)
    st = srv.stats()
    srv.close()
    at100 = [r for r in sweep if r['load'] == 1.0]
    host = {'plan_ms_per_frame': st.plan_ms / max(1, st.completed),
            'launch_ms_per_step': st.launch_ms / max(1, st.steps),
            'frames_per_step': st.stepped_frames / max(1, st.steps)}
    return {
        'metric': 'p50/p99 frame ms and delivered Mpx/s (64 streams, Poisson arrivals)',
        'streams': '19x 640x360 8-bit, 22x 1280x720 8-bit, 16x 1920x1080 10-bit, 7x 3840x2160 10-bit; '
                   'all tools, key frame every %d, half at 30 and half at 60 frames/s, NV12 out'
                   % SERVE_GOP,
        'latency': 'arrival (submit) to the device completion of the frame\'s step, host clock; '
                   'host planning included',
        'capacity_mpx_s': capacity, 'capacity_run': cap, 'natural_load_mpx_s': natural,
        'seconds_per_load': duration, 'sweep': sweep,
        'p99_1080p_ms_at_100': at100[0]['by_class'].get('1080p', {}).get('p99_ms') if at100 else None,
        'steps': st.steps, 'frames': st.completed, 'hbm_reserved_gb': st.hbm_used / 1e9,
        'host': host,
    }


def cpu_baseline(blobs, geo, frames=3):
    """The reference CPU backend on the first `frames` frames of the workload
    (the key frame and two inter frames), all host threads, through its public
    API (decode_reference + to_nv12)."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import refdec
    if not refdec.available():
        return None
    lib = refdec.ref_lib()
    lib.av1ref_set_threads(os.cpu_count() or 1)
    ref = refdec.RefDecoder()
    stream = refdec.Stream(ref)
    own = [refdec.RefBlob(b.to_bytes()) for b in blobs[:frames]]
    t0 = time.perf_counter()
    for k, b in enumerate(own):
        slot, _ = stream.decode(k, b, read_back=True)
        ref.to_nv12(slot, PITCH, geo['w'], geo['h'])
    dt = time.perf_counter() - t0
    return {'value': frames / dt, 'unit': UNIT, 'cores': lib.av1ref_max_threads(),
            'kind': 'reference',
            'sample': '%d frames (1 key + %d inter) of the %dx%d workload, decode_reference + '
                      'to_nv12, %.1f s' % (frames, frames - 1, geo['w'], geo['h'], dt)}


def main():
    args = parse()
    if args.impl == 'reference':
        return run_reference(args)
    return run_ours(args)


if __name__ == '__main__':
    sys.exit(main())
