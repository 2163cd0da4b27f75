"""Benchmark: bit-exact 4K 10-bit AV1 reconstruction fps on B200.

Workload: the headline single-stream configuration - coded 2880x2160 10-bit
4:2:0, superres to 3840x2160, 128x128 superblocks, every tool (64-point
transforms, all transform types, CFL, palette, filter intra, compound with
wedge / difference-weighted masks, OBMC, global warp, deblocking, CDEF, loop
restoration after superres, film grain) and an NV12 output at pitch 4096.
Synthetic FrameSyntax from a seed (the workload generator in
av1ongpu_b200/csrc/synth.cpp); no bitstream is involved.

A step is one group of pictures: one key frame and 29 inter frames (the
configuration's key interval), each decoded into a reference slot and packed
to NV12.

  value   frames/s with every frame's syntax already planned and resident in
          HBM (av1b_plan_frame before the timed region), device work only:
          reconstruction, filters, reference store, grain, NV12 into device
          memory. Per-frame inputs (~40-75 MB) and pictures exceed the 126 MB
          L2 over a step, so no flush is needed between steps.
  e2e     frames/s through the public API with host buffers: every frame's
          serialized syntax is read from pinned host memory, planned,
          uploaded, decoded, and its NV12 read back to the host. The API's
          plan / decode split is used as intended: two threads plan frames
          k + 1 .. k + 3 (av1b_plan_frame) while frame k decodes, and frame
          k - 1's NV12 (packed on the device) is read back meanwhile.

Multi-GPU (torchrun): replicas only - each rank decodes its own stream; the
timing is the max over ranks and `value` sums all ranks' frames.

`--impl reference` times the reference's own CPU backend (oracle/_ref, built
from the reference sources) on the host cores, one frame per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
from concurrent.futures import ThreadPoolExecutor
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'bit-exact 4K 10-bit fps (3840x2160 superres 2880->3840, all tools, NV12 pitch 4096)'
UNIT = 'frames/s'
PITCH = 4096
GOP = 30
SEED = 20261203


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=2)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--scale', type=int, default=1, help='divide the picture size (tests only)')
    ap.add_argument('--frames', type=int, default=GOP, help='frames per step')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true', help='skip the end-to-end leg (profiling runs)')
    return ap.parse_args()


def rank_info():
    return (int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1')),
            int(os.environ.get('LOCAL_RANK', '0')))


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.device), '--query-gpu=' + self.FIELDS,
                 '--format=csv,noheader,nounits', '-lms', '200'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            f = [x.strip() for x in ln.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        return {'sm_mhz': statistics.median(sm) if sm else None,
                'sm_max_mhz': max(smax) if smax else None, 'reasons': sorted(reasons),
                'samples': len(sm)}


def workload_blobs(av1b, scale, frames, seed):
    return [av1b.synth_frame(3, scale, seed, k) for k in range(frames)]


def stage_bytes(L, stage):
    """Algorithmic bytes one launch of `stage` moves for a frame of geometry L
    (a dict: coded / display sample counts, NV12 bytes). Samples are 2 bytes."""
    nc, nd, nv12 = L['coded'], L['display'], L['nv12']
    return {
        'deblock_v': 4 * nc, 'deblock_h': 4 * nc,       # read + write every coded sample
        'cdef': 4 * nc,                                  # snapshot read + picture write
        'upscale': 2 * nc + 2 * nd,                      # coded read, display write
        'lr': 4 * nd,                                    # CDEF snapshot read + write
        'grain_blend': 4 * nd,                           # picture read + display write
        'nv12': 2 * nd + nv12,                           # picture read + NV12 write
        'inter': 2 * nc + 4 * nd,                        # write + two references read once
        'units': 6 * nc,                                 # residual read (4 B) + picture write
        'itx': 4 * nc + 4 * nc,                          # coefficients (4 B) + picture read/write
    }.get(stage)


def geometry(av1b, blob):
    w, cw, h, bd, sx, sy = blob.header
    cw = cw if cw > 0 else w
    c = cw * h + 2 * ((cw + 1) // 2) * ((h + 1) // 2)
    d = w * h + 2 * ((w + 1) // 2) * ((h + 1) // 2)
    return {'w': w, 'h': h, 'coded_w': cw, 'coded': c, 'display': d,
            'nv12': av1b.nv12_size(w, h, sx, sy, PITCH)}


def read_traffic():
    """traffic per launch of the dominant kernel, from the committed ncu summary."""
    path = os.path.join(ROOT, 'profiles', 'traffic.json')
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def cpu_baseline(av1b, scale, seed, frames=3):
    """The reference CPU backend on the first `frames` frames of the workload,
    all host threads, through its public API (decode_reference + to_nv12)."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import refdec
    if not refdec.available():
        return None
    lib = refdec.ref_lib()
    lib.av1ref_set_threads(os.cpu_count() or 1)
    ref = refdec.RefDecoder()
    stream = refdec.Stream(ref)
    blobs = workload_blobs(av1b, scale, frames, seed)
    geo = geometry(av1b, blobs[0])
    t0 = time.perf_counter()
    for k, b in enumerate(blobs):
        slot, _ = stream.decode(k, b, read_back=True)
        ref.to_nv12(slot, PITCH, geo['w'], geo['h'])
    dt = time.perf_counter() - t0
    return {'value': frames / dt, 'unit': UNIT, 'cores': lib.av1ref_max_threads(),
            'kind': 'reference',
            'sample': '%d frames (1 key + %d inter) of the %dx%d workload, decode_reference + '
                      'to_nv12, %.1f s' % (frames, frames - 1, geo['w'], geo['h'], dt)}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return 0
    import av1ongpu_b200 as av1b
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import refdec
    if not refdec.available():
        print(json.dumps({'impl': 'reference', 'unavailable': 'oracle/_ref/libav1ref.so not built'}))
        return 0
    lib = refdec.ref_lib()
    lib.av1ref_set_threads(os.cpu_count() or 1)
    cores = lib.av1ref_max_threads()
    ref = refdec.RefDecoder()
    stream = refdec.Stream(ref)
    n = args.warmup + args.steps
    blobs = workload_blobs(av1b, args.scale, n, SEED)
    geo = geometry(av1b, blobs[0])
    times = []
    for k, b in enumerate(blobs):
        t0 = time.perf_counter()
        slot, _ = stream.decode(k, b, read_back=True)
        ref.to_nv12(slot, PITCH, geo['w'], geo['h'])
        times.append(time.perf_counter() - t0)
    timed = times[args.warmup:]
    fps = len(timed) / sum(timed)
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': fps, 'unit': UNIT, 'n_gpus': args.gpus,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * sum(timed) / len(timed),
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'int32',
        'data': 'synthetic FrameSyntax (seeded)',
        'config': {'workload': 'config3: %dx%d (coded %d) 10-bit 4:2:0 superres, 128x128 SB, all '
                               'tools, NV12 pitch %d' % (geo['w'], geo['h'], geo['coded_w'], PITCH),
                   'step': 'one frame (bounded CPU sample)', 'frames_per_step': 1},
        'cpu_baseline': {'value': fps, 'unit': UNIT, 'cores': cores, 'kind': 'reference',
                         'sample': 'frames %d..%d of the workload, one per step' % (args.warmup, n - 1)},
        'e2e': {'value': fps, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    import ctypes
    import numpy as np
    import torch
    import av1ongpu_b200 as av1b

    rank, world, local = rank_info()
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    seed = SEED + 7919 * rank
    F = args.frames

    blobs = workload_blobs(av1b, args.scale, F, seed)
    geo = geometry(av1b, blobs[0])
    dec = av1b.Decoder(local)
    stream = torch.cuda.ExternalStream(dec.stream(), device=local)

    # ---- value: planned frames resident in HBM ---------------------------------------------
    ring = [dec.reserve_reference() for _ in range(4)]
    plans = []
    for k, b in enumerate(blobs):
        dists = b.get_refs()
        b.set_refs([ring[(k - d) % 4] for d in dists])
        plans.append(dec.plan(b))
        b.set_refs(dists)
    nv12_dev = torch.empty(geo['nv12'], dtype=torch.uint8, device='cuda:%d' % local)

    def device_step():
        for k, pl in enumerate(plans):
            s = ring[k % 4]
            dec.decode_planned(pl, slot=s, keep=True, wait=False)
            dec.to_nv12_device(s, PITCH, nv12_dev.data_ptr(), geo['nv12'])

    for _ in range(args.warmup):
        device_step()
    dec.sync()

    def barrier():
        if dist is not None:
            dist.barrier()

    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        device_step()
    e1.record(stream)
    dec.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms], device='cuda:%d' % local)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        barrier()
    frames_total = F * args.steps * world
    value = frames_total / (ms / 1e3)
    launches_per_frame = dec.stats().kernel_launches + 1  # + the NV12 pack

    # ---- per-stage device times (a separate profiled pass over the same step) ----------
    dec.set_profiling(True)
    device_step()
    dec.sync()
    prof = dec.profile()
    dec.set_profiling(False)
    # the dominant kernel on the frame's critical path: the grain templates
    # run on a side stream, overlapped with reconstruction
    kernels = {k: v for k, v in prof.items()
               if k not in ('copy', 'grain_template') and not k.endswith('_host') and v[1] > 0}
    dom = max(kernels, key=lambda k: kernels[k][0]) if kernels else None
    peaks = {}
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get('hbm_gbs')
    peak_note = 'measured' if hbm_peak else 'fallback'
    hbm_peak = hbm_peak or 6650.0
    roofline = None
    if dom:
        avg_ms = kernels[dom][0] / kernels[dom][1]
        bytes_per_launch = stage_bytes(geo, dom)
        achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9 if bytes_per_launch else None
        tr = read_traffic().get(dom)
        roofline = {'bound': 'hbm', 'kernel': dom, 'achieved': achieved, 'peak': hbm_peak,
                    'peak_source': peak_note, 'unit': 'GB/s',
                    'frac': achieved / hbm_peak if achieved else None,
                    'traffic': tr, 'algorithmic_bytes_per_launch': bytes_per_launch,
                    'avg_launch_ms': avg_ms}
    stage_ms = {k: round(v[0] / F, 4) for k, v in prof.items() if v[1] > 0}

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
            h = ctypes.c_void_p()
            rc = av1b.lib().av1b_plan_frame(e2e_dec.h, view, ctypes.byref(h))
            b.set_refs(dists)
            if rc:
                raise av1b.Av1bError(rc, 'plan_frame')
            return h

        packs = []
        with ThreadPoolExecutor(max_workers=3) as ex:
            futs = {k: ex.submit(plan, k) for k in range(min(ahead, n))}
            for k in range(n):
                h = futs.pop(k).result()
                if k + ahead < n:
                    futs[k + ahead] = ex.submit(plan, k + ahead)
                got = ctypes.c_int(-1)
                rc = av1b.lib().av1b_decode_planned(e2e_dec.h, h, e2e_ring[k % 4], 1, None,
                                                     ctypes.byref(got), 0)
                if rc:
                    raise av1b.Av1bError(rc, 'decode_planned')
                av1b.lib().av1b_plan_free(e2e_dec.h, h)
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
    if dist is not None:
        t = torch.tensor([e2e_s], device='cuda:%d' % local)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {'value': F * e2e_steps * world / e2e_s, 'unit': UNIT, 'h2d_bytes_per_step': h2d,
           'd2h_bytes_per_step': geo['nv12'] * F, 'frames_timed': F * e2e_steps}

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(av1b, args.scale, SEED)

    for pl in plans:
        dec.free_plan(pl)
    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'int32',
            'data': 'synthetic FrameSyntax (seeded generator), device-resident plans',
            'config': {'workload': 'config3: %dx%d (coded %d) 10-bit 4:2:0 superres, 128x128 SB, '
                                   'all tools, film grain, NV12 pitch %d' %
                                   (geo['w'], geo['h'], geo['coded_w'], PITCH),
                       'frames_per_step': F, 'gop': '1 key + %d inter' % (F - 1),
                       'l2': 'inputs larger than L2 (per-step syntax + pictures > 126 MB)',
                       'parallelism': 'replicas x%d' % world},
            'e2e': e2e, 'roofline': roofline, 'cpu_baseline': base,
            'clocks': clk, 'gpu_launches': launches_per_frame * F * args.steps,
            'stage_ms_per_frame': stage_ms,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == 'reference':
        return run_reference(args)
    return run_ours(args)


if __name__ == '__main__':
    sys.exit(main())
