"""bench.py's reference arm on the CPU: it times the reference's CPU backend
on the same GOP and configuration as the GPU arm, and its process maps the
reference's library only - the workload is written by a separate process, so
neither this repository's decoder nor its generator is loaded."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r'''
import sys
sys.argv = ['bench.py', '--impl', 'reference', '--scale', '8', '--frames', '3', '--steps', '1',
            '--warmup', '1']
import bench
bench.main()
maps = open('/proc/self/maps').read()
print('MAPS', 'libav1b.so' in maps, 'libav1synth.so' in maps, 'libav1ref.so' in maps)
'''


def test_reference_arm_maps_only_the_oracle(oracle):
    r = subprocess.run([sys.executable, '-c', PROBE], capture_output=True, text=True, cwd=ROOT,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert line['impl'] == 'reference' and line['value'] > 0
    assert line['config']['gop'] == '1 key + 2 inter' and line['config']['frames_per_step'] == 3
    assert line['cpu_baseline']['kind'] == 'reference'
    assert line['e2e']['h2d_bytes_per_step'] == 0
    assert lines[1] == 'MAPS False False True'


def test_both_arms_name_the_same_config():
    sys.path.insert(0, ROOT)
    import bench
    a = bench.config_dict(3840, 2160, 2880, 30, 1)
    assert a['gop'] == '1 key + 29 inter' and a['seed'] == bench.SEED
    assert 'film grain' in a['workload']


def _replica_rank(rank, world, port, q):
    """One rank of a two-replica job on the CPU (gloo): each rank's time is
    different; every rank must get the slowest one and the whole-job rate."""
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update({'MASTER_ADDR': '127.0.0.1', 'MASTER_PORT': str(port), 'RANK': str(rank),
                       'WORLD_SIZE': str(world)})
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = bench.slowest_rank(100.0 + 50.0 * rank, dist, 'cpu')
        e2e = bench.slowest_rank(2.0 - rank, dist, 'cpu')   # the same reduction, called again in order
        q.put((rank, ms, e2e, bench.replica_rate(30, world, ms / 1e3), bench.rank_info()[:2]))
    finally:
        dist.destroy_process_group()


def test_replicas_report_the_slowest_rank_and_all_frames():
    """bench.py --gpus N runs one replica per rank (no data exchange): its
    time is the maximum over ranks and its value all ranks' frames over that
    time. Two gloo ranks on the CPU stand in for two GPUs."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    procs = [ctx.Process(target=_replica_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, e2e, rate, (r, w) in got:
        assert (r, w) == (rank, 2)
        assert ms == 150.0 and e2e == 2.0
        assert abs(rate - 60 / 0.150) < 1e-9     # 2 ranks x 30 frames in the slowest 150 ms


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun only rank 0 times the reference; another rank exits 0
    at once, printing nothing."""
    env = dict(os.environ, RANK='1', WORLD_SIZE='2', LOCAL_RANK='1')
    r = subprocess.run([sys.executable, 'bench.py', '--impl', 'reference', '--gpus', '2'],
                       capture_output=True, text=True, cwd=ROOT, env=env, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ''


def test_clock_samples_only_from_the_timed_region():
    """Clock samples whose own timestamps fall before begin() (the warm-up)
    or after stop() do not count, whenever their lines were read; throttle
    reasons come from the timed region's samples only."""
    import datetime
    import statistics
    import bench

    def row(t, sm, cap):
        stamp = datetime.datetime.fromtimestamp(t).strftime('%Y/%m/%d %H:%M:%S.%f')[:-3]
        return '%s, 0, %d, 1965, 700, 0x0, Not Active, Not Active, Not Active, %s' % (stamp, sm, cap)

    t0 = 1_800_000_000.0
    lines = [row(t0 - 5.0, 900, 'Active'),        # warm-up
             row(t0 + 0.2, 1965, 'Not Active'),
             row(t0 + 0.3, 1950, 'Not Active'),
             row(t0 + 9.0, 800, 'Active'),         # after the region
             'garbage line']
    out = bench.ClockSampler.summarize(lines, t0, t0 + 1.0)
    assert out['samples'] == 2
    assert out['sm_mhz'] == statistics.median([1965.0, 1950.0])
    assert out['reasons'] == []
    assert bench.ClockSampler.summarize(lines, t0 - 6.0, t0 + 1.0)['reasons'] == ['sw_power_cap']
