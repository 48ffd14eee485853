"""The reference arm of bench.py on the CPU: one JSON line with the contract's keys, timing the oracle's
restatement of the reference arithmetic (the translation workload is the cheapest to sample)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    cmd = [sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--workload', 'translation',
           '--steps', '1', '--warmup', '0']
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better',
                'scaling', 'vs_baseline', 'dtype', 'data', 'config', 'cpu_baseline', 'e2e'):
        assert key in d, key
    assert d['impl'] == 'reference' and d['value'] > 0 and d['unit'] == 'recons/s'
    assert d['cpu_baseline']['kind'] in ('port', 'reference') and d['cpu_baseline']['cores'] >= 1
    assert d['cpu_baseline']['value'] == d['value']
    assert d['e2e'] == {'value': d['value'], 'unit': d['unit'], 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}
    assert 'workload' in d['config']


def test_batched_reference_arm_times_a_whole_reconstruction():
    """The batched workload's reference arm: each timed step is one whole oracle reconstruction of one batch scan
    (here the smallest, scan 3), scaled across scans only."""
    cmd = [sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--workload', 'batched',
           '--steps', '1', '--warmup', '1', '--cpu-sample-scan', '3']
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d['impl'] == 'reference' and d['value'] > 0 and d['steps'] == 1
    sample = d['cpu_baseline']['sample']
    assert 'whole reconstruction of scan 3' in sample and 'across scans' in sample
    assert d['config']['num_scans'] == 24
