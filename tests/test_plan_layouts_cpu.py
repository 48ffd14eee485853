"""The forward projector's shared-memory plans (walk, replay, and the smaller walk the replay kernel uses for tiles
a build could not store) hold what each mode reads and fit the memory each launch gets, and the back projector's
plans cover their work within their shared memory and row cache, for a sweep of parallel, cone and translation
geometries: a host-only program over fp_cb.cuh and bp_fast.cuh, compiled with nvcc and run on the CPU."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _nvcc():
    path = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    return path if os.path.exists(path) else None


def test_projector_plans_fit_their_shared_memory(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip('nvcc is not available')
    exe = str(tmp_path / 'plan_layout_check')
    subprocess.run([nvcc, '-std=c++17', '--expt-relaxed-constexpr', '-gencode', 'arch=compute_100a,code=sm_100a',
                    '-o', exe, os.path.join(HERE, 'plan_layout_check.cu')], check=True, capture_output=True)
    res = subprocess.run([exe], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.startswith('ok ') and int(res.stdout.split()[1]) > 50000
