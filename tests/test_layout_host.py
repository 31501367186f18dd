"""Population-plane index arithmetic of the step kernels (csrc/lattice.cuh, csrc/fused.cuh): the neighbour offsets the
kernels form from a cell's own offset (lvl_nbr) against the direct formula (lvl at the neighbour), for the
level-paired 16-bit planes and the plain 32-bit planes, and the numbering of a level pair's 38 source words. Checked
on the CPU by compiling tests/lvl_check.cu as host code with nvcc."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, 'ashburn_heat_twin_b200', 'csrc')


def test_neighbour_offsets_and_pair_slots(tmp_path):
    nvcc = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(nvcc):
        pytest.skip('nvcc not available')
    exe = str(tmp_path / 'lvl_check')
    subprocess.check_call([nvcc, '-gencode', 'arch=compute_100a,code=sm_100a', '-std=c++17', '--expt-relaxed-constexpr',
                           '-I', CSRC, '-I',
                           os.path.join(ROOT, 'include'), os.path.join(HERE, 'lvl_check.cu'), '-o', exe])
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith('ok ')
