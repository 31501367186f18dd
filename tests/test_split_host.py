"""Column split of a step launch (csrc/split.h, the mapping step_block uses to give each thread its column): checked
on the CPU for whole domains, y-slabs of a larger domain and bands of rows, with and without strips, by compiling
tests/split_check.cpp with the host compiler and walking every thread of each launch grid."""
import itertools
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), 'ashburn_heat_twin_b200', 'csrc')


@pytest.fixture(scope='module')
def split_check(tmp_path_factory):
    cxx = shutil.which('g++') or shutil.which('c++')
    if cxx is None:
        pytest.skip('no host C++ compiler')
    exe = str(tmp_path_factory.mktemp('split') / 'split_check')
    subprocess.check_call([cxx, '-O1', '-std=c++17', '-I', CSRC, os.path.join(HERE, 'split_check.cpp'), '-o', exe])
    return exe


def run(exe, cases):
    args = [str(v) for c in cases for v in c]
    r = subprocess.run([exe] + args, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == f'ok {len(cases)}'


def test_whole_domains(split_check):
    cases = [(nx, ny, 0, ny, 0, ny, 0, ws, rows, 0)
             for nx, ny in [(1, 1), (2, 2), (3, 5), (16, 4), (17, 3), (31, 7), (32, 2), (33, 9), (47, 6), (48, 5),
                            (49, 4), (64, 3), (100, 11), (200, 13), (600, 6)]
             for ws in (0, 8, 16, 32) for rows in (1, 2, 4, 8)]
    run(split_check, cases)


def test_slabs_and_bands(split_check):
    cases = []
    for nyg, parts, nx in itertools.product((12, 19), (1, 2, 3), (20, 40, 70)):
        edges = [round(nyg * p / parts) for p in range(parts + 1)]
        for a, b in zip(edges[:-1], edges[1:]):
            h = 2 if parts > 1 else 0
            lo, hi = max(0, a - h), min(nyg, b + h)
            ny, jg0, jlo, jhi = hi - lo, lo, a - lo, b - lo
            for ws in (0, 16):
                cases.append((nx, ny, jg0, nyg, jlo, jhi, 0, ws, 4, 0))
                # bands of rows of the slab (a step split into boundary rows and interior rows)
                for j0, j1 in [(jlo, min(jhi, jlo + 1)), (jlo + 1, jhi), (jlo, jhi - 1), (jhi - 1, jhi)]:
                    if j0 < j1:
                        cases.append((nx, ny, jg0, nyg, j0, j1, j0, ws, 4, 0))
    run(split_check, cases)


def test_staged_grid(split_check):
    """The TMA-staged paired step's grid (main blocks from the first main row, 8- or 16-column strips): whole domains
    and y-slabs, every column exactly once, no face column in a main warp."""
    cases = [(nx, ny, 0, ny, 0, ny, 0, ws, rows, 1)
             for nx, ny in [(17, 3), (33, 9), (48, 5), (49, 4), (64, 3), (100, 11), (200, 13), (300, 300), (600, 6)]
             for rows in (4, 8) for ws in (8, 16)]
    for nyg, parts, nx in itertools.product((12, 19), (1, 2, 3), (20, 40, 70)):
        edges = [round(nyg * p / parts) for p in range(parts + 1)]
        for a, b in zip(edges[:-1], edges[1:]):
            h = 2 if parts > 1 else 0
            lo, hi = max(0, a - h), min(nyg, b + h)
            cases.append((nx, hi - lo, lo, nyg, a - lo, b - lo, 0, 16, 4, 1))
    run(split_check, cases)
