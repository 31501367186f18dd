"""Build libahx.so (the CUDA backend, sm_100a) in-tree with nvcc.

Translation units and their arithmetic flags:
  step_unit.cu      compiled 14 times, once per (arithmetic variant, population storage):
                    exact  -fmad=false, IEEE division and square root: every f32 expression individually rounded
                           (bit-identical to the CPU restatement of the reference kernels)
                    fast   -fmad=true, approximate division and square root, the paired collision
  step_dispatch.cu  the precision switch of each variant (compiled twice)
  aux.cu         -fmad=false  read-back, init, re-init, stats, layout conversion
  api.cu                      the C ABI (include/ahx.h)
  batch.cu                    batched stepping (ahx_batch_*: tile tables, CUDA graph, stream ordering)
  noalloc.cu                  diagnostics over caller-owned buffers without allocation
  server.cu                   the serving scheduler thread (ahx_server_*: admission, batched chunks, read-back)
  domain.cu      -fmad=false  the domain builder (ahx_static_*, ahx_domain_build: decode, aggregate, campus raster,
                              build rules, column records)
All use -ftz=true (f32 subnormals flushed, as the CPU restatement does); all but the fast variant use IEEE division
and square root.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')
LIB = os.path.join(HERE, 'libahx.so')
OBJDIR = os.path.join(HERE, '_build')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
COMMON = ['-O3', '-std=c++17', '--expt-relaxed-constexpr', '-lineinfo', '-ftz=true', '-Xcompiler', '-fPIC', '-I',
          INCLUDE]
IEEE = ['-prec-div=true', '-prec-sqrt=true']
EXACT = ['-fmad=false'] + IEEE + ['-DAHX_STEP_NS=exact']
FAST = ['-fmad=true', '-prec-div=false', '-prec-sqrt=false', '-DAHX_STEP_NS=fast', '-DAHX_STEP_FAST=1']
# (object name, source, flags); the storages are the ahx_precision values 0 .. 6
UNITS = [(f'step_{v}_p{p}', 'step_unit.cu', flags + [f'-DAHX_STEP_PREC={p}'])
         for v, flags in (('exact', EXACT), ('fast', FAST)) for p in range(7)] + [
    ('step_exact_dispatch', 'step_dispatch.cu', EXACT),
    ('step_fast_dispatch', 'step_dispatch.cu', FAST),
    ('aux', 'aux.cu', ['-fmad=false'] + IEEE),
    ('api', 'api.cu', ['-fmad=false'] + IEEE),
    ('noalloc', 'noalloc.cu', ['-fmad=false'] + IEEE),
    ('batch', 'batch.cu', ['-fmad=false'] + IEEE),
    ('server', 'server.cu', ['-fmad=false'] + IEEE),
    ('domain', 'domain.cu', ['-fmad=false'] + IEEE),
]


def nvcc():
    p = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(p):
        raise RuntimeError('nvcc not found: the CUDA toolkit is required to build libahx.so')
    return p


def _deps_mtime():
    files = glob.glob(os.path.join(CSRC, '*')) + glob.glob(os.path.join(INCLUDE, '*.h')) + [__file__]
    return max(os.path.getmtime(f) for f in files)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    """Compile (if out of date) and return the path of libahx.so."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps_mtime() and not ptxas_v:
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    cc = nvcc()

    def one(unit):
        name, src, flags = unit
        obj = os.path.join(OBJDIR, name + '.o')
        cmd = [cc] + ARCH + COMMON + flags + (['-Xptxas', '-v'] if ptxas_v else []) + \
            ['-c', os.path.join(CSRC, src), '-o', obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f'nvcc failed on {name} ({src}):\n{r.stderr[-6000:]}')
        return obj, r.stderr

    # the longest units (the step instantiations) first
    with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        results = list(ex.map(one, UNITS))
    if verbose or ptxas_v:
        for _, err in results:
            sys.stderr.write(err)
    tmp = LIB + '.tmp'
    cmd = [cc] + ARCH + ['-shared', '-o', tmp] + [o for o, _ in results] + ['-lcudart']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'link failed:\n{r.stderr[-4000:]}')
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True, ptxas_v='-v' in sys.argv))
