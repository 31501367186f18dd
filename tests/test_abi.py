"""The C-ABI library loads and exports every entry point include/*.h declares (no compute: no GPU needed)."""
import ctypes
import glob
import os
import re

from ashburn_heat_twin_b200 import _build
from ashburn_heat_twin_b200 import cuda_device as CD

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, 'include', '*.h')):
        src = open(h).read()
        src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
        names |= set(re.findall(r'\b(ahx_[a-z0-9_]+)\s*\(', src))
    return names


def test_library_exports_every_declared_symbol():
    lib = _build.build()
    L = ctypes.CDLL(lib)
    decl = declared_symbols()
    assert 'ahx_step' in decl and 'ahx_create' in decl
    missing = [n for n in sorted(decl) if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding declares the same set
    assert set(CD.SYMBOLS) | {'ahx_last_error'} >= decl


def test_create_without_gpu_fails_cleanly():
    """With no CUDA device, ahx_create returns an error status and a message instead of aborting."""
    import torch
    if torch.cuda.is_available():
        return
    L = CD.load_library(_build.build())
    d = CD.Dims(nx=8, ny=8, nz=8, precision=0, device_ordinal=-1, arith=0)
    h = ctypes.c_void_p()
    st = L.ahx_create(ctypes.byref(d), ctypes.byref(h))
    assert st == 4
    assert b'no CUDA device' in L.ahx_last_error()


def test_bad_arguments_rejected_before_touching_the_gpu():
    L = CD.load_library(_build.build())
    h = ctypes.c_void_p()
    d = CD.Dims(nx=1, ny=8, nz=8, precision=0, device_ordinal=-1, arith=0)
    assert L.ahx_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d = CD.Dims(nx=8, ny=8, nz=8, precision=9, device_ordinal=-1, arith=0)
    assert L.ahx_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d = CD.Dims(nx=20000, ny=20000, nz=64, precision=0, device_ordinal=-1, arith=0)
    assert L.ahx_create(ctypes.byref(d), ctypes.byref(h)) == 1
    assert b'too large' in L.ahx_last_error()
    assert L.ahx_step(None, 1, 0) == 1


def test_struct_layouts_match_the_header(tmp_path):
    """Every struct the Python binding passes through the C ABI has the header's size and field offsets (checked
    against a C program compiled from include/ahx.h with the system compiler)."""
    import subprocess
    structs = {'ahx_dims': CD.Dims, 'ahx_info_out': CD.InfoOut, 'ahx_stats_out': CD.StatsOut,
               'ahx_budget_out': CD.BudgetOut, 'ahx_server_config': CD.ServerConfig, 'ahx_request': CD.RequestIn,
               'ahx_server_result': CD.ServerResult, 'ahx_server_stats_out': CD.ServerStats,
               'ahx_batch_info_out': CD.BatchInfoOut}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ahx.h"', 'int main(void) {']
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ['  return 0;', '}']
    src = tmp_path / 'layout.c'
    src.write_text('\n'.join(lines))
    exe = tmp_path / 'layout'
    subprocess.check_call(['gcc', '-I', os.path.join(ROOT, 'include'), str(src), '-o', str(exe)])
    out = subprocess.check_output([str(exe)], text=True).split('\n')
    got = {}
    for ln in out:
        if ln:
            c, f, v = ln.split()
            got[(c, f)] = int(v)
    for cname, py in structs.items():
        assert got[(cname, 'size')] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_server_rejects_bad_configuration_and_requests():
    """ahx_server_create validates its configuration before touching a device; without a GPU it fails cleanly."""
    L = CD.load_library(_build.build())
    h = ctypes.c_void_p()
    cfg = CD.ServerConfig(device_ordinal=-1, precision=9, arith=1, chunk=8, max_cells=1000, hbm_budget_bytes=0,
                          batch_mode=0, tune=0, depth=2, pad=0)
    assert L.ahx_server_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    cfg.precision, cfg.batch_mode = 0, 7
    assert L.ahx_server_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert L.ahx_server_submit(None, None, None) == 1
    assert L.ahx_server_poll(None, 1, 0, None, None, None, None, None) == 1
    import torch
    if not torch.cuda.is_available():
        cfg.batch_mode = 0
        assert L.ahx_server_create(ctypes.byref(cfg), ctypes.byref(h)) == 4
