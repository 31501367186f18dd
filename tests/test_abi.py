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
