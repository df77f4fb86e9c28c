"""The C-ABI library builds, loads without a GPU, and exports every entry point include/oi_b200.h declares."""
import os
import re
import subprocess

from opticalimaging_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, 'include', 'oi_b200.h')).read()
    return sorted(set(re.findall(r'^OI_API\s+[\w\s\*]*?\b(oi_\w+)\s*\(', src, flags=re.M)))


def test_header_declares_entry_points():
    names = declared()
    assert 'oi_coherent_coarse' in names and 'oi_last_error' in names
    assert len(names) >= 9


def test_library_exports_declared_symbols():
    lib = N.load()
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(['nm', '-D', '--defined-only', N.lib_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r'\bT (oi_\w+)', out))
    assert set(declared()) <= exported
    # nothing but the ABI is exported
    assert all(s.startswith('oi_') for s in exported)


def test_binding_covers_header():
    assert set(declared()) <= set(N.exported_symbols())


def test_errors_are_reported_not_raised_in_c():
    lib = N.load()
    rc = lib.oi_twiddle(None, 0, 0, 0, 0, 0, 1, 1.0, None)
    assert rc == -1
    assert b'oi_twiddle' in lib.oi_last_error()
    assert lib.oi_version() >= 1


def test_every_literal_call_matches_its_signature():
    """Each N.call('oi_...', ...) in the package, the bench and the tests passes as many arguments as the
    entry point's ctypes signature (and so as include/oi_b200.h) declares."""
    import ast
    import glob
    import os
    from opticalimaging_b200 import _native as N
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    files = glob.glob(os.path.join(root, 'opticalimaging_b200', '*.py')) + glob.glob(os.path.join(root, 'tests', '*.py'))
    files.append(os.path.join(root, 'bench.py'))
    seen = 0
    for f in files:
        for node in ast.walk(ast.parse(open(f).read())):
            if (isinstance(node, ast.Call) and getattr(node.func, 'attr', None) == 'call' and node.args
                    and isinstance(node.args[0], ast.Constant) and node.args[0].value in N._SIGS
                    and not any(isinstance(a, ast.Starred) for a in node.args)):
                name = node.args[0].value
                assert len(node.args) - 1 == len(N._SIGS[name]), f'{f}:{node.lineno} {name}'
                seen += 1
    assert seen > 10


def test_noalloc_path_names_no_allocator():
    """oi_band_spectrum_noalloc and the scratch lookup it calls name no device allocator (checked in the source,
    so a later change that adds one fails here on the CPU, not only on the GPU)."""
    src = open(os.path.join(ROOT, 'opticalimaging_b200', 'csrc', 'spectrum.cu')).read()
    start = src.index('static __device__ __align__(256) float2 g_static_scratch')
    end = src.index('return oi_band_spectrum(', start)
    section = src[start:end]
    assert 'cudaGetSymbolAddress' in section
    for name in ('cudaMalloc', 'cudaFree', 'cudaMallocAsync', 'cudaFreeAsync', 'cuMemAlloc', 'malloc(', 'new '):
        assert name not in section, name
    # the scratch-form entry point it forwards to takes the caller's scratch and allocates nothing either
    body = src[src.index('extern "C" int oi_band_spectrum('):src.index('// Band spectrum for callers that cannot')]
    assert 'cudaMalloc' not in body and 'cudaFree' not in body
