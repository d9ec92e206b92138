"""The C-ABI library loads here (no GPU needed to load it) and exports every entry point include/*.h declares;
the Python binding declares a signature for each of them."""
import ctypes
import glob
import os
import re

from conftest import ROOT


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, 'include', '*.h')):
        src = open(h).read()
        src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
        names |= set(re.findall(r'\b(blml_\w+)\s*\(', src))
    return names


def test_library_exports_every_declared_symbol():
    from blml_b200 import _lib
    assert os.path.exists(_lib.LIB_PATH), 'build the library first: python -m blml_b200.build'
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = declared()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    from blml_b200 import _lib
    assert declared() == set(_lib.EXPORTS)


def test_load_and_query_without_gpu():
    from blml_b200 import _lib
    L = _lib.lib()
    assert L.blml_abi_version() == 1
    assert L.blml_reduce_blocks() > 0
    assert L.blml_last_error() is not None


def test_split_constant_matches_header():
    """The host's copy of BLML_SEG_SPLIT_BLOCKS (the history kernels' block count, used to size their partials)."""
    from blml_b200 import _lib
    hdr = open(os.path.join(ROOT, 'include', 'blml_b200.h')).read()
    assert int(re.search(r'#define BLML_SEG_SPLIT_BLOCKS (\d+)', hdr).group(1)) == _lib.SEG_SPLIT_BLOCKS
