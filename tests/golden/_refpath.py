"""Where the golden-fixture scripts find the reference: the checkout given as the first argument (or in
BLML_REFERENCE). The reference's numba kernels cache their compiled code (cache=True), so NUMBA_CACHE_DIR defaults to
a fresh temporary directory: the checkout itself may be read-only."""
import os
import sys
import tempfile


def reference_checkout():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('BLML_REFERENCE')
    if not ref or not os.path.isdir(ref):
        raise SystemExit(f'usage: python {os.path.basename(sys.argv[0])} <reference checkout> '
                         '(or set BLML_REFERENCE)')
    os.environ.setdefault('NUMBA_CACHE_DIR', tempfile.mkdtemp(prefix='numba-cache-'))
    return ref
