"""CPU oracle for the BLML binned path: test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's
CPU-baseline leg). Never imported by the product package."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
