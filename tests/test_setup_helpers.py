"""Digest of a golden case's setup, shared by the setup tests and the fixture generator."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))


def setup_digests(rn, name):
    import make_golden
    s, _ = make_golden.case_setup(rn, name)
    return make_golden.setup_record(s)
