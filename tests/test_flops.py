"""The algorithmic work constants used for roofline reporting equal the counting oracle's."""
from oracle import flopcount

from gradsolve_b200 import flops


def test_flop_constants_match_counting_oracle():
    assert flopcount.all_counts() == flops.COUNTS
