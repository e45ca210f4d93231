"""CPU oracle for the FDZB soft-shadow path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() (as the checker) and bench.py's CPU
baseline leg use this package.  The product (the 4dzb_b200 package and
libfdzb.so) never imports or calls it.
"""
from .orc import (  # noqa: F401
    OrcFrame, exhaustive_fp32, exhaustive_fp64, frame, light_setup, load, mask_words,
)
