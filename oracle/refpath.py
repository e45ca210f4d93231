"""Where the reference project's sources lie -- TEST INFRASTRUCTURE ONLY.

The build recipes of oracle/ref_emu and oracle/ref_gpu, __graft_entry__.build()
and the tests that rebuild from the reference's sources read them from one
place: $FDZB_REFERENCE, else the checkout this recipe was written against.
Nothing at run time (the library, the GPU tests, bench.py) reads them.
"""
import os

DEFAULT_REFERENCE = "/root/reference"


def reference_root() -> str:
    """The reference checkout (the directory holding 4DZB/)."""
    return os.environ.get("FDZB_REFERENCE", DEFAULT_REFERENCE)


def reference_present() -> bool:
    """True where the reference's soft-shadow sources can be read."""
    return os.path.isdir(os.path.join(reference_root(), "4DZB", "FDZB_Soft_Shadow"))
