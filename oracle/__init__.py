"""TEST INFRASTRUCTURE: CPU restatement of the reference's uniform-patch step.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this package, as the checker. The product (dclaw_b200) never imports it.
"""
from .oracle import Oracle, build, lib_path  # noqa: F401
