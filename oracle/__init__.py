"""The oracle: a CPU restatement of the reference's traversal and BVH-build arithmetic.

Test infrastructure only. The tests, the smoke check and bench.py's CPU-baseline leg use it as the
checker for the CUDA path; the product package never imports it.
"""
