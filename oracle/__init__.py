"""CPU oracle for the warp-fdtd uniform-grid FDTD path.

TEST INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this package as the checker; warp_fdtd_b200 (the
product) never imports, links or runs anything under oracle/.

Parity pin: the restatement reproduces the reference's own Warp float32
outputs committed in warp-fdtd (results/warp/forward50_gpu/fields.npz,
results/warp/hann20/*), copied to tests/golden/ by tests/golden/make_golden.py.
The reference itself (NVIDIA Warp kernels) cannot run in this environment:
warp-lang is not installed and there is no network, so there is no oracle/_ref
build.
"""
