"""CPU oracle for the gwb200 hot path: TEST INFRASTRUCTURE ONLY.

A numpy (float32/float64) restatement of the reference's algorithm for each stage of the matched-filter path, each
function citing the reference file:line it follows (paths within gw-gpu-search). Only tests/, the smoke check in
__graft_entry__.py and bench.py's CPU baseline and reference arm may import this package; the product (gwb200) never
does. Its pins: tests/golden/*.npz, written by tests/golden/make_golden.py from the reference's own code run on the
same seeded inputs (see that script for which stages were pinned and how).
"""
