"""The measurement helpers of bench.py that need no GPU: algorithmic bytes of the
level-0 SpMV and the DRAM traffic read from the committed ncu summary."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_spmv_algorithmic_bytes():
    # 9 FP32 values + a 4-byte (or 2-byte) column index per block, row pointers, x and y
    nnzb, nbrow = 7_189_057, 274_625
    assert bench.spmv_bytes(nnzb, nbrow, 3, 4) == 295_251_784
    assert bench.spmv_bytes(nnzb, nbrow, 3, 4, 2) == 295_251_784 - 2 * nnzb


def test_traffic_of_the_captured_launch_and_of_another_size():
    alg = bench.spmv_bytes(7_189_057, 274_625, 3, 4, 2)
    t, src = bench.ncu_traffic("bsr_spmv_kernel<float,3,0>", alg)
    assert t is not None and "this launch" in src
    assert alg <= t <= 1.02 * alg          # the capture reads what the algorithm needs
    t2, src2 = bench.ncu_traffic("bsr_spmv_kernel<float,3,0>", 10 * alg)
    assert abs(t2 - 10 * t) <= 1e-6 * t2 and "scaled" in src2
    assert bench.ncu_traffic("no_such_kernel", alg) == (None, None)
