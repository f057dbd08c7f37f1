"""The reference arm's inputs: oracle.reference_inputs builds the benchmark workload without
the product library (receptor grids restated in oracle/cdk_oracle.cpp, quaternions and slots
from the reference's own helpers), and it must equal the product's synthetic workload bit for
bit, so that both arms search the same receptor, ligand and rotations."""
import subprocess
import sys

import numpy as np

from cdocker_b200 import synth
from oracle import oracle as O


def test_reference_inputs_equal_product_workload():
    d = O.reference_inputs("c0_32", seed=3, n_conf=2, n_q=40)
    w = synth.make_workload("c0_32", seed=3, n_conf=2, n_q=40)
    assert np.array_equal(d["all_grids"].view(np.uint32), w.all_grids.view(np.uint32))
    assert np.array_equal(d["grids"].view(np.uint32), w.grids.view(np.uint32))
    assert np.array_equal(d["quats"].view(np.uint32), w.quats.view(np.uint32))
    assert np.array_equal(d["coor"], w.coor) and np.array_equal(d["slot"], w.slot)
    assert np.array_equal(d["charge"], w.charge) and np.array_equal(d["eps"], w.eps)


def test_reference_inputs_load_no_product_library():
    code = ("from oracle import oracle as O\n"
            "O.reference_inputs('c0_32', seed=0, n_conf=1, n_q=8)\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('PRODUCT' if 'libcdock_b200' in maps else 'CLEAN')\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300,
                         cwd=O.HERE + "/..")
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip().splitlines()[-1] == "CLEAN"
