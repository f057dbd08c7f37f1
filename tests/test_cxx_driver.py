"""The C++ drop-in: tests/cxx/tranrota_driver.cpp restates the reference driver's search block
(src/TranRotaConfSearchNoMini.cu:96-487) with calls into include/cdock_b200.hpp and links
libcdock_b200.so. The CPU test builds it (the header compiles and every cdk:: symbol it uses
resolves); the GPU test runs it on config 0 and checks its output against the C-ABI search
(cdk_search) bit for bit, the FP64 oracle within the FP32 tolerance, the sort order of the
per-rotation minima, and the rebuilt poses against their definition."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from cdocker_b200 import Receptor, quaternion_uniform_sampling, synth
from cdocker_b200.build import LIB as PRODUCT_LIB
from oracle import oracle as O
from tests.parity import check_search

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cxx", "tranrota_driver.cpp")


def _build(out_dir) -> str:
    exe = os.path.join(str(out_dir), "tranrota_driver")
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++14", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", os.path.dirname(PRODUCT_LIB), "-lcdock_b200",
           "-Wl,-rpath," + os.path.dirname(PRODUCT_LIB), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_driver_builds_against_the_cxx_api(tmp_path):
    exe = _build(tmp_path)
    assert os.path.exists(exe)


def _write_input(path, w, n_conf, n_rota, max_nq, n_lowest, seed):
    with open(path, "wb") as f:
        f.write(struct.pack("<7i", w.n, w.all_grids.shape[0], w.coor.shape[1], n_conf, n_rota,
                            max_nq, n_lowest))
        f.write(struct.pack("<Q", seed))
        f.write(struct.pack("<7f", w.spacing, *w.mid, *w.length))
        for arr in (w.grid_radii, w.all_grids, w.coor[:n_conf], w.charge, w.eps, w.radii):
            f.write(np.ascontiguousarray(arr, np.float32).tobytes())


def _read_output(path, n_conf, n_atom):
    buf = open(path, "rb").read()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(buf, dtype, count, off)
        off += a.nbytes
        return a

    K = int(take("<i4", 1)[0])
    confs = []
    for _ in range(n_conf):
        nu = int(take("<i4", 1)[0])
        q = take("<f4", 4 * nu).reshape(nu, 4)
        e = take("<f4", nu)
        i = take("<i4", 3 * nu).reshape(nu, 3)
        npose = int(take("<i4", 1)[0])
        poses = []
        for _ in range(npose):
            iq = int(take("<i4", 1)[0])
            poses.append((iq, take("<f8", 3 * n_atom).reshape(n_atom, 3)))
        confs.append({"q": q, "e": e, "i": i, "poses": poses})
    assert off == len(buf)
    return K, confs


@pytest.mark.gpu
def test_driver_matches_c_abi_search(tmp_path, c0):
    w = c0
    n_conf, n_rota, n_lowest, seed = 1, 500, 8, 4242
    exe = _build(tmp_path)
    inp, out = os.path.join(tmp_path, "in.bin"), os.path.join(tmp_path, "out.bin")
    # maxNQ >= nRotaSample: the filter keeps every rotation without its rand()-driven shuffle, so
    # the two processes keep the same rotations whatever their rand() state
    _write_input(inp, w, n_conf, n_rota, n_rota, n_lowest, seed)
    subprocess.run([exe, inp, out], check=True, timeout=600)
    K, confs = _read_output(out, n_conf, w.coor.shape[1])
    assert K == w.K
    quats = quaternion_uniform_sampling(seed, n_conf, n_rota)
    h = 0.5
    with Receptor(w.grids, w.spacing) as rec:
        for c, got in enumerate(confs):
            assert np.array_equal(got["q"].view(np.uint32), quats[c].view(np.uint32))
            e, i = rec.search(w.coor[c:c + 1], w.charge, w.eps, w.slot, quats[c:c + 1])
            # the same library search on the same inputs: bit for bit
            assert np.array_equal(got["e"].view(np.uint32), e.view(np.uint32))
            assert np.array_equal(got["i"], i)
            _, ridx, r64 = O.search_direct(w.grids, w.spacing, w.coor[c:c + 1], w.charge, w.eps,
                                           w.slot, quats[c:c + 1], prec=1)
            check_search(got["e"], got["i"], r64, ridx,
                         lambda r: O.energy_map(w.grids, w.spacing, w.coor[c], w.charge, w.eps,
                                                w.slot, quats[c, r]))
            # sort_index: ascending minima (ties in any order, as std::sort leaves them)
            iq = [p[0] for p in got["poses"]]
            assert len(iq) == n_lowest
            kth = np.sort(got["e"])[:n_lowest]
            assert np.array_equal(np.sort(got["e"][iq]), kth)
            assert all(got["e"][iq[k]] <= got["e"][iq[k + 1]] for k in range(n_lowest - 1))
            # pose: rotated float coordinates + (gridMin - mincoor + idx * spacing) in double,
            # gridMin = mid - len/2 in float (src/TranRotaConfSearchNoMini.cu:149-151, :473-487)
            grid_min = (w.mid - w.length / np.float32(2)).astype(np.float32).astype(np.float64)
            for q_idx, pose in got["poses"]:
                rot, mn, _ = O.rotate_bbox(w.coor[c], quats[c, q_idx][None])
                step = (got["i"][q_idx].astype(np.float32) * np.float32(h)).astype(np.float64)
                want = rot[0].astype(np.float64) + (grid_min - mn[0].astype(np.float64) + step)
                assert np.array_equal(pose, want)
