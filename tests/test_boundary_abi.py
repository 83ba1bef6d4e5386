"""The drop-ins against the reference's own plug-in headers, without a GPU.

- Layout: oracle/boundary_abi.cpp built on the reference's
  Readers/StateReader.h + Managers/BaseManager.h and on gexs_b200/host/'s
  re-declarations prints the same vtable slot for every virtual function
  and the same member offsets and sizes, so an object built on ours is used
  unchanged through the reference's StateReader* / BaseManager*
  (Profiles/BaseProfile.cpp:42-71,143-234).  A copy of our StateReader.h
  with a virtual destructor (the earlier mistake) is caught by the same
  comparison.
- Link and dispatch: oracle/boundary_driver.cpp, compiled on the reference's
  headers alone, calls every virtual of both interfaces through base-class
  pointers on objects from the product library (drive_so) and on the
  drop-in sources compiled against the reference's headers (drive_src).
  With no device visible each call takes its error path: no record, Q = 0,
  OpenFile false, CloseFile true, nothing written to the caller's buffer.
  tests/test_gpu_boundary.py runs the same binaries on a GPU.

The binaries are built by oracle/Makefile (target boundary) from the
reference tree when it is present; without the tree and without prebuilt
binaries the tests are skipped.
"""
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BND = os.path.join(ROOT, "oracle", "_ref", "boundary")


def _bin(name):
    p = os.path.join(BND, name)
    if not os.path.exists(p):
        r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "boundary"],
                           capture_output=True, text=True)
        if r.returncode != 0 or not os.path.exists(p):
            pytest.skip("boundary binaries need the reference tree: " + r.stderr[-300:])
    return p


def _json(cmd, env=None):
    p = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=120)
    assert p.returncode == 0, (cmd, p.returncode, p.stdout[-500:], p.stderr[-500:])
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_layout_matches_the_reference_headers():
    ref = _json([_bin("abi_ref")])
    ours = _json([_bin("abi_ours")])
    assert ours == ref
    # every virtual of StateReader.h:13-17 and BaseManager.h:22-35 in order
    assert [ref["StateReader"][k] for k in ("OpenFile", "CloseFile", "ReadNextState6",
                                            "ReadNextState4", "ComputePartition")] == \
        [0, 8, 16, 24, 32]
    assert ref["BaseManager"]["ReadyForWork"] == 80


def test_layout_probe_catches_a_virtual_destructor(tmp_path):
    """A planted mistake in a copy of the header, compiled here on the CPU."""
    src = os.path.join(ROOT, "gexs_b200", "host")
    for h in ("StateReader.h", "BaseManager.h"):
        shutil.copy(os.path.join(src, h), str(tmp_path))
    p = os.path.join(str(tmp_path), "StateReader.h")
    txt = open(p).read()
    assert "    ~StateReader() {}" in txt
    open(p, "w").write(txt.replace("    ~StateReader() {}", "    virtual ~StateReader() {}"))
    exe = os.path.join(str(tmp_path), "abi_bad")
    subprocess.run(["g++", "-std=c++11", "-w", "-I" + str(tmp_path), "-o", exe,
                    os.path.join(ROOT, "oracle", "boundary_abi.cpp")], check=True)
    bad = _json([exe])
    ref = _json([_bin("abi_ref")])
    assert bad["StateReader"]["OpenFile"] != ref["StateReader"]["OpenFile"]


@pytest.mark.parametrize("variant", ["drive_so", "drive_src"])
def test_every_virtual_through_reference_pointers_without_a_device(tmp_path, variant):
    exe = _bin(variant)
    st, tr = os.path.join(str(tmp_path), "a.states"), os.path.join(str(tmp_path), "a.trans")
    open(st, "w").write("1 0.0 1 0\n2 100.0 3 1\n")
    open(tr, "w").write("2 1 1.0\n")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = _json([exe, st, tr, str(tmp_path), "1500", "1", "800", "0.1", "18", "50", "0.1",
               "1000", "0"], env=env)
    assert r == {"q1": 0, "q2": 0, "opened": 0, "records": 0, "closed": 1, "reopened": 0,
                 "got4": 0, "match4": 0, "closed2": 1, "ntrans_capacity": 0, "ready": 0,
                 "ntrans_capacity2": 0, "deprecated_left_buffer": 1}
