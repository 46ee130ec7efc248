"""The C ABI: the library loads, exports every symbol of include/*.h, and the
host-side logic (validation, compilation, FLOP model) is right.  No GPU needed."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import oracle_ref
from conftest import ROOT, golden_lattice, has_gpu, tp

abi = tp._abi
W = __import__("trackpad_b200.workloads", fromlist=["x"])


def header_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"TP_API\s+[\w\s\*]+?\b(tp_\w+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_header_symbol():
    lib = abi.lib()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_struct_layouts_match_header(tmp_path):
    """The ctypes declarations have the sizes and field offsets the C compiler
    gives the header's structs."""
    import subprocess
    structs = {"tp_elem": abi.TpElem, "tp_misalign": abi.TpMisalign, "tp_opts": abi.TpOpts, "tp_stats": abi.TpStats,
               "tp_loss_spec": abi.TpLossSpec, "tp_adjoint_stats": abi.TpAdjointStats,
               "tp_tpsa_stats": abi.TpTpsaStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "trackpad_b200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} @sizeof %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    seen = 0
    for line in filter(None, out):
        cname, what, val = line.split()
        py = structs[cname]
        got = C.sizeof(py) if what == "@sizeof" else getattr(py, what).offset
        assert got == int(val), (cname, what, got, val)
        seen += 1
    assert seen == sum(1 + len(p._fields_) for p in structs.values())


def test_version_and_strerror():
    lib = abi.lib()
    assert lib.tp_abi_version() == 1
    for st in range(0, -9, -1):
        assert lib.tp_strerror(st)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_ctx_create_without_device_fails_cleanly():
    h = C.c_void_p()
    assert abi.lib().tp_ctx_create(0, C.byref(h)) == abi.TP_ENODEV
    assert not h.value


def test_beam_beti_matches_reference():
    v = C.c_double()
    assert abi.lib().tp_beam_beti(3.0e9, tp.M_ELECTRON, C.byref(v)) == 0
    assert v.value == tp.beti(tp.Beam(3.0e9))
    assert abi.lib().tp_beam_beti(-1.0, tp.M_ELECTRON, C.byref(v)) == abi.TP_EINVAL


def _create(elems, mis=None):
    arr = abi.elem_array(elems)
    h = C.c_void_p()
    nm = 0 if mis is None else len(mis)
    marr = None if mis is None else (abi.TpMisalign * nm)(*mis)
    st = abi.lib().tp_lattice_create(arr, len(elems), marr, nm, C.byref(h))
    return st, h


def test_lattice_validation():
    st, h = _create([dict(kind=99)])
    assert st == abi.TP_EUNSUPPORTED
    st, h = _create([dict(kind="QUADRUPOLE", L=0.5, k=1.0, max_order=4, num_int_steps=10)])
    assert st == abi.TP_EINVAL
    st, h = _create([dict(kind="DRIFT", L=1.0, misalign_index=0)])
    assert st == abi.TP_EINVAL  # no misalignment table
    st, h = _create([dict(kind="RFCAVITY", misalign_index=0)], mis=[abi.TpMisalign()])
    assert st == abi.TP_EINVAL  # RFCavity has no misalignment fields
    st, h = _create([dict(kind="DRIFT", L=1.0)])
    assert st == 0
    n = C.c_int64()
    assert abi.lib().tp_lattice_length(h, C.byref(n)) == 0 and n.value == 1
    assert abi.lib().tp_lattice_destroy(h) == 0


def test_null_arguments_are_rejected():
    lib = abi.lib()
    assert lib.tp_lattice_create(None, 3, None, 0, C.byref(C.c_void_p())) == abi.TP_EINVAL
    assert lib.tp_ringpass(None, None, None, 0, None, None, None, 1.0, 1, 0.0, 0.0, 0, None) == abi.TP_EINVAL
    assert lib.tp_last_stats(None, None) == abi.TP_EINVAL


@pytest.mark.parametrize("lat_name", ["fodo", "dba", "golden"])
def test_flop_model_matches_oracle_op_count(lat_name, golden):
    """tp_lattice_flops (the library's algorithmic FLOP model) equals the
    oracle's op-counting scalar, element by element."""
    if lat_name == "fodo":
        lats = [(W.fodo_ring(), 1e9)]
    elif lat_name == "dba":
        lats = [(W.dba_ring(cells=2), 3e9)]
    else:
        for c in golden["cases"]:
            lat = golden_lattice(c)  # element records and misalignment rows
            ref, _ = oracle_ref.count_flops(lat, float.fromhex(c["beti"]))
            assert lat.flops_per_element().tolist() == ref.tolist(), c["name"]
        return
    for lat, e in lats:
        ref, _ = oracle_ref.count_flops(lat, tp.beti(tp.Beam(e)))
        assert lat.flops_per_element().tolist() == ref.tolist()


def test_schedule_validation():
    lat = tp.Lattice([tp.Drift(1.0), tp.Quadrupole(0.4, 0.6)])
    lib = abi.lib()
    f = np.array([5, 1], dtype=np.int32)
    v = np.zeros((2, 1))
    st = lib.tp_lattice_set_schedule(lat.handle, f.ctypes.data_as(C.c_void_p), 1, 0, 2, v.ctypes.data_as(C.c_void_p))
    assert st == abi.TP_EINVAL  # element index out of range
    f = np.array([1, 1], dtype=np.int32)
    st = lib.tp_lattice_set_schedule(lat.handle, f.ctypes.data_as(C.c_void_p), 1, 0, 2, v.ctypes.data_as(C.c_void_p))
    assert st == 0
    assert lib.tp_lattice_set_schedule(lat.handle, None, 0, 0, 0, None) == 0
