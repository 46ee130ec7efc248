"""The CPU oracle against the golden fixtures (bit for bit).

The fixtures come from an independent pure-Python transcription of the
reference maps (tests/golden/make_golden.py) on the reference's own parity
cases (test/verify_elements.jl, verify_fodo.jl, verify_dba.jl, verify_bend.jl,
verify_exact_bend.jl).  Two transcriptions with IEEE arithmetic and the same
libm must agree exactly.
"""
import importlib.util
import os

import numpy as np
import pytest

import oracle_ref
from conftest import ROOT, golden_lattice, unhex


def _cases(golden):
    return [c["name"] for c in golden["cases"]]


def test_fixture_regenerates(golden, tmp_path):
    """The committed fixture is what the generator produces."""
    spec = importlib.util.spec_from_file_location("mg", os.path.join(ROOT, "tests", "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    mis = [c for c in golden["cases"] if c.get("misalign")]
    for c in golden["cases"][:8] + mis[:2]:
        inp = unhex(c["input"]).tolist()
        rows = [{k: [float.fromhex(v) for v in row[k]] for k in ("t1", "t2", "r1", "r2")}
                for row in c.get("misalign", [])]
        out, lost, lt, le = mg.ringpass(c["elements"], inp, float.fromhex(c["beti"]), c["nturns"],
                                        tuple(c["aperture"]), rows)
        assert [[float(v).hex() for v in r] for r in out] == c["output"]


def test_oracle_matches_golden_bitwise(golden):
    assert len(golden["cases"]) >= 40
    for c in golden["cases"]:
        coords = np.asfortranarray(unhex(c["input"]))
        lost = np.zeros(coords.shape[0], dtype=np.int64)
        lt = np.full(coords.shape[0], -1, dtype=np.int32)
        le = np.full(coords.shape[0], -1, dtype=np.int32)
        beti = float.fromhex(c["beti"])
        oracle_ref.ringpass(golden_lattice(c), coords, lost, beti, c["nturns"], aperture=tuple(c["aperture"]),
                            lost_turn=lt, lost_elem=le)
        ref = unhex(c["output"])
        same = (coords == ref) | (np.isnan(coords) & np.isnan(ref))
        assert same.all(), f"{c['name']}: oracle differs from the golden fixture"
        assert lost.tolist() == c["lost"], c["name"]
        assert lt.tolist() == c["lost_turn"], c["name"]
        assert le.tolist() == c["lost_elem"], c["name"]


def test_golden_covers_reference_suite(golden):
    names = set(_cases(golden))
    # test/verify_elements.jl cases the engine supports, plus the lattice tests
    for n in ["Marker", "Drift", "Quadrupole", "Sextupole", "Octupole", "ThinMultipole", "SBend", "RBend", "ExactSBend",
              "ERBend", "RFCavity", "CrabCavity", "AccelCavity", "LongitudinalRFMap", "Solenoid", "Corrector",
              "HKicker", "VKicker", "Translation", "YRotation", "LorentzBoost", "InvLorentzBoost", "DriftSC",
              "QuadrupoleSC", "SextupoleSC", "OctupoleSC", "SBendSC", "RBendSC", "SpaceCharge", "FODO_line",
              "DBA_line", "Bend_pi4", "ExactBend_pi9"]:
        assert n in names, n


def test_loss_cases_have_losses(golden):
    by = {c["name"]: c for c in golden["cases"]}
    for name in ("FODO_ring_losses", "FODO_sext_losses"):
        c = by[name]
        assert 0 < sum(c["lost"]) < len(c["lost"])
    assert max(by["FODO_sext_losses"]["lost_turn"]) > 0


def test_golden_has_misalignment_cases(golden):
    """Offsets (t1, t2), rolls and general non-orthogonal r1/r2 matrices, on
    single elements and on the DBA line over several passes."""
    mis = [c for c in golden["cases"] if c.get("misalign")]
    assert len(mis) >= 6
    rows = mis[0]["misalign"]
    assert any(float.fromhex(v) != 0.0 for r in rows for v in r["t1"])
    assert any(float.fromhex(v) != 0.0 for r in rows for v in r["t2"])
    general = [r for r in rows if any(float.fromhex(v) != 0.0 for v in r["r1"])]
    assert general
    by = {c["name"]: c for c in mis}
    assert by["MisalignedDBA_line_3passes"]["nturns"] == 3
