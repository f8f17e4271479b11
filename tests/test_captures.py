"""The capture tooling: the reference's equivalence gate restated
(tools/testkit/equivalence/harness.py:86-185) over this package's captures,
and the HDF5 converter's dependency gate.  CPU only."""

from __future__ import annotations

import json

import numpy as np
import pytest

from lattice_boltzmann_d3q19_b200 import captures as CAP
from lattice_boltzmann_d3q19_b200.sim import write_capture


def _frames(seed, steps=(0, 5, 10), scale=1.0):
    rng = np.random.default_rng(seed)
    out = []
    for s in steps:
        rho = 1.0 + 0.01 * rng.standard_normal((4, 3, 2))
        u = scale * 0.05 * rng.standard_normal((3, 4, 3, 2))
        out.append((s, {"rho": rho, "u": u}, {"rho_min": float(rho.min())}))
    return out


def _manifest(name="lattice-boltzmann-d3q19", category="lattice"):
    return {"schema_version": "1.0.0", "sim": {"name": name, "category": category, "variant": "bgk-d3q19-qian-1992"},
            "stack": {"name": "test"}, "config": {"seed": 42}}


def _write(tmp_path, tag, frames, **kw):
    return write_capture(frames, _manifest(**kw), tmp_path / tag, "cap")


def test_identical_captures_pass_with_the_lbm_tolerance(tmp_path):
    fr = _frames(1)
    v = CAP.compare_captures(_write(tmp_path, "a", fr), _write(tmp_path, "b", fr))
    assert v.within_tolerance
    assert v.tolerance_table_used == {"category": "lbm", "relative": 1e-5, "absolute": 0.0}
    assert all(d["max_abs_err"] == 0.0 for d in v.per_field_diff.values())
    assert set(v.per_field_diff) == {f"step:{s}:{k}" for s in (0, 5, 10) for k in ("rho", "u")}


def test_tolerance_is_relative_to_the_right_capture_peak(tmp_path):
    fr = _frames(2)
    a = _write(tmp_path, "a", fr)
    # an error just below / above 1e-5 of max|u| in one entry of one frame
    for factor, ok in ((0.9, True), (1.1, False)):
        fr2 = [(s, {k: v.copy() for k, v in st.items()}, d) for s, st, d in fr]
        peak = np.abs(fr2[1][1]["u"]).max()
        fr2[1][1]["u"][0, 1, 1, 1] += factor * 1e-5 * peak
        v = CAP.compare_captures(a, _write(tmp_path, f"b{factor}", fr2))
        assert v.within_tolerance is ok, factor
        assert v.per_field_diff["step:5:u"]["max_abs_err"] > 0


def test_structural_mismatches_fail(tmp_path):
    fr = _frames(3)
    a = _write(tmp_path, "a", fr)
    v = CAP.compare_captures(a, _write(tmp_path, "steps", fr[:2]))
    assert not v.within_tolerance and "step:set-mismatch" in v.per_field_diff
    v = CAP.compare_captures(a, _write(tmp_path, "sim", fr, category="other"))
    assert not v.within_tolerance and "sim:category-mismatch" in v.per_field_diff
    fr_missing = [(s, {"rho": st["rho"]}, d) for s, st, d in fr]
    v = CAP.compare_captures(a, _write(tmp_path, "missing", fr_missing))
    assert not v.within_tolerance and "step:0:u:missing" in v.per_field_diff
    fr_shape = [(s, {"rho": st["rho"][:2], "u": st["u"]}, d) for s, st, d in fr]
    v = CAP.compare_captures(a, _write(tmp_path, "shape", fr_shape))
    assert not v.within_tolerance and "step:0:rho:shape-mismatch" in v.per_field_diff


def test_dtype_mismatch_raises(tmp_path):
    fr = _frames(4)
    a = CAP.load_capture(_write(tmp_path, "a", fr))
    b = CAP.load_capture(_write(tmp_path, "b", fr))
    b.frames[0]["state"]["rho"] = b.frames[0]["state"]["rho"].astype(np.float32)
    with pytest.raises(TypeError):
        CAP.compare_captures(a, b)


def test_load_capture_reads_the_payload_keys(tmp_path):
    fr = _frames(5)
    cap = CAP.load_capture(_write(tmp_path, "a", fr))
    assert cap.steps() == [0, 5, 10]
    assert np.array_equal(cap.frames[5]["state"]["u"], fr[1][1]["u"])
    assert float(cap.frames[10]["diagnostics"]["rho_min"]) == fr[2][2]["rho_min"]
    assert cap.manifest["sim"]["name"] == "lattice-boltzmann-d3q19"


def test_hdf5_converter(tmp_path):
    fr = _frames(6)
    m = _write(tmp_path, "a", fr)
    try:
        import h5py  # noqa: F401
    except ImportError:
        with pytest.raises(ImportError, match="h5py"):
            CAP.to_hdf5(m, tmp_path / "h5")
        return
    out = CAP.to_hdf5(m, tmp_path / "h5")
    man = json.loads(out.read_text())
    assert man["payload"]["path"].endswith(".h5") and man["payload"]["checksum"].startswith("sha256:")
    assert CAP.compare_captures(m, out).within_tolerance
