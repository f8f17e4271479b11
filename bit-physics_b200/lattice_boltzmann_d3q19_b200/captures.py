"""Captures: load, compare against the reference's equivalence gate, convert
to the reference's HDF5 capture format.

A capture is what the canonical runners write (``sim.write_capture``): a
manifest ``<descriptor>.json`` and a payload holding
``steps/{N}/state/{field}`` and ``steps/{N}/diagnostics/{check}`` -- the
reference's capture-v1 layout (tools/testkit/capture/writer.py:36-92,
common_warp/capture/model.py:36-46).  This package writes the payload as
``.npz`` (no h5py dependency); ``to_hdf5`` writes the reference's ``.h5``
payload where h5py is installed, and ``load_capture`` reads either.

``compare_captures`` restates the reference's cross-stack gate
(tools/testkit/equivalence/harness.py:86-185): the same field-by-field
verdict, with the tolerance the reference's table resolves for this
simulation (tools/testkit/equivalence/tolerance.toml:38-40 and 146-147:
sim ``lattice-boltzmann-d3q19`` -> category ``lbm``, relative 1e-5,
absolute 0).
"""

from __future__ import annotations

import hashlib
import json
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any

import numpy as np

# The reference's tolerance table, as far as this simulation resolves it:
# [defaults.lbm] and [overrides.lattice-boltzmann-d3q19].
TOLERANCE_DEFAULTS = {"lbm": {"relative": 1e-5, "absolute": 0.0}}
TOLERANCE_OVERRIDES = {"lattice-boltzmann-d3q19": {"category": "lbm"}}


@dataclass
class Capture:
    manifest: dict[str, Any]
    # step -> {"state": {field: array}, "diagnostics": {check: float}}
    frames: dict[int, dict[str, dict[str, Any]]]

    def steps(self) -> list[int]:
        return sorted(self.frames)


@dataclass
class EquivalenceVerdict:
    """Outcome of compare_captures: ``per_field_diff`` maps a field key to
    ``{max_abs_err, max_rel_err}``; ``tolerance_table_used`` records the
    resolved ``{category, relative, absolute}``."""

    within_tolerance: bool
    per_field_diff: dict[str, dict[str, float]] = field(default_factory=dict)
    tolerance_table_used: dict[str, Any] = field(default_factory=dict)


def _frames_from_items(items) -> dict[int, dict[str, dict[str, Any]]]:
    frames: dict[int, dict[str, dict[str, Any]]] = {}
    for key, value in items:
        parts = key.strip("/").split("/")
        if len(parts) != 4 or parts[0] != "steps" or parts[2] not in ("state", "diagnostics"):
            continue
        fr = frames.setdefault(int(parts[1]), {"state": {}, "diagnostics": {}})
        fr[parts[2]][parts[3]] = np.asarray(value)
    return frames


def load_capture(manifest_path) -> Capture:
    """Read a capture from its manifest (payload ``.npz`` or ``.h5`` next to it)."""
    manifest_path = Path(manifest_path)
    manifest = json.loads(manifest_path.read_text())
    payload = manifest_path.parent / Path(manifest["payload"]["path"]).name
    if payload.suffix == ".npz":
        with np.load(payload) as z:
            frames = _frames_from_items((k, z[k]) for k in z.files)
    else:
        h5py = _h5py()
        items = []
        with h5py.File(payload, "r") as h:
            for step, sg in h["steps"].items():
                for kind in ("state", "diagnostics"):
                    if kind in sg:
                        for name, ds in sg[kind].items():
                            items.append((f"steps/{step}/{kind}/{name}", ds[()]))
        frames = _frames_from_items(items)
    return Capture(manifest, frames)


def _resolve_tolerance(sim_name: str, sim_category: str) -> dict[str, Any]:
    """{category, relative, absolute} for (sim, category), harness.py:61-82."""
    if sim_name in TOLERANCE_OVERRIDES:
        ov = TOLERANCE_OVERRIDES[sim_name]
        base = TOLERANCE_DEFAULTS.get(ov["category"], {})
        return {"category": ov["category"], "relative": float(ov.get("relative", base.get("relative", 0.0))),
                "absolute": float(ov.get("absolute", base.get("absolute", 0.0)))}
    if sim_category not in TOLERANCE_DEFAULTS:
        raise KeyError(f"no tolerance for category {sim_category!r} (sim {sim_name!r})")
    d = TOLERANCE_DEFAULTS[sim_category]
    return {"category": sim_category, "relative": float(d["relative"]), "absolute": float(d["absolute"])}


def _inf() -> dict[str, float]:
    return {"max_abs_err": float("inf"), "max_rel_err": float("inf")}


def compare_captures(left, right) -> EquivalenceVerdict:
    """Field-by-field diff of two captures against the resolved tolerance
    (harness.py:86-185).  The sim name and category come from the left
    manifest and must match the right's; the step sets must match; per
    step and state field, max_abs_err = max |a - b| and max_rel_err =
    max |a - b| / max(|a|, |b|) over entries with a nonzero denominator; a
    field fails when max_abs_err > absolute + relative * max |b| (b: the
    right capture).  Mismatched dtypes raise TypeError."""
    lc = left if isinstance(left, Capture) else load_capture(left)
    rc = right if isinstance(right, Capture) else load_capture(right)
    lsim, rsim = lc.manifest.get("sim", {}), rc.manifest.get("sim", {})
    if lsim.get("category") != rsim.get("category") or lsim.get("name") != rsim.get("name"):
        return EquivalenceVerdict(False, {"sim:category-mismatch": _inf()}, {})
    resolved = _resolve_tolerance(str(lsim.get("name", "")), str(lsim.get("category", "")))
    rtol, atol = resolved["relative"], resolved["absolute"]
    if lc.steps() != rc.steps():
        return EquivalenceVerdict(False, {"step:set-mismatch": _inf()}, resolved)
    per_field: dict[str, dict[str, float]] = {}
    within = True
    for n in lc.steps():
        ls, rs = lc.frames[n]["state"], rc.frames[n]["state"]
        for k in sorted(set(ls) | set(rs)):
            if k not in ls or k not in rs:
                per_field[f"step:{n}:{k}:missing"] = _inf()
                within = False
                continue
            a, b = ls[k], rs[k]
            if a.shape != b.shape:
                per_field[f"step:{n}:{k}:shape-mismatch"] = _inf()
                within = False
                continue
            if a.dtype != b.dtype:
                raise TypeError(f"compare_captures: dtype mismatch on field {k!r}: {a.dtype} vs {b.dtype}")
            a64, b64 = a.astype(np.float64), b.astype(np.float64)
            diff = np.abs(a64 - b64)
            abs_err = float(diff.max()) if diff.size else 0.0
            denom = np.maximum(np.abs(a64), np.abs(b64))
            with np.errstate(divide="ignore", invalid="ignore"):
                rel = np.where(denom > 0, diff / denom, 0.0)
            per_field[f"step:{n}:{k}"] = {"max_abs_err": abs_err, "max_rel_err": float(rel.max()) if rel.size else 0.0}
            scale = float(np.abs(b64).max()) if b64.size else 0.0
            if abs_err > atol + rtol * scale:
                within = False
    return EquivalenceVerdict(within, per_field, resolved)


def _h5py():
    try:
        import h5py
    except ImportError as e:  # the converter needs it; nothing else does
        raise ImportError("to_hdf5 / .h5 captures need h5py, which is not installed") from e
    return h5py


def to_hdf5(manifest_path, out_dir) -> Path:
    """Write the capture as the reference's capture-v1 HDF5 payload
    (writer.py:36-92: ``/steps/{N}/state/{field}``,
    ``/steps/{N}/diagnostics/{check}``, ``/metadata`` attributes) plus its
    manifest, with ``payload.path`` and the payload's sha256 ``checksum``.
    Returns the new manifest path.  Needs h5py."""
    h5py = _h5py()
    cap = load_capture(manifest_path)
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    descriptor = Path(cap.manifest["payload"]["path"]).stem
    payload = out_dir / f"{descriptor}.h5"
    with h5py.File(payload, "w", libver="earliest") as h:
        steps = h.create_group("steps", track_order=False)
        for n in cap.steps():
            sg = steps.create_group(str(n), track_order=False)
            st = sg.create_group("state", track_order=False)
            for name, arr in cap.frames[n]["state"].items():
                st.create_dataset(name, data=np.asarray(arr), track_times=False)
            dg = sg.create_group("diagnostics", track_order=False)
            for name, val in cap.frames[n]["diagnostics"].items():
                dg.create_dataset(name, data=np.asarray(val), track_times=False)
        meta = h.create_group("metadata", track_order=False)
        m = cap.manifest
        meta.attrs["schema_version"] = m.get("schema_version", "")
        meta.attrs["sim_name"] = m.get("sim", {}).get("name", "")
        meta.attrs["sim_category"] = m.get("sim", {}).get("category", "")
        meta.attrs["sim_variant"] = m.get("sim", {}).get("variant", "")
        meta.attrs["stack_name"] = m.get("stack", {}).get("name", "")
        meta.attrs["seed"] = int(m.get("config", {}).get("seed", 0))
    digest = hashlib.sha256(payload.read_bytes()).hexdigest()
    manifest = dict(cap.manifest)
    manifest["payload"] = {"format": "hdf5", "path": payload.name, "checksum": f"sha256:{digest}"}
    out = out_dir / f"{descriptor}.json"
    out.write_text(json.dumps(manifest, indent=2, sort_keys=True) + "\n")
    return out


__all__ = ["Capture", "EquivalenceVerdict", "compare_captures", "load_capture", "to_hdf5"]
