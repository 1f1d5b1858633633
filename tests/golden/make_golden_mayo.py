"""Generate tests/golden/mayo_ref.npz from the reference's own Mayo loader.

Run where the XRecon reference tree is importable, naming its root in
XRECON_REFERENCE_ROOT:

    XRECON_REFERENCE_ROOT=<reference tree> python tests/golden/make_golden_mayo.py

The reference's xrecon/utils/mayo.py and xrecon/utils/mayo_fdk.py import
pydicom, which is not installed here.  A stand-in ``pydicom`` module serves
their ``dcmread`` calls with the values pydicom presents for an implicit-VR
DICOM-CT-PD file (tests/golden/mayo_series.py: private tags as raw bytes,
pixel-module tags decoded, the stored pixels), keyed by file path; the files
themselves are written with the library's writer so that the reference's
own file globbing and selection run on them.  Everything else is the
reference's code: read_mayo_geometry, choose_files, load_projection_stack,
normalize_angles, order_views, volume_z_center, detector_shift, to_hu,
make_projector (mayo.py) and make_source_pos, load_mayo_problem,
make_helical_projector (mayo_fdk.py), with the reference's
HelicalProjector3d (xrecon_C served by its C++ CPU kernels).

Recorded per case: the geometry, chosen file names, sinogram, angles, source
z and offsets, detector shifts, source_pos, the driver projector's options /
weight / filter, make_projector's options, and the SHA-256 of every written
file (pins the writer that the tests use to recreate the series).
"""
from __future__ import annotations

import hashlib
import importlib
import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
if not os.environ.get("XRECON_REFERENCE_ROOT"):
    sys.exit("set XRECON_REFERENCE_ROOT to the XRecon reference tree")
REF_ROOT = Path(os.environ["XRECON_REFERENCE_ROOT"])
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

import mayo_series as MS  # noqa: E402
from oracle import refcpu  # noqa: E402

_REGISTRY: dict = {}


class _Value:
    def __init__(self, v):
        self.value = v


class _Dataset:
    """What the reference's loader touches of a pydicom Dataset."""

    def __init__(self, tags, pixels, rescale):
        self._tags = tags
        self._pixels = pixels
        self.RescaleSlope, self.RescaleIntercept = rescale

    def __contains__(self, tag):
        return tuple(tag) in self._tags

    def __getitem__(self, tag):
        return _Value(self._tags[tuple(tag)])

    @property
    def pixel_array(self):
        return self._pixels.copy()


def _dcmread(path, stop_before_pixels=False):
    return _REGISTRY[str(Path(path).resolve())]


def import_reference():
    stub = types.ModuleType("pydicom")
    stub.dcmread = _dcmread
    sys.modules["pydicom"] = stub
    sys.modules["xrecon_C"] = refcpu.RefXreconC()
    sys.path.insert(0, str(REF_ROOT))
    rmayo = importlib.import_module("xrecon.utils.mayo")
    rfdk = importlib.import_module("xrecon.utils.mayo_fdk")
    return rmayo, rfdk


def _digest(p: Path) -> str:
    return hashlib.sha256(p.read_bytes()).hexdigest()


def run_case(rmayo, rfdk, case: str, out: dict, tmp: Path) -> None:
    root = tmp / case
    paths = MS.write_series(root, case)
    geometry, views = MS.series(case)
    for p, v in zip(paths, views):
        _REGISTRY[str(p.resolve())] = _Dataset(*MS.pydicom_view(case, geometry, v))
    out[f"{case}_sha256"] = np.array([_digest(p) for p in paths])

    # driver settings: the reference's defaults, then the case's
    defaults = {name: getattr(rfdk, name) for name in MS.DRIVER_NAMES.values()}
    for field, value in MS.CASES[case]["config"].items():
        setattr(rfdk, MS.DRIVER_NAMES[field], value)
    rfdk.DATA_DIR = root
    rfdk.FILE_PATTERN = "*.dcm"
    try:
        g, chosen, sino, angles, sz, shz, sha, shr, binshift = rfdk.load_mayo_problem()
        out[f"{case}_geometry_num"] = np.array([g.num_det_col, g.num_det_row, g.det_col_size, g.det_row_size,
                                                g.iso_source, g.source_detector, g.det_center_col,
                                                g.det_center_row, g.views_per_rotation,
                                                np.nan if g.water_mu is None else g.water_mu], np.float64)
        out[f"{case}_geometry_text"] = np.array([g.detector_type, g.trajectory, g.beam_type])
        out[f"{case}_files"] = np.array([Path(p).name for p in chosen])
        for k, a in (("sino", sino), ("angles", angles), ("source_z", sz), ("shift_z", shz),
                     ("shift_angle", sha), ("shift_radius", shr)):
            out[f"{case}_{k}"] = np.asarray(a)
        out[f"{case}_binshift"] = np.array(binshift, np.float64)
        sp = rfdk.make_source_pos(sz, shz, sha, shr, torch.device("cpu"))
        out[f"{case}_source_pos"] = sp.numpy()
        P = rfdk.make_helical_projector(g, sino.shape, binshift, torch.device("cpu"))
        out[f"{case}_proj_options"] = P.options.numpy()
        out[f"{case}_proj_weight"] = P.weight.numpy()
        out[f"{case}_proj_filter"] = P.filter.numpy()
        # the reference's pipeline in mayo.py alone (no driver): stack, unwrap,
        # order, the other z-centre modes, make_projector
        files = rmayo._dicom_files(root, "*.dcm")
        stack = rmayo.load_projection_stack(files[:7], 1, 1)
        out[f"{case}_stack7_sino"] = stack[0]
        out[f"{case}_stack7_angles"] = stack[1]
        un = rmayo.normalize_angles(stack[1])
        out[f"{case}_stack7_unwrapped"] = un
        dec = rmayo.order_views(*(stack[0], un) + tuple(stack[2:]), "decreasing")
        out[f"{case}_stack7_decreasing_angles"] = dec[1]
        out[f"{case}_stack7_decreasing_sino"] = dec[0]
        out[f"{case}_zc"] = np.array([rmayo.volume_z_center(stack[2], m, None) for m in ("mean", "middle", "first")])
        args = types.SimpleNamespace(image_size=16, num_slices=4, pixel_size=1.5, slice_spacing=2.0,
                                     det_col_stride=1, det_row_stride=2, volume_z_shift=1.0, filter="shepplogan")
        Q = rmayo.make_projector(args, g, sino.shape[2], sino.shape[1], binshift)
        out[f"{case}_make_projector_options"] = Q.options.numpy()
        out[f"{case}_make_projector_filter"] = Q.filter.numpy()
    finally:
        for name, value in defaults.items():
            setattr(rfdk, name, value)


def helpers(rmayo, out: dict) -> None:
    """Stand-alone helpers on fixed inputs."""
    ds = []
    for center, count, stride, origin, start in ((368.625, 736, 1, 1.0, 0), (368.625, 368, 2, 1.0, 0),
                                                 (32.5, 64, 1, 0.0, 0), (40.25, 32, 2, 1.0, 8),
                                                 (12.0, 7, 3, 0.5, 1)):
        ds.append(rmayo.detector_shift(center, count, stride, origin, start))
    out["helper_detector_shift"] = np.array(ds, np.float64)
    sel = []
    for first, num, stride in ((1, 0, 1), (3, 5, 2), (10, 100, 3), (17, 1, 1), (1, 4, 7)):
        sel.append(",".join(str(i) for i in rmayo.choose_files(list(range(20)), first, num, stride)))
    out["helper_choose_files"] = np.array(sel)
    rec = np.linspace(-0.01, 0.04, 11, dtype=np.float32)
    out["helper_to_hu"] = np.stack([rmayo.to_hu(rec, 0.0192, False), rmayo.to_hu(rec, 0.0192, True),
                                    rmayo.to_hu(rec, None, False), rmayo.to_hu(rec, -1.0, False)])


def main() -> None:
    rmayo, rfdk = import_reference()
    out: dict = {}
    with tempfile.TemporaryDirectory() as d:
        for case in MS.CASES:
            run_case(rmayo, rfdk, case, out, Path(d))
    helpers(rmayo, out)
    np.savez_compressed(HERE / "mayo_ref.npz", **out)
    print("mayo fixtures written to", HERE / "mayo_ref.npz")


if __name__ == "__main__":
    main()
