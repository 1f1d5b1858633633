"""Seeded synthetic DICOM-CT-PD projection series for the Mayo ingest tests.

``series(case)`` gives the scan geometry and the per-view values (angle,
source z, focal-spot offsets, rescale, stored pixels); ``write_series``
writes them as files with ``xrecon_b200.mayo.write_projection_file``;
``pydicom_view`` gives the same view as pydicom presents an implicit-VR
file to the reference's loader (private tags, and the water coefficient
tag, as the raw little-endian bytes of their values; pixel-module tags
decoded; RescaleSlope / RescaleIntercept as numbers).  The byte layout is
built here with ``struct``, independently of the library's writer.

Angles are stored modulo 2 pi, as a scanner stores them, so unwrapping is
exercised; the source rises by ``pitch`` per turn with seeded jitter.
"""
from __future__ import annotations

import math
import struct
from pathlib import Path

import numpy as np

CASES = {
    # increasing angles across the 2 pi wrap; default driver settings
    "increasing": dict(views=40, per_turn=24, start=2 * math.pi - 0.9, sign=+1.0, nu=24, nv=6,
                       slope=0.25, intercept=-3.0, det_center=(12.875, 3.5), pitch=6.0, z0=-40.0,
                       water_mu=0.0192, omit=(), seed=1,
                       config=dict(first_view=3, num_views=30, image_size=32, num_slices=8, pixel_size=0.9,
                                   slice_spacing=1.25)),
    # decreasing angles reordered to increasing, every second view, every
    # second detector column, columns flipped, source offsets used, shifts
    # from the file, z centre at the middle view, no source-z smoothing
    "decreasing": dict(views=33, per_turn=16, start=0.4, sign=-1.0, nu=24, nv=6,
                       slope=0.0005, intercept=0.0, det_center=(13.25, 3.75), pitch=5.0, z0=10.0,
                       water_mu=0.0187, omit=(), seed=2,
                       config=dict(first_view=1, num_views=0, view_stride=2, det_col_stride=2,
                                   flip_det_cols=True, flip_det_rows=False, use_source_shifts=True,
                                   smooth_source_z_for_fdk=False, z_center_mode="middle", binshift_u=None,
                                   binshift_v=None, image_size=24, num_slices=6, pixel_size=1.1,
                                   slice_spacing=1.0, helical_view_mode="auto", helical_weight_mode="tang3d",
                                   filter_type="hann")),
    # file order kept, z centre given, rows strided, optional tags absent
    # (water coefficient, trajectory, beam type, source offsets)
    "dicom_order": dict(views=20, per_turn=12, start=1.0, sign=+1.0, nu=20, nv=8,
                        slope=1.0, intercept=0.0, det_center=(10.5, 4.5), pitch=4.0, z0=0.0,
                        water_mu=None, seed=3,
                        omit=((0x7037, 0x1009), (0x7037, 0x100A), (0x7033, 0x100B), (0x7033, 0x100C),
                              (0x7033, 0x100D)),
                        config=dict(first_view=2, num_views=15, angle_order="dicom", z_center_value=2.5,
                                    det_row_stride=2, detector_index_origin=0.0, image_size=20, num_slices=4,
                                    pixel_size=1.0, slice_spacing=2.0, helical_view_mode="half",
                                    filter_type="ramp")),
}

# the reference driver's module-level names for MayoFdkConfig fields
DRIVER_NAMES = {
    "first_view": "FIRST_VIEW", "num_views": "NUM_VIEWS", "view_stride": "VIEW_STRIDE",
    "angle_order": "ANGLE_ORDER", "image_size": "IMAGE_SIZE", "pixel_size": "PIXEL_SIZE",
    "num_slices": "NUM_SLICES", "slice_spacing": "SLICE_SPACING", "volume_z_shift": "VOLUME_Z_SHIFT",
    "z_center_mode": "Z_CENTER_MODE", "z_center_value": "Z_CENTER_VALUE", "det_col_stride": "DET_COL_STRIDE",
    "det_row_stride": "DET_ROW_STRIDE", "detector_index_origin": "DETECTOR_INDEX_ORIGIN",
    "binshift_u": "BINSHIFT_U", "binshift_v": "BINSHIFT_V", "flip_det_cols": "FLIP_DET_COLS",
    "flip_det_rows": "FLIP_DET_ROWS", "use_source_shifts": "USE_SOURCE_SHIFTS",
    "smooth_source_z_for_fdk": "SMOOTH_SOURCE_Z_FOR_FDK", "filter_type": "FILTER_TYPE",
    "direct_fdk_scale": "DIRECT_FDK_SCALE", "helical_view_mode": "HELICAL_VIEW_MODE",
    "helical_view_turns": "HELICAL_VIEW_TURNS", "helical_halfscan_coef": "HELICAL_HALFSCAN_COEF",
    "helical_weight_mode": "HELICAL_WEIGHT_MODE", "helical_tang_k": "HELICAL_TANG_K",
    "helical_tang_blend": "HELICAL_TANG_BLEND",
}


def series(case: str):
    """(geometry, views): the MayoGeometry written to every file and one
    dict per view (angle, source_z, shift_z, shift_angle, shift_radius,
    slope, intercept, pixels [num_det_col, num_det_row] uint16)."""
    from xrecon_b200.mayo import MayoGeometry
    c = CASES[case]
    rng = np.random.default_rng(c["seed"])
    V, nu, nv = c["views"], c["nu"], c["nv"]
    geometry = MayoGeometry(num_det_col=nu, num_det_row=nv, det_col_size=1.2858, det_row_size=1.0947,
                            iso_source=595.0, source_detector=1085.6, det_center_col=c["det_center"][0],
                            det_center_row=c["det_center"][1], views_per_rotation=c["per_turn"],
                            detector_type="cylindrical", trajectory="helical", beam_type="fanbeam",
                            water_mu=c["water_mu"])
    k = np.arange(V, dtype=np.float64)
    ang = np.mod(c["start"] + c["sign"] * k * (2 * math.pi / c["per_turn"]), 2 * math.pi).astype(np.float32)
    sz = (c["z0"] + k * c["pitch"] / c["per_turn"] + rng.normal(0.0, 0.01, V)).astype(np.float32)
    shz = rng.normal(0.0, 0.3, V).astype(np.float32)
    sha = rng.normal(0.0, 5e-4, V).astype(np.float32)
    shr = rng.normal(0.0, 1.0, V).astype(np.float32)
    pixels = rng.integers(0, 4096, (V, nu, nv), dtype=np.uint16)
    views = [dict(angle=float(ang[i]), source_z=float(sz[i]), shift_z=float(shz[i]), shift_angle=float(sha[i]),
                  shift_radius=float(shr[i]), slope=c["slope"], intercept=c["intercept"], pixels=pixels[i])
             for i in range(V)]
    return geometry, views


def file_name(i: int) -> str:
    return f"proj_{i:05d}.dcm"


def write_series(root: Path, case: str, transfer_syntax=None, private_vr=None) -> list:
    """Write the series as files root/proj_00000.dcm ...; returns the paths."""
    from xrecon_b200 import dicom, mayo
    geometry, views = series(case)
    root = Path(root)
    root.mkdir(parents=True, exist_ok=True)
    paths = []
    for i, v in enumerate(views):
        p = root / file_name(i)
        mayo.write_projection_file(p, geometry, v["pixels"], v["angle"], v["source_z"], v["shift_z"],
                                   v["shift_angle"], v["shift_radius"], v["slope"], v["intercept"],
                                   transfer_syntax=transfer_syntax or dicom.IMPLICIT_LE,
                                   private_vr=private_vr, omit=CASES[case]["omit"])
        paths.append(p)
    return paths


def _f32(*v) -> bytes:
    return struct.pack("<" + "f" * len(v), *v)


def _i16(v) -> bytes:
    return struct.pack("<h", v)


def _text(s: str) -> bytes:
    b = s.upper().encode("ascii")
    return b + b" " if len(b) % 2 else b


def pydicom_view(case: str, geometry, view) -> tuple:
    """(tags, pixels, rescale): the view as pydicom presents an implicit-VR
    file to the reference, tags keyed by (group, element)."""
    g = geometry
    tags = {
        (0x7029, 0x1002): _f32(g.det_col_size), (0x7029, 0x1006): _f32(g.det_row_size),
        (0x7029, 0x100B): _text(g.detector_type), (0x7029, 0x1010): _i16(g.num_det_row),
        (0x7029, 0x1011): _i16(g.num_det_col), (0x7031, 0x1001): _f32(view["angle"]),
        (0x7031, 0x1002): _f32(view["source_z"]), (0x7031, 0x1003): _f32(g.iso_source),
        (0x7031, 0x1031): _f32(g.source_detector), (0x7031, 0x1033): _f32(g.det_center_col, g.det_center_row),
        (0x7033, 0x100B): _f32(view["shift_z"]), (0x7033, 0x100C): _f32(view["shift_angle"]),
        (0x7033, 0x100D): _f32(view["shift_radius"]), (0x7033, 0x1013): _i16(g.views_per_rotation),
        (0x7037, 0x1009): _text(g.trajectory), (0x7037, 0x100A): _text(g.beam_type),
        (0x0028, 0x0010): int(view["pixels"].shape[0]), (0x0028, 0x0011): int(view["pixels"].shape[1]),
    }
    if g.water_mu is not None:
        tags[(0x0018, 0x0061)] = _f32(g.water_mu)
    for t in CASES[case]["omit"]:
        tags.pop(tuple(t), None)
    return tags, view["pixels"].copy(), (float(view["slope"]), float(view["intercept"]))
