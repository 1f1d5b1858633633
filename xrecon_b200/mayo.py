"""DICOM-CT-PD (Mayo low-dose CT projection data) ingest for the helical
projector.

Same functions, arguments and results as the reference's
``xrecon/utils/mayo.py:21-300`` (tag table, ``MayoGeometry``,
``read_mayo_geometry``, ``choose_files``, ``detector_shift``,
``load_projection_stack``, ``normalize_angles``, ``order_views``,
``volume_z_center``, ``to_hu``, ``save_metadata_csv``, ``make_projector``),
plus the loading half of ``xrecon/utils/mayo_fdk.py:86-172``
(``make_source_pos``, ``load_mayo_problem``, ``make_helical_projector``,
``direct_fdk``) with its module-level settings gathered in
:class:`MayoFdkConfig`.  Files are parsed by :mod:`xrecon_b200.dicom` (the
reference calls pydicom).  The matplotlib previews of the reference
(``save_preview``, ``save_auto_preview``, ``save_projection_preview``) are
display code and are not provided.

Tag decoding follows the reference's rules for values stored as raw bytes
(implicit-VR files and private tags of VR UN/OB, which is how the
DICOM-CT-PD private tags reach the reference): a 4-byte value is one
little-endian float32, a 2-byte value one little-endian int16, a pair
two float32.  A value of an explicitly numeric VR (FL, FD, US, SS, UL, SL)
or a decimal string (DS, IS) is decoded by its VR.

:func:`write_projection_file` writes the inverse: one view of a DICOM-CT-PD
style file with these tags, for exporting projections and for synthetic
test series.
"""
from __future__ import annotations

import csv
from dataclasses import dataclass
from pathlib import Path
from typing import Iterable, Optional, Sequence, Tuple, Union

import numpy as np

from . import dicom

TAG_DET_DU = (0x7029, 0x1002)
TAG_DET_DV = (0x7029, 0x1006)
TAG_DET_TYPE = (0x7029, 0x100B)
TAG_NUM_ROWS = (0x7029, 0x1010)
TAG_NUM_COLS = (0x7029, 0x1011)
TAG_ANGLE = (0x7031, 0x1001)
TAG_SOURCE_Z = (0x7031, 0x1002)
TAG_SOD = (0x7031, 0x1003)
TAG_SDD = (0x7031, 0x1031)
TAG_DET_CENTER = (0x7031, 0x1033)
TAG_SOURCE_SHIFT_Z = (0x7033, 0x100B)
TAG_SOURCE_SHIFT_ANGLE = (0x7033, 0x100C)
TAG_SOURCE_SHIFT_RADIUS = (0x7033, 0x100D)
TAG_VIEWS_PER_ROT = (0x7033, 0x1013)
TAG_SCAN_TRAJECTORY = (0x7037, 0x1009)
TAG_BEAM_TYPE = (0x7037, 0x100A)
TAG_WATER_MU = (0x0018, 0x0061)

# VRs whose stored bytes the decoders below interpret themselves
_RAW_VRS = (None, "UN", "OB", "OW")


@dataclass(frozen=True)
class MayoGeometry:
    num_det_col: int
    num_det_row: int
    det_col_size: float
    det_row_size: float
    iso_source: float
    source_detector: float
    det_center_col: float
    det_center_row: float
    views_per_rotation: int
    detector_type: str
    trajectory: str
    beam_type: str
    water_mu: Optional[float]


def dicom_files(root: Union[str, Path], pattern: str) -> list:
    """Files under ``root`` matching ``pattern``, sorted by name
    (mayo.py:57-61); raises FileNotFoundError when none match."""
    root = Path(root)
    files = sorted(root.glob(pattern))
    if not files:
        raise FileNotFoundError(f"No DICOM files matched {root / pattern}")
    return files


_dicom_files = dicom_files


def _raw(ds: dicom.DicomFile, tag) -> bytes:
    el = ds[tag]
    if el.vr in _RAW_VRS:
        return el.raw
    return str(el.value).encode("ascii", errors="ignore")


def _float32(ds: dicom.DicomFile, tag, default: Optional[float] = None) -> float:
    """mayo.py:73-81: a 4-byte raw value is one float32; anything else is
    read as a number."""
    if tag not in ds:
        if default is None:
            raise KeyError(tag)
        return float(default)
    el = ds[tag]
    if el.vr in _RAW_VRS:
        if len(el.raw) == 4:
            return float(np.frombuffer(el.raw, dtype="<f4", count=1)[0])
        return float(el.raw)
    v = el.value
    if isinstance(v, list):
        raise ValueError(f"tag {tag} holds {len(v)} values, one expected")
    return float(v)


def _float32_pair(ds: dicom.DicomFile, tag) -> Tuple[float, float]:
    """mayo.py:84-89: two float32 values."""
    el = ds[tag]
    if el.vr in _RAW_VRS:
        values = np.frombuffer(el.raw, dtype="<f4", count=2)
    else:
        v = el.value
        values = np.asarray(v if isinstance(v, list) else [v], dtype=np.float64)
    if values.size != 2:
        raise ValueError(f"Expected two float32 values in tag {tag}")
    return float(values[0]), float(values[1])


def _int16(ds: dicom.DicomFile, tag) -> int:
    """mayo.py:92-96: a 2-byte raw value is one int16; anything else is
    read as an integer."""
    el = ds[tag]
    if el.vr in _RAW_VRS:
        if len(el.raw) == 2:
            return int(np.frombuffer(el.raw, dtype="<i2", count=1)[0])
        return int(el.raw)
    v = el.value
    if isinstance(v, list):
        raise ValueError(f"tag {tag} holds {len(v)} values, one expected")
    return int(v)


def _text(ds: dicom.DicomFile, tag, default: str = "") -> str:
    """mayo.py:99-102: the value as lower-case ASCII text without padding."""
    if tag not in ds:
        return default
    return _raw(ds, tag).rstrip(b"\x00 ").decode("ascii", errors="ignore").strip().lower()


def read_mayo_geometry(first_file: Union[str, Path]) -> MayoGeometry:
    """The scan geometry from one projection file (mayo.py:105-125)."""
    ds = dicom.dcmread(first_file, stop_before_pixels=True)
    det_center_col, det_center_row = _float32_pair(ds, TAG_DET_CENTER)
    water_mu = _float32(ds, TAG_WATER_MU, default=np.nan)
    if not np.isfinite(water_mu) or water_mu <= 0:
        water_mu = None
    return MayoGeometry(
        num_det_col=_int16(ds, TAG_NUM_COLS),
        num_det_row=_int16(ds, TAG_NUM_ROWS),
        det_col_size=_float32(ds, TAG_DET_DU),
        det_row_size=_float32(ds, TAG_DET_DV),
        iso_source=_float32(ds, TAG_SOD),
        source_detector=_float32(ds, TAG_SDD),
        det_center_col=det_center_col,
        det_center_row=det_center_row,
        views_per_rotation=_int16(ds, TAG_VIEWS_PER_ROT),
        detector_type=_text(ds, TAG_DET_TYPE, "cylindrical"),
        trajectory=_text(ds, TAG_SCAN_TRAJECTORY, "helical"),
        beam_type=_text(ds, TAG_BEAM_TYPE, "fanbeam"),
        water_mu=water_mu,
    )


def choose_files(files: Sequence, first_view: int, num_views: int, view_stride: int) -> list:
    """Views ``first_view`` (one-based), every ``view_stride``-th, at most
    ``num_views`` of them (all when <= 0) (mayo.py:128-136)."""
    if first_view < 1:
        raise ValueError("first-view is one-based and should be >= 1")
    start = first_view - 1
    stop = len(files) if num_views <= 0 else min(len(files), start + num_views * view_stride)
    chosen = list(files[start:stop:view_stride])
    if not chosen:
        raise ValueError("No views selected")
    return chosen


def detector_shift(center: float, count: int, stride: int, origin: float, start: int = 0) -> float:
    """Detector shift in bins, from the file's central element index with
    origin ``origin``, after taking every ``stride``-th element from
    ``start`` (mayo.py:139-142)."""
    new_center = (center - origin - start) / stride
    default_center = count / 2.0 - 0.5
    return -(new_center - default_center)


def _view(ds: dicom.DicomFile, det_col_stride: int, det_row_stride: int) -> np.ndarray:
    raw = ds.pixel_array.astype(np.float32)
    slope = float(ds.RescaleSlope) if dicom.RESCALE_SLOPE in ds else 1.0
    intercept = float(ds.RescaleIntercept) if dicom.RESCALE_INTERCEPT in ds else 0.0
    projection = raw * slope + intercept
    projection = projection[::det_col_stride, ::det_row_stride].T
    return np.ascontiguousarray(projection)


def _load_stack_native(files: Sequence, det_col_stride, det_row_stride, threads: Optional[int]):
    """The series through the library's multi-threaded reader
    (``xr_ctpd_load``); None when it does not take these files."""
    import ctypes
    import operator
    import os

    from . import _native
    try:
        cs, rs = operator.index(det_col_stride), operator.index(det_row_stride)
    except TypeError:
        return None
    if not files or cs < 1 or rs < 1:
        return None
    try:
        head = dicom.dcmread(files[0], stop_before_pixels=True)
    except (OSError, dicom.DicomError):
        return None
    rows = head[dicom.ROWS].value if dicom.ROWS in head else None
    cols = head[dicom.COLUMNS].value if dicom.COLUMNS in head else None
    if not (isinstance(rows, int) and isinstance(cols, int) and rows > 0 and cols > 0):
        return None
    n = len(files)
    sino = np.empty((n, -(-cols // rs), -(-rows // cs)), dtype=np.float32)
    views = np.empty((n, 5), dtype=np.float32)
    paths = (ctypes.c_char_p * n)(*[os.fsencode(str(p)) for p in files])
    failed = ctypes.c_int(-1)
    rc = _native.lib().xr_ctpd_load(paths, n, rows, cols, cs, rs, int(threads or 0), sino.ctypes.data,
                                    views.ctypes.data, ctypes.byref(failed))
    if rc != 0:
        return None
    return (sino,) + tuple(np.ascontiguousarray(views[:, k]) for k in range(5))


def load_projection_stack(files: Sequence, det_col_stride: int, det_row_stride: int,
                          threads: Optional[int] = None, native: bool = True):
    """sino [V, Nv, Nu] (rescaled pixel values, detector columns and rows
    strided, stored rows = detector columns transposed to the last axis),
    angles, source_z, source_shift_z, source_shift_angle,
    source_shift_radius [V] float32 (mayo.py:145-170).

    The files are read by the library's multi-threaded reader
    (``xr_ctpd_load``, ``threads`` workers, one per core by default); a
    series it does not take (deflated encoding, unusual tag forms) or
    ``native=False`` goes through :mod:`xrecon_b200.dicom` one file at a
    time.  Both give the same arrays, bit for bit, and the second raises
    the errors of a malformed series."""
    if native:
        out = _load_stack_native(files, det_col_stride, det_row_stride, threads)
        if out is not None:
            return out
    n = len(files)
    sinos = []
    angles = np.empty(n, dtype=np.float32)
    source_z = np.empty(n, dtype=np.float32)
    source_shift_z = np.empty(n, dtype=np.float32)
    source_shift_angle = np.empty(n, dtype=np.float32)
    source_shift_radius = np.empty(n, dtype=np.float32)
    for i, path in enumerate(files):
        ds = dicom.dcmread(path, stop_before_pixels=False)
        sinos.append(_view(ds, det_col_stride, det_row_stride))
        angles[i] = _float32(ds, TAG_ANGLE)
        source_z[i] = _float32(ds, TAG_SOURCE_Z)
        source_shift_z[i] = _float32(ds, TAG_SOURCE_SHIFT_Z, default=0.0)
        source_shift_angle[i] = _float32(ds, TAG_SOURCE_SHIFT_ANGLE, default=0.0)
        source_shift_radius[i] = _float32(ds, TAG_SOURCE_SHIFT_RADIUS, default=0.0)
    sino = np.stack(sinos, axis=0)
    return sino, angles, source_z, source_shift_z, source_shift_angle, source_shift_radius


def normalize_angles(angles: np.ndarray) -> np.ndarray:
    """Angles unwrapped in float64, returned as float32 (mayo.py:173-175)."""
    return np.ascontiguousarray(np.unwrap(angles.astype(np.float64)).astype(np.float32))


def order_views(sino, angles, source_z, source_shift_z, source_shift_angle, source_shift_radius, mode: str):
    """Reverse all per-view arrays when ``mode`` is "increasing" and the
    angles decrease, or "decreasing" and they increase; "dicom" keeps file
    order (mayo.py:178-202)."""
    mode = mode.lower()
    arrays = (sino, angles, source_z, source_shift_z, source_shift_angle, source_shift_radius)
    if mode == "dicom" or angles.size < 2:
        return arrays
    decreasing = angles[-1] < angles[0]
    if (mode == "increasing" and decreasing) or (mode == "decreasing" and not decreasing):
        return tuple(np.ascontiguousarray(a[::-1]) for a in arrays)
    return arrays


def volume_z_center(source_z: np.ndarray, mode: str, value: Optional[float]) -> float:
    """``value`` if given, else the mean, middle or first source z
    (mayo.py:205-215)."""
    if value is not None:
        return float(value)
    mode = mode.lower()
    if mode == "mean":
        return float(source_z.mean())
    if mode == "middle":
        return float(source_z[len(source_z) // 2])
    if mode == "first":
        return float(source_z[0])
    raise ValueError(f"Unsupported z-center mode: {mode}")


def to_hu(recon: np.ndarray, water_mu: Optional[float], force_raw: bool) -> np.ndarray:
    """Attenuation to Hounsfield units, 1000 (mu / mu_water - 1); unchanged
    without a positive water coefficient or with ``force_raw``
    (mayo.py:218-221)."""
    if force_raw or water_mu is None or water_mu <= 0:
        return recon
    return 1000.0 * (recon / water_mu - 1.0)


def save_metadata_csv(path: Union[str, Path], rows: Iterable[Tuple[str, object]]) -> None:
    """key,value rows in a CSV file (mayo.py:272-276)."""
    with Path(path).open("w", newline="", encoding="utf-8") as f:
        writer = csv.writer(f)
        writer.writerow(["key", "value"])
        writer.writerows(rows)


def make_projector(args, geometry: MayoGeometry, nu: int, nv: int, binshift: Tuple[float, float]):
    """The helical projector for a loaded series from command-line style
    ``args`` (image_size, num_slices, pixel_size, slice_spacing,
    det_col_stride, det_row_stride, volume_z_shift, filter)
    (mayo.py:279-299)."""
    from .projector import HelicalProjector3d
    image_size = (args.image_size, args.image_size, args.num_slices)
    pix_size = (args.pixel_size, args.pixel_size, args.slice_spacing)
    det_size = (geometry.det_col_size * args.det_col_stride, geometry.det_row_size * args.det_row_stride)
    return HelicalProjector3d(image_size, (nu, nv), pix_size, det_size, geometry.iso_source,
                              geometry.source_detector,
                              pixshift=(0.0, 0.0, args.volume_z_shift / args.slice_spacing), binshift=binshift,
                              scan_type="arc", pitch=0.0, z0=0.0, filter_type=args.filter)


# ---------------------------------------------------------------------------
# the loading half of the reference's Mayo FDK driver


@dataclass
class MayoFdkConfig:
    """The settings of the reference's Mayo FDK driver
    (mayo_fdk.py:22-83), with its defaults."""
    data_dir: Union[str, Path] = "data/mayo/full_DICOM-CT-PD"
    file_pattern: str = "*"
    first_view: int = 1000
    num_views: int = 6912
    view_stride: int = 1
    angle_order: str = "increasing"
    image_size: int = 512
    pixel_size: float = 0.68
    num_slices: int = 64
    slice_spacing: float = 1.0
    volume_z_shift: float = 0.0
    z_center_mode: str = "mean"
    z_center_value: Optional[float] = None
    det_col_stride: int = 1
    det_row_stride: int = 1
    detector_index_origin: float = 1.0
    binshift_u: Optional[float] = -1.625
    binshift_v: Optional[float] = -0.5
    flip_det_cols: bool = False
    flip_det_rows: bool = True
    use_source_shifts: bool = False
    smooth_source_z_for_fdk: bool = True
    filter_type: str = "cosine"
    direct_fdk_scale: float = 1.0
    helical_view_mode: str = "one_turn"
    helical_view_turns: float = 1.0
    helical_halfscan_coef: float = 1.0
    helical_weight_mode: str = "2d"
    helical_tang_k: float = 5.0
    helical_tang_blend: float = 0.0
    water_mu: float = 0.0192


def make_source_pos(source_z, source_shift_z, source_shift_angle, source_shift_radius, device):
    """source_pos [4, V] = (source_z, shift_radius, shift_angle, shift_z)
    (mayo_fdk.py:86-98)."""
    import torch
    rows = (source_z, source_shift_radius, source_shift_angle, source_shift_z)
    sp = torch.zeros((4, np.asarray(source_z).size), dtype=torch.float32)
    for i, r in enumerate(rows):
        sp[i] = torch.from_numpy(np.ascontiguousarray(r, dtype=np.float32))
    return sp.to(device).contiguous()


@dataclass
class MayoProblem:
    geometry: MayoGeometry
    files: list
    sino: np.ndarray
    angles: np.ndarray
    source_z: np.ndarray
    shift_z: np.ndarray
    shift_angle: np.ndarray
    shift_radius: np.ndarray
    binshift: Tuple[float, float]

    def __iter__(self):
        """Unpacks like the reference's 9-tuple."""
        return iter((self.geometry, self.files, self.sino, self.angles, self.source_z, self.shift_z,
                     self.shift_angle, self.shift_radius, self.binshift))


def load_mayo_problem(config: Optional[MayoFdkConfig] = None) -> MayoProblem:
    """Read, select, order, flip and centre a series (mayo_fdk.py:101-145):
    unwrapped angles in the requested order, detector rows/columns flipped
    as configured, source offsets zeroed unless used, source z relative to
    the volume centre and (by default) replaced by its least-squares line
    in the angle, detector shifts from the file or the configured values."""
    c = config or MayoFdkConfig()
    files = dicom_files(c.data_dir, c.file_pattern)
    geometry = read_mayo_geometry(files[0])
    chosen = choose_files(files, c.first_view, c.num_views, c.view_stride)
    sino, angles, source_z, shift_z, shift_angle, shift_radius = load_projection_stack(
        chosen, c.det_col_stride, c.det_row_stride)
    angles = normalize_angles(angles)
    reverse_files = False
    if c.angle_order != "dicom" and angles.size > 1:
        decreasing = angles[-1] < angles[0]
        reverse_files = (c.angle_order == "increasing" and decreasing) or (
            c.angle_order == "decreasing" and not decreasing)
    sino, angles, source_z, shift_z, shift_angle, shift_radius = order_views(
        sino, angles, source_z, shift_z, shift_angle, shift_radius, c.angle_order)
    if reverse_files:
        chosen = list(reversed(chosen))
    if c.flip_det_cols:
        sino = np.ascontiguousarray(sino[:, :, ::-1])
    if c.flip_det_rows:
        sino = np.ascontiguousarray(sino[:, ::-1, :])
    if not c.use_source_shifts:
        shift_z.fill(0.0)
        shift_angle.fill(0.0)
        shift_radius.fill(0.0)
    z_center = volume_z_center(source_z, c.z_center_mode, c.z_center_value)
    source_z = np.ascontiguousarray(source_z - z_center)
    if c.smooth_source_z_for_fdk and source_z.size > 1:
        slope, intercept = np.polyfit(angles.astype(np.float64), source_z.astype(np.float64), 1)
        source_z = np.ascontiguousarray((slope * angles + intercept).astype(np.float32))
    nv, nu = sino.shape[1:]
    binshift_u = detector_shift(geometry.det_center_col, nu, c.det_col_stride, c.detector_index_origin)
    binshift_v = detector_shift(geometry.det_center_row, nv, c.det_row_stride, c.detector_index_origin)
    if c.binshift_u is not None:
        binshift_u = float(c.binshift_u)
    if c.binshift_v is not None:
        binshift_v = float(c.binshift_v)
    return MayoProblem(geometry, chosen, sino, angles, source_z, shift_z, shift_angle, shift_radius,
                       (binshift_u, binshift_v))


def make_helical_projector(geometry: MayoGeometry, sino_shape, binshift, device,
                           config: Optional[MayoFdkConfig] = None):
    """The helical projector of the direct-FDK route (mayo_fdk.py:148-167)."""
    from .projector import HelicalProjector3d
    c = config or MayoFdkConfig()
    _, nv, nu = sino_shape
    return HelicalProjector3d(
        (c.image_size, c.image_size, c.num_slices), (nu, nv), (c.pixel_size, c.pixel_size, c.slice_spacing),
        (geometry.det_col_size * c.det_col_stride, geometry.det_row_size * c.det_row_stride),
        geometry.iso_source, geometry.source_detector, pixshift=(0.0, 0.0, c.volume_z_shift / c.slice_spacing),
        binshift=binshift, scan_type="arc", filter_type=c.filter_type, helical_view_mode=c.helical_view_mode,
        helical_view_turns=c.helical_view_turns, helical_halfscan_coef=c.helical_halfscan_coef,
        helical_weight_mode=c.helical_weight_mode, helical_tang_k=c.helical_tang_k,
        helical_tang_blend=c.helical_tang_blend).to(device)


def direct_fdk(projector, sino, angles, source_pos, config: Optional[MayoFdkConfig] = None):
    """Helical FDK of a loaded series, scaled (mayo_fdk.py:170-172)."""
    c = config or MayoFdkConfig()
    recon = projector.filtered_backprojection(sino, angles, source_pos, filter_type=c.filter_type)
    return recon * c.direct_fdk_scale


# ---------------------------------------------------------------------------
# writing projection files


def write_projection_file(path: Union[str, Path], geometry: MayoGeometry, pixels: np.ndarray, angle: float,
                          source_z: float, shift_z: float = 0.0, shift_angle: float = 0.0,
                          shift_radius: float = 0.0, slope: float = 1.0, intercept: float = 0.0,
                          transfer_syntax: str = dicom.IMPLICIT_LE, private_vr: Optional[str] = None,
                          omit: Sequence = ()) -> None:
    """One view as a DICOM-CT-PD style file: ``pixels`` [num_det_col,
    num_det_row] unsigned 16-bit stored values (the layout
    :func:`load_projection_stack` transposes), the tags read by
    :func:`read_mayo_geometry` and :func:`load_projection_stack`, and the
    rescale slope and intercept.  Private tags are written as raw
    little-endian bytes (VR ``private_vr``: None = implicit/UN, or "OB").
    Tags listed in ``omit`` are left out."""
    px = np.ascontiguousarray(pixels, dtype="<u2")
    if px.ndim != 2:
        raise ValueError("pixels should be [num_det_col, num_det_row]")
    pv = private_vr

    def f32(*v):
        return np.asarray(v, dtype="<f4").tobytes()

    def i16(v):
        return np.asarray([v], dtype="<i2").tobytes()

    def text(s):
        b = s.encode("ascii")
        return b + b" " if len(b) % 2 else b

    els = [
        ((0x0008, 0x0016), "UI", "1.2.840.10008.5.1.4.1.1.66"),
        ((0x0008, 0x0060), "CS", "CT"),
        ((0x0028, 0x0002), "US", 1),
        ((0x0028, 0x0004), "CS", "MONOCHROME2"),
        (dicom.ROWS, "US", px.shape[0]),
        (dicom.COLUMNS, "US", px.shape[1]),
        (dicom.BITS_ALLOCATED, "US", 16),
        (dicom.BITS_STORED, "US", 16),
        (dicom.HIGH_BIT, "US", 15),
        (dicom.PIXEL_REPRESENTATION, "US", 0),
        (dicom.RESCALE_INTERCEPT, "DS", float(intercept)),
        (dicom.RESCALE_SLOPE, "DS", float(slope)),
        ((0x7029, 0x0010), "LO", "DICOM-CT-PD"),
        ((0x7031, 0x0010), "LO", "DICOM-CT-PD"),
        ((0x7033, 0x0010), "LO", "DICOM-CT-PD"),
        ((0x7037, 0x0010), "LO", "DICOM-CT-PD"),
        (TAG_DET_DU, pv, f32(geometry.det_col_size)),
        (TAG_DET_DV, pv, f32(geometry.det_row_size)),
        (TAG_DET_TYPE, pv, text(geometry.detector_type.upper())),
        (TAG_NUM_ROWS, pv, i16(geometry.num_det_row)),
        (TAG_NUM_COLS, pv, i16(geometry.num_det_col)),
        (TAG_ANGLE, pv, f32(angle)),
        (TAG_SOURCE_Z, pv, f32(source_z)),
        (TAG_SOD, pv, f32(geometry.iso_source)),
        (TAG_SDD, pv, f32(geometry.source_detector)),
        (TAG_DET_CENTER, pv, f32(geometry.det_center_col, geometry.det_center_row)),
        (TAG_SOURCE_SHIFT_Z, pv, f32(shift_z)),
        (TAG_SOURCE_SHIFT_ANGLE, pv, f32(shift_angle)),
        (TAG_SOURCE_SHIFT_RADIUS, pv, f32(shift_radius)),
        (TAG_VIEWS_PER_ROT, pv, i16(geometry.views_per_rotation)),
        (TAG_SCAN_TRAJECTORY, pv, text(geometry.trajectory.upper())),
        (TAG_BEAM_TYPE, pv, text(geometry.beam_type.upper())),
        (dicom.PIXEL_DATA, "OW", px.tobytes()),
    ]
    if geometry.water_mu is not None:
        els.append((TAG_WATER_MU, pv, f32(geometry.water_mu)))
    skip = {tuple(t) for t in omit}
    dicom.write(path, [e for e in els if e[0] not in skip], transfer_syntax)
