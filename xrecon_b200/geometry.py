"""Scan geometry descriptions, API-compatible with ``xrecon.projector.geometry``
(XRecon xrecon/projector/geometry.py:28-270).

The public names, fields and derived quantities are kept identical so user
code constructing ``Volume3d(...)``/``ConeBeam3d(...)`` works unchanged:

* ``effective_det_spacing`` -- 2D flat ``du*SOD/SDD``, 2D arc
  ``2*atan(du/(2*SDD))`` (geometry.py:105-109); 3D flat ``du*SOD/SDD``, 3D
  arc ``du/SDD`` (geometry.py:198-203);
* ``effective_det_shift`` -- the bin shift times the effective spacing;
* ``scan_id`` -- 0 parallel, 1 flat, 2 arc.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Tuple, Union

Number = Union[int, float]


def _pair(value, name: str) -> Tuple[Number, Number]:
    if isinstance(value, (tuple, list)):
        if len(value) != 2:
            raise ValueError(f"{name} should be a scalar or a 2-tuple/list")
        return value[0], value[1]
    return value, value


def _triple(value, name: str) -> Tuple[Number, Number, Number]:
    if isinstance(value, (tuple, list)):
        if len(value) != 3:
            raise ValueError(f"{name} should be a scalar or a 3-tuple/list")
        return value[0], value[1], value[2]
    return value, value, value


def _freeze(obj, **fields):
    for k, v in fields.items():
        object.__setattr__(obj, k, v)


@dataclass(frozen=True, init=False)
class Volume2d:
    """Image grid: ``size`` (W, H) in pixels, ``spacing`` (dx, dy) in mm,
    ``shift`` in pixels."""
    size: Tuple[int, int]
    spacing: Tuple[float, float]
    shift: Tuple[float, float]

    def __init__(self, size, spacing, shift=0.0) -> None:
        w, h = _pair(size, "size")
        dx, dy = _pair(spacing, "spacing")
        sx, sy = _pair(shift, "shift")
        _freeze(self, size=(int(w), int(h)), spacing=(float(dx), float(dy)), shift=(float(sx), float(sy)))


@dataclass(frozen=True, init=False)
class Detector2d:
    """Linear detector: ``count`` bins of ``spacing`` mm, ``shift`` in bins."""
    count: int
    spacing: float
    shift: float

    def __init__(self, count: int, spacing: float, shift: float = 0.0) -> None:
        _freeze(self, count=int(count), spacing=float(spacing), shift=float(shift))


@dataclass(frozen=True)
class ParallelBeam2d:
    detector: Detector2d
    scan_type: str = "parallel"
    iso_source: float = 0.0
    source_detector: float = 0.0

    @property
    def scan_id(self) -> int:
        return 0

    @property
    def effective_det_spacing(self) -> float:
        return self.detector.spacing

    @property
    def effective_det_shift(self) -> float:
        return self.detector.shift * self.effective_det_spacing


@dataclass(frozen=True, init=False)
class FanBeam2d:
    detector: Detector2d
    iso_source: float
    source_detector: float
    detector_type: str

    def __init__(self, detector: Detector2d, iso_source: float, source_detector: float,
                 detector_type: str = "flat") -> None:
        kind = detector_type.lower().strip()
        if kind not in ("flat", "arc"):
            raise ValueError("detector_type should be 'flat' or 'arc'")
        _freeze(self, detector=detector, iso_source=float(iso_source),
                source_detector=float(source_detector), detector_type=kind)

    @property
    def scan_type(self) -> str:
        return self.detector_type

    @property
    def scan_id(self) -> int:
        return 1 if self.detector_type == "flat" else 2

    @property
    def effective_det_spacing(self) -> float:
        du = self.detector.spacing
        if self.detector_type == "flat":
            return du * self.iso_source / self.source_detector
        return 2.0 * math.atan(du / self.source_detector / 2.0)

    @property
    def effective_det_shift(self) -> float:
        return self.detector.shift * self.effective_det_spacing


Geometry2d = Union[ParallelBeam2d, FanBeam2d]


def make_geometry2d(scan_type: str, num_det: int, det_size: float, iso_source: float,
                    source_detector: float, binshift: float = 0.0) -> Geometry2d:
    kind = scan_type.lower().strip()
    kind = "parallel" if kind == "para" else kind
    det = Detector2d(num_det, det_size, binshift)
    if kind == "parallel":
        return ParallelBeam2d(det)
    if kind in ("flat", "arc"):
        return FanBeam2d(det, iso_source, source_detector, kind)
    raise ValueError(f"Unsupported scan_type: {scan_type}")


@dataclass(frozen=True, init=False)
class Volume3d:
    """Volume grid: ``size`` (W, H, D) voxels, ``spacing`` (dx, dy, dz) mm,
    ``shift`` in voxels."""
    size: Tuple[int, int, int]
    spacing: Tuple[float, float, float]
    shift: Tuple[float, float, float]

    def __init__(self, size, spacing, shift=0.0) -> None:
        w, h, d = _triple(size, "size")
        dx, dy, dz = _triple(spacing, "spacing")
        sx, sy, sz = _triple(shift, "shift")
        _freeze(self, size=(int(w), int(h), int(d)), spacing=(float(dx), float(dy), float(dz)),
                shift=(float(sx), float(sy), float(sz)))


@dataclass(frozen=True, init=False)
class Detector3d:
    """Area detector: ``count`` (Nu, Nv), ``spacing`` (du, dv) mm, ``shift``
    in bins."""
    count: Tuple[int, int]
    spacing: Tuple[float, float]
    shift: Tuple[float, float]

    def __init__(self, count, spacing, shift=0.0) -> None:
        nu, nv = _pair(count, "count")
        du, dv = _pair(spacing, "spacing")
        su, sv = _pair(shift, "shift")
        _freeze(self, count=(int(nu), int(nv)), spacing=(float(du), float(dv)), shift=(float(su), float(sv)))


@dataclass(frozen=True, init=False)
class ConeBeam3d:
    detector: Detector3d
    iso_source: float
    source_detector: float
    detector_type: str

    def __init__(self, detector: Detector3d, iso_source: float, source_detector: float,
                 detector_type: str = "flat") -> None:
        kind = detector_type.lower().strip()
        if kind not in ("flat", "arc"):
            raise ValueError("detector_type should be 'flat' or 'arc'")
        _freeze(self, detector=detector, iso_source=float(iso_source),
                source_detector=float(source_detector), detector_type=kind)

    @property
    def scan_type(self) -> str:
        return self.detector_type

    @property
    def scan_id(self) -> int:
        return 1 if self.detector_type == "flat" else 2

    @property
    def effective_det_spacing(self) -> Tuple[float, float]:
        du, dv = self.detector.spacing
        if self.detector_type == "flat":
            return du * self.iso_source / self.source_detector, dv
        return du / self.source_detector, dv

    @property
    def effective_det_shift(self) -> Tuple[float, float]:
        du, dv = self.effective_det_spacing
        su, sv = self.detector.shift
        return su * du, sv * dv


@dataclass(frozen=True)
class ParallelBeam3d:
    detector: Detector3d
    scan_type: str = "parallel"

    @property
    def scan_id(self) -> int:
        return 0

    @property
    def effective_det_spacing(self) -> Tuple[float, float]:
        return self.detector.spacing

    @property
    def effective_det_shift(self) -> Tuple[float, float]:
        du, dv = self.detector.spacing
        su, sv = self.detector.shift
        return su * du, sv * dv


@dataclass(frozen=True, init=False)
class HelicalConeBeam3d(ConeBeam3d):
    """Helical trajectory: cone-beam geometry plus the source's rise per turn
    (``pitch``) and its z at the first view (``z0``), as the reference's
    geometry.py:233-248; used by :class:`~xrecon_b200.HelicalProjector3d`."""
    pitch: float
    z0: float

    def __init__(self, detector: Detector3d, iso_source: float, source_detector: float,
                 detector_type: str = "arc", pitch: float = 0.0, z0: float = 0.0) -> None:
        super().__init__(detector, iso_source, source_detector, detector_type)
        _freeze(self, pitch=float(pitch), z0=float(z0))


Geometry3d = Union[ParallelBeam3d, ConeBeam3d, HelicalConeBeam3d]


def make_geometry3d(scan_type: str, num_det, det_size, iso_source: float, source_detector: float,
                    binshift=0.0) -> Geometry3d:
    kind = scan_type.lower().strip()
    kind = "parallel" if kind == "para" else kind
    det = Detector3d(num_det, det_size, binshift)
    if kind == "parallel":
        return ParallelBeam3d(det)
    if kind in ("flat", "arc"):
        return ConeBeam3d(det, iso_source, source_detector, kind)
    raise ValueError(f"Unsupported 3D scan_type: {scan_type}")


def pack_options2d(volume: Volume2d, geometry: Geometry2d) -> list:
    """The 12 packed options of Projector2d (projector.py:97-110):
    [W, H, Nu, dx, dy, du_eff, SOD, SDD, shift_x mm, shift_y mm, shift_u_eff, scan_id]."""
    W, H = volume.size
    dx, dy = volume.spacing
    shx, shy = volume.shift
    return [W, H, geometry.detector.count, dx, dy, geometry.effective_det_spacing,
            float(geometry.iso_source), float(geometry.source_detector), shx * dx, shy * dy,
            geometry.effective_det_shift, geometry.scan_id]


def pack_options3d(volume: Volume3d, geometry: Geometry3d) -> list:
    """The 18 packed options of Projector3d (projector3d.py:73-107).  Flat
    detectors pass the raw du and raw shift (mm) and the kernels scale by
    SOD/SDD; arc detectors pass du/SDD (rad); parallel the raw values."""
    W, H, D = volume.size
    dx, dy, dz = volume.spacing
    shx, shy, shz = volume.shift
    Nu, Nv = geometry.detector.count
    raw_du, raw_dv = geometry.detector.spacing
    raw_shu, raw_shv = geometry.detector.shift
    shu_eff, _ = geometry.effective_det_shift
    du_eff, _ = geometry.effective_det_spacing
    scan = geometry.scan_type.lower()
    kernel_du = raw_du if scan == "flat" else du_eff
    kernel_shu = raw_shu * raw_du if scan == "flat" else shu_eff
    return [W, H, D, Nu, Nv, dx, dy, dz, kernel_du, raw_dv,
            float(getattr(geometry, "iso_source", 0.0)), float(getattr(geometry, "source_detector", 0.0)),
            shx * dx, shy * dy, shz * dz, kernel_shu, raw_shv * raw_dv, geometry.scan_id]
