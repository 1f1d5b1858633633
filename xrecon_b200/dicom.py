"""Minimal DICOM Part 10 reader and writer for projection files.

Reads what a DICOM-CT-PD projection file holds (the format of the Mayo
low-dose CT projection data): the 128-byte preamble and ``DICM`` prefix, the
file meta group (always explicit VR little endian), then a data set in
implicit VR little endian, explicit VR little endian or deflated explicit VR
little endian, with native (uncompressed) pixel data.  Sequences of defined
and undefined length, and undefined-length UN elements, are walked and kept
as raw bytes.  Big-endian and encapsulated (compressed) transfer syntaxes
raise ``DicomError``.

This stands in for the ``pydicom.dcmread`` calls of the reference's
``xrecon/utils/mayo.py:106,157``: every element keeps the bytes of its value
as stored, so the reader of a private tag decides how to decode it, exactly
as the reference does with the bytes pydicom hands it for private tags it
has no dictionary entry for.  Standard tags that the projection loader needs
(image size, bits, rescale) carry their VR even in implicit-VR files.

The layout rules followed are those of DICOM PS3.10 §7 (file format) and
PS3.5 §7 (data element encoding), §7.5 (sequences and items), §8 (pixel
data) and §A (transfer syntaxes).
"""
from __future__ import annotations

import hashlib
import struct
import zlib
from dataclasses import dataclass
from pathlib import Path
from typing import Dict, Iterable, Iterator, Optional, Tuple, Union

import numpy as np

Tag = Tuple[int, int]

IMPLICIT_LE = "1.2.840.10008.1.2"
EXPLICIT_LE = "1.2.840.10008.1.2.1"
DEFLATED_LE = "1.2.840.10008.1.2.1.99"
EXPLICIT_BE = "1.2.840.10008.1.2.2"

# VRs whose explicit encoding has two reserved bytes and a 32-bit length
_LONG_VRS = frozenset({"OB", "OD", "OF", "OL", "OV", "OW", "SQ", "SV", "UC", "UN", "UR", "UT", "UV"})
_TEXT_VRS = frozenset({"AE", "AS", "CS", "DA", "DS", "DT", "IS", "LO", "LT", "PN", "SH", "ST", "TM", "UC",
                       "UI", "UR", "UT"})
_NUMERIC = {"US": "<u2", "SS": "<i2", "UL": "<u4", "SL": "<i4", "FL": "<f4", "FD": "<f8", "UV": "<u8",
            "SV": "<i8", "OF": "<f4", "OD": "<f8", "OL": "<u4"}
_UNDEFINED = 0xFFFFFFFF
_ITEM = (0xFFFE, 0xE000)
_ITEM_END = (0xFFFE, 0xE00D)
_SEQ_END = (0xFFFE, 0xE0DD)

PIXEL_DATA = (0x7FE0, 0x0010)
ROWS = (0x0028, 0x0010)
COLUMNS = (0x0028, 0x0011)
SAMPLES_PER_PIXEL = (0x0028, 0x0002)
NUMBER_OF_FRAMES = (0x0028, 0x0008)
BITS_ALLOCATED = (0x0028, 0x0100)
BITS_STORED = (0x0028, 0x0101)
HIGH_BIT = (0x0028, 0x0102)
PIXEL_REPRESENTATION = (0x0028, 0x0103)
RESCALE_INTERCEPT = (0x0028, 0x1052)
RESCALE_SLOPE = (0x0028, 0x1053)
TRANSFER_SYNTAX = (0x0002, 0x0010)

# VRs of the standard tags that are read by value in implicit-VR data sets
# (the DICOM data dictionary, PS3.6); every other implicit-VR element keeps
# VR None and its raw bytes.
_IMPLICIT_VR = {
    ROWS: "US", COLUMNS: "US", SAMPLES_PER_PIXEL: "US", NUMBER_OF_FRAMES: "IS", BITS_ALLOCATED: "US",
    BITS_STORED: "US", HIGH_BIT: "US", PIXEL_REPRESENTATION: "US", RESCALE_INTERCEPT: "DS",
    RESCALE_SLOPE: "DS", PIXEL_DATA: "OW", (0x0008, 0x0016): "UI", (0x0008, 0x0018): "UI",
    (0x0008, 0x0060): "CS", (0x0028, 0x0004): "CS",
}

# keyword access used by the projection loader (``ds.RescaleSlope``)
_KEYWORDS = {"Rows": ROWS, "Columns": COLUMNS, "SamplesPerPixel": SAMPLES_PER_PIXEL,
             "NumberOfFrames": NUMBER_OF_FRAMES, "BitsAllocated": BITS_ALLOCATED, "BitsStored": BITS_STORED,
             "HighBit": HIGH_BIT, "PixelRepresentation": PIXEL_REPRESENTATION,
             "RescaleIntercept": RESCALE_INTERCEPT, "RescaleSlope": RESCALE_SLOPE}


class DicomError(ValueError):
    """A file that is not DICOM Part 10, is truncated, or uses an encoding
    this reader does not decode."""


@dataclass(frozen=True)
class Element:
    """One data element: its tag, VR (None for an implicit-VR element the
    reader has no dictionary entry for) and the bytes of its value as stored
    (for a sequence, the bytes of all its items)."""
    tag: Tag
    vr: Optional[str]
    raw: bytes

    @property
    def value(self):
        """The decoded value: numbers for numeric VRs (a scalar for one
        value, a list for several), text for string VRs (DS and IS as
        numbers), the raw bytes otherwise (OB, OW, UN, SQ and unknown)."""
        return decode_value(self.vr, self.raw)


def decode_value(vr: Optional[str], raw: bytes):
    if vr in _NUMERIC:
        dt = np.dtype(_NUMERIC[vr])
        n = len(raw) // dt.itemsize
        vals = np.frombuffer(raw, dtype=dt, count=n).tolist()
        return vals[0] if n == 1 else vals
    if vr in ("DS", "IS"):
        parts = [p.strip(" \x00") for p in raw.decode("ascii", errors="replace").split("\\")]
        conv = float if vr == "DS" else int
        vals = [conv(p) for p in parts if p]
        if not vals:
            return None
        return vals[0] if len(vals) == 1 else vals
    if vr in _TEXT_VRS:
        text = raw.decode("latin-1").rstrip(" \x00")
        return text.split("\\") if "\\" in text and vr not in ("LT", "ST", "UT", "UR") else text
    return raw


class _Cursor:
    __slots__ = ("buf", "pos", "end")

    def __init__(self, buf: bytes, pos: int, end: int):
        self.buf, self.pos, self.end = buf, pos, end

    def take(self, n: int) -> bytes:
        if n < 0 or self.pos + n > self.end:
            raise DicomError(f"truncated data: need {n} bytes at offset {self.pos}, {self.end - self.pos} left")
        b = self.buf[self.pos:self.pos + n]
        self.pos += n
        return bytes(b)

    def u16(self) -> int:
        return struct.unpack("<H", self.take(2))[0]

    def u32(self) -> int:
        return struct.unpack("<I", self.take(4))[0]


def _header(cur: _Cursor, explicit: bool) -> Tuple[Tag, Optional[str], int]:
    """Tag, VR and value length of the next element (PS3.5 §7.1)."""
    tag = (cur.u16(), cur.u16())
    if tag[0] == 0xFFFE:  # item and delimitation tags carry no VR
        return tag, None, cur.u32()
    if not explicit:
        return tag, _IMPLICIT_VR.get(tag), cur.u32()
    vr = cur.take(2).decode("ascii", errors="replace")
    if vr in _LONG_VRS:
        cur.take(2)
        return tag, vr, cur.u32()
    if not (vr.isalpha() and vr.isupper()):
        raise DicomError(f"invalid VR {vr!r} for tag ({tag[0]:04X},{tag[1]:04X}) at offset {cur.pos - 6}")
    return tag, vr, cur.u16()


def _skip_items(cur: _Cursor, explicit: bool, depth: int) -> None:
    """Walk the items of an undefined-length sequence up to its
    sequence delimitation item (PS3.5 §7.5.2)."""
    if depth > 32:
        raise DicomError("sequences nested more than 32 deep")
    while True:
        tag, _, length = _header(cur, explicit)
        if tag == _SEQ_END:
            return
        if tag != _ITEM:
            raise DicomError(f"expected an item tag in a sequence, got ({tag[0]:04X},{tag[1]:04X})")
        if length != _UNDEFINED:
            cur.take(length)
            continue
        # undefined-length item: a nested data set up to the item delimiter
        while True:
            start = cur.pos
            t, vr, ln = _header(cur, explicit)
            if t == _ITEM_END:
                break
            if ln == _UNDEFINED:
                if vr not in ("SQ", "UN", None):
                    raise DicomError(f"undefined length on VR {vr} at offset {start}")
                # an undefined-length UN holds implicit-VR items (PS3.5 §6.2.2)
                _skip_items(cur, explicit and vr == "SQ", depth + 1)
            else:
                cur.take(ln)


def _read_elements(cur: _Cursor, explicit: bool, stop_before_pixels: bool,
                   out: Dict[Tag, Element]) -> bool:
    """Read top-level elements into ``out``; return True if the pixel data
    are encapsulated."""
    encapsulated = False
    while cur.pos < cur.end:
        if cur.end - cur.pos < 8:
            if cur.buf[cur.pos:cur.end].strip(b"\x00"):
                raise DicomError(f"{cur.end - cur.pos} stray bytes at the end of the data set")
            break
        start = cur.pos
        tag, vr, length = _header(cur, explicit)
        if stop_before_pixels and tag >= PIXEL_DATA:
            cur.pos = start
            break
        if length == _UNDEFINED:
            if tag == PIXEL_DATA:
                encapsulated = True
                vstart = cur.pos
                _skip_items(cur, explicit, 0)
                out[tag] = Element(tag, vr, bytes(cur.buf[vstart:cur.pos]))
                continue
            if vr not in ("SQ", "UN", None):
                raise DicomError(f"undefined length on VR {vr} at offset {start}")
            vstart = cur.pos
            _skip_items(cur, explicit and vr == "SQ", 0)
            out[tag] = Element(tag, vr, bytes(cur.buf[vstart:cur.pos]))
            continue
        out[tag] = Element(tag, vr, bytes(cur.take(length)))
    return encapsulated


class DicomFile:
    """A parsed DICOM Part 10 file: ``meta`` (group 0002) and the data set,
    both keyed by ``(group, element)`` tuples.

    ``tag in f``, ``f[tag]`` (an :class:`Element`, whose ``.value`` decodes
    it), ``f.get(tag)``, keyword attributes for the pixel-module tags
    (``f.Rows``, ``f.RescaleSlope``, ...) and :attr:`pixel_array`.
    """

    def __init__(self, meta: Dict[Tag, Element], elements: Dict[Tag, Element], transfer_syntax: str,
                 encapsulated: bool, path: Optional[str] = None):
        self.meta = meta
        self.elements = elements
        self.transfer_syntax = transfer_syntax
        self.encapsulated = encapsulated
        self.path = path

    def __contains__(self, tag) -> bool:
        return tuple(tag) in self.elements

    def __getitem__(self, tag) -> Element:
        try:
            return self.elements[tuple(tag)]
        except KeyError:
            raise KeyError(tag) from None

    def get(self, tag, default=None):
        return self.elements.get(tuple(tag), default)

    def __iter__(self) -> Iterator[Element]:
        return iter(self.elements.values())

    def __len__(self) -> int:
        return len(self.elements)

    def __getattr__(self, name: str):
        tag = _KEYWORDS.get(name)
        if tag is None or tag not in self.__dict__.get("elements", {}):
            raise AttributeError(name)
        return self.elements[tag].value

    @property
    def pixel_array(self) -> np.ndarray:
        """The stored pixel values, [Rows, Columns] (or [frames, Rows,
        Columns]), as unsigned or signed integers of BitsAllocated bits by
        PixelRepresentation (PS3.5 §8).  Signed values with BitsStored below
        BitsAllocated are sign-extended from bit BitsStored - 1; unsigned
        values are returned as stored."""
        if PIXEL_DATA not in self.elements:
            raise DicomError("the file has no pixel data (or was read with stop_before_pixels)")
        if self.encapsulated:
            raise DicomError(f"encapsulated (compressed) pixel data, transfer syntax {self.transfer_syntax}")
        rows, cols = int(self[ROWS].value), int(self[COLUMNS].value)
        spp = int(self[SAMPLES_PER_PIXEL].value) if SAMPLES_PER_PIXEL in self else 1
        if spp != 1:
            raise DicomError(f"{spp} samples per pixel; projection data have one")
        frames = int(self[NUMBER_OF_FRAMES].value) if NUMBER_OF_FRAMES in self else 1
        bits = int(self[BITS_ALLOCATED].value)
        signed = PIXEL_REPRESENTATION in self and int(self[PIXEL_REPRESENTATION].value) == 1
        if bits not in (8, 16, 32):
            raise DicomError(f"BitsAllocated {bits} is not decoded (8, 16 or 32)")
        dt = np.dtype(("<i" if signed else "<u") + str(bits // 8))
        n = rows * cols * frames
        raw = self[PIXEL_DATA].raw
        if len(raw) < n * dt.itemsize:
            raise DicomError(f"pixel data hold {len(raw)} bytes, {n * dt.itemsize} expected")
        arr = np.frombuffer(raw, dtype=dt, count=n)
        stored = int(self[BITS_STORED].value) if BITS_STORED in self else bits
        if signed and stored < bits:
            shift = bits - stored
            arr = (arr << shift) >> shift
        shape = (rows, cols) if frames == 1 else (frames, rows, cols)
        return arr.reshape(shape)


def read_bytes(data: bytes, stop_before_pixels: bool = False, path: Optional[str] = None) -> DicomFile:
    """Parse a DICOM Part 10 file held in memory."""
    buf = memoryview(data)
    if len(buf) < 132 or bytes(buf[128:132]) != b"DICM":
        raise DicomError(f"{path or 'data'}: no DICM prefix after the 128-byte preamble (not DICOM Part 10)")
    cur = _Cursor(buf, 132, len(buf))
    meta: Dict[Tag, Element] = {}
    # the file meta group is explicit VR little endian; its length is in (0002,0000)
    first = cur.pos
    tag, vr, length = _header(cur, True)
    if tag != (0x0002, 0x0000):
        cur.pos = first
        while cur.pos < cur.end:
            save = cur.pos
            t, v, ln = _header(cur, True)
            if t[0] != 0x0002:
                cur.pos = save
                break
            meta[t] = Element(t, v, bytes(cur.take(ln)))
    else:
        glen = struct.unpack("<I", cur.take(length))[0]
        meta[tag] = Element(tag, vr, struct.pack("<I", glen))
        sub = _Cursor(buf, cur.pos, min(cur.pos + glen, len(buf)))
        _read_elements(sub, True, False, meta)
        cur.pos = sub.end
    if TRANSFER_SYNTAX not in meta:
        raise DicomError(f"{path or 'data'}: file meta group has no transfer syntax (0002,0010)")
    ts = str(meta[TRANSFER_SYNTAX].value).strip("\x00 ")
    if ts == IMPLICIT_LE:
        explicit = False
    elif ts == EXPLICIT_LE:
        explicit = True
    elif ts == DEFLATED_LE:
        try:
            body = zlib.decompress(bytes(buf[cur.pos:]), -15)
        except zlib.error as exc:
            raise DicomError(f"{path or 'data'}: deflated data set does not inflate: {exc}") from None
        buf = memoryview(body)
        cur = _Cursor(buf, 0, len(buf))
        explicit = True
    elif ts == EXPLICIT_BE:
        raise DicomError(f"{path or 'data'}: big-endian transfer syntax {ts} is not decoded")
    else:
        explicit = True  # every other syntax encapsulates its pixel data in explicit VR LE
    elements: Dict[Tag, Element] = {}
    encapsulated = _read_elements(cur, explicit, stop_before_pixels, elements)
    if ts not in (IMPLICIT_LE, EXPLICIT_LE, DEFLATED_LE) and not encapsulated and PIXEL_DATA in elements:
        raise DicomError(f"{path or 'data'}: unknown transfer syntax {ts}")
    return DicomFile(meta, elements, ts, encapsulated, path)


def dcmread(path: Union[str, Path], stop_before_pixels: bool = False) -> DicomFile:
    """Read a DICOM Part 10 file (the pydicom.dcmread call of the
    reference's loader)."""
    p = Path(path)
    return read_bytes(p.read_bytes(), stop_before_pixels, str(p))


# ---------------------------------------------------------------------------
# writer


def _uid_for(content: bytes) -> str:
    """A UID under the 2.25 root (a UUID as a decimal integer, PS3.5 §B.2),
    derived from ``content`` so equal files get equal UIDs."""
    return "2.25." + str(int.from_bytes(hashlib.sha256(content).digest()[:16], "big") >> 6)


def _encode_value(vr: Optional[str], value) -> bytes:
    if isinstance(value, (bytes, bytearray, memoryview)):
        raw = bytes(value)
    elif isinstance(value, np.ndarray) and vr not in _NUMERIC:
        raw = np.ascontiguousarray(value).tobytes()
    elif vr in _NUMERIC:
        raw = np.asarray(value, dtype=_NUMERIC[vr]).reshape(-1).tobytes()
    elif vr in ("DS", "IS") or vr in _TEXT_VRS:
        if isinstance(value, (list, tuple)):
            text = "\\".join(_num_text(vr, v) for v in value)
        else:
            text = _num_text(vr, value)
        raw = text.encode("latin-1")
    else:
        raise TypeError(f"cannot encode {type(value).__name__} as VR {vr}")
    if len(raw) % 2:
        raw += b"\x00" if vr in ("UI", "OB", "UN", None) else b" "
    return raw


def _num_text(vr: str, v) -> str:
    if vr == "DS" and not isinstance(v, str):
        t = repr(float(v))
        return t[:-2] if t.endswith(".0") else t
    if vr == "IS" and not isinstance(v, str):
        return str(int(v))
    return str(v)


def _encode_element(tag: Tag, vr: Optional[str], raw: bytes, explicit: bool) -> bytes:
    head = struct.pack("<HH", tag[0], tag[1])
    if not explicit:
        return head + struct.pack("<I", len(raw)) + raw
    if vr is None:
        vr = "UN"
    if vr in _LONG_VRS:
        return head + vr.encode("ascii") + b"\x00\x00" + struct.pack("<I", len(raw)) + raw
    if len(raw) > 0xFFFF:
        raise ValueError(f"value of ({tag[0]:04X},{tag[1]:04X}) is too long for VR {vr}")
    return head + vr.encode("ascii") + struct.pack("<H", len(raw)) + raw


def encode(elements: Iterable[Tuple[Tag, Optional[str], object]], transfer_syntax: str = IMPLICIT_LE,
           sop_class: str = "1.2.840.10008.5.1.4.1.1.66") -> bytes:
    """A DICOM Part 10 file holding ``elements`` = (tag, VR, value) in the
    given transfer syntax (implicit, explicit or deflated explicit VR little
    endian).  VR None writes an implicit-VR element as raw bytes, or an
    explicit one as UN.  The SOP class defaults to Raw Data Storage."""
    if transfer_syntax not in (IMPLICIT_LE, EXPLICIT_LE, DEFLATED_LE):
        raise ValueError(f"transfer syntax {transfer_syntax} is not written")
    explicit = transfer_syntax != IMPLICIT_LE
    body = bytearray()
    for tag, vr, value in sorted(elements, key=lambda e: e[0]):
        body += _encode_element(tuple(tag), vr, _encode_value(vr, value), explicit)
    if transfer_syntax == DEFLATED_LE:
        co = zlib.compressobj(6, zlib.DEFLATED, -15)
        body = bytearray(co.compress(bytes(body)) + co.flush())
    uid = _uid_for(bytes(body))
    meta = bytearray()
    for tag, vr, value in (((0x0002, 0x0001), "OB", b"\x00\x01"), ((0x0002, 0x0002), "UI", sop_class),
                           ((0x0002, 0x0003), "UI", uid), ((0x0002, 0x0010), "UI", transfer_syntax),
                           ((0x0002, 0x0012), "UI", "2.25.1")):
        meta += _encode_element(tag, vr, _encode_value(vr, value), True)
    group = _encode_element((0x0002, 0x0000), "UL", struct.pack("<I", len(meta)), True)
    return bytes(128) + b"DICM" + group + bytes(meta) + bytes(body)


def write(path: Union[str, Path], elements: Iterable[Tuple[Tag, Optional[str], object]],
          transfer_syntax: str = IMPLICIT_LE) -> None:
    Path(path).write_bytes(encode(elements, transfer_syntax))
