"""DICOM-CT-PD ingest (xrecon_b200.dicom, xrecon_b200.mayo) on the CPU.

* the DICOM reader on files of the library's writer (implicit, explicit and
  deflated explicit VR little endian) and on byte strings laid out by hand
  from the standard (sequences of defined and undefined length, nested
  items, undefined-length UN, signed pixels, errors);
* the Mayo loader against the reference's own loader
  (tests/golden/mayo_ref.npz, made by tests/golden/make_golden_mayo.py from
  xrecon/utils/mayo.py and mayo_fdk.py): geometry, view selection and
  order, sinogram, angles, source z and offsets, detector shifts,
  source_pos and the helical projector it builds -- bit for bit;
* the series written in explicit VR, with private tags as OB, loads the
  same as the implicit-VR series.
"""
import hashlib
import struct
import sys
import types
from pathlib import Path

import numpy as np
import pytest
import torch

from conftest import GOLDEN, load_golden

sys.path.insert(0, str(GOLDEN))
import mayo_series as MS  # noqa: E402

from xrecon_b200 import dicom, mayo  # noqa: E402


def _config(case: str, root: Path) -> "mayo.MayoFdkConfig":
    return mayo.MayoFdkConfig(data_dir=root, file_pattern="*.dcm", **MS.CASES[case]["config"])


# ---------------------------------------------------------------------------
# the DICOM reader


@pytest.mark.parametrize("ts", [dicom.IMPLICIT_LE, dicom.EXPLICIT_LE, dicom.DEFLATED_LE])
def test_dicom_round_trip(tmp_path, ts):
    px = np.arange(7 * 5, dtype=np.uint16).reshape(7, 5) * 1000
    els = [((0x0008, 0x0060), "CS", "CT"), (dicom.ROWS, "US", 7), (dicom.COLUMNS, "US", 5),
           (dicom.BITS_ALLOCATED, "US", 16), (dicom.PIXEL_REPRESENTATION, "US", 0),
           (dicom.RESCALE_SLOPE, "DS", 0.5), (dicom.RESCALE_INTERCEPT, "DS", -1024.0),
           ((0x0018, 0x0050), "DS", [1.25, 2.5]), ((0x7031, 0x1033), None, struct.pack("<ff", 368.625, 32.5)),
           ((0x7029, 0x100B), None, b"CYLINDRICAL "), (dicom.PIXEL_DATA, "OW", px.tobytes())]
    p = tmp_path / "a.dcm"
    dicom.write(p, els, ts)
    f = dicom.dcmread(p)
    assert f.transfer_syntax == ts
    assert (f.Rows, f.Columns, f.RescaleSlope, f.RescaleIntercept) == (7, 5, 0.5, -1024.0)
    assert f[(0x7031, 0x1033)].raw == struct.pack("<ff", 368.625, 32.5)
    assert f[(0x7029, 0x100B)].raw == b"CYLINDRICAL "
    assert (0x0008, 0x0060) in f and f[(0x0008, 0x0060)].value == "CT"
    if ts != dicom.IMPLICIT_LE:  # the VR travels with explicit-VR data only
        assert f[(0x0018, 0x0050)].value == [1.25, 2.5]
        assert f[(0x7031, 0x1033)].vr == "UN"
    np.testing.assert_array_equal(f.pixel_array, px)
    head = dicom.dcmread(p, stop_before_pixels=True)
    assert dicom.PIXEL_DATA not in head and head.Rows == 7
    with pytest.raises(dicom.DicomError):
        head.pixel_array


def _el_explicit(group, elem, vr, value: bytes) -> bytes:
    h = struct.pack("<HH", group, elem) + vr.encode()
    if vr in ("OB", "OW", "SQ", "UN", "UT"):
        return h + b"\0\0" + struct.pack("<I", len(value)) + value
    return h + struct.pack("<H", len(value)) + value


def _el_implicit(group, elem, value: bytes, length=None) -> bytes:
    return struct.pack("<HHI", group, elem, len(value) if length is None else length) + value


def _file(body: bytes, ts: str) -> bytes:
    uid = ts.encode() + (b"\0" if len(ts) % 2 else b"")
    meta = _el_explicit(0x0002, 0x0010, "UI", uid)
    return bytes(128) + b"DICM" + _el_explicit(0x0002, 0x0000, "UL", struct.pack("<I", len(meta))) + meta + body


UNDEF = 0xFFFFFFFF
ITEM, ITEM_END, SEQ_END = (0xFFFE, 0xE000), (0xFFFE, 0xE00D), (0xFFFE, 0xE0DD)


def _tag(t, length) -> bytes:
    return struct.pack("<HHI", t[0], t[1], length)


def test_dicom_sequences_explicit():
    """Defined- and undefined-length sequences with nested items, and an
    undefined-length UN (implicit-VR items inside), before the elements that
    follow them (PS3.5 §7.5)."""
    inner = _el_explicit(0x0008, 0x0100, "SH", b"ABCD")
    nested = (_el_explicit(0x0040, 0xA730, "SQ", b"")[:-4] + struct.pack("<I", UNDEF)
              + _tag(ITEM, UNDEF) + inner + _tag(ITEM_END, 0) + _tag(SEQ_END, 0))
    seq_undef = (_el_explicit(0x0008, 0x1140, "SQ", b"")[:-4] + struct.pack("<I", UNDEF)
                 + _tag(ITEM, len(inner)) + inner
                 + _tag(ITEM, UNDEF) + nested + _tag(ITEM_END, 0) + _tag(SEQ_END, 0))
    item = _tag(ITEM, len(inner)) + inner
    seq_def = _el_explicit(0x0008, 0x1150, "SQ", item + item)
    un_items = _tag(ITEM, UNDEF) + _el_implicit(0x0010, 0x0010, b"NAME") + _tag(ITEM_END, 0) + _tag(SEQ_END, 0)
    un_undef = _el_explicit(0x0009, 0x1001, "UN", b"")[:-4] + struct.pack("<I", UNDEF) + un_items
    body = (_el_explicit(0x0008, 0x0060, "CS", b"CT") + seq_undef + seq_def + un_undef
            + _el_explicit(0x0028, 0x0010, "US", struct.pack("<H", 3))
            + _el_explicit(0x0028, 0x0011, "US", struct.pack("<H", 2))
            + _el_explicit(0x0028, 0x0100, "US", struct.pack("<H", 16))
            + _el_explicit(0x0028, 0x0103, "US", struct.pack("<H", 1))
            + _el_explicit(0x7FE0, 0x0010, "OW", np.array([-1, 2, -3, 4, -5, 6], "<i2").tobytes()))
    f = dicom.read_bytes(_file(body, dicom.EXPLICIT_LE))
    assert f[(0x0008, 0x1140)].vr == "SQ" and f[(0x0008, 0x1150)].raw == item + item
    assert f[(0x0009, 0x1001)].raw == un_items
    assert f.Rows == 3 and f.Columns == 2
    np.testing.assert_array_equal(f.pixel_array, [[-1, 2], [-3, 4], [-5, 6]])


def test_dicom_sequences_implicit_and_pixel_forms():
    inner = _el_implicit(0x0008, 0x0100, b"ABCD")
    seq = _el_implicit(0x0008, 0x1140, b"", UNDEF) + _tag(ITEM, UNDEF) + inner + _tag(ITEM_END, 0) + \
        _tag(ITEM, len(inner)) + inner + _tag(SEQ_END, 0)
    vals = np.array([0x0FFF, 0x0800, 0x07FF, 0x0001], "<u2")  # 12-bit two's complement
    body = (seq + _el_implicit(0x0028, 0x0010, struct.pack("<H", 2)) + _el_implicit(0x0028, 0x0011, struct.pack("<H", 2))
            + _el_implicit(0x0028, 0x0100, struct.pack("<H", 16)) + _el_implicit(0x0028, 0x0101, struct.pack("<H", 12))
            + _el_implicit(0x0028, 0x0103, struct.pack("<H", 1))
            + _el_implicit(0x0028, 0x1053, b"2.5 ") + _el_implicit(0x7FE0, 0x0010, vals.tobytes()))
    f = dicom.read_bytes(_file(body, dicom.IMPLICIT_LE))
    assert f.RescaleSlope == 2.5
    np.testing.assert_array_equal(f.pixel_array, [[-1, -2048], [2047, 1]])
    # 8- and 32-bit unsigned, two frames
    for bits, dt in ((8, "<u1"), (32, "<u4")):
        px = np.arange(12, dtype=dt) * 7
        body = (_el_implicit(0x0028, 0x0008, b"2 ") + _el_implicit(0x0028, 0x0010, struct.pack("<H", 2))
                + _el_implicit(0x0028, 0x0011, struct.pack("<H", 3))
                + _el_implicit(0x0028, 0x0100, struct.pack("<H", bits)) + _el_implicit(0x7FE0, 0x0010, px.tobytes()))
        np.testing.assert_array_equal(dicom.read_bytes(_file(body, dicom.IMPLICIT_LE)).pixel_array,
                                      px.reshape(2, 2, 3))


def test_dicom_errors():
    ok = _el_implicit(0x0028, 0x0010, struct.pack("<H", 2))
    with pytest.raises(dicom.DicomError, match="DICM"):
        dicom.read_bytes(bytes(200))
    with pytest.raises(dicom.DicomError, match="big-endian"):
        dicom.read_bytes(_file(ok, dicom.EXPLICIT_BE))
    with pytest.raises(dicom.DicomError, match="truncated"):
        dicom.read_bytes(_file(ok + _el_implicit(0x0028, 0x0011, b"")[:-4] + struct.pack("<I", 64) + b"xx",
                               dicom.IMPLICIT_LE))
    # encapsulated (JPEG baseline) pixel data: parsed, not decoded
    frag = b"\xff\xd8\xff\xd9"
    enc = (_el_explicit(0x0028, 0x0010, "US", struct.pack("<H", 1)) + _el_explicit(0x0028, 0x0011, "US", struct.pack("<H", 1))
           + _el_explicit(0x0028, 0x0100, "US", struct.pack("<H", 16))
           + _el_explicit(0x7FE0, 0x0010, "OB", b"")[:-4] + struct.pack("<I", UNDEF)
           + _tag(ITEM, 0) + _tag(ITEM, len(frag)) + frag + _tag(SEQ_END, 0))
    f = dicom.read_bytes(_file(enc, "1.2.840.10008.1.2.4.50"))
    assert f.encapsulated
    with pytest.raises(dicom.DicomError, match="compressed"):
        f.pixel_array
    # short pixel data
    short = ok + _el_implicit(0x0028, 0x0011, struct.pack("<H", 2)) + \
        _el_implicit(0x0028, 0x0100, struct.pack("<H", 16)) + _el_implicit(0x7FE0, 0x0010, b"\0\0")
    with pytest.raises(dicom.DicomError, match="pixel data hold"):
        dicom.read_bytes(_file(short, dicom.IMPLICIT_LE)).pixel_array


# ---------------------------------------------------------------------------
# the Mayo loader against the reference's


@pytest.mark.parametrize("case", sorted(MS.CASES))
def test_mayo_loader_matches_reference(tmp_path, case):
    g = load_golden("mayo_ref")
    paths = MS.write_series(tmp_path, case)
    # the files are the ones the reference loaded
    assert [hashlib.sha256(p.read_bytes()).hexdigest() for p in paths] == list(g[f"{case}_sha256"])
    cfg = _config(case, tmp_path)
    prob = mayo.load_mayo_problem(cfg)
    geo = prob.geometry
    num = np.array([geo.num_det_col, geo.num_det_row, geo.det_col_size, geo.det_row_size, geo.iso_source,
                    geo.source_detector, geo.det_center_col, geo.det_center_row, geo.views_per_rotation,
                    np.nan if geo.water_mu is None else geo.water_mu], np.float64)
    np.testing.assert_array_equal(num, g[f"{case}_geometry_num"])
    assert [geo.detector_type, geo.trajectory, geo.beam_type] == list(g[f"{case}_geometry_text"])
    assert [Path(p).name for p in prob.files] == list(g[f"{case}_files"])
    for k in ("sino", "angles", "source_z", "shift_z", "shift_angle", "shift_radius"):
        got = getattr(prob, k)
        assert got.dtype == g[f"{case}_{k}"].dtype, k
        np.testing.assert_array_equal(got, g[f"{case}_{k}"], err_msg=k)
    np.testing.assert_array_equal(np.array(prob.binshift, np.float64), g[f"{case}_binshift"])
    sp = mayo.make_source_pos(prob.source_z, prob.shift_z, prob.shift_angle, prob.shift_radius, "cpu")
    np.testing.assert_array_equal(sp.numpy(), g[f"{case}_source_pos"])
    P = mayo.make_helical_projector(geo, prob.sino.shape, prob.binshift, "cpu", cfg)
    np.testing.assert_array_equal(P.options.numpy(), g[f"{case}_proj_options"])
    np.testing.assert_allclose(P.weight.numpy(), g[f"{case}_proj_weight"], rtol=1e-6, atol=0)
    ref_f = g[f"{case}_proj_filter"]
    np.testing.assert_allclose(P.filter.numpy(), ref_f, rtol=2e-6, atol=1e-7 * np.abs(ref_f).max())
    # the pieces of mayo.py on their own
    files = mayo.dicom_files(tmp_path, "*.dcm")
    stack = mayo.load_projection_stack(files[:7], 1, 1)
    np.testing.assert_array_equal(stack[0], g[f"{case}_stack7_sino"])
    np.testing.assert_array_equal(stack[1], g[f"{case}_stack7_angles"])
    un = mayo.normalize_angles(stack[1])
    np.testing.assert_array_equal(un, g[f"{case}_stack7_unwrapped"])
    dec = mayo.order_views(*(stack[0], un) + tuple(stack[2:]), "decreasing")
    np.testing.assert_array_equal(dec[1], g[f"{case}_stack7_decreasing_angles"])
    np.testing.assert_array_equal(dec[0], g[f"{case}_stack7_decreasing_sino"])
    zc = [mayo.volume_z_center(stack[2], m, None) for m in ("mean", "middle", "first")]
    np.testing.assert_array_equal(np.array(zc), g[f"{case}_zc"])
    args = types.SimpleNamespace(image_size=16, num_slices=4, pixel_size=1.5, slice_spacing=2.0, det_col_stride=1,
                                 det_row_stride=2, volume_z_shift=1.0, filter="shepplogan")
    Q = mayo.make_projector(args, geo, prob.sino.shape[2], prob.sino.shape[1], prob.binshift)
    np.testing.assert_array_equal(Q.options.numpy(), g[f"{case}_make_projector_options"])
    ref_q = g[f"{case}_make_projector_filter"]
    np.testing.assert_allclose(Q.filter.numpy(), ref_q, rtol=2e-6, atol=1e-7 * np.abs(ref_q).max())


def test_mayo_helpers_match_reference():
    g = load_golden("mayo_ref")
    got = [mayo.detector_shift(*a) for a in ((368.625, 736, 1, 1.0, 0), (368.625, 368, 2, 1.0, 0),
                                              (32.5, 64, 1, 0.0, 0), (40.25, 32, 2, 1.0, 8), (12.0, 7, 3, 0.5, 1))]
    np.testing.assert_array_equal(np.array(got), g["helper_detector_shift"])
    sel = [",".join(str(i) for i in mayo.choose_files(list(range(20)), *a))
           for a in ((1, 0, 1), (3, 5, 2), (10, 100, 3), (17, 1, 1), (1, 4, 7))]
    assert sel == list(g["helper_choose_files"])
    rec = np.linspace(-0.01, 0.04, 11, dtype=np.float32)
    hu = np.stack([mayo.to_hu(rec, 0.0192, False), mayo.to_hu(rec, 0.0192, True), mayo.to_hu(rec, None, False),
                   mayo.to_hu(rec, -1.0, False)])
    np.testing.assert_array_equal(hu, g["helper_to_hu"])
    with pytest.raises(ValueError):
        mayo.choose_files([1, 2], 0, 1, 1)
    with pytest.raises(ValueError):
        mayo.choose_files([1, 2], 5, 1, 1)
    with pytest.raises(ValueError):
        mayo.volume_z_center(np.zeros(3, np.float32), "median", None)
    with pytest.raises(FileNotFoundError):
        mayo.dicom_files(GOLDEN, "*.no_such_suffix")


@pytest.mark.parametrize("ts,vr", [(dicom.EXPLICIT_LE, None), (dicom.EXPLICIT_LE, "OB"), (dicom.DEFLATED_LE, None)])
def test_mayo_encodings_load_alike(tmp_path, ts, vr):
    """Explicit-VR (private tags UN or OB) and deflated series load exactly
    as the implicit-VR series the reference read."""
    g = load_golden("mayo_ref")
    case = "decreasing"
    MS.write_series(tmp_path, case, transfer_syntax=ts, private_vr=vr)
    prob = mayo.load_mayo_problem(_config(case, tmp_path))
    np.testing.assert_array_equal(prob.sino, g[f"{case}_sino"])
    np.testing.assert_array_equal(prob.angles, g[f"{case}_angles"])
    np.testing.assert_array_equal(prob.source_z, g[f"{case}_source_z"])
    np.testing.assert_array_equal(np.array(prob.binshift), g[f"{case}_binshift"])


def test_mayo_typed_private_tags(tmp_path):
    """Private tags written with numeric VRs (FL pair, US) decode by VR."""
    els = [((0x7031, 0x1033), "FL", [368.625, 32.5]), ((0x7029, 0x1010), "US", 64),
           ((0x7029, 0x1002), "FD", 1.2858), ((0x0018, 0x0061), "DS", 0.0192)]
    p = tmp_path / "t.dcm"
    dicom.write(p, els, dicom.EXPLICIT_LE)
    ds = dicom.dcmread(p)
    assert mayo._float32_pair(ds, mayo.TAG_DET_CENTER) == (368.625, 32.5)
    assert mayo._int16(ds, mayo.TAG_NUM_ROWS) == 64
    assert mayo._float32(ds, mayo.TAG_DET_DU) == 1.2858
    assert mayo._float32(ds, mayo.TAG_WATER_MU) == 0.0192
    assert mayo._float32(ds, mayo.TAG_SOURCE_Z, default=0.0) == 0.0
    with pytest.raises(KeyError):
        mayo._float32(ds, mayo.TAG_SOURCE_Z)
    assert mayo._text(ds, mayo.TAG_BEAM_TYPE, "fanbeam") == "fanbeam"


def test_mayo_metadata_csv(tmp_path):
    p = tmp_path / "m.csv"
    mayo.save_metadata_csv(p, [("views", 3), ("sod", 595.0)])
    assert p.read_text().splitlines() == ["key,value", "views,3", "sod,595.0"]


def test_mayo_problem_unpacks_like_the_reference(tmp_path):
    MS.write_series(tmp_path, "dicom_order")
    prob = mayo.load_mayo_problem(_config("dicom_order", tmp_path))
    geometry, chosen, sino, angles, source_z, shift_z, shift_angle, shift_radius, binshift = prob
    assert sino is prob.sino and binshift == prob.binshift and len(chosen) == sino.shape[0] == angles.size
    assert isinstance(mayo.make_source_pos(source_z, shift_z, shift_angle, shift_radius, "cpu"), torch.Tensor)


# ---------------------------------------------------------------------------
# the library's multi-threaded reader (xr_ctpd_load) against the Python reader


def _both(files, cs, rs, threads=None):
    nat = mayo._load_stack_native(files, cs, rs, threads)
    py = mayo.load_projection_stack(files, cs, rs, native=False)
    return nat, py


def _same(a, b):
    return all(x.dtype == y.dtype and x.shape == y.shape and np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("ts,vr", [(dicom.IMPLICIT_LE, None), (dicom.EXPLICIT_LE, None), (dicom.EXPLICIT_LE, "OB")])
@pytest.mark.parametrize("strides", [(1, 1), (2, 1), (1, 2), (3, 5), (30, 30)])
def test_native_reader_matches_python_reader(tmp_path, ts, vr, strides):
    files = MS.write_series(tmp_path, "decreasing", transfer_syntax=ts, private_vr=vr)
    for threads in (1, 3, None):
        nat, py = _both(files, *strides, threads)
        assert nat is not None, "the native reader declined a plain series"
        assert _same(nat, py)


def _pixel_file(path, px, bits, signed, stored, slope="0.0005 ", intercept="-7.25", ts=dicom.IMPLICIT_LE,
                tags=None):
    els = [(dicom.ROWS, "US", px.shape[0]), (dicom.COLUMNS, "US", px.shape[1]), (dicom.BITS_ALLOCATED, "US", bits),
           (dicom.BITS_STORED, "US", stored), (dicom.PIXEL_REPRESENTATION, "US", int(signed)),
           (dicom.RESCALE_SLOPE, "DS", slope), (dicom.RESCALE_INTERCEPT, "DS", intercept),
           (mayo.TAG_ANGLE, None, struct.pack("<f", 1.5)), (mayo.TAG_SOURCE_Z, None, struct.pack("<f", -2.0)),
           (dicom.PIXEL_DATA, "OB" if bits == 8 else "OW", px.tobytes())]
    if tags:
        els = [e for e in els if e[0] not in {t[0] for t in tags}] + list(tags)
    dicom.write(path, els, ts)


def test_native_reader_pixel_forms(tmp_path):
    """8/16/32-bit, signed with fewer stored bits (sign extension), DS text
    with padding, typed private tags (FL, FD, US, DS, IS) and raw tags of
    other lengths read as decimal text."""
    rng = np.random.default_rng(7)
    cases = [
        (rng.integers(0, 255, (9, 4), dtype=np.uint8), 8, False, 8, {}),
        (rng.integers(-128, 127, (9, 4), dtype=np.int8), 8, True, 6, {}),
        (rng.integers(0, 65535, (9, 4), dtype="<u2"), 16, False, 12, {}),
        (rng.integers(-32768, 32767, (9, 4), dtype="<i2"), 16, True, 12, {}),
        (rng.integers(0, 2**31, (9, 4), dtype="<u4") * 2, 32, False, 32, {}),
        (rng.integers(-2**31, 2**31 - 1, (9, 4), dtype="<i4"), 32, True, 20, {}),
    ]
    typed = [((mayo.TAG_ANGLE), "FL", 0.3), ((mayo.TAG_SOURCE_Z), "FD", -1.0 / 3.0),
             ((mayo.TAG_SOURCE_SHIFT_Z), "US", 7), ((mayo.TAG_SOURCE_SHIFT_ANGLE), "DS", " 1.25e-3 "),
             ((mayo.TAG_SOURCE_SHIFT_RADIUS), "IS", "-4")]
    raw_text = [((mayo.TAG_ANGLE), None, b"2.515 "), ((mayo.TAG_SOURCE_Z), None, b" -0.125 ")]
    for i, (px, bits, signed, stored, _) in enumerate(cases):
        for j, tags in enumerate((None, typed, raw_text)):
            ts = dicom.EXPLICIT_LE if tags is typed else dicom.IMPLICIT_LE
            p = tmp_path / f"p{i}_{j}.dcm"
            _pixel_file(p, px, bits, signed, stored, ts=ts, tags=tags)
            nat, py = _both([p, p], 2, 1, 1)
            assert nat is not None, (bits, signed, stored, j)
            assert _same(nat, py), (bits, signed, stored, j)


def test_native_reader_declines_what_it_does_not_take(tmp_path):
    """Deflated files, multi-valued or oddly typed tags, frames, a different
    matrix: the native reader declines and the Python reader decides."""
    g, views = MS.series("increasing")
    v = views[0]
    mayo.write_projection_file(tmp_path / "d.dcm", g, v["pixels"], v["angle"], v["source_z"],
                               transfer_syntax=dicom.DEFLATED_LE)
    assert mayo._load_stack_native([tmp_path / "d.dcm"], 1, 1, 1) is None
    assert mayo.load_projection_stack([tmp_path / "d.dcm"], 1, 1)[0].shape == (1, 6, 24)
    px = np.arange(12, dtype="<u2").reshape(4, 3)
    odd = {
        "two_slopes": [(dicom.RESCALE_SLOPE, "DS", [1.0, 2.0])],
        # raw values of 4 bytes are float32s; these are text of other lengths
        "hex_text": [(mayo.TAG_ANGLE, None, b"0x1p3 ")],
        "nul_in_raw_text": [(mayo.TAG_ANGLE, None, b"1.50\0\0")],
        "lo_angle": [(mayo.TAG_ANGLE, "LO", "1.5")],
        "two_frames": [((0x0028, 0x0008), "IS", 2)],
        "no_angle": [(mayo.TAG_ANGLE, None, None)],
    }
    for name, tags in odd.items():
        p = tmp_path / f"{name}.dcm"
        if name == "no_angle":
            dicom.write(p, [e for e in [(dicom.ROWS, "US", 4), (dicom.COLUMNS, "US", 3),
                                        (dicom.BITS_ALLOCATED, "US", 16), (mayo.TAG_SOURCE_Z, None, bytes(4)),
                                        (dicom.PIXEL_DATA, "OW", px.tobytes())]], dicom.EXPLICIT_LE)
        else:
            _pixel_file(p, px, 16, False, 16, ts=dicom.EXPLICIT_LE, tags=tags)
        assert mayo._load_stack_native([p], 1, 1, 1) is None, name
    # a different matrix in the second file
    _pixel_file(tmp_path / "a.dcm", px, 16, False, 16)
    _pixel_file(tmp_path / "b.dcm", np.zeros((5, 3), "<u2"), 16, False, 16)
    assert mayo._load_stack_native([tmp_path / "a.dcm", tmp_path / "b.dcm"], 1, 1, 1) is None
    with pytest.raises(ValueError):
        mayo.load_projection_stack([tmp_path / "a.dcm", tmp_path / "b.dcm"], 1, 1)


def test_native_reader_on_damaged_files(tmp_path):
    """Every truncation and 1500 random byte changes of a projection file
    (implicit and explicit VR, with a sequence before the pixel data): the
    native reader either declines or returns exactly what the Python reader
    returns; it never reads out of bounds (the process would die)."""
    import ctypes
    from xrecon_b200 import _native
    L = _native.lib()
    g, views = MS.series("dicom_order")
    v = views[0]
    rng = np.random.default_rng(11)
    for ts in (dicom.IMPLICIT_LE, dicom.EXPLICIT_LE):
        src = tmp_path / "src.dcm"
        mayo.write_projection_file(src, g, v["pixels"], v["angle"], v["source_z"], 0.5, -0.25, 3.0, 1.5, -2.0,
                                   transfer_syntax=ts)
        good = bytearray(src.read_bytes())
        # a defined-length sequence in front of the rows (0008,1140)
        item = struct.pack("<HHI", 0xFFFE, 0xE000, 0)
        if ts == dicom.EXPLICIT_LE:
            seq = struct.pack("<HH", 0x0008, 0x1140) + b"SQ\0\0" + struct.pack("<I", len(item)) + item
        else:
            seq = struct.pack("<HHI", 0x0008, 0x1140, len(item)) + item
        f0 = dicom.read_bytes(bytes(good))
        meta_len = 132 + 12 + struct.unpack("<I", f0.meta[(0x0002, 0x0000)].raw)[0]
        good = good[:meta_len] + seq + good[meta_len:]
        rows, cols = int(f0.Rows), int(f0.Columns)
        nv, nu = cols, rows
        p = tmp_path / "m.dcm"

        def check(data: bytes):
            p.write_bytes(data)
            sino = np.zeros((1, nv, nu), np.float32)
            vw = np.zeros((1, 5), np.float32)
            paths = (ctypes.c_char_p * 1)(str(p).encode())
            failed = ctypes.c_int(-1)
            rc = L.xr_ctpd_load(paths, 1, rows, cols, 1, 1, 1, sino.ctypes.data, vw.ctypes.data, ctypes.byref(failed))
            if rc != 0:
                assert rc == 4 and failed.value == 0
                return False
            py = mayo.load_projection_stack([p], 1, 1, native=False)
            assert _same((sino,) + tuple(vw[:, k] for k in range(5)), py)
            return True

        assert check(bytes(good))
        for cut in range(0, len(good) - 1, 3):
            check(bytes(good[:cut]))
        accepted = 0
        for _ in range(1500):
            bad = bytearray(good)
            for _k in range(int(rng.integers(1, 4))):
                pos = int(rng.integers(0, len(bad) - nv * nu * 2)) if rng.random() < 0.9 else int(rng.integers(0, len(bad)))
                bad[pos] = int(rng.integers(0, 256))
            accepted += check(bytes(bad))
        assert accepted > 100  # the changes that keep a readable file are compared, not only declined
