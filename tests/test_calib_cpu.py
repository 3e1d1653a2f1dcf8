"""The reference's calibration files on the host (include/pfd_calib.h):
CalibInfo.xml read and written, intrinsics.xml read, each against text laid
out as the reference's reader walks it (DepthSolver.cpp:872-1340), with its
quirks: sscanf conversions, the last pitch value winning, later lenses with
the same key replacing earlier ones, unlisted blur types reading radius 0."""
import numpy as np
import pytest

CALIB = """<?xml version="1.0" encoding="UTF-8"?>
<!-- written by hand in the reference's layout -->
<Calib>
    <BlurInfo>
        <pose><r>1,0,0,1</r><t>0.5,-0.5</t></pose>
        <MLAType id="0">0.6</MLAType>
        <MLAType id="1">1.0</MLAType>
    </BlurInfo>
    <MLAInfo>
        <MLA><key>2,3</key><center>100.5,200.25</center><MLAType>1</MLAType><aera>350</aera></MLA>
        <MLA><key>0,7</key><center> 11.125 , 12.5</center><MLAType>0</MLAType><aera>401.5</aera></MLA>
        <MLA><key>2,3</key><center>101.5,201.25</center><MLAType>2</MLAType><aera>351</aera></MLA>
        <MLA><key>0x1,010</key><center>55,66</center><MLAType>1</MLAType><aera/></MLA>
    </MLAInfo>
</Calib>
"""

INTRINSICS = """<?xml version="1.0"?>
<_>
  <D>1.25</D>
  <d>0.75</d>
  <sensor>
    <pose>
      <rotation>
        <_><_>1</_><_>2</_><_>3</_></_>
        <_><_>4</_><_>5</_><_>6</_></_>
        <_><_>7</_><_>8</_><_>9</_></_>
      </rotation>
      <translation><_><_>0.1</_><_>0.2</_><_>0.3</_></_></translation>
    </pose>
    <scale>0.0055</scale>
  </sensor>
  <main_lens><f>50.5</f></main_lens>
  <mia>
    <mesh>
      <width>174</width>
      <height>151</height>
      <pitch><_><_>23.21</_><_>23.19</_></_></pitch>
    </mesh>
  </mia>
  <distortions>
    <depth><_><_>0.01</_><_>0.02</_><_>0.03</_></_></depth>
    <radial><_><_>-0.1</_><_>0.2</_><_>-0.3</_></_></radial>
    <tangential><_><_>0.004</_><_>0.005</_></_></tangential>
  </distortions>
</_>
"""


def f32(x):
    return float(np.float32(x))


def test_read_calib_follows_the_reference(pfd):
    m = pfd.read_calib_xml(CALIB)
    # map order (row, column); the second (2,3) replaces the first; key 0x1,010 is row 1, column 8
    assert [(int(r), int(c)) for r, c in zip(m["row"], m["col"])] == [(0, 7), (1, 8), (2, 3)]
    a, b, c = m
    # "%f,%f" needs the comma right after the first number: " 11.125 , 12.5" reads x only
    assert (a["cx"], a["cy"], a["type"], a["area"]) == (f32(11.125), 0.0, 0, f32(401.5))
    assert a["blur_radius"] == f32(0.6)
    assert (b["cx"], b["cy"], b["area"], b["blur_radius"]) == (55.0, 66.0, 0.0, f32(1.0))
    assert (c["cx"], c["cy"], c["type"], c["area"]) == (f32(101.5), f32(201.25), 2, f32(351))
    assert c["blur_radius"] == 0.0                       # type 2 is not in BlurInfo


def test_write_calib_is_the_reference_layout(pfd):
    L = np.zeros(3, pfd.MLA_ENTRY)
    L[0] = (4, 1, 1234.5678, 12.0, 0, 100.125, 0)
    L[1] = (2, 0, 7.25, 8.5, 0, 99.0, 0)
    L[2] = (9, 9, 1.0, 2.0, 0, 3.0, 0)
    txt = pfd.write_calib_xml(L, abandon=[0, 0, 1])
    assert txt == (
        "<Calib>\n    <BlurInfo>\n"
        '        <MLAType id="0">0</MLAType>\n        <MLAType id="1">1</MLAType>\n'
        '        <MLAType id="2">2</MLAType>\n    </BlurInfo>\n    <MLAInfo>\n'
        "        <MLA>\n            <key>0,2</key>\n            <center>7.25,8.5</center>\n"
        "            <MLAType>1</MLAType>\n            <aera>99</aera>\n        </MLA>\n"
        "        <MLA>\n            <key>1,4</key>\n            <center>1234.57,12</center>\n"
        "            <MLAType>1</MLAType>\n            <aera>100.125</aera>\n        </MLA>\n"
        "    </MLAInfo>\n</Calib>\n")
    back = pfd.read_calib_xml(txt)
    assert list(back["col"]) == [2, 4] and list(back["cx"]) == [f32(7.25), f32(1234.57)]
    assert list(back["blur_radius"]) == [f32(1.0), f32(1.0)]      # MLAType 1 written, radius text "1"


def test_detected_centres_survive_the_file_round_trip(pfd, oracle):
    """Centres from the MLA detection (the oracle's restatement, pinned to
    OpenCV) written and read back keep their keys and six significant digits."""
    from test_mla_cpu import white_image
    img, _ = white_image(240, 200, 23.2, seed=3)
    ent, _ = oracle.mla_centers(img, 23.2, 12, 10)
    L = np.zeros(len(ent["col"]), pfd.MLA_ENTRY)
    L["col"], L["row"], L["cx"], L["cy"], L["area"] = ent["col"], ent["row"], ent["cx"], ent["cy"], ent["area"]
    back = pfd.read_calib_xml(pfd.write_calib_xml(L, abandon=ent["abandon"]))
    keep = np.asarray(ent["abandon"]) == 0
    order = np.lexsort((L["col"][keep], L["row"][keep]))
    kept = L[keep][order]
    assert len(back) == len(kept) > 10
    assert np.array_equal(back["col"], kept["col"]) and np.array_equal(back["row"], kept["row"])
    for name in ("cx", "cy", "area"):
        want = np.array([f32(float("%.6g" % v)) for v in kept[name]], np.float32)
        assert np.array_equal(back[name], want), name


def test_read_intrinsics_follows_the_reference(pfd):
    d = pfd.read_intrinsics_xml(INTRINSICS)
    assert d["D"] == f32(1.25) and d["d"] == f32(0.75)
    # one "_" per column: element (row i) of column j
    assert d["sensor_rotation"] == [1, 4, 7, 2, 5, 8, 3, 6, 9]
    assert d["sensor_translate"] == [0.1, 0.2, 0.3]
    assert d["sensor_pixel_size"] == f32(0.0055) and d["mainlen_focal_length"] == f32(50.5)
    assert (d["mla_u_size"], d["mla_v_size"]) == (174, 151)
    assert d["baseline"] == f32(23.19)                   # the last pitch value wins
    assert d["distor_depth"] == [0.01, 0.02, 0.03] and d["distor_radial"] == [-0.1, 0.2, -0.3]
    assert d["distor_tangential"] == [0.004, 0.005] and d["has_mia"] == 1


@pytest.mark.parametrize("bad", [
    "<Root><MLAInfo/></Root>",                                            # wrong root
    "<Calib><BlurInfo><MLAType>1</MLAType></BlurInfo></Calib>",           # type without id
    "<Calib><MLAInfo><MLA><key>1,2</key></MLA></Calib>",                  # unbalanced
    "<Calib><MLAInfo><MLA><key><x/></key></MLA></MLAInfo></Calib>",       # element where text is read
])
def test_read_calib_rejects_what_the_reference_cannot_read(pfd, bad):
    with pytest.raises(pfd.PfdError):
        pfd.read_calib_xml(bad)


def test_read_intrinsics_rejects_missing_values(pfd):
    with pytest.raises(pfd.PfdError):
        pfd.read_intrinsics_xml("<_><distortions><depth><_><_>1</_></_></depth></distortions></_>")
    with pytest.raises(pfd.PfdError):
        pfd.read_intrinsics_xml("<Calib/>")
