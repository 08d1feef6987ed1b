"""CPU tests: the reference's CSV universe format, the viewport mapping, the
render oracle's coverage and blending rules, and the PNG writer."""
import struct
import zlib

import numpy as np
import pytest


def test_csv_round_trip_is_exact(nbp, tmp_path):
    m, p, v = nbp.universes.exponential_disc(500, 3)
    b = nbp.Bodies(m, p, v, ids=[f"body-{i}" for i in range(500)])
    f = tmp_path / "u.csv"
    nbp.csvio.write_csv(f, b)
    lines = f.read_text().splitlines()
    assert lines[0] == "id,mass,x,y,vel_x,vel_y" and len(lines) == 501
    r = nbp.csvio.read_csv(f)
    assert r.ids == b.ids
    assert np.array_equal(r.mass, b.mass) and np.array_equal(r.pos, b.pos)
    assert np.array_equal(r.vel, b.vel)


@pytest.mark.parametrize("value,text", [(100000.0, "100000"), (1e-05, "1e-05"), (0.1, "0.1"),
                                        (1e16, "1e+16"), (-0.0, "-0"), (2.5e-320, "2.5e-320"),
                                        (5.972e24, "5.972e+24"), (123.456, "123.456")])
def test_numbers_are_written_shortest(nbp, value, text):
    assert nbp.csvio.format_double(value) == text
    assert float(text) == value


def test_csv_rejects_duplicate_ids_and_short_rows(nbp, tmp_path):
    f = tmp_path / "d.csv"
    f.write_text("id,mass,x,y,vel_x,vel_y\na,1,0,0,0,0\nb,1,1,0,0,0\na,2,0,1,0,0\n")
    with pytest.raises(ValueError, match="duplicate"):
        nbp.csvio.read_csv(f)
    f.write_text("id,mass,x,y,vel_x,vel_y\na,1,0,0\n")
    with pytest.raises(ValueError, match="6 columns"):
        nbp.csvio.read_csv(f)


def test_viewport_matches_the_reference_arithmetic(nbp):
    vp = nbp.render.ViewPort(800, 600, 0.05)
    assert (vp.x, vp.y, vp.width, vp.height) == (-20.0, -15.0, 40.0, 30.0)
    q = vp.coords_to_pos_on_viewport(np.array([[0.0, 0.0], [-20.0, -15.0], [10.0, 7.5]]))
    assert np.array_equal(q, np.array([[400, 300], [0, 0], [600, 450]], dtype=np.float32))
    vp.zoom(True, 400.0, 300.0)  # about the centre: the centre stays put
    c = vp.coords_to_pos_on_viewport(np.array([[0.0, 0.0]]))[0]
    assert np.allclose(c, [400, 300], atol=1e-3)
    vp.pan(80.0, 0.0)
    assert vp.coords_to_pos_on_viewport(np.array([[0.0, 0.0]]))[0][0] == pytest.approx(320, abs=1e-3)


def test_render_oracle_rules(orc_render):
    t = orc_render.blend_table()
    # 8-bit blending with rounding to nearest settles at 254: 120 + 254 * 135/255
    # = 254.47 rounds back to 254
    assert t[0] == 0 and t[1] == 120 and t[2] == 184 and t[255] == 254
    assert (np.diff(t.astype(int)) >= 0).all()
    # diameter 1: exactly the pixel whose centre is within half a pixel
    pos = np.array([[0.25, 0.25], [0.25, 0.25], [3.9, 2.1]])
    c = orc_render.coverage(pos, 0.0, 0.0, 8.0, 8.0, 8, 8, 1.0)
    assert c.sum() == 3 and c[0, 0] == 2 and c[2, 3] == 1
    # diameter 3 centred on a pixel centre: the 3 x 3 square minus nothing
    # (corners at distance sqrt(2)/3 < 1/2 from the sprite centre stay)
    c = orc_render.coverage(np.array([[4.5, 4.5]]), 0.0, 0.0, 8.0, 8.0, 8, 8, 3.0)
    assert c.sum() == 9 and c[3:6, 3:6].all()
    # diameter 5: the circle clip removes the four corners of the 5 x 5 square
    c = orc_render.coverage(np.array([[4.5, 4.5]]), 0.0, 0.0, 10.0, 10.0, 10, 10, 5.0)
    assert c.sum() == 21 and c[2, 2] == 0 and c[4, 2] == 1


def test_png_writer(nbp, tmp_path):
    img = np.zeros((3, 4, 4), dtype=np.uint8)
    img[1, 2] = (255, 120, 7, 255)
    f = tmp_path / "x.png"
    nbp.render.write_png(f, img)
    data = f.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    w, h = struct.unpack(">II", data[16:24])
    assert (w, h) == (4, 3)
    idat = data.index(b"IDAT")
    n = struct.unpack(">I", data[idat - 4:idat])[0]
    raw = zlib.decompress(data[idat + 4:idat + 4 + n])
    rows = np.frombuffer(raw, dtype=np.uint8).reshape(3, 1 + 16)
    assert (rows[:, 0] == 0).all() and np.array_equal(rows[:, 1:].reshape(3, 4, 4), img)
