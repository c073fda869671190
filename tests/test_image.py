"""Film output and film filters (host-only C ABI, no GPU):
* PFM as write_image_pfm writes it (core/imageio.rs:264-310): header, rows
  bottom to top, little-endian, bit-exact round trip, either byte order read;
* the filters of the filters/ directory and the film's 16 x 16 weight table
  (core/film.rs:70-82) against a float32 numpy restatement of the same
  expressions (exact where the arithmetic is + - * /, a few ulps where it
  calls exp or sin)."""
import os

import numpy as np
import pytest

from rs_illume_b200 import image

F = np.float32


def test_pfm_layout_and_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    img = rng.standard_normal((2, 3, 3)).astype(np.float32)
    p = str(tmp_path / "a.pfm")
    image.write_pfm(p, img)
    raw = open(p, "rb").read()
    head = b"PF\n3 2\n-1\n"
    assert raw.startswith(head)
    body = np.frombuffer(raw[len(head):], "<f4").reshape(2, 3, 3)
    assert np.array_equal(body[0], img[1]) and np.array_equal(body[1], img[0])    # bottom row first
    assert image.read_pfm(p).tobytes() == img.tobytes()


def test_pfm_reads_big_endian(tmp_path):
    img = np.arange(2 * 2 * 3, dtype=np.float32).reshape(2, 2, 3)
    p = str(tmp_path / "b.pfm")
    with open(p, "wb") as f:
        f.write(b"PF\n2 2\n1.0\n" + img[::-1].astype(">f4").tobytes())
    assert np.array_equal(image.read_pfm(p), img)


def test_pfm_rejects_bad_files(tmp_path):
    p = str(tmp_path / "c.pfm")
    with open(p, "wb") as f:
        f.write(b"P6\n2 2\n255\n" + bytes(12))
    with pytest.raises(Exception):
        image.read_pfm(p)
    with pytest.raises(Exception):
        image.read_pfm(str(tmp_path / "missing.pfm"))


def table_points(radius):
    x = ((np.arange(16, dtype=F) + F(0.5)) * F(radius[0])) / F(16)
    y = ((np.arange(16, dtype=F) + F(0.5)) * F(radius[1])) / F(16)
    return np.meshgrid(x, y)


def mitchell1d(x, b, c):
    b, c = F(b), F(c)
    x = np.abs(F(2) * x)
    far = ((-b - F(6) * c) * x * x * x + (F(6) * b + F(30) * c) * x * x + (F(-12) * b - F(48) * c) * x +
           (F(8) * b + F(24) * c)) * (F(1) / F(6))
    near = ((F(12) - F(9) * b - F(6) * c) * x * x * x + (F(-18) + F(12) * b + F(6) * c) * x * x +
            (F(6) - F(2) * b)) * (F(1) / F(6))
    return np.where(x > F(1), far, near).astype(F)


def test_box_and_triangle_tables_exact():
    t = image.filter_table(image.filter_desc("box", (0.5, 0.5)))
    assert np.all(t == 1.0)
    r = (2.0, 1.5)
    x, y = table_points(r)
    want = np.maximum(F(r[0]) - np.abs(x), F(0)) * np.maximum(F(r[1]) - np.abs(y), F(0))
    assert image.filter_table(image.filter_desc("triangle", r)).tobytes() == want.astype(F).tobytes()


def test_mitchell_table_exact():
    r, b, c = (2.0, 2.0), 1.0 / 3.0, 1.0 / 3.0
    x, y = table_points(r)
    inv = F(1) / F(2.0)
    want = mitchell1d(x * inv, b, c) * mitchell1d(y * inv, b, c)
    got = image.filter_table(image.filter_desc("mitchell", r, b, c))
    assert got.tobytes() == want.astype(F).tobytes()
    # mitchell1d(0) = (6 - 2B) / 6
    assert image.filter_evaluate(image.filter_desc("mitchell", r, b, c), 0.0, 0.0) == pytest.approx(
        ((6 - 2 * b) / 6) ** 2, rel=1e-6)


def test_gaussian_and_lanczos_tables():
    r, alpha = (1.5, 1.5), 2.0
    x, y = table_points(r)
    e = np.exp(F(-alpha) * F(r[0]) * F(r[0]))
    g = lambda d: np.maximum(np.exp(F(-alpha) * d * d) - e, F(0))
    got = image.filter_table(image.filter_desc("gaussian", r, alpha))
    np.testing.assert_allclose(got, g(x) * g(y), rtol=4e-7, atol=1e-9)
    r, tau = (3.0, 3.0), 3.0
    x, y = table_points(r)

    def sinc(v):
        v = np.abs(v)
        return np.where(v < F(1e-5), F(1), np.sin(F(np.pi) * v) / (F(np.pi) * v))

    def wsinc(v, rad):
        v = np.abs(v)
        return np.where(v > F(rad), F(0), sinc(v) * sinc(v / F(tau)))
    got = image.filter_table(image.filter_desc("lanczos", r, tau))
    np.testing.assert_allclose(got, wsinc(x, r[0]) * wsinc(y, r[1]), rtol=2e-6, atol=1e-7)
    assert image.filter_evaluate(image.filter_desc("lanczos", r, tau), 0.0, 0.0) == 1.0
    assert image.filter_evaluate(image.filter_desc("lanczos", r, tau), 3.5, 0.0) == 0.0


def test_filter_rejects_bad_descriptions():
    with pytest.raises(Exception):
        image.filter_table(image.filter_desc("box", (0.0, 1.0)))
    with pytest.raises(Exception):
        image.filter_table(image.filter_desc("lanczos", (1.0, 1.0), 0.0))


def test_golden_render_as_pfm():
    here = os.path.join(os.path.dirname(__file__), "golden")
    g = np.load(os.path.join(here, "golden.npz"))
    assert image.read_pfm(os.path.join(here, "pt_tile.pfm")).tobytes() == g["pt_image"].tobytes()
