"""PNG output of tone-mapped films (host code, no GPU)."""
import numpy as np

from wayland_b200.png import read_png, write_png


def test_png_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, (37, 53, 4), dtype=np.uint8)
    path = tmp_path / "a.png"
    write_png(path, img)
    back = read_png(path)
    assert np.array_equal(back, img[::-1])  # stored flipped vertically, as the reference does
    write_png(path, img, flip=False)
    assert np.array_equal(read_png(path), img)
    raw = open(path, "rb").read()
    assert raw[:8] == b"\x89PNG\r\n\x1a\n" and b"IHDR" in raw[:16] and raw[-8:-4] == b"IEND"
