"""Time-lapse ingest on the CPU: the native TIFF reader against the arrays
written (PIL's writer and a minimal writer of this suite for the layouts PIL
does not write: big-endian, tiles, PackBits on every type), and the frame
source's read-ahead ring."""
import numpy as np
import pytest

from multi_quickpiv_b200 import _lib
from multi_quickpiv_b200.ingest import FrameSource, TiffFile, read_tiff, tiff_info
from tests.tiff_writer import write_tiff


def _pages(dtype, n=3, shape=(37, 53), seed=0):
    g = np.random.default_rng(seed)
    if np.dtype(dtype).kind == "f":
        return [g.normal(100, 40, shape).astype(dtype) for _ in range(n)]
    info = np.iinfo(dtype)
    return [g.integers(info.min, info.max, shape, endpoint=True).astype(dtype) for _ in range(n)]


def _check(path, pages):
    vol = read_tiff(path, 0, len(pages), dtype=np.float64)
    assert vol.shape == pages[0].shape + (len(pages),) and vol.flags.f_contiguous
    for k, p in enumerate(pages):
        assert np.array_equal(vol[:, :, k], p.astype(np.float64))
    one = read_tiff(path, len(pages) - 1)
    assert one.dtype == np.float32 and np.array_equal(one, pages[-1].astype(np.float32))


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float32])
@pytest.mark.parametrize("compression", [None, "packbits"])
def test_reads_pil_stacks(tmp_path, dtype, compression):
    from PIL import Image
    pages = _pages(dtype)
    path = str(tmp_path / "stack.tif")
    ims = [Image.fromarray(p) for p in pages]
    kw = {"compression": compression} if compression else {}
    ims[0].save(path, save_all=True, append_images=ims[1:], **kw)
    _check(path, pages)
    info = tiff_info(path)
    assert info["pages"] == 3 and info["width"] == 53 and info["height"] == 37 and info["uniform"] == 1


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.uint16, np.int32, np.uint32, np.float32, np.float64])
@pytest.mark.parametrize("layout", ["le_strips", "be_strips", "le_tiles_packbits", "be_tiles"])
def test_reads_every_layout(tmp_path, dtype, layout):
    pages = _pages(dtype, seed=3)
    path = str(tmp_path / "stack.tif")
    kw = {"le_strips": dict(byteorder="<", rows_per_strip=5),
          "be_strips": dict(byteorder=">", rows_per_strip=8, compress=True),
          "le_tiles_packbits": dict(byteorder="<", tile=(16, 16), compress=True),
          "be_tiles": dict(byteorder=">", tile=(16, 32))}[layout]
    write_tiff(path, pages, **kw)
    _check(path, pages)


def test_frame_source_reads_ahead_in_order(tmp_path):
    pages = _pages(np.uint16, n=7, shape=(24, 20), seed=5)
    path = str(tmp_path / "t.tif")
    write_tiff(path, pages, rows_per_strip=4)
    with FrameSource(path, ring=3) as src:
        assert src.frames == 7 and src.shape == (24, 20)
        got = [(k, f.copy()) for k, f in src]
    assert [k for k, _ in got] == list(range(7))
    for k, f in got:
        assert np.array_equal(f, pages[k].astype(np.float32))
    # 3D+t: frames of 3 pages; the trailing page that does not fill a frame is left out
    with FrameSource(path, pages_per_frame=3, dtype=np.float64, ring=2) as src:
        assert src.frames == 2 and src.shape == (24, 20, 3)
        k, f = src.next()
        assert np.array_equal(f, np.stack(pages[:3], -1).astype(np.float64))
        k, f = src.next()
        assert k == 1 and np.array_equal(f, np.stack(pages[3:6], -1).astype(np.float64))
        assert src.next() is None


def test_errors_are_reported(tmp_path):
    bad = tmp_path / "bad.tif"
    bad.write_bytes(b"not a tiff at all")
    with pytest.raises(_lib.MQPError):
        read_tiff(str(bad))
    with pytest.raises(_lib.MQPError):
        read_tiff(str(tmp_path / "missing.tif"))
    pages = _pages(np.uint8, n=2)
    path = str(tmp_path / "s.tif")
    write_tiff(path, pages)
    with TiffFile(path) as t:
        with pytest.raises(_lib.MQPError):
            t.read(1, 2)  # beyond the last page
