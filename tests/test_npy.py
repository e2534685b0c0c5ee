"""`.npy` interchange (nmx_npy_save / nmx_npy_load / nmx_npy_header) on host
tensors, against numpy's own reader and writer.

numpy.lib.format is the oracle here: every file the library writes must be
byte-identical to numpy.save's for the same array, and every file numpy.save
writes must load to the same values.  The cases follow numax's own tests of
the format (numax tests/io/test_npy.mojo:122-305): numpy-written rank-1 f32
and rank-2 i32 files, byte identity of a saved rank-1 f32 array (144
bytes), the rank-2 header text, round trips, load_dyn, and the failures
numax raises on -- Fortran order, a big-endian descr, a dtype or shape
mismatch, a rank the file does not have, a non-.npy (.npz) file.  No GPU:
host tensors take the library's no-CUDA path."""
import io
import os
import struct
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "numax_b200", "libnmxla.so")),
    reason="libnmxla.so not built")

NP_OF = {torch.float32: np.float32, torch.float64: np.float64, torch.float16: np.float16,
         torch.int8: np.int8, torch.int16: np.int16, torch.int32: np.int32,
         torch.int64: np.int64, torch.uint8: np.uint8, torch.uint16: np.uint16,
         torch.uint32: np.uint32, torch.uint64: np.uint64, torch.bool: np.bool_}


def np_bytes(a: np.ndarray) -> bytes:
    b = io.BytesIO()
    np.save(b, a)
    return b.getvalue()


def sample(np_dtype, shape, seed=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    n = int(np.prod(shape)) if len(shape) else 1
    if np_dtype == np.bool_:
        v = rng.integers(0, 2, n).astype(np.bool_)
    elif np.issubdtype(np_dtype, np.floating):
        v = rng.standard_normal(n).astype(np_dtype)
    else:
        info = np.iinfo(np_dtype)
        v = rng.integers(info.min, info.max, n, dtype=np_dtype, endpoint=True)
    return v.reshape(shape)


@pytest.fixture
def npx():
    from numax_b200.io import numpy as npx
    return npx


SHAPES = [(4,), (2, 3), (), (0,), (3, 0, 2), (2, 3, 4, 5), (1,) * 8, (7, 1, 9)]


@pytest.mark.parametrize("tdt", list(NP_OF))
@pytest.mark.parametrize("shape", SHAPES)
def test_save_is_byte_identical_to_numpy(npx, tmp_path, tdt, shape):
    a = sample(NP_OF[tdt], shape, seed=len(shape))
    p = tmp_path / "a.npy"
    npx.save(torch.from_numpy(a.copy()), p)
    assert p.read_bytes() == np_bytes(a)


@pytest.mark.parametrize("tdt", list(NP_OF))
@pytest.mark.parametrize("shape", SHAPES)
def test_load_reads_numpy_files(npx, tmp_path, tdt, shape):
    a = sample(NP_OF[tdt], shape, seed=3 + len(shape))
    p = tmp_path / "a.npy"
    np.save(p, a)
    got = npx.load(p, tdt, *shape)
    assert tuple(got.shape) == shape and got.dtype == tdt
    assert got.numpy().tobytes() == a.tobytes()
    dyn = npx.load_dyn(p, tdt, len(shape))
    assert tuple(dyn.shape) == shape and dyn.numpy().tobytes() == a.tobytes()


def test_numax_fixture_f32_rank1(npx, tmp_path):
    # numax's fixture: float32([1.5, -2.25, 3.0, 0.125]) -> a 144-byte file
    # (10-byte prelude, 118-byte header, 16-byte payload).
    a = np.array([1.5, -2.25, 3.0, 0.125], np.float32)
    p = tmp_path / "f.npy"
    npx.save(torch.from_numpy(a), p)
    data = p.read_bytes()
    assert len(data) == 144 and data == np_bytes(a)
    assert data[:10] == b"\x93NUMPY\x01\x00" + struct.pack("<H", 118)
    assert data[10:].startswith(b"{'descr': '<f4', 'fortran_order': False, 'shape': (4,), }  ")
    assert data[127:128] == b"\n"
    assert npx.load(p, torch.float32, 4).tolist() == [1.5, -2.25, 3.0, 0.125]


def test_numax_fixture_i32_rank2_and_f64_header(npx, tmp_path):
    p = tmp_path / "i.npy"
    np.save(p, np.array([[1, 2], [3, 4]], np.int32))
    assert npx.load(p, torch.int32, 2, 2).tolist() == [[1, 2], [3, 4]]
    q = tmp_path / "d.npy"
    npx.save(torch.arange(6, dtype=torch.float64).reshape(2, 3), q)
    data = q.read_bytes()
    assert len(data) == 10 + 118 + 48
    assert data[10:].startswith(b"{'descr': '<f8', 'fortran_order': False, 'shape': (2, 3), }  ")


def test_growth_padding_across_a_64_byte_boundary(npx, tmp_path):
    # numpy adds 21 - digits(shape[0]) spaces after the dict; with a long
    # shape that pushes the header past the next 64-byte boundary.
    shape = (0,) + (1,) * 15
    a = np.empty(shape, np.float32)
    p = tmp_path / "g.npy"
    npx.save(torch.empty(shape, dtype=torch.float32), p)
    assert p.read_bytes() == np_bytes(a)
    assert len(np_bytes(a)) == 192


def test_load_accepts_format_2_and_native_order_descr(npx, tmp_path):
    a = sample(np.float64, (3, 5), seed=11)
    p = tmp_path / "v2.npy"
    with open(p, "wb") as f:
        np.lib.format.write_array(f, a, version=(2, 0))
    assert npx.load(p, torch.float64, 3, 5).numpy().tobytes() == a.tobytes()
    # '=f8' (native order) and '<u1'/'|u1' name the same types as '<f8' / '|u1'.
    raw = np_bytes(a).replace(b"'<f8'", b"'=f8'")
    (tmp_path / "eq.npy").write_bytes(raw)
    assert npx.load(tmp_path / "eq.npy", torch.float64, 3, 5).numpy().tobytes() == a.tobytes()
    b = np.arange(6, dtype=np.uint8)
    raw = np_bytes(b).replace(b"'|u1'", b"'<u1'")
    (tmp_path / "u1.npy").write_bytes(raw)
    assert npx.load(tmp_path / "u1.npy", torch.uint8, 6).tolist() == list(range(6))


def test_round_trip_bits_and_large_payload(npx, tmp_path):
    # 40 MiB: several 8 MiB chunks over the worker threads.
    a = torch.from_numpy(sample(np.float64, (5, 1024, 1024), seed=2))
    p = tmp_path / "big.npy"
    npx.save(a, p)
    assert p.read_bytes() == np_bytes(a.numpy())
    b = npx.load(p, torch.float64, 5, 1024, 1024)
    assert torch.equal(a.view(torch.int64), b.view(torch.int64))
    c = np.load(p)
    assert c.tobytes() == a.numpy().tobytes()


def test_header_reports_dtype_rank_shape(tmp_path):
    import ctypes as C
    from numax_b200 import _lib
    p = tmp_path / "h.npy"
    np.save(p, np.zeros((3, 4, 5), np.int16))
    code, rank, off = C.c_int(), C.c_int(), C.c_int64()
    shape = (C.c_int64 * 8)()
    assert _lib.load().nmx_npy_header(os.fsencode(p), C.byref(code), C.byref(rank), shape, 8,
                                      C.byref(off)) == 0
    assert (code.value, rank.value, list(shape[:3]), off.value) == (4, 3, [3, 4, 5], 128)
    np.save(p, np.zeros(2, np.complex64))
    assert _lib.load().nmx_npy_header(os.fsencode(p), C.byref(code), C.byref(rank), shape, 8,
                                      None) == 0
    assert code.value == -1


def _expect(npx, path, dtype, dims, text, dyn=False):
    from numax_b200.io import NpyError
    with pytest.raises(NpyError) as e:
        if dyn:
            npx.load_dyn(path, dtype, dims)
        else:
            npx.load(path, dtype, *dims)
    assert text in str(e.value), str(e.value)


def test_load_raises_like_numax(npx, tmp_path):
    a = np.array([1.5, -2.25, 3.0, 0.125], np.float32)
    good = np_bytes(a)
    p = tmp_path / "x.npy"
    # Fortran order.
    f = np_bytes(np.asfortranarray(np.zeros((2, 3), np.float32)))
    assert b"'fortran_order': True" in f
    p.write_bytes(f)
    _expect(npx, p, torch.float32, (2, 3), "Fortran-ordered .npy")
    # Big-endian descr.
    p.write_bytes(np_bytes(a.astype(">f4")))
    _expect(npx, p, torch.float32, (4,), "big-endian .npy (descr '>f4')")
    # dtype mismatch.
    p.write_bytes(good)
    _expect(npx, p, torch.int32, (4,), "dtype mismatch -- the file holds '<f4' but '<i4'")
    # Shape and rank mismatch.
    _expect(npx, p, torch.float32, (2, 2), "rank mismatch -- the file is rank 1, rank 2")
    _expect(npx, p, torch.float32, (5,), "shape mismatch")
    _expect(npx, p, torch.float32, 2, "rank mismatch", dyn=True)
    # Not a .npy file (an .npz archive is a zip container).
    p.write_bytes(b"PK\x03\x04 this is a zip, i.e. an .npz")
    _expect(npx, p, torch.float32, (4,), "bad magic bytes -- not a .npy file")
    z = tmp_path / "z.npz"
    np.savez(z, a=a)
    _expect(npx, z, torch.float32, (4,), "bad magic bytes")
    # Short payload, short file, unknown version, missing file.
    p.write_bytes(good[:-4])
    _expect(npx, p, torch.float32, (4,), "payload size doesn't match the header")
    p.write_bytes(good[:6])
    _expect(npx, p, torch.float32, (4,), "file too short to be a .npy file")
    p.write_bytes(good[:6] + b"\x03\x00" + good[8:])
    _expect(npx, p, torch.float32, (4,), "unsupported .npy format version")
    p.write_bytes(good[:40])
    _expect(npx, p, torch.float32, (4,), "truncated .npy header")
    _expect(npx, tmp_path / "missing.npy", torch.float32, (4,), "cannot open")


def test_save_rejects_bfloat16(npx, tmp_path):
    from numax_b200.io import NpyError
    with pytest.raises(NpyError, match="bfloat16 has no NumPy dtype"):
        npx.save(torch.zeros(3, dtype=torch.bfloat16), tmp_path / "b.npy")
    p = tmp_path / "f.npy"
    np.save(p, np.zeros(3, np.float32))
    with pytest.raises(NpyError, match="bfloat16 has no NumPy dtype"):
        npx.load(p, torch.bfloat16, 3)


def test_save_of_a_strided_tensor_writes_its_c_order(npx, tmp_path):
    # numax writes a tensor in row-major order whatever its view; a
    # transposed torch view is saved as its C-order copy.
    a = torch.arange(12, dtype=torch.float64).reshape(3, 4).t()
    p = tmp_path / "t.npy"
    npx.save(a, p)
    assert p.read_bytes() == np_bytes(np.ascontiguousarray(a.numpy()))
    assert npx.load(p, torch.float64, 4, 3).tolist() == a.tolist()
