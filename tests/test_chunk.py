"""The detector chunk codec (sf_chunk_*; the reference's decompress::image,
src/decompress.cc:85-134): HDF5 filter framing, LZ4 blocks and the
bitshuffle transpose.

The reference links the bitshuffle library and liblz4 for these, neither of
which is vendored (its third_party/bitshuffle submodule is empty). The LZ4
blocks are pinned against the system's liblz4 (LZ4_compress_default /
LZ4_decompress_safe, called through its public API) where it is installed;
the bit transpose against a numpy restatement of the published layout (bit
k of byte j of element e at bit e mod 8 of byte e / 8 of row 8j + k) and
against a chunk worked out by hand from the published formats.
Host tests need no device; the device decoder's tests are marked gpu."""

import ctypes
import ctypes.util
import struct

import numpy as np
import pytest

from dials_metal_spotfinder_b200 import chunk as C
from dials_metal_spotfinder_b200._lib import BadArgument


def liblz4():
    for name in ("lz4", "liblz4.so.1"):
        path = ctypes.util.find_library(name) if name == "lz4" else name
        if not path:
            continue
        try:
            lib = ctypes.CDLL(path)
        except OSError:
            continue
        lib.LZ4_compress_default.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                             ctypes.c_int]
        lib.LZ4_decompress_safe.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                            ctypes.c_int]
        return lib
    return None


LZ4 = liblz4()
needs_liblz4 = pytest.mark.skipif(LZ4 is None, reason="liblz4 is not installed")


def frames():
    rng = np.random.default_rng(11)
    out = []
    for h, w in [(1, 1), (1, 7), (3, 5), (17, 31), (64, 128), (257, 511), (1062, 1028)]:
        img = rng.poisson(1.5, (h, w)).astype(np.uint16)
        img[rng.random((h, w)) < 0.01] = rng.integers(100, 60000)
        if w > 10:
            img[:, w // 3] = 0xFFFF  # a module gap
        out.append(img)
    big = rng.integers(0, 2 ** 32, (130, 77), dtype=np.uint64).astype(np.uint32)
    out.append(big)
    out.append(np.zeros((40, 40), np.uint32))
    return out


def split_blocks(raw, n_coded):
    size, block = struct.unpack(">QI", raw[:12])
    at, done, out = 12, 0, []
    while done < n_coded:
        (cs,) = struct.unpack(">I", raw[at:at + 4])
        out.append(raw[at + 4:at + 4 + cs])
        at += 4 + cs
        done += min(block, n_coded - done)
    return size, block, out, raw[at:]


def bit_transpose(block: np.ndarray) -> bytes:
    """The published bitshuffle layout of one block (numpy restatement)."""
    n = len(block)
    s = block.dtype.itemsize
    b = block.view(np.uint8).reshape(n, s)                  # [element][byte]
    bits = np.unpackbits(b, axis=1, bitorder="little")       # [element][8*byte + bit]
    rows = bits.T.reshape(8 * s, n // 8, 8)                 # [row][group][element % 8]
    return np.packbits(rows, axis=2, bitorder="little").reshape(-1).tobytes()


def liblz4_chunk(img: np.ndarray, algorithm: str, block_bytes: int) -> np.ndarray:
    """A chunk in the HDF5 filter framing with any block size, its blocks
    compressed by liblz4 and, for bslz4, bit-transposed by the numpy
    restatement above (the trailing elements past a multiple of 8 copied
    as they are)."""
    s = img.dtype.itemsize
    flat = img.reshape(-1)
    raw = flat.view(np.uint8).tobytes()
    out = bytearray(struct.pack(">QI", len(raw), block_bytes))

    def emit(src: bytes):
        dst = ctypes.create_string_buffer(len(src) + len(src) // 255 + 64)
        cs = LZ4.LZ4_compress_default(src, dst, len(src), len(dst))
        assert cs > 0
        out.extend(struct.pack(">I", cs) + dst.raw[:cs])

    if algorithm == "lz4":
        for at in range(0, len(raw), block_bytes):
            emit(raw[at:at + block_bytes])
    else:
        per = block_bytes // s
        coded = len(flat) - len(flat) % 8
        for at in range(0, coded, per):
            emit(bit_transpose(flat[at:min(at + per, coded)]))
        out.extend(flat[coded:].view(np.uint8).tobytes())
    return np.frombuffer(bytes(out), np.uint8)


# A bitshuffle + LZ4 chunk worked out by hand from the published formats,
# not by any encoder here. The frame is 1 x 8 uint16 pixels
#     0x0001 0x0003 0x0000 0x8000 0x00ff 0x0100 0x0000 0xffff
# Low bytes by element:  01 03 00 00 ff 00 00 ff; high bytes: 00 00 00 80 00 01 00 ff.
# Bitshuffle writes, for byte j and bit k of the element, row 8j + k: one bit
# per element, element e at bit e mod 8 of byte e / 8 (8 elements: one byte
# per row, 16 rows).
#   row 0 (bit 0 of the low bytes): elements 0, 1, 4, 7    -> 0b10010011 = 0x93
#   row 1 (bit 1):                  elements 1, 4, 7       -> 0x92
#   rows 2-7:                       elements 4, 7          -> 0x90 each
#   row 8 (bit 0 of the high bytes): elements 5, 7         -> 0xa0
#   rows 9-14:                      element 7              -> 0x80 each
#   row 15 (bit 7):                 elements 3, 7          -> 0x88
# The LZ4 block holds those 16 bytes as one literals-only sequence: token
# 0xf0 (15 literals and more, no match), length byte 0x01 (15 + 1 = 16),
# then the 16 bytes. The HDF5 bitshuffle filter's framing before it: the
# uncompressed size as 8 big-endian bytes (16), the block size as 4 (8192
# bytes), then the block's compressed length as 4 (18).
HAND_FRAME = np.array([[0x0001, 0x0003, 0x0000, 0x8000, 0x00ff, 0x0100, 0x0000, 0xffff]],
                      np.uint16)
HAND_ROWS = bytes([0x93, 0x92] + [0x90] * 6 + [0xa0] + [0x80] * 6 + [0x88])
HAND_CHUNK = bytes.fromhex("0000000000000010" "00002000" "00000012" "f001") + HAND_ROWS


def test_hand_derived_bitshuffle_chunk_decodes():
    assert bit_transpose(HAND_FRAME.reshape(-1)) == HAND_ROWS
    got = C.decode(np.frombuffer(HAND_CHUNK, np.uint8), HAND_FRAME.shape, np.uint16, "bslz4")
    assert np.array_equal(got, HAND_FRAME)
    # the same eight pixels with two more after them: those two are not
    # transposed (not a whole group of 8) and follow the blocks as they are
    frame10 = np.concatenate([HAND_FRAME, [[0x1234, 0xabcd]]], axis=1).astype(np.uint16)
    chunk10 = (bytes.fromhex("0000000000000014" "00002000" "00000012" "f001") + HAND_ROWS +
               bytes.fromhex("3412" "cdab"))
    got = C.decode(np.frombuffer(chunk10, np.uint8), frame10.shape, np.uint16, "bslz4")
    assert np.array_equal(got, frame10)


@needs_liblz4
def test_our_bslz4_chunk_of_the_hand_frame_is_the_hand_rows():
    chunk = bytes(C.encode(HAND_FRAME, "bslz4"))
    size, block, parts, rest = split_blocks(chunk, 16)
    assert (size, len(parts), rest) == (16, 1, b"")
    dst = ctypes.create_string_buffer(16)
    assert LZ4.LZ4_decompress_safe(parts[0], dst, len(parts[0]), 16) == 16
    assert dst.raw == HAND_ROWS


@needs_liblz4
@pytest.mark.parametrize("algorithm", ["lz4", "bslz4"])
def test_liblz4_chunks_with_small_blocks_decode_with_ours(algorithm):
    for img in frames():
        chunk = liblz4_chunk(img, algorithm, 256 * img.dtype.itemsize)
        assert np.array_equal(C.decode(chunk, img.shape, img.dtype, algorithm), img)


@pytest.mark.parametrize("algorithm", ["raw", "lz4", "bslz4"])
def test_round_trip(algorithm):
    for img in frames():
        chunk = C.encode(img, algorithm)
        back = C.decode(chunk, img.shape, img.dtype, algorithm)
        assert np.array_equal(back, img), (algorithm, img.shape, img.dtype)


def test_synthetic_frames_compress():
    from dials_metal_spotfinder_b200 import synth
    img = synth.eiger_4m(frames=1).frame(0)
    chunk = C.encode(img, "bslz4")
    assert len(chunk) < img.nbytes / 2.5  # the high bit planes are almost all zero
    assert np.array_equal(C.decode(chunk, img.shape), img)


@needs_liblz4
@pytest.mark.parametrize("algorithm", ["lz4", "bslz4"])
def test_our_blocks_decode_with_liblz4(algorithm):
    for img in frames():
        n = img.size
        s = img.dtype.itemsize
        raw = bytes(C.encode(img, algorithm))
        coded = (n - n % 8) * s if algorithm == "bslz4" else n * s
        size, block, parts, rest = split_blocks(raw, coded)
        assert size == img.nbytes and block == 8192
        flat = img.reshape(-1)
        at = 0
        for part in parts:
            nbytes = min(block, coded - at)
            dst = ctypes.create_string_buffer(nbytes)
            got = LZ4.LZ4_decompress_safe(part, dst, len(part), nbytes)
            assert got == nbytes
            if algorithm == "bslz4":
                elems = flat[at // s:(at + nbytes) // s]
                assert dst.raw == bit_transpose(elems)
            else:
                assert dst.raw == flat.view(np.uint8)[at:at + nbytes].tobytes()
            at += nbytes
        assert rest == flat.view(np.uint8)[coded:].tobytes()


@needs_liblz4
def test_liblz4_blocks_decode_with_ours():
    rng = np.random.default_rng(5)
    img = rng.poisson(0.7, (300, 333)).astype(np.uint16)
    img[::7, ::5] = 4000
    n, s = img.size, 2
    flat = img.reshape(-1)
    coded = (n - n % 8) * s
    out = bytearray(struct.pack(">QI", img.nbytes, 8192))
    for at in range(0, coded, 8192):
        nbytes = min(8192, coded - at)
        src = bit_transpose(flat[at // s:(at + nbytes) // s])
        dst = ctypes.create_string_buffer(nbytes + nbytes // 255 + 64)
        cs = LZ4.LZ4_compress_default(src, dst, nbytes, len(dst))
        assert cs > 0
        out += struct.pack(">I", cs) + dst.raw[:cs]
    out += flat.view(np.uint8)[coded:].tobytes()
    back = C.decode(np.frombuffer(bytes(out), np.uint8), img.shape, np.uint16, "bslz4")
    assert np.array_equal(back, img)


@needs_liblz4
@pytest.mark.parametrize("block", [65536, 1 << 30])
def test_large_lz4_blocks_decode_on_the_host(block):
    """HDF5's LZ4 filter writes blocks far beyond 8 KB (1 GB by default, so a
    frame is one block): liblz4's blocks of 64 KB and of the whole frame
    decode to the frame, and a block cut short is refused."""
    rng = np.random.default_rng(12)
    img = rng.poisson(0.9, (333, 517)).astype(np.uint16)
    img[::11, ::3] = 4000
    raw = img.reshape(-1).view(np.uint8).tobytes()
    out = bytearray(struct.pack(">QI", len(raw), block))
    for at in range(0, len(raw), block):
        src = raw[at:at + block]
        dst = ctypes.create_string_buffer(len(src) + len(src) // 255 + 64)
        cs = LZ4.LZ4_compress_default(src, dst, len(src), len(dst))
        assert cs > 0
        out += struct.pack(">I", cs) + dst.raw[:cs]
    good = np.frombuffer(bytes(out), np.uint8)
    assert np.array_equal(C.decode(good, img.shape, np.uint16, "lz4"), img)
    with pytest.raises(BadArgument):
        C.decode(good[:-1], img.shape, np.uint16, "lz4")


def test_malformed_chunks_are_refused():
    rng = np.random.default_rng(2)
    img = rng.poisson(2.0, (100, 90)).astype(np.uint16)
    good = C.encode(img, "bslz4")
    with pytest.raises(BadArgument):
        C.decode(good[:-3], img.shape)                     # truncated
    with pytest.raises(BadArgument):
        C.decode(good, (100, 91))                          # header size mismatch
    with pytest.raises(BadArgument):
        C.decode(C.encode(img, "raw"), img.shape, algorithm="lz4")
    bad = good.copy()
    bad[16] ^= 0xF0                                        # a corrupted token
    try:
        back = C.decode(bad, img.shape)
    except BadArgument:
        pass
    else:
        assert not np.array_equal(back, img)
    with pytest.raises(BadArgument):
        C.decode(good, img.shape, algorithm=7)


# -- the device decoder ------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("algorithm", ["raw", "lz4", "bslz4"])
def test_device_decode_feeds_the_engine(gpu_lib, algorithm):
    from dials_metal_spotfinder_b200 import synth
    from dials_metal_spotfinder_b200.engine import Engine
    from oracle import oracle as O
    shapes = [(2162, 2068), (257, 511), (1062, 1028)]
    rng = np.random.default_rng(7)
    imgs = [synth.eiger_4m(frames=1).frame(0)]
    for h, w in shapes[1:]:
        img = rng.poisson(1.2, (h, w)).astype(np.uint16)
        img[rng.random((h, w)) < 0.003] = 5000
        imgs.append(img)
    chunks = [C.encode(img, algorithm) for img in imgs]
    with Engine(shapes, np.uint16, slots=2) as eng:
        for rep in range(2):  # reuse of the staging buffers
            for f, ch in enumerate(chunks):
                eng.upload_chunk(rep % 2, f, ch, algorithm)
            eng.run(rep % 2)
            eng.synchronize()
            for f, img in enumerate(imgs):
                assert eng.signal(rep % 2, f).tobytes() == O.dext(img)[1].tobytes()


@pytest.mark.gpu
def test_device_decodes_the_hand_derived_chunk(gpu_lib):
    import torch
    dev = torch.zeros(HAND_FRAME.shape, dtype=torch.uint16, device="cuda")
    C.decode_device(np.frombuffer(HAND_CHUNK, np.uint8), HAND_FRAME.shape, np.uint16,
                    dev.data_ptr())
    assert np.array_equal(dev.cpu().numpy(), HAND_FRAME)


@pytest.mark.gpu
def test_device_decode_u32(gpu_lib):
    from dials_metal_spotfinder_b200.engine import Engine
    from oracle import oracle as O
    rng = np.random.default_rng(9)
    img = rng.poisson(3.0, (333, 517)).astype(np.uint32)
    img[rng.random(img.shape) < 0.002] = 2_000_000
    with Engine([img.shape], np.uint32) as eng:
        eng.upload_chunk(0, 0, C.encode(img, "bslz4"))
        eng.run(0)
        eng.synchronize()
        assert eng.signal(0, 0).tobytes() == O.dext(img)[1].tobytes()


@pytest.mark.gpu
def test_device_reports_a_malformed_block(gpu_lib):
    from dials_metal_spotfinder_b200._lib import DeviceError
    from dials_metal_spotfinder_b200.engine import Engine
    rng = np.random.default_rng(3)
    img = rng.poisson(2.0, (256, 384)).astype(np.uint16)
    good = C.encode(img, "bslz4")
    size, block, parts, rest = split_blocks(bytes(good), img.nbytes)
    # framing intact, first block's content replaced by a match whose offset
    # reaches before the start of the output
    first = bytes([0x0F, 0xFF, 0xFF]) + parts[0][3:]
    bad = bytearray(good[:12]) + struct.pack(">I", len(first)) + first
    bad += bytes(good[12 + 4 + len(parts[0]):])
    with Engine([img.shape], np.uint16) as eng:
        eng.upload_chunk(0, 0, np.frombuffer(bytes(bad), np.uint8))
        eng.run(0)
        with pytest.raises(DeviceError):
            eng.synchronize()
        eng.upload_chunk(0, 0, good)  # and the engine still works
        eng.run(0)
        eng.synchronize()


@pytest.mark.gpu
@pytest.mark.parametrize("algorithm", ["raw", "lz4", "bslz4"])
@pytest.mark.parametrize("dtype", [np.uint16, np.uint32])
def test_device_decode_is_exact(gpu_lib, algorithm, dtype):
    """Every byte of the decoded frame, at a pitch wider than the row and at
    the row's own length: widths whose rows end inside a group of eight
    elements, single columns, frames shorter than one block, a raw tail."""
    import torch
    rng = np.random.default_rng(11)
    shapes = [(1, 1), (3, 5), (7, 3), (1, 9), (41, 465), (257, 511), (300, 4148 // 4),
              (1062, 1028), (64, 4099)]
    for h, w in shapes:
        img = rng.poisson(1.5, (h, w)).astype(dtype)
        img[rng.random((h, w)) < 0.01] = np.iinfo(dtype).max
        img[rng.random((h, w)) < 0.005] = rng.integers(1000, 60000)
        ch = C.encode(img, algorithm)
        eb = img.dtype.itemsize
        for pitch in (w * eb, ((w * eb + 127) // 128) * 128 + 16):
            dev = torch.full((h * pitch,), 0xA5, dtype=torch.uint8, device="cuda")
            C.decode_device(ch, img.shape, dtype, dev.data_ptr(), pitch, algorithm)
            got = dev.cpu().numpy().reshape(h, pitch)
            rows = got[:, : w * eb].copy().view(dtype)
            assert np.array_equal(rows, img), (algorithm, h, w, pitch)
            # the bytes between rows are untouched
            assert (got[:, w * eb:] == 0xA5).all(), (algorithm, h, w, pitch)


@pytest.mark.gpu
def test_device_decode_16m_frame(gpu_lib):
    import torch
    from dials_metal_spotfinder_b200 import synth
    img = synth.eiger_16m(frames=1).frame(0)
    h, w = img.shape
    ch = C.encode(img, "bslz4")
    dev = torch.empty((h, 4224), dtype=torch.uint16, device="cuda")
    C.decode_device(ch, img.shape, np.uint16, dev.data_ptr(), 4224 * 2)
    assert np.array_equal(dev[:, :w].cpu().numpy(), img)


@pytest.mark.gpu
def test_device_decode_refuses_a_malformed_block(gpu_lib):
    import torch
    from dials_metal_spotfinder_b200._lib import DeviceError
    rng = np.random.default_rng(3)
    img = rng.poisson(2.0, (256, 384)).astype(np.uint16)
    good = C.encode(img, "bslz4")
    size, block, parts, rest = split_blocks(bytes(good), img.nbytes)
    first = bytes([0x0F, 0xFF, 0xFF]) + parts[0][3:]
    bad = bytearray(good[:12]) + struct.pack(">I", len(first)) + first
    bad += bytes(good[12 + 4 + len(parts[0]):])
    dev = torch.empty(img.shape, dtype=torch.uint16, device="cuda")
    with pytest.raises(DeviceError):
        C.decode_device(np.frombuffer(bytes(bad), np.uint8), img.shape, np.uint16, dev.data_ptr())
    C.decode_device(good, img.shape, np.uint16, dev.data_ptr())
    assert np.array_equal(dev.cpu().numpy(), img)


@pytest.mark.gpu
@needs_liblz4
@pytest.mark.parametrize("block", [65536, 0])
def test_device_decode_large_lz4_blocks(gpu_lib, block):
    """Plain LZ4 chunks whose blocks exceed shared memory (HDF5's LZ4 filter
    writes up to 1 GB blocks; 0 here: the whole frame in one block), made by
    liblz4, decode on the device exactly as on the host."""
    import torch
    rng = np.random.default_rng(8)
    img = rng.poisson(0.8, (517, 1031)).astype(np.uint16)
    img[::9, ::4] = 3000
    raw = img.reshape(-1).view(np.uint8).tobytes()
    bs = block or len(raw)
    out = bytearray(struct.pack(">QI", len(raw), bs))
    for at in range(0, len(raw), bs):
        src = raw[at:at + bs]
        dst = ctypes.create_string_buffer(len(src) + len(src) // 255 + 64)
        cs = LZ4.LZ4_compress_default(src, dst, len(src), len(dst))
        assert cs > 0
        out += struct.pack(">I", cs) + dst.raw[:cs]
    ch = np.frombuffer(bytes(out), np.uint8)
    assert np.array_equal(C.decode(ch, img.shape, np.uint16, "lz4"), img)
    pitch = 1031 * 2 + 50
    dev = torch.zeros((517 * pitch,), dtype=torch.uint8, device="cuda")
    C.decode_device(ch, img.shape, np.uint16, dev.data_ptr(), pitch, "lz4")
    got = dev.cpu().numpy().reshape(517, pitch)[:, :1031 * 2].copy().view(np.uint16)
    assert np.array_equal(got, img)


@pytest.mark.gpu
@needs_liblz4
@pytest.mark.parametrize("algorithm", ["lz4", "bslz4"])
def test_batched_chunk_uploads_match_the_oracle(gpu_lib, algorithm):
    """upload_chunks: every frame of the batch, in any frame order, gives the
    oracle's list, as per-frame upload_chunk does. Eight batches of six
    chunks (48 uploads) wrap the 32-deep block-table ring; the last three
    batches use frames with smaller LZ4 blocks, so more blocks per chunk,
    and a table still in use must grow."""
    from dials_metal_spotfinder_b200.engine import Engine
    from oracle import oracle as O
    rng = np.random.default_rng(21)
    shape = (517, 733)
    imgs = []
    for _ in range(6):
        img = rng.poisson(1.4, shape).astype(np.uint16)
        img[rng.random(shape) < 0.004] = rng.integers(200, 30000)
        imgs.append(img)
    chunks = [C.encode(img, algorithm) for img in imgs]
    # 1 KB blocks: eight times as many per chunk as the encoder's 8 KB
    small = [liblz4_chunk(img, algorithm, 1024) for img in imgs]
    order = [3, 0, 5, 1, 4, 2]
    with Engine([shape] * 6, np.uint16, slots=2) as eng:
        for rep in range(8):
            use = small if rep >= 5 else chunks
            eng.upload_chunks(rep % 2, [use[f] for f in order], frames=order,
                              algorithm=algorithm)
            eng.run(rep % 2)
            eng.synchronize()
            for f, img in enumerate(imgs):
                assert eng.signal(rep % 2, f).tobytes() == O.dext(img)[1].tobytes()


@pytest.mark.gpu
def test_batched_chunk_uploads_refuse_every_chunk_for_one_bad_one(gpu_lib):
    from dials_metal_spotfinder_b200.engine import Engine
    from oracle import oracle as O
    rng = np.random.default_rng(22)
    shape = (256, 384)
    imgs = [rng.poisson(2.0, shape).astype(np.uint16) for _ in range(3)]
    good = [C.encode(img, "bslz4") for img in imgs]
    bad = good[:]
    bad[1] = good[1][:-3]  # framing no longer describes the frame
    with Engine([shape] * 3, np.uint16) as eng:
        with pytest.raises(BadArgument):
            eng.upload_chunks(0, bad)
        eng.upload_chunks(0, good)
        eng.run(0)
        eng.synchronize()
        for f, img in enumerate(imgs):
            assert eng.signal(0, f).tobytes() == O.dext(img)[1].tobytes()
