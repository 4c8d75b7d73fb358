"""The CLI's PNG encoder (optimizec_b200/cli/png_writer.h) on the CPU: a small harness writes
known RGB images of several shapes (one and several 65535-byte stored deflate blocks); Python's
zlib decodes them, which checks the zlib header and the Adler-32, and every chunk CRC-32 is
recomputed."""
import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = r'''
#include "png_writer.h"
#include <cstdlib>
int main(int argc, char **argv)
{
    const int w = std::atoi(argv[2]), h = std::atoi(argv[3]);
    std::vector<unsigned char> rgb((size_t)w * h * 3);
    for (size_t i = 0; i < rgb.size(); ++i) rgb[i] = (unsigned char)((i * 7 + i / 13) & 255);
    return PngWriter().write(argv[1], w, h, rgb.data()) ? 0 : 1;
}
'''


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("png")
    src = d / "h.cpp"
    src.write_text(HARNESS)
    exe = d / "h"
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I", os.path.join(REPO, "optimizec_b200", "cli"),
                           "-o", str(exe), str(src)])
    return str(exe)


def decode(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, chunks = 8, b"", []
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        typ, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(typ + body) & 0xFFFFFFFF == crc
        chunks.append(typ)
        if typ == b"IHDR":
            w, h, depth, ctype, comp, filt, inter = struct.unpack(">IIBBBBB", body)
            assert (depth, ctype, comp, filt, inter) == (8, 2, 0, 0, 0)
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    assert chunks == [b"IHDR", b"IDAT", b"IEND"] and pos == len(data)
    raw = np.frombuffer(zlib.decompress(idat), dtype=np.uint8).reshape(h, 3 * w + 1)
    assert np.all(raw[:, 0] == 0)
    return raw[:, 1:].reshape(h, w, 3)


@pytest.mark.parametrize("w,h", [(1, 1), (7, 5), (200, 150), (3000, 40), (257, 257)])
def test_png_roundtrip(harness, tmp_path, w, h):
    path = str(tmp_path / "f.png")
    subprocess.check_call([harness, path, str(w), str(h)])
    img = decode(path)
    i = np.arange(w * h * 3, dtype=np.int64)
    ref = ((i * 7 + i // 13) & 255).astype(np.uint8).reshape(h, w, 3)
    assert np.array_equal(img, ref)
    # stored blocks: the file is the raw scanlines plus fixed framing (5 bytes a 65535-byte block)
    raw = (3 * w + 1) * h
    assert os.path.getsize(path) == 8 + 25 + 12 + 2 + raw + 5 * max(1, -(-raw // 65535)) + 4 + 12
