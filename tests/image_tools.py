"""Decoders for the image files of the film-output tests: Radiance .hdr
(flat and run-length scanlines) to RGBE bytes; .png and .bmp through PIL."""
import numpy as np


def read_hdr_rgbe(path):
    """RGBE bytes (h, w, 4) of a Radiance .hdr file with a -Y h +X w header."""
    data = open(path, "rb").read()
    pos = 0
    while True:  # header lines up to the resolution line
        end = data.index(b"\n", pos)
        line = data[pos:end].decode("ascii", "replace")
        pos = end + 1
        if line.startswith("-Y "):
            _, h, _, w = line.split()
            h, w = int(h), int(w)
            break
    out = np.zeros((h, w, 4), np.uint8)
    for y in range(h):
        if 8 <= w <= 32767 and data[pos] == 2 and data[pos + 1] == 2 and not (data[pos + 2] & 0x80):
            assert (data[pos + 2] << 8 | data[pos + 3]) == w
            pos += 4
            for c in range(4):
                x = 0
                while x < w:
                    n = data[pos]
                    pos += 1
                    if n > 128:
                        out[y, x:x + n - 128, c] = data[pos]
                        pos += 1
                        x += n - 128
                    else:
                        out[y, x:x + n, c] = np.frombuffer(data[pos:pos + n], np.uint8)
                        pos += n
                        x += n
        else:
            out[y] = np.frombuffer(data[pos:pos + 4 * w], np.uint8).reshape(w, 4)
            pos += 4 * w
    return out


def read_rgb8(path):
    from PIL import Image
    return np.asarray(Image.open(path).convert("RGB"))
