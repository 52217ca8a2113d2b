"""CPU restatement of the reference's frame file format -- test infrastructure.

NuiFileIOUtilities::writeFrameImage / readFrameImageHeader / readFrameImageBuffer
(src/Foundation/NuiFileIOUtilities.cpp:13-118): int64 timestamp, uint32 width, uint32 height,
uint32 stored size, payload.  Written compressed, the payload is zlib's compress2 at
Z_BEST_SPEED (level 1) of the pixels and the stored size is its length; otherwise the raw
pixels with their size.  The reader decompresses whenever the stored size differs from the
expected pixel bytes.  writeCamera / readCamera (:120-161): four floats fx, fy, cx, cy.
"""
import struct
import zlib

import numpy as np


def write_frame(path, pixels, timestamp, compressed):
    a = np.ascontiguousarray(pixels)
    h, w = a.shape[:2]
    raw = a.tobytes()
    payload = zlib.compress(raw, 1) if compressed else raw
    with open(path, "wb") as f:
        f.write(struct.pack("<qIII", timestamp, w, h, len(payload)))
        f.write(payload)


def read_frame(path, dtype, channels=1):
    with open(path, "rb") as f:
        ts, w, h, stored = struct.unpack("<qIII", f.read(20))
        payload = f.read(stored)
    nbytes = w * h * channels * np.dtype(dtype).itemsize
    raw = payload if stored == nbytes else zlib.decompress(payload)
    shape = (h, w) if channels == 1 else (h, w, channels)
    return ts, np.frombuffer(raw, dtype).reshape(shape).copy(), stored


def write_camera(path, fx, fy, cx, cy):
    with open(path, "wb") as f:
        f.write(struct.pack("<4f", fx, fy, cx, cy))


def read_camera(path):
    with open(path, "rb") as f:
        return struct.unpack("<4f", f.read(16))
