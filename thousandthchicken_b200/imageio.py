"""Output writers for decoded images: PNM (PGM/PPM) and PGX.

The reference's decoder hands its components to the host and writes them out
through its test harness.  These writers close the same loop for the planar
samples this package decodes.  PGX is the JPEG 2000 conformance format: one
file per component with a "PG ML +|- <depth> <width> <height>" header and
big-endian samples.  PNM covers 1 component (PGM) and 3 components (PPM),
with a maximum value of 2^bits - 1 and big-endian 16-bit samples above
8 bits.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np


def _planes(planes: np.ndarray) -> np.ndarray:
    planes = np.asarray(planes)
    return planes[None] if planes.ndim == 2 else planes


def write_pnm(path, planes: np.ndarray, bits: int) -> None:
    """planes [1 or 3, h, w] unsigned samples of `bits` bits -> .pgm/.ppm."""
    planes = _planes(planes)
    c, h, w = planes.shape
    if c not in (1, 3) or not 1 <= bits <= 16:
        raise ValueError("PNM holds 1 or 3 components of 1 to 16 bits")
    dt = ">u1" if bits <= 8 else ">u2"
    body = np.ascontiguousarray(np.moveaxis(planes, 0, -1)).astype(dt)
    Path(path).write_bytes(f"{'P5' if c == 1 else 'P6'}\n{w} {h}\n{(1 << bits) - 1}\n".encode() + body.tobytes())


def read_pnm(path):
    """-> (planes [c, h, w], bits) of a binary PGM/PPM."""
    data = Path(path).read_bytes()
    fields, pos = [], 0
    while len(fields) < 4:
        while data[pos:pos + 1].isspace():
            pos += 1
        if data[pos:pos + 1] == b"#":
            pos = data.index(b"\n", pos) + 1
            continue
        end = pos
        while not data[end:end + 1].isspace():
            end += 1
        fields.append(data[pos:end])
        pos = end
    magic, w, h, mx = fields[0], int(fields[1]), int(fields[2]), int(fields[3])
    c = {b"P5": 1, b"P6": 3}[magic]
    dt = ">u1" if mx < 256 else ">u2"
    a = np.frombuffer(data, dt, count=w * h * c, offset=pos + 1).reshape(h, w, c)
    return np.moveaxis(a, -1, 0).astype(np.uint8 if mx < 256 else np.uint16), mx.bit_length()


def write_pgx(prefix, planes: np.ndarray, bits: int, signed: bool = False) -> list:
    """One <prefix>_<c>.pgx per component; returns the paths."""
    planes = _planes(planes)
    paths = []
    for c, plane in enumerate(planes):
        p = Path(f"{prefix}_{c}.pgx")
        h, w = plane.shape
        dt = (">i1" if signed else ">u1") if bits <= 8 else (">i2" if signed else ">u2")
        hdr = f"PG ML {'-' if signed else '+'} {bits} {w} {h}\n".encode()
        p.write_bytes(hdr + np.ascontiguousarray(plane).astype(dt).tobytes())
        paths.append(p)
    return paths


def read_pgx(path):
    """-> (plane [h, w], bits, signed) of one PGX file."""
    data = Path(path).read_bytes()
    nl = data.index(b"\n")
    tok = data[:nl].split()
    if tok[0] != b"PG" or tok[1] not in (b"ML", b"LM"):
        raise ValueError("not a PGX file")
    big = tok[1] == b"ML"
    if tok[2] in (b"+", b"-"):
        signed, rest = tok[2] == b"-", tok[3:]
    else:
        signed, rest = False, tok[2:]
    bits, w, h = int(rest[0]), int(rest[1]), int(rest[2])
    dt = np.dtype(("i" if signed else "u") + ("1" if bits <= 8 else "2")).newbyteorder(">" if big else "<")
    a = np.frombuffer(data, dt, count=w * h, offset=nl + 1).reshape(h, w)
    return a.astype(dt.newbyteorder("=")), bits, signed


def write_image(path, planes: np.ndarray, bits: int, signed: bool = False):
    """By extension: .pgm/.ppm/.pnm -> PNM, .pgx -> one PGX per component
    (path without the extension as the prefix)."""
    path = Path(path)
    if path.suffix.lower() in (".pgm", ".ppm", ".pnm"):
        if signed:
            raise ValueError("PNM holds unsigned samples")
        write_pnm(path, planes, bits)
        return [path]
    if path.suffix.lower() == ".pgx":
        return write_pgx(path.with_suffix(""), planes, bits, signed)
    raise ValueError(f"unknown image extension: {path.suffix}")
