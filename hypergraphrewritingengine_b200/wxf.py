"""Decoder of the Wolfram Exchange Format (WXF) replies the GPU backend writes
(include/hgx/gpu_backend.hpp, include/hgx/wxf.hpp).

Covers the expressions a reply holds -- integers (8/16/32/64-bit), reals, strings, symbols,
List[...] and other functions, associations -- and returns Python values: int, float, str,
``Symbol`` for symbols, list for List[...], ``(head, args)`` for other functions, dict for
associations (rule order kept).
"""
from __future__ import annotations

import struct


class Symbol(str):
    """A WXF symbol (as opposed to a string)."""


class WXFError(ValueError):
    pass


def loads(data: bytes):
    """Decode one WXF expression (with its "8:" header)."""
    data = bytes(data)
    if data[:2] != b"8:":
        raise WXFError("not a WXF stream (missing the 8: header)")
    value, pos = _read(data, 2, 0)
    if pos != len(data):
        raise WXFError(f"{len(data) - pos} trailing bytes after the expression")
    return value


def _varint(data: bytes, pos: int):
    value, shift = 0, 0
    while True:
        if pos >= len(data):
            raise WXFError("truncated varint")
        b = data[pos]
        pos += 1
        value |= (b & 0x7F) << shift
        shift += 7
        if not b & 0x80:
            return value, pos


_INTS = {ord("C"): ("<b", 1), ord("j"): ("<h", 2), ord("i"): ("<i", 4), ord("L"): ("<q", 8)}


def _read(data: bytes, pos: int, depth: int):
    if depth > 512:
        raise WXFError("expression nested too deeply")
    if pos >= len(data):
        raise WXFError("truncated expression")
    tok = data[pos]
    pos += 1
    if tok in _INTS:
        fmt, n = _INTS[tok]
        return struct.unpack_from(fmt, data, pos)[0], pos + n
    if tok == ord("r"):
        return struct.unpack_from("<d", data, pos)[0], pos + 8
    if tok in (ord("S"), ord("s")):
        n, pos = _varint(data, pos)
        text = data[pos:pos + n].decode("utf-8")
        return (text if tok == ord("S") else Symbol(text)), pos + n
    if tok == ord("f"):
        n, pos = _varint(data, pos)
        head, pos = _read(data, pos, depth + 1)
        args = []
        for _ in range(n):
            a, pos = _read(data, pos, depth + 1)
            args.append(a)
        if isinstance(head, Symbol) and head == "List":
            return args, pos
        return (head, args), pos
    if tok == ord("A"):
        n, pos = _varint(data, pos)
        out = {}
        for _ in range(n):
            if data[pos] not in (ord("-"), ord(":")):
                raise WXFError(f"expected a rule in an association at byte {pos}")
            k, pos = _read(data, pos + 1, depth + 1)
            v, pos = _read(data, pos, depth + 1)
            out[k] = v
        return out, pos
    raise WXFError(f"unsupported token 0x{tok:02x} at byte {pos - 1}")
