"""The Rust FFI block a bevy_lux maintainer adds (the `extern "C"` block of the
integration guide at the repository root) against the C header and the
library: every function of include/lux.h is declared with
the header's parameter count and exported by liblux.so, and every #[repr(C)]
record has the field names, order and size of the binding's records (which
mirror the header).  No GPU needed."""
import ctypes as C
import os
import re

import pytest

import bevy_penumbra_b200 as bp
from bevy_penumbra_b200 import _native as N
from tests.test_abi import ROOT, declared_functions


def rust_block() -> str:
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```rust\n(.*?)```", text, flags=re.S)
    assert len(blocks) == 1
    return blocks[0]


def split_params(params: str) -> list[str]:
    params = params.strip()
    if not params or params == "void":
        return []
    return [p for p in (x.strip() for x in params.split(",")) if p]


def rust_functions() -> dict[str, int]:
    body = re.sub(r"//[^\n]*", "", rust_block())
    return {name: len(split_params(params))
            for name, params in re.findall(r"pub fn (lux_\w+)\((.*?)\)\s*(?:->|;)", body, flags=re.S)}


def header_functions() -> dict[str, int]:
    text = open(os.path.join(ROOT, "include", "lux.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for name in declared_functions():
        m = re.search(r"\b" + name + r"\s*\(([^;]*?)\)\s*;", text, flags=re.S)
        assert m, name
        out[name] = len(split_params(m.group(1)))
    return out


def test_every_header_function_is_declared_with_its_arity():
    rust, header = rust_functions(), header_functions()
    assert set(rust) == set(header), (sorted(set(header) - set(rust)), sorted(set(rust) - set(header)))
    wrong = {n: (rust[n], header[n]) for n in header if rust[n] != header[n]}
    assert not wrong, wrong


def test_every_declared_function_is_exported():
    lib = C.CDLL(N.LIB_PATH)
    missing = [n for n in rust_functions() if not hasattr(lib, n)]
    assert not missing, missing


SCALARS = {"f32": 4, "u32": 4, "i32": 4, "u16": 2, "u8": 1, "u64": 8, "f64": 8, "usize": 8}


def rust_structs() -> dict[str, list[tuple[str, str]]]:
    body = re.sub(r"///[^\n]*", "", rust_block())
    out = {}
    for name, fields in re.findall(r"#\[repr\(C\)\](?:\s*#\[derive\([^\]]*\)\])?\s*pub struct (\w+)\s*\{(.*?)\}",
                                   body, flags=re.S):
        parsed = re.findall(r"(?:pub\s+)?(\w+)\s*:\s*(\[[^\]]*\]|[^,]+)", fields)
        out[name] = [(f, t.strip()) for f, t in parsed]
    return out


def layout(ty: str, structs) -> tuple[int, int]:
    """(size, alignment) of a Rust field type under #[repr(C)]."""
    ty = ty.strip()
    if ty.startswith("*"):
        return 8, 8
    m = re.fullmatch(r"\[(.+);\s*(\w+)\]", ty)
    if m:
        size, align = layout(m.group(1), structs)
        count = 12 if m.group(2) == "LUX_MAX_LEVELS" else int(m.group(2))
        return size * count, align
    if ty in SCALARS:
        return SCALARS[ty], SCALARS[ty]
    return struct_layout(structs[ty], structs)


def struct_layout(fields, structs) -> tuple[int, int]:
    offset, align = 0, 1
    for _, ty in fields:
        size, a = layout(ty, structs)
        offset = (offset + a - 1) // a * a + size
        align = max(align, a)
    return (offset + align - 1) // align * align, align


def test_records_match_the_binding_layouts():
    structs = rust_structs()
    records = {name: fields for name, fields in structs.items() if fields != [("_p", "[u8; 0]")]}
    opaque = {name for name, fields in structs.items() if fields == [("_p", "[u8; 0]")]}
    assert {"LuxContext", "LuxScene", "LuxView", "LuxPackedScene", "LuxBatch", "LuxCache", "LuxScreen"} <= opaque
    checked = 0
    for name, fields in records.items():
        size, _ = struct_layout(fields, structs)
        names = [f for f, _ in fields]
        if name == "LuxCacheSample":
            assert names == list(bp.CACHE_SAMPLE_DTYPE.names)
            assert size == bp.CACHE_SAMPLE_DTYPE.itemsize == 64
        else:
            ct = getattr(N, name)
            assert names == [f[0] for f in ct._fields_], name
            assert size == C.sizeof(ct), (name, size, C.sizeof(ct))
        checked += 1
    assert checked >= 19
