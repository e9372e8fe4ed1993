"""The C ABI's structs as the bindings see them: every field of each `typedef struct` in
include/galaxy_b200.h at the same offset, with the same size, in the ctypes mirror
(galaxy_b200/_lib.py) and in the Rust FFI crate's #[repr(C)] mirrors
(galaxy_b200/rust/galaxy-b200/src/lib.rs). The C side is measured by a small program
built here with the system compiler (offsetof / sizeof); the Rust side is laid out from
its declarations with the C rules #[repr(C)] follows (the crate itself cannot be
compiled here)."""

import ctypes as C
import json
import os
import re
import shutil
import subprocess

import pytest

from galaxy_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "galaxy_b200.h")
RUST = os.path.join(ROOT, "galaxy_b200", "rust", "galaxy-b200", "src", "lib.rs")


def _c_structs():
    """{struct name: [field names]} of the header's struct definitions."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for name, body in re.findall(r"typedef struct (\w+) \{(.*?)\} \1;", text, flags=re.S):
        out[name] = re.findall(r"\b(\w+)\s*(?:\[[^\]]*\])?\s*;", body)
    return out


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    """{struct: {"size": n, "fields": {field: (offset, size)}}} measured by the compiler."""
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = _c_structs()
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {",
             'printf("{");']
    first = True
    for s, fields in structs.items():
        sep = "" if first else ","
        first = False
        lines.append(f'printf("{sep}\\"{s}\\": {{\\"size\\": %zu, \\"fields\\": {{", sizeof({s}));')
        for i, f in enumerate(fields):
            comma = "," if i else ""
            lines.append(f'printf("{comma}\\"{f}\\": [%zu, %zu]", offsetof({s}, {f}), sizeof((({s}*)0)->{f}));')
        lines.append('printf("}}");')
    lines += ['printf("}\\n");', "return 0; }"]
    d = tmp_path_factory.mktemp("layout")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines))
    subprocess.run([cc, "-std=c11", "-o", str(exe), str(src)], check=True)
    return json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)


CTYPES = {"gx_options": _lib.Options, "gx_stats": _lib.Stats, "gx_sph_params": _lib.SphParams,
          "gx_tuning": _lib.Tuning, "gx_batch_stats": _lib.BatchStats, "gx_snap_opts": _lib.SnapOpts,
          "gx_server_stats": _lib.ServerStats}


def test_every_header_struct_has_a_ctypes_mirror(c_layout):
    assert set(c_layout) == set(CTYPES)


@pytest.mark.parametrize("name", sorted(CTYPES))
def test_ctypes_mirror_matches_the_header(c_layout, name):
    cls, c = CTYPES[name], c_layout[name]
    assert [f[0] for f in cls._fields_] == list(c["fields"]), name
    for f, _ in cls._fields_:
        assert (getattr(cls, f).offset, getattr(cls, f).size) == tuple(c["fields"][f]), (name, f)
    assert C.sizeof(cls) == c["size"], name


RUST_SIZES = {"u8": 1, "i8": 1, "u16": 2, "i16": 2, "u32": 4, "i32": 4, "c_int": 4, "f32": 4, "u64": 8, "i64": 8,
              "f64": 8, "usize": 8, "isize": 8}


def _rust_structs():
    """{Rust struct: [(field, type)]} of the crate's #[repr(C)] structs with fields."""
    text = open(RUST).read()
    out = {}
    for name, body in re.findall(r"#\[repr\(C\)\]\s*(?:#\[derive\([^)]*\)\]\s*)?pub struct (\w+) \{(.*?)\n\}", text,
                                 flags=re.S):
        fields = re.findall(r"pub (\w+):\s*([\w:]+)", body)
        if fields:
            out[name] = fields
    return out


def _c_rules(fields):
    """Offsets and total size of a #[repr(C)] struct of scalar fields."""
    off, align, lay = 0, 1, {}
    for f, t in fields:
        size = RUST_SIZES[t.split("::")[-1]]
        off = (off + size - 1) // size * size
        lay[f] = (off, size)
        off += size
        align = max(align, size)
    return lay, (off + align - 1) // align * align


def test_rust_mirrors_match_the_header(c_layout):
    rust = _rust_structs()
    names = {"GxOptions": "gx_options", "GxSphParams": "gx_sph_params"}
    assert set(rust) == set(names), sorted(rust)
    for r, c_name in names.items():
        lay, size = _c_rules(rust[r])
        c = c_layout[c_name]
        assert [f for f, _ in rust[r]] == list(c["fields"]), r
        assert lay == {f: tuple(v) for f, v in c["fields"].items()}, r
        assert size == c["size"], r
