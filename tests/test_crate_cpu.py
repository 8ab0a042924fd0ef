"""The Rust crate's declarations (crates/continuum-cuda/src/ffi.rs, shipped as
source: no Rust toolchain here) follow include/continuum_cuda.h one for one:
the same functions with the same number of parameters, and the same structs
with the same number of fields."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / "include" / "continuum_cuda.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"CC_API\s+[\w\s\*]+?\b(cc_\w+)\s*\(([^)]*)\)\s*;", text, flags=re.S):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def rust_functions():
    text = (ROOT / "crates" / "continuum-cuda" / "src" / "ffi.rs").read_text()
    block = text[text.index('unsafe extern "C"'):]
    out = {}
    for m in re.finditer(r"pub fn (cc_\w+)\(([^)]*)\)", block, flags=re.S):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if not args else args.rstrip(",").count(",") + 1
    return out


def fields(text, pattern):
    return {m.group(1): len([l for l in m.group(2).split(";" if pattern == "c" else ",") if l.strip()])
            for m in re.finditer(r"typedef struct (cc_\w+) \{(.*?)\} \1;" if pattern == "c"
                                 else r"pub struct (cc_\w+) \{(.*?)\n\}", text, flags=re.S)}


def test_every_header_function_is_declared_with_its_parameters():
    h, r = header_functions(), rust_functions()
    assert len(h) >= 50
    assert set(h) == set(r), (set(h) ^ set(r))
    for name, n in h.items():
        assert r[name] == n, name


def test_structs_have_the_headers_fields():
    ht = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "continuum_cuda.h").read_text(), flags=re.S)
    rt = (ROOT / "crates" / "continuum-cuda" / "src" / "ffi.rs").read_text()
    hc, rc = fields(ht, "c"), fields(rt, "rust")
    for name, n in hc.items():
        assert rc.get(name) == n, (name, n, rc.get(name))
