"""INTEGRATION.md's Rust FFI block against include/propaq_cuda.h: every entry
point the header declares is in the block with the same parameters (names,
order and types), and every #[repr(C)] struct has the header struct's fields
in the header's order with the same types.  A Rust caller built from the
document therefore passes each argument in its slot."""

from __future__ import annotations

import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

C_SCALARS = {"uint32_t": "u32", "uint64_t": "u64", "int64_t": "i64", "int32_t": "i32", "size_t": "usize",
             "int": "c_int", "double": "f64", "char": "c_char", "void": "c_void"}
C_NAMED = {"pq_engine": "PqEngine", "pq_plugin": "PqPlugin", "pq_run_config": "PqRunConfig",
           "pq_result": "PqResult", "pq_instance": "PqInstance", "pq_batch_tuning": "PqBatchTuning",
           "pq_engine_limits": "PqEngineLimits", "pq_gate_record": "PqGateRecord",
           "pq_noise_factor_fn": "PqNoiseFactorFn"}


def c_to_rust(ctype: str) -> str:
    """The Rust spelling of a C parameter type."""
    t = ctype.replace("const ", "const_").strip()
    stars = t.count("*")
    base = t.replace("*", "").strip()
    is_const = base.startswith("const_")
    base = base.replace("const_", "").strip()
    rust = C_SCALARS.get(base) or C_NAMED[base]
    if stars == 0:
        return rust
    # the first pointer level carries the const of the pointee
    out = ("*const " if is_const else "*mut ") + rust
    for _ in range(stars - 1):
        out = "*mut " + out
    return out


def header_functions():
    text = (ROOT / "include" / "propaq_cuda.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"typedef[^;]*;", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\n([A-Za-z_][\w \*]*?)\s*\b(pq_\w+)\(([^)]*)\);", text):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3)
        params = []
        for a in filter(None, (x.strip() for x in args.split(","))):
            pm = re.match(r"(.*?)(\w+)$", a)
            params.append((pm.group(2), c_to_rust(pm.group(1))))
        ret_rust = None if ret == "void" else c_to_rust(ret)
        out[name] = (params, ret_rust)
    return out


def header_structs():
    text = (ROOT / "include" / "propaq_cuda.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", text, flags=re.S):
        fields = []
        for decl in filter(None, (d.strip() for d in m.group(2).split(";"))):
            dm = re.match(r"(const\s+)?(\w+)\s*(\**)\s*(.*)", decl, flags=re.S)
            ctype = (dm.group(1) or "") + dm.group(2) + dm.group(3)
            for n in dm.group(4).split(","):
                n = n.strip()
                stars = n.count("*")
                fields.append((n.replace("*", "").strip(), c_to_rust(ctype + "*" * stars)))
        out[C_NAMED[m.group(1)]] = fields
    return out


def rust_block():
    text = (ROOT / "INTEGRATION.md").read_text()
    m = re.search(r"```rust\n(.*?)```", text, flags=re.S)
    assert m, "INTEGRATION.md has no rust block"
    return m.group(1)


def rust_functions():
    block = rust_block()
    ext = block[block.index('extern "C" {'):]
    out = {}
    for m in re.finditer(r"fn (pq_\w+)\((.*?)\)\s*(->\s*([^;]+))?;", ext, flags=re.S):
        params = []
        for a in filter(None, (x.strip() for x in m.group(2).split(","))):
            n, t = a.split(":", 1)
            params.append((n.strip().rstrip("_"), " ".join(t.split())))
        out[m.group(1)] = (params, m.group(4).strip() if m.group(4) else None)
    return out


def rust_structs():
    block = rust_block()
    out = {}
    for m in re.finditer(r"pub struct (\w+)\s*\{(.*?)\}", block, flags=re.S):
        body = re.sub(r"//[^\n]*", "", m.group(2))
        fields = []
        for f in filter(None, (x.strip() for x in body.split(","))):
            n, t = f.split(":", 1)
            fields.append((n.replace("pub", "").strip(), " ".join(t.split())))
        out[m.group(1)] = fields
    return out


def test_every_entry_point_is_declared_alike():
    hdr, rs = header_functions(), rust_functions()
    assert len(hdr) >= 20
    assert set(hdr) == set(rs), f"only in header: {set(hdr) - set(rs)}; only in the doc: {set(rs) - set(hdr)}"
    for name, (params, ret) in hdr.items():
        rparams, rret = rs[name]
        assert [n for n, _ in params] == [n for n, _ in rparams], f"{name}: parameter names/order differ"
        assert [t for _, t in params] == [t for _, t in rparams], f"{name}: parameter types differ"
        assert ret == rret, f"{name}: return type {ret} vs {rret}"


def test_every_struct_has_the_header_layout():
    hdr, rs = header_structs(), rust_structs()
    for name, fields in hdr.items():
        assert name in rs, f"{name} missing from INTEGRATION.md"
        assert fields == rs[name], f"{name}: fields differ\nheader {fields}\ndoc    {rs[name]}"


def test_doc_has_no_stale_claims():
    text = (ROOT / "INTEGRATION.md").read_text()
    assert "not run by the CUDA engine" not in text
    assert "runs four of them" not in text
