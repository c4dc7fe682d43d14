"""CPU checks of the Rust drop-in crate under rust/ (no Rust toolchain exists
here, so the crate is checked as text): its `extern "C"` block declares every
entry point of include/cfgmm.h with the same argument count and the same
argument types and widths, every name it binds is exported by libcfgmm.so, its
#[repr(C)] structs match the header's, and the safe wrappers keep the
reference's public names (src/impl_matmul.rs:155-248,
src/impl_aodmao2rho.rs:171-261, src/impl_matmul_non0tab.rs:210-326)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "cfgmm.h")
FFI = os.path.join(ROOT, "rust", "src", "ffi.rs")
LIB_RS = os.path.join(ROOT, "rust", "src", "lib.rs")

# C spelling -> canonical Rust spelling (after pointer normalisation)
_C_SCALARS = {
    "double": "f64", "float": "f32", "size_t": "usize", "uint8_t": "u8", "int": "i32",
    "uint64_t": "u64", "void": "void", "char": "char",
    "cfgmm_aodm_plan": "cfgmm_aodm_plan", "cfgmm_aodm_batch": "cfgmm_aodm_batch",
    "cfgmm_server": "cfgmm_server", "cfgmm_request_stats": "cfgmm_request_stats",
}
_RUST_SCALARS = {"c_int": "i32", "c_void": "void", "c_char": "char", "i32": "i32", "u8": "u8",
                 "usize": "usize", "u64": "u64", "f64": "f64", "f32": "f32"}


def _canon_c(t: str) -> str:
    """'const double*' -> '*const f64'; 'void* const*' -> '*const *mut void';
    'cfgmm_aodm_plan**' -> '*mut *mut cfgmm_aodm_plan'."""
    t = " ".join(t.replace("*", " * ").split())
    toks = t.split()
    # base type with its own const, then a chain of '*' each optionally followed by const
    i = 0
    base_const = False
    if toks[i] == "const":
        base_const, i = True, i + 1
    base = toks[i]
    i += 1
    if i < len(toks) and toks[i] == "const":
        base_const, i = True, i + 1
    ptrs = []  # const-ness of each pointer level, innermost first
    while i < len(toks):
        assert toks[i] == "*", t
        i += 1
        c = False
        if i < len(toks) and toks[i] == "const":
            c, i = True, i + 1
        ptrs.append(c)
    out = _C_SCALARS[base]
    # the pointee of the first '*' is const when the base type is const;
    # the pointee of each further '*' is const when the previous '*' is const
    pointee_const = base_const
    for c in ptrs:
        out = ("*const " if pointee_const else "*mut ") + out
        pointee_const = c
    return out


def _canon_rust(t: str) -> str:
    t = " ".join(t.split())
    m = re.match(r"^\*(const|mut)\s+(.*)$", t)
    if m:
        return f"*{m.group(1)} " + _canon_rust(m.group(2))
    return _RUST_SCALARS.get(t, t)


def _header_functions():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    text = re.sub(r"^\s*#.*$", "", text, flags=re.M)
    out = {}
    for ret, name, args in re.findall(r"([A-Za-z_][\w\s\*]*?)\s*\b(cfgmm_\w+)\s*\(([^)]*)\)\s*;",
                                      text):
        ret = " ".join(ret.split())
        if ret.startswith("typedef"):
            continue
        params = []
        a = " ".join(args.split())
        if a and a != "void":
            for p in a.split(","):
                p = p.strip()
                m = re.match(r"^(.*?)\s*\b(\w+)$", p)
                params.append(_canon_c(m.group(1)))
        out[name] = (_canon_c(ret), params)
    return out


def _rust_functions():
    text = open(FFI).read()
    block = re.search(r'extern\s+"C"\s*\{(.*)\n\}', text, flags=re.S).group(1)
    block = re.sub(r"//[^\n]*", "", block)
    out = {}
    for name, args, ret in re.findall(
            r"pub\s+fn\s+(cfgmm_\w+)\s*\((.*?)\)\s*(?:->\s*([^;]+))?;", block, flags=re.S):
        params = []
        for p in [x.strip() for x in args.split(",") if x.strip()]:
            _, t = p.split(":", 1)
            params.append(_canon_rust(t))
        out[name] = (_canon_rust(ret.strip()) if ret else "void", params)
    return out


def test_canonical_forms():
    assert _canon_c("const double*") == "*const f64"
    assert _canon_c("double*") == "*mut f64"
    assert _canon_c("void* const*") == "*const *mut void"
    assert _canon_c("cfgmm_aodm_plan**") == "*mut *mut cfgmm_aodm_plan"
    assert _canon_c("const cfgmm_aodm_plan*") == "*const cfgmm_aodm_plan"
    assert _canon_rust("*const *mut c_void") == "*const *mut void"
    assert _canon_rust("c_int") == "i32"


def test_every_header_function_is_bound_with_the_same_signature():
    h = _header_functions()
    r = _rust_functions()
    assert len(h) >= 40
    missing = sorted(set(h) - set(r))
    extra = sorted(set(r) - set(h))
    assert not missing, f"not bound in rust/src/ffi.rs: {missing}"
    assert not extra, f"bound but not declared in cfgmm.h: {extra}"
    for name, (ret, params) in h.items():
        rret, rparams = r[name]
        assert rret == ret, f"{name}: return {rret} vs {ret}"
        assert len(rparams) == len(params), f"{name}: {len(rparams)} args vs {len(params)}"
        for i, (a, b) in enumerate(zip(rparams, params)):
            assert a == b, f"{name} argument {i}: {a} vs {b}"


def test_every_bound_name_is_exported(cm):
    lib = ctypes.CDLL(cm.library_path)
    missing = [n for n in _rust_functions() if not hasattr(lib, n)]
    assert not missing, missing


def _c_struct_fields(name):
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef\s+struct\s+" + name + r"\s*\{(.*?)\}\s*" + name + r"\s*;", text,
                     flags=re.S).group(1)
    fields = []
    for decl in [d.strip() for d in body.split(";") if d.strip()]:
        m = re.match(r"^(.*?)\s*\b(\w+(?:\s*,\s*\w+)*)$", " ".join(decl.split()))
        t, names = m.group(1), m.group(2)
        for n in names.split(","):
            fields.append((n.strip(), _canon_c(t)))
    return fields


def _rust_struct_fields(name):
    text = open(FFI).read()
    body = re.search(r"pub\s+struct\s+" + name + r"\s*\{(.*?)\n\}", text, flags=re.S).group(1)
    return [(n, _canon_rust(t.strip())) for n, t in re.findall(r"pub\s+(\w+)\s*:\s*([^,]+),",
                                                                body)]


@pytest.mark.parametrize("name", ["cfgmm_aodm_batch", "cfgmm_request_stats"])
def test_repr_c_structs_match(name):
    assert _rust_struct_fields(name) == _c_struct_fields(name)


def test_constants_match_header():
    h = open(HEADER).read()
    r = open(FFI).read()
    for name, val in re.findall(r"#define\s+(CFGMM_(?:OK|ERR_\w+|PREC_\w+|PLAN_\w+))\s+\(?(-?\d+)\)?",
                                h):
        m = re.search(r"pub const " + name + r":\s*c_int\s*=\s*(-?\d+);", r)
        assert m and int(m.group(1)) == int(val), name
    m = re.search(r"#define CFGMM_NOALLOC_SCRATCH_BYTES \((\d+)u << (\d+)\)", h)
    assert f"CFGMM_NOALLOC_SCRATCH_BYTES: usize = {m.group(1)} << {m.group(2)};" in r


def test_safe_wrappers_keep_the_reference_names():
    text = open(LIB_RS).read()
    for sig in [
        r"pub fn matmul_loop_parallel_mnk_pack_a\(\s*c: &mut \[f64\], a: &\[f64\], b: &\[f64\], "
        r"m: usize, n: usize, k: usize, lda: usize,\s*ldb: usize, ldc: usize, transa: bool, "
        r"transb: bool,",
        r"pub fn matmul_loop_parallel_mnk_pack_a_non0tab<const BLKSIZE: usize>\(",
        r"pub fn aodmao2rho_loop_parallel<const BLKSIZE: usize>\(\s*rhos: &mut \[f64\], "
        r"dms: &\[f64\], ao_lhs: &\[f64\], ao_rhs: &\[f64\], strides: \[usize; 2\],\s*"
        r"shape: \[usize; 2\], nset: usize, tab: &\[bool\], ldtab: usize,",
        r"pub fn matmul_loop_macro_mb<const MB: usize>\(",
        r"pub fn matmul_anyway_full\(",
        r"pub fn matmul_anyway_full_non0tab\(",
        r"pub fn aodmao2rho_anyway\(",
        r"pub mod impl_matmul\b", r"pub mod impl_aodmao2rho\b", r"pub mod impl_matmul_non0tab\b",
        r"pub struct MatmulLoops<\s*T,\s*const MC: usize,\s*const KC: usize,\s*const NC: usize,"
        r"\s*const MR: usize,\s*const NR_LANE: usize,\s*const LANE: usize,\s*>",
    ]:
        assert re.search(sig, text), sig
    cargo = open(os.path.join(ROOT, "rust", "Cargo.toml")).read()
    assert 'name = "cfgable_matmul"' in cargo and 'build = "build.rs"' in cargo
    build = open(os.path.join(ROOT, "rust", "build.rs")).read()
    assert "build.py" in build and "rustc-link-lib=dylib=cfgmm" in build
