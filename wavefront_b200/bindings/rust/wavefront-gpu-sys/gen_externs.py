"""Regenerates the `extern "C"` block of src/lib.rs from include/wavefront_gpu.h.

Every function the header declares becomes one Rust declaration, in the
header's order, with the header's types mapped to Rust's (int -> c_int,
int32_t -> i32, const T * -> *const T, T (*p)[N] -> *const [T; N], ...).
Run from anywhere: python gen_externs.py
"""
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(HERE, "..", "..", "..", "..", "include", "wavefront_gpu.h")
LIB_RS = os.path.join(HERE, "src", "lib.rs")

TYPES = {"int": "c_int", "int32_t": "i32", "int64_t": "i64", "uint8_t": "u8", "uint64_t": "u64",
         "float": "f32", "double": "f64", "void": "c_void", "char": "c_char",
         "wf_status": "wf_status", "wf_handle": "wf_handle", "wf_batch": "wf_batch",
         "wf_tiling": "wf_tiling", "wf_grid_desc": "wf_grid_desc",
         "wf_snapshot_writer": "wf_snapshot_writer", "unsigned": "u32"}
RESERVED = {"type", "ref", "in", "loop", "move", "fn", "mod", "use", "box"}


def rust_type(t: str) -> str:
    t = " ".join(t.split())
    const = t.startswith("const ")
    base = t[6:] if const else t
    nptr = base.count("*")
    r = TYPES[base.replace("*", "").strip()]
    for i in range(nptr):
        r = ("*const " if (const and i == nptr - 1) else "*mut ") + r
    return r


def param(p: str) -> str:
    p = " ".join(p.split())
    m = re.match(r"(.*?)\(\s*\*\s*(\w+)\s*\)\s*\[(\d+)\]$", p)  # T (*name)[N]
    if m:
        const = m.group(1).strip().startswith("const")
        base = m.group(1).replace("const", "").strip()
        return f"{m.group(2)}: *{'const' if const else 'mut'} [{rust_type(base)}; {m.group(3)}]"
    m = re.match(r"(.*?)\b(\w+)\s*\[(\d*)\]$", p)  # T name[N]
    if m:
        const = m.group(1).strip().startswith("const")
        base = m.group(1).replace("const", "").strip()
        return f"{m.group(2)}: *{'const' if const else 'mut'} {rust_type(base)}"
    m = re.match(r"(.*?[\s\*])(\w+)$", p)
    name = m.group(2) + ("_" if m.group(2) in RESERVED else "")
    return f"{name}: {rust_type(m.group(1))}"


def externs() -> str:
    body = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = []
    for ret, name, params in re.findall(
            r"^\s*([A-Za-z_][\w \*]*?)\s*\b(wf_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", body, flags=re.M):
        params = params.strip()
        ps = [] if params in ("", "void") else [param(p) for p in params.split(",")]
        r = rust_type(ret)
        out.append(f"    pub fn {name}({', '.join(ps)}){'' if r == 'c_void' else ' -> ' + r};")
    return "\n".join(out) + "\n"


if __name__ == "__main__":
    src = open(LIB_RS).read()
    i = src.index('extern "C" {\n') + len('extern "C" {\n')
    open(LIB_RS, "w").write(src[:i] + externs() + "}\n")
    print("wrote", LIB_RS)
