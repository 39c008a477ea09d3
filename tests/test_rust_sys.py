"""The Rust FFI crate (crates/sr-cuda-sys) against the C header it binds (include/sr_cuda.h): every struct the header
defines has the same fields in the same order with the same widths, every function the header declares is declared in
the crate's `extern "C"` block with the same argument and return types, and the ABI version and enum constants agree.
No Rust toolchain is needed: both files are parsed as text."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sr_cuda.h")
CRATE = os.path.join(ROOT, "crates", "sr-cuda-sys")

C_SCALARS = {"uint32_t": "u32", "int32_t": "i32", "uint64_t": "u64", "int64_t": "i64", "double": "f64",
             "float": "f32", "char": "c_char", "void": "c_void", "sr_status": "sr_status"}


def strip_c_comments(s):
    s = re.sub(r"/\*.*?\*/", "", s, flags=re.S)
    return re.sub(r"//[^\n]*", "", s)


def rust_type_of_c(t: str) -> str:
    t = " ".join(t.split())
    stars = t.count("*")
    base = t.replace("*", " ").split()
    const = base[0] == "const"
    base = [w for w in base if w != "const"]
    name = C_SCALARS.get(base[0], base[0])
    if stars == 0:
        return "()" if name == "c_void" else name
    out = name
    for k in range(stars):
        # the innermost pointer keeps the C const; outer ones are mutable
        out = ("*const " if (k == 0 and const) else "*mut ") + out
    return out


def c_structs(src):
    out = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} (\w+);", src, flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            ty, names = decl.split(" ", 1)
            for name in names.split(","):
                name = name.strip()
                arr = re.match(r"(\w+)\[(\d+)\]", name)
                if arr:
                    fields.append((arr.group(1), f"[{C_SCALARS[ty]}; {arr.group(2)}]"))
                else:
                    fields.append((name, C_SCALARS[ty]))
        out[m.group(1)] = fields
    return out


def c_functions(src):
    out = {}
    for m in re.finditer(r"^([\w ]+?\**)\s*(sr_\w+)\(([^)]*)\);", src, flags=re.M | re.S):
        ret, name, args = m.group(1).strip(), m.group(2), " ".join(m.group(3).split())
        params = []
        if args != "void":
            for a in args.split(","):
                a = a.strip()
                pm = re.match(r"(.*?)(\w+)$", a)
                params.append((pm.group(2), rust_type_of_c(pm.group(1))))
        out[name] = (params, rust_type_of_c(ret))
    return out


def rust_structs(src):
    out = {}
    for m in re.finditer(r"pub struct (\w+) \{(.*?)\n\}", src, flags=re.S):
        fields = re.findall(r"pub (\w+): ([^,\n]+),", m.group(2))
        if fields:
            out[m.group(1)] = [(n, t.strip()) for n, t in fields]
    return out


def rust_functions(src):
    block = re.search(r'extern "C" \{(.*?)\n\}', src, flags=re.S).group(1)
    out = {}
    for m in re.finditer(r"pub fn (\w+)\((.*?)\)(?: -> ([^;]+))?;", block, flags=re.S):
        args = " ".join(m.group(2).split())
        params = []
        if args:
            for a in re.split(r",\s*(?=\w+:)", args):
                a = a.strip().rstrip(",")
                n, t = a.split(":", 1)
                params.append((n.strip(), t.strip()))
        out[m.group(1)] = (params, (m.group(3) or "()").strip())
    return out


def load():
    with open(HEADER) as f:
        h = strip_c_comments(f.read())
    with open(os.path.join(CRATE, "src", "lib.rs")) as f:
        r = f.read()
    return h, r


def test_the_crate_has_its_manifest_and_build_script():
    for name in ("Cargo.toml", "build.rs", os.path.join("src", "lib.rs")):
        assert os.path.exists(os.path.join(CRATE, name)), name
    with open(os.path.join(CRATE, "build.rs")) as f:
        b = f.read()
    assert "arch=compute_100a,code=sm_100a" in b
    # the build script compiles every source the Python build compiles
    from sandbox_reactions_b200 import build as lib_build
    for src in lib_build.SOURCES:
        assert f'"{src}"' in b, src


def test_every_struct_matches_the_header_field_for_field():
    h, r = load()
    cs, rs = c_structs(h), rust_structs(r)
    assert set(cs) <= set(rs), set(cs) - set(rs)
    for name, fields in cs.items():
        assert rs[name] == fields, name


def test_every_function_matches_the_header_signature():
    h, r = load()
    cf, rf = c_functions(h), rust_functions(r)
    assert cf, "no declarations parsed from the header"
    assert set(cf) == set(rf), (set(cf) ^ set(rf))
    for name, (params, ret) in cf.items():
        rparams, rret = rf[name]
        assert [t for _, t in rparams] == [t for _, t in params], name
        assert [n for n, _ in rparams] == [n for n, _ in params], name
        assert rret == ret, name


def test_constants_and_the_abi_version_agree():
    h, r = load()
    version = re.search(r"#define SR_ABI_VERSION (\d+)u", h).group(1)
    assert re.search(rf"pub const SR_ABI_VERSION: u32 = {version};", r)
    for enum in re.finditer(r"enum \{([^}]*)\}", h):
        for name, value in re.findall(r"(SR_\w+) = (\d+)", enum.group(1)):
            assert re.search(rf"pub const {name}: \w+ = {value};", r), name
    body = re.search(r"typedef enum sr_status \{(.*?)\} sr_status;", h, flags=re.S).group(1)
    for name, value in re.findall(r"(SR_\w+) = (\d+)", body):
        assert re.search(rf"pub const {name}: sr_status = {value};", r), name
