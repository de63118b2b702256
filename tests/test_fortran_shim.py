"""The Fortran ISO_C_BINDING interfaces against the C header, on the CPU.

The image has no Fortran compiler, so rsdft_gpu_mod.f90 cannot be built
here; this test reads it.  Every `bind(C, name=...)` interface must name an
entry of include/rsdft_gpu.h and pass the same arguments in the same order:
`type(c_ptr), value` for a C pointer, `integer(c_int), value` for int,
`integer(c_long), value` for long, `real(c_double), value` for double
(every dummy by value: a by-reference dummy would hand C the address of the
Fortran variable instead).  The return kinds must match as well.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rsdft_gpu.h")
SHIM = os.path.join(ROOT, "rsdft_b200", "fortran", "rsdft_gpu_mod.f90")


def c_kind(decl: str) -> str:
    decl = decl.strip()
    if "*" in decl:
        return "ptr"
    words = decl.replace("const ", "").split()
    base = " ".join(words[:-1]) if len(words) > 1 else words[0]
    return {"int": "int", "long": "long", "long long": "longlong", "double": "double"}[base]


def header_entries():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"(?m)^\s*([A-Za-z_][\w\s\*]*?)\b(rsdft_gpu_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, args = m.group(1), m.group(2), m.group(3).strip()
        params = [] if args in ("", "void") else [c_kind(a) for a in args.split(",")]
        out[name] = (c_kind(ret + " x"), params)
    return out


F_KINDS = {"type(c_ptr)": "ptr", "integer(c_int)": "int", "integer(c_long)": "long", "real(c_double)": "double"}


def shim_interfaces():
    text = open(SHIM).read()
    text = re.sub(r"&\s*\n\s*", " ", text)  # join continuation lines
    block = text[text.index("interface"):text.index("end interface")]
    out = {}
    for m in re.finditer(r"(?s)(type\(c_ptr\)|integer\(c_int\))\s+function\s+(\w+)\s*\(([^)]*)\)\s*"
                         r"bind\(C,\s*name=\"(\w+)\"\)(.*?)end function", block):
        ret, fname, dummies, cname, body = m.groups()
        order = [d.strip().lower() for d in dummies.split(",") if d.strip()]
        kind_of, by_value = {}, {}
        for line in body.splitlines():
            dm = re.match(r"\s*(type\(c_ptr\)|integer\(c_int\)|integer\(c_long\)|real\(c_double\))\s*(,\s*value)?\s*::"
                          r"\s*(.+)", line, flags=re.I)
            if not dm:
                continue
            for v in dm.group(3).split(","):
                v = v.strip().lower()
                kind_of[v] = F_KINDS[dm.group(1).lower()]
                by_value[v] = bool(dm.group(2))
        out[cname] = (fname, F_KINDS[ret.lower()], order, kind_of, by_value)
    return out


def test_shim_parses_every_interface():
    shim = shim_interfaces()
    text = open(SHIM).read()
    assert len(shim) == text.count("bind(C, name=") > 10


def test_shim_interfaces_match_header():
    hdr = header_entries()
    for cname, (fname, ret, order, kind_of, by_value) in shim_interfaces().items():
        assert fname == cname, (fname, cname)
        assert cname in hdr, f"{cname} is not declared in the header"
        cret, cparams = hdr[cname]
        # const char* last_error comes back as type(c_ptr)
        assert ret == cret or (ret == "ptr" and cret == "ptr"), (cname, ret, cret)
        assert len(order) == len(cparams), (cname, order, cparams)
        for i, (dummy, ck) in enumerate(zip(order, cparams)):
            assert dummy in kind_of, f"{cname}: dummy {dummy} has no declaration"
            assert kind_of[dummy] == ck, f"{cname} argument {i + 1} ({dummy}): Fortran {kind_of[dummy]}, C {ck}"
            assert by_value[dummy], f"{cname}: dummy {dummy} is not passed by value"


def test_header_parser_sees_the_entries():
    hdr = header_entries()
    assert hdr["rsdft_gpu_set_vloc"] == ("int", ["ptr", "long", "int"])
    assert hdr["rsdft_gpu_last_error"][0] == "ptr" and hdr["rsdft_gpu_last_error"][1] == []
    assert hdr["rsdft_gpu_set_grid"][1] == ["ptr", "int", "double", "ptr", "ptr", "ptr", "double"]
