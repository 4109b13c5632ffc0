"""The Julia binding (julia/SSGB200/src/SSGB200.jl) cannot run here -- no
Julia runtime -- so its struct mirrors are checked against the C header's
structs as text: same fields, same order, same widths.  The ctypes mirrors
are checked against the compiled header layout in test_abi.py; this compares
the Julia ones with those, and checks that every entry point the binding
calls is one the header declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "julia", "SSGB200", "src", "SSGB200.jl")

JL_TYPES = {"Int32": ctypes.c_int32, "Int64": ctypes.c_int64, "Float64": ctypes.c_double}


def julia_struct(text, name):
    m = re.search(r"(?:mutable\s+)?struct\s+" + name + r"\s*\n(.*?)\nend", text, flags=re.S)
    assert m, name
    fields = []
    for line in m.group(1).splitlines():
        line = line.split("#")[0].strip()
        if not line:
            continue
        f, t = [x.strip() for x in line.split("::")]
        tup = re.fullmatch(r"NTuple\{(\d+),(\w+)\}", t)
        fields.append((f, (int(tup.group(1)), JL_TYPES[tup.group(2)]) if tup else (1, JL_TYPES[t])))
    return fields


def ctypes_fields(cls):
    out = []
    for f, t in cls._fields_:
        if issubclass(t, ctypes.Array):
            out.append((f, (t._length_, t._type_)))
        else:
            out.append((f, (1, t)))
    return out


def test_julia_structs_match_the_c_abi(ssg):
    text = open(JL).read()
    L = ssg._lib
    for jl, cls in (("SsgConfig", L.SsgConfig), ("MaStats", L.SsgMaStats), ("StepStats", L.SsgStepStats),
                    ("Diagnostics", L.SsgDiagnostics), ("AdjointStats", L.SsgAdjointStats)):
        assert julia_struct(text, jl) == ctypes_fields(cls), jl


def test_julia_binding_calls_declared_entry_points(ssg):
    text = open(JL).read()
    called = set(re.findall(r"ccall\(\(:(ssg_[a-z_]+), lib\)", text))
    assert called and called <= set(ssg._lib.EXPORTED_SYMBOLS), called - set(ssg._lib.EXPORTED_SYMBOLS)
