"""The Julia binding (tesserae.jl_b200/julia/TesseraeB200Ext.jl) against the C
ABI, without Julia: every library symbol it calls is declared in
include/tesserae_b200.h with the same argument list, and every POD descriptor
it declares has the header struct's field names, offsets and size (C layout
rules applied to the Julia field types, offsets from a compiled C probe)."""
import ctypes as C
import pathlib
import re
import subprocess
import tempfile

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
JL = ROOT / "tesserae.jl_b200" / "julia" / "TesseraeB200Ext.jl"
HEADER = ROOT / "include" / "tesserae_b200.h"

STRUCTS = {"TbMesh": "tb_mesh", "TbParticles": "tb_particles", "TbGrid": "tb_grid", "TbPartition": "tb_partition",
           "TbWeights": "tb_weights", "TbParams": "tb_step_params", "TbAdjoint": "tb_adjoint",
           "TbKernelTime": "tb_kernel_time"}
# the C field names the Julia side spells differently (none: kept alike on purpose)
SCALAR = {"Int32": (4, 4), "Int64": (8, 8), "Float64": (8, 8), "UInt8": (1, 1), "Cvoid": (0, 1)}


def jl_source():
    # drop comments and docstrings
    text = JL.read_text()
    text = re.sub(r'"""(.*?)"""', "", text, flags=re.S)
    return "\n".join(l.split("#", 1)[0] for l in text.splitlines())


def jl_type_layout(t: str):
    t = t.strip()
    if t.startswith("Ptr{") or t == "Cstring":
        return 8, 8
    m = re.fullmatch(r"NTuple\{(\d+),\s*(.+)\}", t)
    if m:
        n = int(m.group(1))
        size, align = jl_type_layout(m.group(2))
        return n * size, align
    return SCALAR[t]


def jl_structs():
    out = {}
    for name, body in re.findall(r"^struct (Tb\w+)\n(.*?)^end", jl_source(), flags=re.S | re.M):
        fields = []
        for line in body.splitlines():
            line = line.strip()
            if not line:
                continue
            fname, ftype = line.split("::", 1)
            fields.append((fname.strip(), ftype.strip()))
        out[name] = fields
    return out


def jl_layout(fields):
    off, maxal, offs = 0, 1, []
    for fname, ftype in fields:
        size, align = jl_type_layout(ftype)
        off = (off + align - 1) // align * align
        offs.append((fname, off))
        off += size
        maxal = max(maxal, align)
    return offs, (off + maxal - 1) // maxal * maxal


def c_layout(cname, fields):
    lines = [f'printf("{f} %zu\\n", offsetof({cname}, {f}));' for f, _ in fields]
    lines.append(f'printf("__size__ %zu\\n", sizeof({cname}));')
    src = (f'#include "{HEADER}"\n#include <stdio.h>\n#include <stddef.h>\nint main(){{' + "".join(lines) + "}\n")
    with tempfile.TemporaryDirectory() as d:
        c = pathlib.Path(d) / "p.c"
        c.write_text(src)
        exe = pathlib.Path(d) / "p"
        subprocess.run(["gcc", str(c), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    vals = dict(zip(out[0::2], (int(v) for v in out[1::2])))
    size = vals.pop("__size__")
    return [(f, vals[f]) for f, _ in fields], size


@pytest.mark.parametrize("jname", sorted(STRUCTS))
def test_descriptor_layouts_match_header(jname):
    structs = jl_structs()
    assert jname in structs, f"{jname} missing from the binding"
    fields = structs[jname]
    joffs, jsize = jl_layout(fields)
    coffs, csize = c_layout(STRUCTS[jname], fields)
    assert joffs == coffs
    assert jsize == csize


def header_symbols():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return set(re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(tb_\w+)\s*\(", text, flags=re.M))


def _balanced(src, i):
    """Index just past the parenthesis that closes the one opened before `i`."""
    depth = 1
    while depth:
        depth += {"(": 1, ")": -1}.get(src[i], 0)
        i += 1
    return i


def ccalls():
    """(symbol names, return type, argument types) of every ccall in the binding."""
    src = jl_source()
    out = []
    for m in re.finditer(r"ccall\(\(", src):
        end = _balanced(src, m.end())
        head = src[m.end():end - 1]
        head = head[:head.rindex(",")]  # drop ", libtb"
        rest = re.match(r"\s*,\s*([\w{}]+)\s*,\s*\(", src[end:])
        assert rest, src[m.start():m.start() + 80]
        a0 = end + rest.end()
        a1 = _balanced(src, a0)
        args = [a.strip() for a in re.split(r",(?![^{]*\})", src[a0:a1 - 1]) if a.strip()]
        names = re.findall(r":(tb_\w+)", head)
        sm = re.match(r"sym\(:(tb_\w+),\s*(.*)\)$", head.strip(), flags=re.S)
        if sm:
            forms = ["f64", "f32", "f32x64"] if sm.group(2).strip() == "form(particles)" else ["f64", "f32"]
            names = [f"{sm.group(1)}_{f}" for f in forms]
        assert names, head
        out.append((names, rest.group(1), args))
    return out


def test_every_called_symbol_is_declared():
    decl = header_symbols()
    called = {n for names, _, _ in ccalls() for n in names}
    assert called, "no ccall found"
    assert called <= decl, sorted(called - decl)


def test_ccall_argument_lists_match_the_abi(tb):
    abi = tb._abi
    sig = {n: (r, a) for n, r, a in abi.SIGNATURES}
    P = C.POINTER
    structs = {j: getattr(abi, c) for j, c in STRUCTS.items()}
    jl2c = {"Ptr{Cvoid}": C.c_void_p, "Int32": C.c_int32, "Int64": C.c_int64, "Float64": C.c_double,
            "Cstring": C.c_char_p, "Cvoid": None}

    def ctype(t):
        m = re.fullmatch(r"Ref\{(\w+)\}", t)
        if m:
            inner = m.group(1)
            return P(structs[inner]) if inner in structs else P(jl2c[inner])
        return jl2c[t]

    for names, ret, args in ccalls():
        for n in names:
            r, a = sig[n]
            assert ctype(ret) == r, (n, ret)
            assert [ctype(t) for t in args] == list(a), (n, args)


def test_binding_covers_the_dispatch_seam():
    src = jl_source()
    for method in ("KernelAbstractions.get_backend(::B200Device)", "Tesserae.has_device(::B200Device)",
                   "Tesserae.free_temporary!(a::CuArray)", "Adapt.adapt_storage(::B200Device",
                   "function Tesserae.update!(bs::GPUBlockStrategy", "function Tesserae.update!(weights::",
                   "function Tesserae.P2G(bodies::P2GBodies", "function Tesserae.foreach_loop(f, device::CUDADevice",
                   "function Tesserae.G2P(f, device::CUDADevice", "function Tesserae.reorder_particles!(",
                   "function Tesserae.block_ordered_particle_contiguity(", "function ChainRulesCore.rrule("):
        assert method in src, method
