"""The C ABI library loads and exports every symbol include/lbm_b200.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

from lbm_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lbm_b200.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(lbm_\w+)\s*\(", txt, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_header_parses():
    names = header_functions()
    assert "lbm_postcoll" in names and "lbm_step" in names and "lbm_boundarycond" in names
    assert len(names) >= 29


def test_library_exports_every_header_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\sT\s(\w+)$", out.stdout, flags=re.M))
    missing = [n for n in header_functions() if n not in exported]
    assert not missing, "not exported: %s" % missing
    for n in header_functions():
        assert hasattr(lib, n)


def test_bindings_cover_header():
    bound = set(_lib.SIGNATURES) | {"lbm_last_error", "lbm_ensemble_last_error"}
    assert set(header_functions()) == bound


def test_fortran_module_binds_every_header_function():
    """include/lbm_b200_iface.F90 has an interface (bind(C, name=...)) for every
    entry point of the header, so a Fortran driver can call all of them."""
    import os
    import re
    src = open(os.path.join(os.path.dirname(_lib.LIB_PATH), "..", "include", "lbm_b200_iface.F90")).read()
    bound = set(re.findall(r'bind\(C,\s*name="(lbm_[a-z0-9_]+)"\)', src))
    assert set(header_functions()) <= bound, sorted(set(header_functions()) - bound)


def test_library_does_not_link_the_oracle(lib):
    out = subprocess.run(["nm", "-D", _lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    assert "orc_" not in out
    ldd = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in ldd


def test_abi_version(lib):
    assert lib.lbm_abi_version() == 1


def test_params_struct_matches_header():
    txt = open(HEADER).read()
    body = re.search(r"typedef struct lbm_params \{(.*?)\} lbm_params;", txt, flags=re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        ty, names = decl.split(None, 1)
        fields += [(n.strip(), ty) for n in names.split(",")]
    py = [(n, t) for n, t in _lib.LbmParams._fields_]
    assert [n for n, _ in fields] == [n for n, _ in py]
    for (n, ty), (_, ct) in zip(fields, py):
        assert (ty == "float") == (ct is ctypes.c_float), n
    assert ctypes.sizeof(_lib.LbmParams) == 4 * len(fields)


def test_null_context_is_an_error_not_a_crash(lib):
    """Every entry point that takes a context (or an ensemble) as its first
    argument answers LBM_ERR_ARG to a null one, before touching the GPU."""
    no_context = {"lbm_create", "lbm_abi_version", "lbm_last_error", "lbm_ensemble_last_error",
                  "lbm_ensemble_create", "lbm_mass_momentum_noalloc", "lbm_ensemble_variant_shape"}
    checked = 0
    for name in header_functions():
        if name in no_context:
            continue
        args = []
        for t in _lib.SIGNATURES[name]:
            if t is ctypes.c_void_p or not hasattr(t, "_type_") or isinstance(t._type_, type):
                args.append(None)                       # pointers, the context first
            elif t._type_ in "fd":
                args.append(0.0)
            else:
                args.append(1)
        assert getattr(lib, name)(*args) == _lib.LBM_ERR_ARG, name
        checked += 1
    assert checked >= 70


def test_ensemble_launch_shapes(lib):
    """The autotuner's launch shapes: distinct (threads, min blocks per SM, tiles
    per block) whose register caps the compiler can meet, out-of-range variants
    refused."""
    t, m, r = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_int32(0)
    shapes = []
    for v in range(_lib.LBM_ENS_VARIANTS):
        assert lib.lbm_ensemble_variant_shape(v, ctypes.byref(t), ctypes.byref(m), ctypes.byref(r)) == _lib.LBM_OK
        assert t.value in (64, 128, 256) and 1 <= m.value and t.value * m.value <= 2048 and r.value in (1, 2, 4)
        shapes.append((t.value, m.value, r.value))
    assert len(set(shapes)) == len(shapes)
    for v in (-1, _lib.LBM_ENS_VARIANTS):
        assert lib.lbm_ensemble_variant_shape(v, ctypes.byref(t), ctypes.byref(m), ctypes.byref(r)) == _lib.LBM_ERR_ARG


def test_create_rejects_bad_params_before_touching_the_gpu(lib):
    h = ctypes.c_void_p()
    for bad in (dict(nl=15), dict(nx=1), dict(ibgk=4), dict(storage=7), dict(ihrr=2)):
        kw = dict(nx=8, ny=8, nz=8, nl=27, ibgk=3, ihrr=1, ivreman=1, ibnd=1, jbnd=0, kbnd=12,
                  iturb_pos=3, storage=0, kinevisc=1e-4, smagorinsky=0.15, rho0=1.0, udir=0.0)
        kw.update(bad)
        p = _lib.LbmParams(**kw)
        rc = lib.lbm_create(ctypes.byref(h), ctypes.byref(p))
        assert rc in (_lib.LBM_ERR_ARG, _lib.LBM_ERR_UNSUPPORTED), (bad, rc)


def test_header_compiles_as_c_and_cxx(tmp_path):
    """The header is plain C: it compiles as C99 and as C++17 with warnings as errors."""
    for cc, std in (("gcc", "-std=c99"), ("g++", "-std=c++17")):
        src = tmp_path / ("probe.c" if cc == "gcc" else "probe.cpp")
        src.write_text('#include "lbm_b200.h"\nint main(void) { return LBM_OK; }\n')
        r = subprocess.run([cc, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                            "-I", os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_plain_c_caller_links_and_runs_without_a_gpu(lib, tmp_path):
    """A C program links against liblbmb200.so the way a Fortran or C driver would,
    and the calls that touch no GPU answer: the ABI version, and lbm_create's
    refusal of bad dimensions with a code instead of a trap."""
    src = tmp_path / "caller.c"
    src.write_text(r'''
#include <stdio.h>
#include "lbm_b200.h"
int main(void) {
    lbm_params p = {0};
    lbm_ctx* ctx = 0;
    p.nx = 1; p.ny = 8; p.nz = 8; p.nl = 19;
    int bad = lbm_create(&ctx, &p);
    printf("%d %d %d\n", lbm_abi_version(), bad, ctx == 0);
    return 0;
}
''')
    exe = tmp_path / "caller"
    libdir = os.path.dirname(_lib.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                        "-L", libdir, "-llbmb200", "-Wl,-rpath," + libdir, "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    version, bad, null = (int(x) for x in out.stdout.split())
    assert version == lib.lbm_abi_version() and bad == _lib.LBM_ERR_ARG and null == 1


def test_fortran_interfaces_match_the_c_signatures():
    """Each bind(C) interface of include/lbm_b200_iface.F90 has the C function's
    argument count, and each argument's declaration passes what the C side
    expects: device and host addresses as type(c_ptr), value (or a Fortran
    variable by reference where C takes int64_t* / double* / a struct),
    integers as integer(c_int32_t / c_int64_t), value, reals as real(c_float /
    c_double), value."""
    src = open(os.path.join(ROOT, "include", "lbm_b200_iface.F90")).read()
    src = re.sub(r"!.*", "", src)                                   # comments
    src = re.sub(r"&\s*\n\s*&?", " ", src)                          # continuation lines
    blocks = re.findall(r'function\s+(lbm_\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name="(lbm_\w+)"\)(.*?)end function',
                        src, flags=re.S)

    def fortran_kind(decl):
        d = decl.replace(" ", "").lower()
        for prefix, k in (("type(c_ptr),value", "ptr"), ("integer(c_int32_t),value", "i32"),
                          ("integer(c_int),value", "i32"), ("integer(c_int64_t),value", "i64"),
                          ("real(c_float),value", "f32"), ("real(c_double),value", "f64")):
            if d.startswith(prefix):
                return k
        return "ref"                                                # passed by reference: a pointer in C

    c_kind = {ctypes.c_void_p: ("ptr", "ref"), ctypes.c_int32: ("i32",), ctypes.c_int64: ("i64",),
              ctypes.c_uint64: ("i64",), ctypes.c_float: ("f32",), ctypes.c_double: ("f64",)}
    checked = 0
    for _, args, cname, body in blocks:
        if cname not in _lib.SIGNATURES:
            continue
        names = [a.strip().lower() for a in args.split(",") if a.strip()]
        sig = _lib.SIGNATURES[cname]
        assert len(names) == len(sig), (cname, names, len(sig))
        kinds = {}
        for line in body.splitlines():
            if "::" in line:
                decl, names_part = line.split("::", 1)
                for v in names_part.split(","):
                    v = v.strip().split("(")[0].strip().lower()
                    if v:
                        kinds[v] = fortran_kind(decl)
        for a, t in zip(names, sig):
            allowed = c_kind.get(t, ("ref",))
            assert kinds.get(a) in allowed, (cname, a, kinds.get(a), allowed)
        checked += 1
    assert checked >= 75
