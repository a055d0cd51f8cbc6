"""CPU checks of the Fortran 77 forms of the C ABI (include/flosic_sic_f77.h):
the lowercase, trailing-underscore names a Fortran host without
iso_c_binding links to, every argument by reference, status in IERR.

The calls are made the way a Fortran caller makes them (ctypes with byref
INTEGER*4 / INTEGER*8 / REAL*8 arguments and a hidden CHARACTER length).
Forwarding is checked against a recording stand-in for the C ABI, compiled
here from the header: every F77 form must pass its scalars' values, its
arrays' addresses, the context handle and device addresses unchanged to the
C entry point of the same name, and return that entry point's status in IERR.
No GPU is touched."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "flosic_sic.h")
F77 = os.path.join(ROOT, "include", "flosic_sic_f77.h")
SRC = os.path.join(ROOT, "publicrelease_2020_b200", "csrc", "fortran_abi.cpp")
LIB = os.path.join(ROOT, "publicrelease_2020_b200", "libflosic_sic_b200.so")
FLOSIC_ERR_ARG = 1


def c_signatures():
    """(name, [(type, argument)]) of every entry point of flosic_sic.h."""
    text = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    out = []
    for m in re.finditer(r"^(?:int|const char\*)\s+(flosic_sic_\w+)\s*\((.*?)\);", text, re.M | re.S):
        params = []
        for p in (" ".join(q.split()) for q in m.group(2).split(",")):
            if p == "void":
                continue
            typ, var = p.rsplit(" ", 1)
            while var.startswith("*"):
                typ, var = typ + "*", var[1:]
            params.append((typ, var))
        out.append((m.group(1), params))
    return out


def f77_names():
    text = re.sub(r"/\*.*?\*/", "", open(F77).read(), flags=re.S)
    return sorted(re.findall(r"^void\s+(flosic_sic_\w+_)\s*\(", text, re.M))


def test_every_entry_point_has_an_f77_form():
    assert f77_names() == sorted(name + "_" for name, _ in c_signatures())


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "publicrelease_2020_b200")], check=True)
    return C.CDLL(LIB)


def test_library_exports_the_f77_forms(lib):
    for name in f77_names():
        assert hasattr(lib, name), name


def test_null_context_status_and_message(lib):
    ctx, mode, ierr = C.c_int64(0), C.c_int32(0), C.c_int32(-1)
    lib.flosic_sic_set_precision_(C.byref(ctx), C.byref(mode), C.byref(ierr))
    assert ierr.value == FLOSIC_ERR_ARG
    msg = C.create_string_buffer(64)
    lib.flosic_sic_last_error_(msg, C.c_size_t(64))
    text = msg.raw.decode()
    assert text.rstrip() == "null context" and text.endswith(" ") and len(text) == 64
    short = C.create_string_buffer(4)
    lib.flosic_sic_last_error_(short, C.c_size_t(4))
    assert short.raw.decode() == "null"


# ---------------------------------------------------------------------------
# forwarding, against a recording stand-in for the C entry points
# ---------------------------------------------------------------------------
def _stub_source(sigs):
    lines = ['#include <stdio.h>', '#include <string.h>', '#include "flosic_sic.h"',
             'static char g_log[4096];', 'static void rec(const char* s) { strncat(g_log, s, 4000); }',
             'extern "C" const char* stub_log(void) { return g_log; }',
             'extern "C" void stub_reset(void) { g_log[0] = 0; }']
    for i, (name, params) in enumerate(sigs):
        if name == "flosic_sic_last_error":
            lines.append('extern "C" const char* flosic_sic_last_error(void) { return "stub message"; }')
            continue
        decl = ", ".join(f"{t} {v}" for t, v in params)
        body = [f'  char b[256]; snprintf(b, sizeof b, "{name}"); rec(b);']
        for t, v in params:
            if t == "int":
                body.append(f'  snprintf(b, sizeof b, " {v}=%d", {v}); rec(b);')
            elif t == "int64_t":
                body.append(f'  snprintf(b, sizeof b, " {v}=%lld", (long long){v}); rec(b);')
            elif t == "flosic_ctx**" and v != "ctxs":
                body.append(f'  *{v} = (flosic_ctx*)0xabc0; snprintf(b, sizeof b, " {v}=set"); rec(b);')
            else:
                body.append(f'  snprintf(b, sizeof b, " {v}=%p", (const void*){v}); rec(b);')
        body.append(f"  return {100 + i};")
        lines.append(f'extern "C" int {name}({decl}) {{\n' + "\n".join(body) + "\n}")
    return "\n".join(lines) + "\n"


@pytest.fixture(scope="module")
def stub(tmp_path_factory):
    d = tmp_path_factory.mktemp("f77")
    src = d / "stub.cpp"
    src.write_text(_stub_source(c_signatures()))
    so = d / "libf77stub.so"
    subprocess.run(["g++", "-std=c++17", "-shared", "-fPIC", "-O1", "-I", os.path.join(ROOT, "include"),
                    "-o", str(so), str(src), SRC], check=True)
    L = C.CDLL(str(so))
    L.stub_log.restype = C.c_char_p
    return L


def test_f77_forms_forward_to_the_c_entry_points(stub):
    for i, (name, params) in enumerate(c_signatures()):
        if name in ("flosic_sic_last_error", "flosic_sic_create", "flosic_sic_destroy"):
            continue
        args, expect, keep = [], [name], []
        for j, (t, v) in enumerate(params):
            if t == "flosic_ctx*":
                h = C.c_int64(0x10000 + 0x100 * i)
                keep.append(h)
                args.append(C.byref(h))
                expect.append(f"{v}={hex(h.value)}")
            elif t == "int":
                x = C.c_int32(7 * i + j - 3)
                keep.append(x)
                args.append(C.byref(x))
                expect.append(f"{v}={x.value}")
            elif t == "int64_t":
                x = C.c_int64(1000003 * i + j)
                keep.append(x)
                args.append(C.byref(x))
                expect.append(f"{v}={x.value}")
            elif v.startswith("d_"):
                a = C.c_int64(0x7f0000000000 + 0x1000 * j)
                keep.append(a)
                args.append(C.byref(a))
                expect.append(f"{v}={hex(a.value)}")
            else:
                addr = 0x200000 + 0x1000 * i + 0x40 * j
                args.append(C.c_void_p(addr))
                expect.append(f"{v}={hex(addr)}")
        ierr = C.c_int32(-1)
        args.append(C.byref(ierr))
        stub.stub_reset()
        getattr(stub, name + "_")(*args)
        assert stub.stub_log().decode() == " ".join(expect), name
        assert ierr.value == 100 + i, name


def test_f77_lifecycle_and_message(stub):
    sigs = [n for n, _ in c_signatures()]
    dev, ctx, ierr = C.c_int32(3), C.c_int64(0), C.c_int32(-1)
    stub.stub_reset()
    stub.flosic_sic_create_(C.byref(dev), C.byref(ctx), C.byref(ierr))
    assert stub.stub_log().decode() == "flosic_sic_create device=3 ctx=set"
    assert ctx.value == 0xabc0 and ierr.value == 100 + sigs.index("flosic_sic_create")
    stub.stub_reset()
    stub.flosic_sic_destroy_(C.byref(ctx), C.byref(ierr))
    assert stub.stub_log().decode() == "flosic_sic_destroy ctx=0xabc0"
    assert ctx.value == 0 and ierr.value == 100 + sigs.index("flosic_sic_destroy")
    msg = C.create_string_buffer(20)
    stub.flosic_sic_last_error_(msg, C.c_size_t(20))
    assert msg.raw.decode() == "stub message" + " " * 8
