"""The C-ABI library without a GPU: it builds, loads, exports every symbol
include/*.h declares, and validates arguments before touching a device."""
import ctypes
import os
import re
import subprocess
import sys

import pytest

import imgrecsrc_b200 as ct
from imgrecsrc_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\([^;{]*\)\s*;", text, re.M):
            names.add(m.group(1))
        for m in re.finditer(r"^extern\s+[\w\s\*]+?\b(\w+)\s*;", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_builds_and_exports_every_declared_symbol():
    path = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    decl = declared_symbols()
    assert {"setup", "gpuPrj", "pConf", "ctprj_forward", "ctprj_backward"} <= set(decl)
    missing = [s for s in decl if s not in exported]
    assert not missing, missing


def test_geometry_struct_matches_header():
    assert ctypes.sizeof(ct.Geometry) == 7 * 4


@pytest.mark.parametrize("geo, status", [
    ((32, 45, 16, 18), ct._lib.CTPRJ_EINVAL),       # prjFull not a multiple of 4
    ((32, 45, 40, 36), ct._lib.CTPRJ_EINVAL),       # np > prjFull
    ((0, 45, 16, 16), ct._lib.CTPRJ_EINVAL),
    ((32, 45, 16, 16, 0.0), ct._lib.CTPRJ_EINVAL),  # dSize
    ((32, 45, 16, 16, 1.0, -1.0), ct._lib.CTPRJ_EINVAL),
    ((70000, 45, 16, 16), ct._lib.CTPRJ_ERANGE),
])
def test_plan_rejects_invalid_geometry_without_a_device(geo, status):
    L = ct.lib()
    g = ct.Geometry(*geo)
    p = ctypes.c_void_p()
    assert L.ctprj_plan_create(ctypes.byref(g), 0, ctypes.byref(p)) == status
    assert not p.value
    assert L.ctprj_last_error()


def test_null_arguments_rejected():
    L = ct.lib()
    assert L.ctprj_plan_create(None, 0, None) == ct._lib.CTPRJ_EINVAL
    assert L.ctprj_forward(None, None, None, None) == ct._lib.CTPRJ_EINVAL
    assert L.ctprj_backward(None, None, None, None) == ct._lib.CTPRJ_EINVAL
    assert L.ctprj_fbp(None, None, None, None) == ct._lib.CTPRJ_EINVAL
    assert L.ctprj_error_string(ct._lib.CTPRJ_ENOTSETUP)


def test_gpuprj_before_setup_reports_not_setup():
    # fresh process: the reference-compatible entry points keep global state
    code = ("import imgrecsrc_b200 as ct; L = ct.lib(); import numpy as np;"
            "a = np.zeros(4, np.float32);"
            "print(L.gpuPrj(a.ctypes.data, a.ctypes.data, bytes([ct.FWD_BIT])))")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert int(r.stdout.strip()) == ct._lib.CTPRJ_ENOTSETUP


def test_no_cpu_fallback_without_a_device():
    """Without a CUDA device a valid geometry fails with a CUDA status and a
    message; nothing computes on the host instead."""
    code = ("import ctypes, imgrecsrc_b200 as ct; L = ct.lib();"
            "g = ct.Geometry(64, 91, 30, 60, 1.0, 1.0, 0.0); p = ctypes.c_void_p();"
            "st = L.ctprj_plan_create(ctypes.byref(g), 0, ctypes.byref(p));"
            "print(st, bool(p.value), L.ctprj_last_error().decode())")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr
    st, made, msg = r.stdout.strip().split(" ", 2)
    assert int(st) == ct._lib.CTPRJ_ECUDA and made == "False" and msg


def test_python_layer_raises_without_a_device():
    code = ("import imgrecsrc_b200 as ct\n"
            "try:\n"
            "    ct.Projector(ct.Geometry(64, 91, 30, 60, 1.0, 1.0, 0.0), device=0)\n"
            "    print('made')\n"
            "except Exception as e:\n"
            "    print(type(e).__name__)\n")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() != "made"
