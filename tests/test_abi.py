"""The C-ABI library loads, exports every declared entry point, and fails
cleanly (no crash, an error status) when there is no sm_100 device.  CPU only:
no compute call is made here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu

HEADER = os.path.join(ROOT, "include", "ft_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(ft_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_reference_api():
    names = set(declared_functions())
    for f in ("ft_plan_sph2fourier", "ft_execute_sph2fourier", "ft_execute_fourier2sph", "ft_destroy_harmonic_plan",
              "ft_plan_tri2cheb", "ft_execute_tri2cheb", "ft_execute_cheb2tri", "ft_plan_disk2cxf",
              "ft_execute_disk2cxf", "ft_execute_cxf2disk", "ft_plan_rotsphere", "ft_execute_sph_hi2lo",
              "ft_execute_sph_lo2hi", "ft_destroy_rotation_plan"):
        assert f in names


def test_library_exports_every_declared_symbol():
    import fasttransforms_b200 as ft
    lib = C.CDLL(ft.library_path)
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_plan_struct_prefix_matches_reference():
    # src/fasttransforms.h:370-385: 5 pointers, 5 doubles, 3 ints
    from oracle.bind import _RefHarmonicPlan
    assert _RefHarmonicPlan.NRP.offset == 5 * 8 + 5 * 8
    assert C.sizeof(_RefHarmonicPlan) == 5 * 8 + 5 * 8 + 3 * 4 + 4


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_device_fails_cleanly():
    import fasttransforms_b200 as ft
    p = ft.lib.ft_plan_sph2fourier(16)
    assert not p
    assert ft.lib.ft_b200_last_status() in (2, 4)
    with pytest.raises(ft.FTB200Error):
        ft.plan_sph2fourier(16)


def test_grid_plan_host_checks():
    """Argument checks that run before any device work: the grid plans' odd-M rule (here before
    the device probe, so it holds on any host), NULL plans in the getters, destroyers and execute
    calls (a status, no crash), and the spin grid's no-op TRANS values."""
    import fasttransforms_b200 as ft
    L = ft.lib
    for plan in (lambda: L.ft_plan_spinsph_synthesis(8, 14, 0, 0), lambda: L.ft_plan_spinsph_analysis(8, 14, 1, 0),
                 lambda: L.ft_plan_sph_synthesis(8, 14, 0), lambda: L.ft_plan_disk_analysis(8, 14, 0)):
        assert not plan()
        assert L.ft_b200_last_status() == 1
    assert L.ft_plan_spinsph_synthesis(0, 15, 0, 0) is None and L.ft_b200_last_status() == 1
    assert L.ft_get_spin_spinsphere_fftw_plan(None) == 0
    L.ft_destroy_spinsphere_fftw_plan(None)
    X = np.zeros(2 * 8 * 15)
    ptr = X.ctypes.data_as(C.POINTER(C.c_double))
    L.ft_execute_spinsph_synthesis(b"N", None, ptr, 8, 15)
    assert L.ft_b200_last_status() == 1
    L.ft_execute_sph_analysis(b"N", None, ptr, 8, 15)
    assert L.ft_b200_last_status() == 1
    assert L.ft_b200_execute_spinsph_grid_dev(None, 0, b"N", None, 8, 15, None) == 1


def test_grid_plans_with_kind_check_their_kinds():
    """ft_plan_*_with_kind accept the kind combinations the grid kernels compute and return NULL
    with FT_B200_EUNSUPPORTED (status 6) for others, before any device work; an
    accepted combination goes on to the device (ENODEV without one, or a plan)."""
    import fasttransforms_b200 as ft
    L = ft.lib
    K = lambda *k: (C.c_int * len(k))(*k)
    R2HC, HC2R, RE01, RE10, RE11, RO01, RO10, RE00 = 0, 1, 4, 5, 6, 8, 9, 3
    bad = [lambda: L.ft_plan_sph_with_kind(8, 15, K(RE01, RO10, HC2R), 0),      # mixed types
           lambda: L.ft_plan_sph_with_kind(8, 15, K(RE00, RO01, HC2R), 0),      # a kind not computed here
           lambda: L.ft_plan_disk_with_kind(8, 29, K(RE01, RE01, HC2R), 0),     # the disk's second kind is REDFT11
           lambda: L.ft_plan_tri_with_kind(8, 8, RE01, RE10, 0),
           lambda: L.ft_plan_annulus_with_kind(8, 29, 0.5, K(RO01, HC2R), 0),
           lambda: L.ft_plan_rectdisk_with_kind(8, 8, K(RE01, RO10, RE01), 0),
           lambda: L.ft_plan_tet_with_kind(4, 4, 4, RE01, RE01, RE10, 0),
           lambda: L.ft_plan_spinsph_with_kind(8, 15, 1, K(RO01, RE01), 2, 0)]   # sign must be +-1
    for b in bad:
        assert not b()
        assert L.ft_b200_last_status() == 6
    good = [(lambda: L.ft_plan_sph_with_kind(8, 15, K(RE01, RO01, HC2R), 0), L.ft_destroy_sphere_fftw_plan),
            (lambda: L.ft_plan_disk_with_kind(8, 29, K(RE10, RE11, R2HC), 0), L.ft_destroy_disk_fftw_plan),
            (lambda: L.ft_plan_tri_with_kind(8, 8, RE10, RE10, 0), L.ft_destroy_triangle_fftw_plan),
            (lambda: L.ft_plan_spinsph_with_kind(8, 15, 1, K(RO01, RE01), 1, 0), L.ft_destroy_spinsphere_fftw_plan)]
    for g, destroy in good:
        p = g()
        if has_gpu():
            assert p
            destroy(p)
        else:
            assert not p and L.ft_b200_last_status() in (2, 4)


def test_thread_settings():
    """ft_set_num_threads (plan-building threads) and the FFTW threading calls take any value."""
    import fasttransforms_b200 as ft
    for n in (4, 0, -1, 1000):
        ft.lib.ft_set_num_threads(n)
    assert ft.lib.ft_fftw_init_threads() == 1
    ft.lib.ft_fftw_plan_with_nthreads(8)
    ft.lib.ft_set_num_threads(0)


def _run_c_caller(tmp_path, src):
    """Compile tests/c/<src> as C99 with -Wall -Werror against include/ft_b200.h, link it with
    -lft_b200 and run it; returns the completed process."""
    import shutil
    import subprocess
    import fasttransforms_b200 as ft
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    libdir = os.path.dirname(ft.library_path)
    exe = str(tmp_path / src[:-2])
    subprocess.run([cc, "-O2", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c", src),
                    "-L", libdir, "-lft_b200", "-Wl,-rpath," + libdir, "-lm", "-o", exe], check=True)
    return subprocess.run([exe], capture_output=True, text=True, timeout=300)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path; the device run is the gpu-marked twin")
@pytest.mark.parametrize("src", ["dropin.c", "families.c", "shared_host.c"])
def test_c_caller_compiles_links_and_runs(tmp_path, src):
    """C programs written against the reference's API (tests/c/dropin.c: sph2fourier;
    tests/c/families.c: every other family and the grids) compile, link and, without a usable
    device, report FT_B200_ENODEV cleanly."""
    r = _run_c_caller(tmp_path, src)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ENODEV"


@pytest.mark.gpu
@pytest.mark.parametrize("src", ["dropin.c", "families.c", "shared_host.c"])
def test_c_caller_round_trips_on_device(tmp_path, src):
    """The same C programs on an sm_100 device: every transform they call returns its input
    (dropin.c and shared_host.c print the sph round-trip error, below 1e-13; families.c prints
    "ok")."""
    r = _run_c_caller(tmp_path, src)
    assert r.returncode == 0, r.stderr
    out = r.stdout.strip()
    assert out == "ok" or float(out) < 1e-13, out


def _prototypes():
    """name -> (return type, [parameter declarations]) for every function the header declares."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    text = "\n".join(line for line in text.splitlines() if not line.lstrip().startswith("#"))
    text = re.sub(r"\s+", " ", text)
    protos = {}
    for m in re.finditer(r"(?:^|(?<=[;{}]))\s*([A-Za-z_][\w \*]*?)\b(ft_\w+)\s*\(([^()]*)\)\s*;", text):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3).strip()
        protos[name] = (ret, [] if params in ("", "void") else [q.strip() for q in params.split(",")])
    return protos


def _kind(decl, named=True):
    """'int' / 'double' / 'char' / 'uint' / 'void' / 'ptr' of a return type or a parameter."""
    if "*" in decl or "[" in decl:
        return "ptr"
    toks = [t for t in decl.split() if t != "const"]
    if named and len(toks) > 1:
        toks = toks[:-1]
    for t, k in (("long", "ull"), ("int", "int"), ("double", "double"), ("char", "char"), ("unsigned", "uint"),
                 ("void", "void")):
        if t in toks:
            return k
    return "ptr"


def test_python_bindings_match_the_header():
    """Every function fasttransforms_b200 binds has the header's arity and scalar types."""
    import ctypes
    import fasttransforms_b200 as ft
    kinds = {ctypes.c_int: "int", ctypes.c_double: "double", ctypes.c_char: "char", ctypes.c_uint: "uint",
             ctypes.c_ulonglong: "ull"}
    protos = _prototypes()
    checked = 0
    for name, (ret, params) in protos.items():
        f = getattr(ft.lib, name, None)
        if f is None or f.argtypes is None:
            continue
        got = [kinds.get(a, "ptr") for a in f.argtypes]
        want = [_kind(q) for q in params]
        assert got == want, (name, got, want)
        r = f.restype
        rk = "void" if r is None else kinds.get(r, "ptr")
        assert rk == _kind(ret, named=False), (name, rk, ret)
        checked += 1
    assert checked > 60
