"""CPU checks of the C ABI: the library loads, exports every declared symbol,
and its host-side logic answers without touching a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import mfix_b200
from mfix_b200 import leq

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(mfixgpu_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    L = mfix_b200.lib()
    names = _declared()
    assert len(names) >= 14
    for nm in names:
        assert hasattr(L, nm), nm


def _gpu_visible():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def test_geometry_validation():
    assert leq.init_geometry(4, 5, 6, 1, 120, 0) == 0
    assert leq.init_geometry(4, 5, 6, 1, 121, 0) == leq.IER_ARGS
    assert leq.init_geometry(4, 5, 2, 0, 40, 0) == leq.IER_ARGS  # 2-D needs KMAX2 = 1
    assert leq.init_geometry(0, 5, 6, 1, 0, 0) == leq.IER_ARGS


def test_options_roundtrip():
    assert leq.set_option("precision", 1) == 0 and leq.get_option("precision") == 1
    assert leq.set_option("precision", 0) == 0
    assert leq.set_option("precision", 3) == leq.IER_ARGS
    assert leq.set_option("no_such_option", 1) == leq.IER_ARGS
    assert leq.get_option("write_back_ab") == 1
    assert leq.get_option("do_transpose") == 0
    assert leq.set_option("do_transpose", 1) == 0 and leq.get_option("do_transpose") == 1
    assert leq.set_option("do_transpose", 0) == 0
    assert leq.get_option("deflate") == 1 and leq.get_option("replace_every") == 20
    assert leq.get_option("staged_matvec") == 2
    assert leq.get_option("restart_growth") == 100
    assert leq.get_option("minimize_dotproducts") == 0 and leq.get_option("icheck_bicgs") == 1
    assert leq.set_option("icheck_bicgs", 0) == leq.IER_ARGS
    assert leq.set_option("restart_growth", 0.5) == leq.IER_ARGS
    assert leq.set_option("restart_growth", 0) == 0 and leq.set_option("restart_growth", 100) == 0
    assert leq.set_option("staged_matvec", 0) == 0 and leq.get_option("staged_matvec") == 0
    assert leq.set_option("staged_matvec", 3) == leq.IER_ARGS
    assert leq.set_option("staged_matvec", 2) == 0
    # lanes per J-line: 1..32
    assert leq.set_option("line_lanes", 32) == 0 and leq.get_option("line_lanes") == 32
    assert leq.set_option("line_lanes", 33) == leq.IER_ARGS
    assert leq.set_option("line_lanes", 64) == leq.IER_ARGS
    assert leq.set_option("line_lanes", 0) == 0


def test_argument_errors_before_device_work():
    a = np.zeros((2, 7, 120))
    b = np.zeros((2, 120))
    x = np.zeros(120)
    assert leq.init_geometry(4, 5, 6, 1, 120, 1) == 0
    assert leq.solve_lin_eq("U_g", 3, x, a, b, 5, 10, 2, "RSRS", 1e-8, "LINE") == leq.IER_ARGS  # M > DIMENSION_M
    assert leq.solve_lin_eq("U_g", 3, x, a, b, 0, 10, 0, "RSRS", 1e-8, "LINE") == leq.IER_UNSUPPORTED
    assert leq.solve_lin_eq("U_g", 3, x, a, b, 0, 10, 6, "RSRS", 1e-8, "LINE") == leq.IER_UNSUPPORTED
    assert leq.solve_lin_eq("U_g", 3, x, a, b, 0, 10, 2, "RSRS", 1e-8, "ILU") == leq.IER_UNSUPPORTED


@pytest.mark.skipif(_gpu_visible(), reason="checks the behaviour without a GPU")
def test_no_cpu_fallback_without_gpu():
    a = np.zeros((7, 120))
    a[3] = -1.0
    b = np.ones(120)
    x = np.zeros(120)
    assert leq.init_geometry(4, 5, 6, 1, 120, 0) == 0
    assert leq.solve_lin_eq("U_g", 3, x, a, b, 0, 10, 2, "RSRS", 1e-8, "LINE") == leq.IER_CUDA
    assert "no CUDA device" in leq.last_error()
    assert not x.any()


def test_fastdiv_formula():
    """The host/device magic-number division used for cell -> (i, j, k)."""
    rng = np.random.default_rng(0)
    for d in list(range(1, 70)) + [193, 194, 258, 386, 1000, 65537]:
        l = 0
        while (1 << l) < d:
            l += 1
        m = ((1 << 32) * ((1 << l) - d)) // d + 1
        m &= 0xFFFFFFFF
        ns = np.concatenate([rng.integers(0, 2**31, 2000), np.arange(0, 5000), [2**31 - 1, 2**32 - 1]])
        for n in ns.tolist():
            q = (((n * m) >> 32) + n) >> l
            assert q == n // d, (d, n)


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors have the sizes and field offsets of include/mfixgpu.h."""
    import ctypes as C
    import subprocess

    structs = {"mfixgpu_stats": leq.Stats, "mfixgpu_geom": leq.Geom, "mfixgpu_system": leq.SystemC,
               "mfixgpu_server_config": leq.ServerConfigC, "mfixgpu_request": leq.RequestC,
               "mfixgpu_server_counters": leq.ServerCountersC}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mfixgpu.h"', 'int main(void){']
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_server_config_errors_before_device_work():
    import ctypes as C

    L = mfix_b200.lib()
    h = C.c_void_p()

    def create(**kw):
        cfg = leq.ServerConfigC(kw.get("precision", 1), 0, 0, 0, 0.0, 0.0, kw.get("sweep", b"RSRS"),
                                kw.get("pc", b"LINE"))
        return L.mfixgpu_server_create(C.byref(cfg), C.byref(h))

    assert create(precision=2) == leq.IER_ARGS
    assert create(pc=b"ILU ") == leq.IER_UNSUPPORTED
    assert create(sweep=b"ISIS") == leq.IER_UNSUPPORTED
    assert create(sweep=b"ASAS") == leq.IER_UNSUPPORTED
    assert L.mfixgpu_server_create(None, None) == leq.IER_ARGS
    if not _gpu_visible():
        assert create() == leq.IER_CUDA
        assert "no CUDA device" in leq.last_error()


@pytest.mark.skipif(_gpu_visible(), reason="checks the behaviour without a GPU")
def test_deferred_calls_without_gpu():
    """mfixgpu_solve_lin_eq_defer_ checks each call at once and queues the
    batchable ones (IER = INCOMPLETE until the flush); the flush writes every
    queued IER, here the no-device code."""
    n = 120
    a = np.zeros((3, 7, n))
    a[:, 3] = -1.0
    b = np.ones((3, n))
    xs = [np.zeros(n) for _ in range(3)]
    assert leq.init_geometry(4, 5, 6, 1, n, 2) == 0
    bad = leq.defer_lin_eq("U_s", 3, xs[0], a, b, 5, 10, 2, "RSRS", 1e-8, "LINE")  # M > DIMENSION_M
    assert bad.value == leq.IER_ARGS and leq.pending_lin_eq() == 0
    cells = [leq.defer_lin_eq("U_s", 3, xs[m], a, b, m, 10, 2, "RSRS", 1e-8, "LINE") for m in range(3)]
    assert [c.value for c in cells] == [leq.IER_INCOMPLETE] * 3 and leq.pending_lin_eq() == 3
    assert leq.flush_lin_eq() == leq.IER_CUDA
    assert [c.value for c in cells] == [leq.IER_CUDA] * 3 and leq.pending_lin_eq() == 0
    assert leq.flush_lin_eq() == 0  # nothing queued


@pytest.mark.skipif(_gpu_visible(), reason="checks the behaviour without a GPU")
def test_deferred_queue_aliasing_geometry_finalize():
    """A deferred call whose VAR or A_M(:,:,M) slice is already queued solves the
    queue first (the earlier call's IER is written, the new call waits alone); a
    geometry registered after a call was queued does not change that call; and
    mfixgpu_finalize drops the queue, leaving its IERs at INCOMPLETE."""
    n = 120
    a = np.zeros((3, 7, n))
    a[:, 3] = -1.0
    b = np.ones((3, n))
    xs = [np.zeros(n) for _ in range(3)]
    assert leq.init_geometry(4, 5, 6, 1, n, 2) == 0
    c0 = leq.defer_lin_eq("U_s", 3, xs[0], a, b, 0, 10, 2, "RSRS", 1e-8, "LINE")
    c1 = leq.defer_lin_eq("U_s", 3, xs[1], a, b, 1, 10, 2, "RSRS", 1e-8, "LINE")
    assert leq.pending_lin_eq() == 2
    same_var = leq.defer_lin_eq("U_s", 3, xs[0], a, b, 2, 10, 2, "RSRS", 1e-8, "LINE")
    assert (c0.value, c1.value) == (leq.IER_CUDA, leq.IER_CUDA)  # the queue was solved first
    assert same_var.value == leq.IER_INCOMPLETE and leq.pending_lin_eq() == 1
    same_slice = leq.defer_lin_eq("U_s", 3, xs[1], a, b, 2, 10, 2, "RSRS", 1e-8, "LINE")
    assert same_var.value == leq.IER_CUDA and same_slice.value == leq.IER_INCOMPLETE
    assert leq.pending_lin_eq() == 1
    # a new geometry: the queued call keeps its own, the flush still runs it
    assert leq.init_geometry(2, 5, 3, 1, 30, 0) == 0
    assert leq.flush_lin_eq() == leq.IER_CUDA and same_slice.value == leq.IER_CUDA
    assert leq.init_geometry(4, 5, 6, 1, n, 2) == 0
    left = leq.defer_lin_eq("U_s", 3, xs[2], a, b, 2, 10, 2, "RSRS", 1e-8, "LINE")
    assert leq.pending_lin_eq() == 1
    leq.finalize()
    assert leq.pending_lin_eq() == 0 and left.value == leq.IER_INCOMPLETE


def test_pp_assembly_argument_checks():
    """The pressure-correction entry points refuse a missing field record, a
    compressible run and missing arrays before any device work."""
    from mfix_b200 import systems as S

    f = S.pp_fields(6, 7, 5, seed=1, mmax=1)
    assert leq.init_geometry(f.imax2, f.jmax2, f.kmax2, f.do_k, f.n, 2) == 0
    a, b, bm = np.zeros((7, f.n)), np.zeros(f.n), np.zeros(f.n)
    L = mfix_b200.lib()
    assert L.mfixgpu_conv_source_pp_g(None, a.ctypes.data, b.ctypes.data, bm.ctypes.data) == leq.IER_ARGS
    c = leq.pp_struct(f)
    if _gpu_visible():
        c.ro_g0_defined = 0
        assert L.mfixgpu_conv_source_pp_g(ctypes.byref(c), a.ctypes.data, b.ctypes.data,
                                          bm.ctypes.data) == leq.IER_UNSUPPORTED
    else:  # without a device every call ends in the no-device code
        assert L.mfixgpu_conv_source_pp_g(ctypes.byref(c), a.ctypes.data, b.ctypes.data,
                                          bm.ctypes.data) == leq.IER_CUDA
        ier, _ = leq.solve_pp_g(f, 0.0, np.zeros(f.n))
        assert ier == leq.IER_CUDA
