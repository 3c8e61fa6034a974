"""The C ABI library: builds, loads, exports what include/std2g.h declares.

No compute call is made here; on a machine without a GPU ``std2g_create``
must fail with STD2G_ENODEV instead of falling back to the CPU.
"""
import ctypes
import os
import re

import pytest

from tests.conftest import ROOT


def header_functions():
    text = open(os.path.join(ROOT, "include", "std2g.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|int64_t|const char \*)\s*\*?\s*(std2g_\w+)\s*\(",
                                 text, re.M)))


def test_header_declares_entry_points():
    names = header_functions()
    assert "std2g_solve" in names and "std2g_create" in names and len(names) >= 11


def test_library_exports_every_declared_symbol():
    from stda_b200.build import build
    path = build()
    lib = ctypes.CDLL(path)
    for name in header_functions():
        assert hasattr(lib, name), name


def test_binding_covers_exports():
    from stda_b200.engine import EXPORTS
    assert sorted(EXPORTS) == sorted(n for n in header_functions() if n in EXPORTS)
    assert set(header_functions()) <= set(EXPORTS), set(header_functions()) - set(EXPORTS)


def test_create_without_gpu_is_an_error_not_a_fallback():
    from stda_b200 import engine
    lib = engine.library()
    ctx = ctypes.c_void_p()
    opts = engine.Opts(0, 0, 0, 0, 0)
    code = lib.std2g_create(ctypes.byref(ctx), ctypes.byref(opts))
    if code == 0:          # a B200 is present: fine, release it
        lib.std2g_destroy(ctx)
    else:
        assert code == 12, engine.STATUS.get(code)
        assert b"sm_100" in lib.std2g_error_string(code) or code == 12


def test_null_arguments_rejected():
    from stda_b200 import engine
    lib = engine.library()
    assert lib.std2g_create(None, None) == 1
    assert lib.std2g_solve(None, None, None) == 1
    assert lib.std2g_error_string(4) == b"no CSF, increase energy threshold (-e option)"


def test_server_arguments_checked_before_any_device_call():
    from stda_b200 import engine
    lib = engine.library()
    srv = ctypes.c_void_p()
    assert lib.std2g_server_create(ctypes.byref(srv), None) == 1
    for slots in (0, 65):
        opts = engine.ServerOpts(0, 1, slots, 0, 0)
        assert lib.std2g_server_create(ctypes.byref(srv), ctypes.byref(opts)) == 1
    assert lib.std2g_server_submit(None, None, None) == 1
    done = ctypes.c_int()
    assert lib.std2g_server_poll(None, 1, ctypes.byref(done)) == 1
    assert lib.std2g_server_wait(None, 1, None, None, None, None) == 1
    assert lib.std2g_set_sm_limit(None, 4) == 1
    lib.std2g_server_destroy(None)       # a null server is ignored


def test_batch_arguments_checked_before_any_device_call():
    """The batched-eigensolve entry points reject null arguments and bad
    devices without touching a device (and so without a GPU)."""
    from stda_b200 import engine
    lib = engine.library()
    one = ctypes.c_int64()
    assert lib.std2g_batch_create(0, None) == 1
    b = ctypes.c_void_p()
    assert lib.std2g_batch_create(-1, ctypes.byref(b)) == 12 and not b.value
    assert lib.std2g_attach_batch(None, None) == 1
    assert lib.std2g_batch_stats(None, ctypes.byref(one), ctypes.byref(one),
                                 ctypes.byref(one), None) == 1
    assert lib.std2g_server_batch_stats(None, ctypes.byref(one), ctypes.byref(one),
                                        ctypes.byref(one), None) == 1
    assert lib.std2g_last_batched(None) == 0
    lib.std2g_batch_destroy(None)         # a null batch is ignored


C_HOST = r"""
#include <stdio.h>
#include <string.h>
#include "std2g.h"
int main(void) {
  std2g_opts o;
  std2g_params p;
  std2g_result r;
  void *ctx = 0;
  int st;
  memset(&o, 0, sizeof o);
  memset(&p, 0, sizeof p);
  memset(&r, 0, sizeof r);
  st = std2g_create(&ctx, &o);
  if (st == STD2G_OK) std2g_destroy(ctx);
  (void)p; (void)r;
  printf("%d %s\n", st, std2g_error_string(st));
  return 0;
}
"""


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c99"), ("g++", "-std=c++11")])
def test_header_serves_plain_c_and_cpp_hosts(tmp_path, compiler, std):
    """A C (or C++) host compiles against include/std2g.h without warnings,
    links libstd2g.so and gets a status code with its message back."""
    import shutil
    import subprocess
    from stda_b200.build import build
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not available")
    lib = build()
    src = tmp_path / ("host.c" if compiler == "gcc" else "host.cpp")
    src.write_text(C_HOST)
    exe = tmp_path / "host"
    libdir = os.path.dirname(lib)
    r = subprocess.run([compiler, std, "-Wall", "-Wextra", "-pedantic", "-Werror",
                        "-I" + os.path.join(ROOT, "include"), str(src), "-L" + libdir, "-lstd2g",
                        "-Wl,-rpath," + libdir, "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    code, msg = out.stdout.split(" ", 1)
    assert int(code) in (0, 12) and msg.strip()
