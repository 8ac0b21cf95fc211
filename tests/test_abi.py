"""The C ABI library: builds for sm_100a, loads, exports every declared symbol."""
import ctypes
import os
import re

import pytest

from tests.conftest import ROOT, cuda_available


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"^\s*(?:ILG_API\s+)?(?:const\s+)?(?:int|void|const char|char)\s*\*?\s*(ilg_\w+)\s*\(", src, re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("ilg_create", "ilg_destroy", "ilg_set_mesh", "ilg_build", "ilg_intersect", "ilg_occluded"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from illuminaprt_b200 import build
    lib = ctypes.CDLL(build.build())
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert missing == []


def test_library_exports_only_the_entry_points():
    import shutil
    import subprocess
    from illuminaprt_b200 import build
    if shutil.which("nm") is None:
        pytest.skip("no nm")
    out = subprocess.run(["nm", "-D", "--defined-only", build.build()], capture_output=True, text=True,
                         check=True).stdout
    code = [ln.split()[-1] for ln in out.splitlines() if len(ln.split()) == 3 and ln.split()[1] == "T"]
    assert code and all(name.startswith("ilg_") for name in code), [n for n in code if not n.startswith("ilg_")][:5]
    assert sorted(code) == sorted(declared_symbols())


def test_binding_lists_every_symbol():
    from illuminaprt_b200.ilg import EXPORTED
    assert sorted(EXPORTED) == sorted(s for s in declared_symbols() if s in EXPORTED)
    assert set(declared_symbols()) <= set(EXPORTED) | {s for s in declared_symbols() if not s.startswith("ilg_")}


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_loudly():
    from illuminaprt_b200.ilg import GpuSpace, IlgError
    with pytest.raises(IlgError):
        GpuSpace()


def test_binding_constants_match_the_header():
    # every #define of the C ABI that the Python binding also names has the
    # same value there (flags, material kinds, sizes)
    from illuminaprt_b200 import ilg
    text = open(os.path.join(ROOT, "include", "ilg.h")).read()
    defines = {m.group(1): int(m.group(2), 0) for m in re.finditer(r"#define (ILG_\w+) (0x[0-9a-fA-F]+|\d+)u", text)}
    shared = [k for k in defines if hasattr(ilg, k)]
    assert {"ILG_MAT_MIRROR", "ILG_MAT_GLASS", "ILG_DEVICE_PTRS", "ILG_WATERTIGHT"} <= set(shared), shared
    for k in shared:
        assert getattr(ilg, k) == defines[k], k
    # the option structs have the header's layout size
    assert ctypes.sizeof(ilg.ilg_render_opts) == 4 * (7 + 3 + 6)
    assert ctypes.sizeof(ilg.ilg_material) == 32


def test_plain_c_client_builds_and_links(tmp_path):
    # the header is plain C99 (what a cgo, JNI or C host includes) and a C
    # program links against the library; without a GPU, ilg_create fails
    # with ILG_ECUDA and leaves the handle null
    import shutil
    import subprocess
    from illuminaprt_b200 import build
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    lib = build.build()
    src = tmp_path / "client.c"
    src.write_text(
        '#include "ilg.h"\n#include <stdio.h>\n'
        "int main(void) {\n"
        "    ilg_ctx *ctx = 0;\n    ilg_opts o = {0};\n"
        "    int rc = ilg_create(&ctx, &o);\n"
        '    printf("create %d %d %s\\n", rc, ctx != 0, ilg_last_error(ctx));\n'
        "    if (rc == ILG_OK) ilg_destroy(ctx);\n    return 0;\n}\n")
    exe = tmp_path / "client"
    libdir = os.path.dirname(lib)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I",
                    os.path.join(ROOT, "include"), str(src), "-L", libdir, "-l:" + os.path.basename(lib),
                    "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120, check=True).stdout.split()
    assert out[0] == "create"
    if not cuda_available():
        assert out[1] == "3" and out[2] == "0"  # ILG_ECUDA, no handle
    else:
        assert out[1] == "0" and out[2] == "1"
