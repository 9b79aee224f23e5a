"""C ABI: the libraries load without a GPU and export every declared symbol;
the Python mirror matches the header.  No compute call is made here."""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

import hunyuansc25_b200 as hp
from hunyuansc25_b200 import _abi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("defined",)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(hp.library_path()):
        build.build_cuda()
    return C.CDLL(hp.library_path())


def test_partition_header_symbols_exported(lib):
    names = declared_functions("hp_partition.h")
    assert "hp_partition" in names and "hunyuangraph_PartitionGraph" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_c_program_links_every_entry_point(lib, tmp_path):
    """A C caller compiled against include/hp_partition.h links libhp_b200.so:
    every declared function resolves at link time (the legacy
    hunyuangraph_PartitionGraph among them), and the entry points that need
    no device run."""
    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("no C compiler")
    names = declared_functions("hp_partition.h")
    refs = "\n".join(f"    (void *)&{n}," for n in names)
    src = tmp_path / "caller.c"
    src.write_text(f"""#include <stdio.h>
#include <string.h>
#include "hp_partition.h"
static void *const entry_points[] = {{
{refs}
}};
int main(void)
{{
    for (size_t i = 0; i < sizeof entry_points / sizeof entry_points[0]; i++)
        if (!entry_points[i]) return 2;
    hp_options o;
    hp_options_default(&o);
    hp_tuning t;
    hp_tuning_default(&t);
    if (o.version != HP_OPTIONS_VERSION || o.match_rounds != 6 || t.small_match_n != 8192) return 3;
    if (strcmp(hp_strerror(HP_ERR_TIMEOUT), hp_strerror(HP_OK)) == 0) return 4;
    printf("linked %zu entry points\\n", sizeof entry_points / sizeof entry_points[0]);
    return 0;
}}
""")
    libdir = os.path.dirname(hp.library_path())
    exe = tmp_path / "caller"
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lhp_b200", f"-Wl,-rpath,{libdir}"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert f"linked {len(names)} entry points" in r.stdout


def test_gen_header_symbols_exported():
    path = build.build_gen()
    lib = C.CDLL(path)
    names = declared_functions("hp_gen.h")
    assert "hp_gen_rmat" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_prototypes_cover_header():
    names = declared_functions("hp_partition.h")
    assert sorted(_abi.PROTOTYPES) == names


def test_load_library_binds_prototypes(lib):
    L = hp.load_library()
    assert L.hp_partition.restype == C.c_int


def test_options_struct_layout():
    # version + 11 int32 fields (48 bytes), then the 8-byte seed; `eager` took the
    # padding slot, so the layout of version-1 callers is unchanged
    assert C.sizeof(_abi.HpOptions) == 56
    assert _abi.HpOptions.eager.offset == 44
    assert _abi.HpOptions.seed.offset == 48
    # the per-class arrays hold HP_PROF_NCLASS (12) entries
    assert _abi.HP_PROF_NCLASS == 12
    assert C.sizeof(_abi.HpStats) == 8 * 3 + 4 * 2 + 8 + 4 * 2 + 4 * 6 + 4 * 12 + 8 * 12 + 4 * 12


def test_options_default_matches_library(lib):
    o = _abi.HpOptions()
    lib.hp_options_default(C.byref(o))
    d = _abi.default_options()
    for name, _ in _abi.HpOptions._fields_:
        assert getattr(o, name) == getattr(d, name), name


def test_strerror(lib):
    lib.hp_strerror.restype = C.c_char_p
    assert lib.hp_strerror(0) == b"ok"
    assert b"device memory" in lib.hp_strerror(_abi.HP_ERR_NOMEM)
    assert lib.hp_strerror(-99) == b"unknown error"


def test_legacy_symbol_signature_comment():
    hdr = open(os.path.join(ROOT, "include", "hp_partition.h")).read()
    assert "void hunyuangraph_PartitionGraph(int *nvtxs, int *xadj, int *adjncy, int *vwgt" in hdr
