"""CPU checks of the C-ABI boundary: the library loads, exports every symbol
include/cdft_b200.h declares, and the ctypes struct layouts equal the C ones
(checked by compiling a probe against the header with gcc)."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cdft_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cdft_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_header_symbols():
    from cdft_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 13
    for n in names:
        assert hasattr(lib, n), f"{n} declared in cdft_b200.h but not exported"
    assert sorted(_lib.EXPORTED) == names
    assert lib.cdft_version().startswith(b"cdft_b200")


def test_last_error_without_gpu_work():
    from cdft_b200 import _lib
    lib = _lib.load()
    buf = ctypes.create_string_buffer(64)
    # invalid call: NULL plan output pointer -> CDFT_E_INVALID, no CUDA call made
    rc = lib.cdft_plan_create(None, None)
    assert rc == _lib.E_INVALID
    assert lib.cdft_last_error(buf, 64) == _lib.E_INVALID
    assert b"NULL" in buf.value


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc missing")
def test_struct_layout_matches_header(tmp_path):
    from cdft_b200 import _lib
    probe = tmp_path / "probe.c"
    probe.write_text(f"""
#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main(void) {{
  printf("%zu %zu %zu %zu\\n", sizeof(cdft_system_desc), sizeof(cdft_solver_opts), sizeof(cdft_result), sizeof(cdft_assoc_pair));
  printf("%zu %zu %zu %zu %zu\\n", offsetof(cdft_system_desc, vext), offsetof(cdft_system_desc, precision),
         offsetof(cdft_system_desc, mu_res_plus_ln_rhob), offsetof(cdft_solver_opts, engine),
         offsetof(cdft_result, history_len));
  return 0;
}}
""")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-o", str(exe), str(probe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    sizes = list(map(int, out[0].split()))
    offs = list(map(int, out[1].split()))
    assert sizes == [ctypes.sizeof(_lib.SystemDesc), ctypes.sizeof(_lib.SolverOpts), ctypes.sizeof(_lib.Result),
                     ctypes.sizeof(_lib.AssocPair)]
    assert offs == [_lib.SystemDesc.vext.offset, _lib.SystemDesc.precision.offset,
                    _lib.SystemDesc.mu_res_plus_ln_rhob.offset, _lib.SolverOpts.engine.offset,
                    _lib.Result.history_len.offset]
    # the oracle's C++ restatement takes the same structs through its own ctypes mirror
    from oracle import cpu
    assert sizes == [ctypes.sizeof(cpu.SystemDesc), ctypes.sizeof(cpu.SolverOpts), ctypes.sizeof(cpu.Result),
                     ctypes.sizeof(cpu.AssocPair)]
    assert offs[:2] == [cpu.SystemDesc.vext.offset, cpu.SystemDesc.precision.offset]


def test_library_is_not_older_than_its_sources():
    """The in-tree library must be rebuilt after any change to its CUDA sources or the ABI header."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("cdft_build", os.path.join(ROOT, "cdft.jl_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert len(mod.DEPS) >= 7
    assert mod.up_to_date(), "libcdft_b200.so is older than its sources: run cdft.jl_b200/build.py"


def test_julia_shim_structs_mirror_the_header():
    """CDFTB200.jl declares the C structs field by field (ccall passes them by value or
    reference): same fields in the same order as include/cdft_b200.h."""
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "cdft_b200.h")).read()
    shim = open(os.path.join(root, "cdft.jl_b200", "julia", "CDFTB200.jl")).read()

    def c_fields(name):
        end = header.index("} " + name + ";")
        body = header[header.rindex("typedef struct {", 0, end) + len("typedef struct {"):end]
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        out = []
        for decl in body.split(";"):
            decl = re.sub(r"\[.*?\]", "", decl).replace("*", " ").strip()
            if not decl:
                continue
            toks = [t for t in re.split(r"[\s,]+", decl) if t]
            skip = 2 if toks[0] in ("const", "unsigned") else 1   # the type ("int icomp, jcomp" declares two)
            out += toks[skip:]
        return out

    def jl_fields(name):
        body = re.search(r"(?:mutable )?struct " + name + r"\n(.*?)\nend", shim, re.S).group(1)
        return [ln.split("::")[0].strip() for ln in body.splitlines() if "::" in ln and not ln.strip().startswith("#")
                and "=" not in ln.split("::")[0]]

    for c, jl in (("cdft_system_desc", "CDFTSystemDesc"), ("cdft_solver_opts", "CDFTSolverOpts"),
                  ("cdft_result", "CDFTResult"), ("cdft_assoc_pair", "CDFTAssocPair")):
        assert jl_fields(jl) == c_fields(c), (c, jl_fields(jl), c_fields(c))
