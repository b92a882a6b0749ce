"""The C ABI library: loads without a GPU, exports every function and
variable that include/*.h declares, and keeps the reference's struct sizes."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import spgemm_b200 as sg

INCLUDE = Path(__file__).resolve().parents[1] / "include"


def declared_symbols():
    names = set()
    for h in INCLUDE.glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?[\s\*]([A-Za-z_]\w*)\s*\([^;{]*\)\s*;",
                             text, flags=re.M):
            if m.group(1) not in ("if", "while", "return"):
                names.add(m.group(1))
        for m in re.finditer(r"^\s*extern\s+[\w\s\*]+?([A-Za-z_]\w*)\s*;", text, flags=re.M):
            names.add(m.group(1))
    return names


def exported():
    out = subprocess.run(["nm", "-D", "--defined-only", str(sg.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_every_declared_symbol_is_exported():
    decl = declared_symbols()
    assert {"cudaCOO2CM", "cudaMergeGEMM", "readMTX", "spgemm_symbolic", "maxWL", "makeWLT"} <= decl
    missing = sorted(decl - exported())
    assert not missing, missing


def test_library_loads_and_reports_version():
    assert sg.version().startswith("spgemm_b200")
    L = sg.lib()
    L.spgemm_status_string.argtypes = [C.c_int]
    assert L.spgemm_status_string(0) == b"ok"
    assert L.spgemm_status_string(6) == b"device-side check failed"


def test_struct_layouts_match_reference():
    # triplet {int,int,float}; coo {ptr,int,int,int,bool}; cm {3 ptr, 3 int, bool}
    assert C.sizeof(sg.Triplet) == 12
    assert C.sizeof(sg.COO) == 24
    assert C.sizeof(sg.CM) == 40
    assert sg.CM.nnz.offset == 24 and sg.CM.type.offset == 36


def test_host_helpers_without_gpu():
    L = sg.lib()
    m = sg.CM()
    L.cmInit.argtypes = [C.POINTER(sg.CM)]
    L.cmInit(C.byref(m))
    assert (m.nnz, m.num_rows, m.num_cols, bool(m.type)) == (0, 0, 0, False)
    L.cmSetNNZ.argtypes = [C.POINTER(sg.CM), C.c_int]
    L.cmGetNNZ.argtypes = [sg.CM]
    L.cmSetNNZ(C.byref(m), 17)
    assert L.cmGetNNZ(m) == 17
