"""The C-ABI library loads and exports every entry point its header declares (CPU)."""
import ctypes
import os
import re

from chapsim2_b200 import build as B
from chapsim2_b200 import solver as S

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "chapsim_gpu.h")


def declared_functions():
    txt = open(HDR).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(chs_[a-z0-9_]+)\s*\(", txt)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(S.EXPORTED)


def test_library_exports_all_symbols():
    B.build()
    lib = ctypes.CDLL(B.LIB)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_create_rejects_bad_config_without_gpu_work():
    """Argument checks run before any device call: an invalid accuracy is refused."""
    from chapsim2_b200 import config as C
    L = S.load()
    cfg = C.taylor_green(16)
    cfg.iacc = 9
    s, keep = S.make_config(cfg)
    h = ctypes.c_void_p()
    rc = L.chs_create(ctypes.byref(s), -1, ctypes.byref(h))
    assert rc != 0 and not h.value


def test_data_file_names_follow_the_reference():
    # generate_pathfile_name (src/io_tools.f90:44-61): <dir>/domain<idom>_<keyword>_<iter>.bin
    assert S.data_file_name("1_data", 1, "qx", 1000) == "1_data/domain1_qx_1000.bin"
    assert S.data_file_name("out", 2, "time_averaged_uv", 7) == "out/domain2_time_averaged_uv_7.bin"
