"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute calls here)."""
import ctypes as C
import os
import re

import pytest

from blaze import device

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(REPO, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(REPO, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:int|void|blaze_sim\s*\*)\s+([A-Za-z_]\w*)\s*\(", src, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_reference_interface():
    names = set(declared_functions())
    for ref_name in ["Device_Set_SimulationData", "Device_DEM_UpdateSim", "Device_Set_Pos",
                     "Device_Set_Pos_Velocity", "Device_Set_System_State", "Device_Set_Tallys",
                     "Device_Get_System_State", "Device_Get_P_Positions", "Device_Get_P_Velocity",
                     "Device_Get_W_Forces", "Device_Get_Energy", "Device_Reset_Energy",
                     "Device_Update_DObjectPostions", "Device_Update_WorldObjectPostions",
                     "Device_OpenHatch", "drum_rotation", "Start_Bin", "Device_AddForce",
                     "Device_SubForce", "Device_ZeroForce", "Device_Clean"]:
        assert ref_name in names, ref_name


def test_library_exports_every_declared_symbol():
    if not os.path.isfile(device.LIB_PATH):
        pytest.fail("libblaze_b200.so not built: run __graft_entry__.build()")
    lib = C.CDLL(device.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_default_options():
    o = device.default_options()
    assert o.max_nbr == 32 and o.skin == 0.0 and o.wall_grid == 1
