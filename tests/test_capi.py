"""The C-ABI library loads and exports every symbol include/erf_b200.h declares,
and the ctypes mirrors have the C struct layouts (no GPU compute here)."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from erf_b200 import config as C
from erf_b200 import dycore

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "erf_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char\s*\*)\s*(erf_b200_\w+)\s*\(", txt, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(dycore.LIB_PATH):
        from erf_b200 import build
        build.build()
    return ctypes.CDLL(dycore.LIB_PATH)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "erf_b200_advance" in names and "erf_b200_create" in names
    assert len(names) >= 16


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_lists_every_symbol():
    assert sorted(dycore.EXPORTS) == declared_functions()


def test_struct_layouts_match_c():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "erf_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(erf_b200_config), sizeof(erf_b200_fab),
         offsetof(erf_b200_config, abl_geo_forcing), offsetof(erf_b200_config, precision),
         offsetof(erf_b200_fab, nstride), offsetof(erf_b200_config, substepping_type),
         offsetof(erf_b200_config, most_zref));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        cpath = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(cpath, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), cpath, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    sc, sf, og, op, on, osub, ozref = map(int, out)
    assert sc == ctypes.sizeof(C.ErfConfig)
    assert sf == ctypes.sizeof(dycore.ErfFab)
    assert og == C.ErfConfig.abl_geo_forcing.offset
    assert op == C.ErfConfig.precision.offset
    assert on == dycore.ErfFab.nstride.offset
    assert osub == C.ErfConfig.substepping_type.offset
    assert ozref == C.ErfConfig.most_zref.offset


def test_config_defaults_match_c(lib):
    c = C.ErfConfig()
    lib.erf_b200_config_defaults.argtypes = [ctypes.c_void_p]
    assert lib.erf_b200_config_defaults(ctypes.byref(c)) == 0
    d = C.defaults()
    for name, _ in C.ErfConfig._fields_:
        if name in ("reserved", "abl_geo_forcing"):
            continue
        assert getattr(c, name) == pytest.approx(getattr(d, name)), name


def test_create_rejects_bad_config_without_gpu(lib):
    # validation happens before any CUDA call
    c = C.defaults()
    c.mri_ratio = 5
    ctx = ctypes.c_void_p()
    lib.erf_b200_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_void_p]
    assert lib.erf_b200_create(ctypes.byref(ctx), ctypes.byref(c), None) == 8  # ERF_B200_ECONFIG


@pytest.mark.parametrize("change", ["terrain", "no_closure", "mlp", "z0_above_zref", "zref_outside",
                                    "most_lid"])
def test_create_rejects_unsupported_most_config(lib, change):
    """A MOST ground is accepted flat and under Smagorinsky or Deardorff,
    with z0 below the snapped reference height, and only as the lower
    boundary; the rest is refused before any CUDA call."""
    c = C.defaults()
    c.zlo_bc = C.BC_MOST
    c.les_type = C.LES_SMAGORINSKY
    c.most_z0, c.most_zref = 0.1, 8.0
    if change == "terrain":
        c.use_terrain = 1
    elif change == "no_closure":
        c.les_type = C.LES_NONE
    elif change == "mlp":
        c.les_type = C.LES_MLP
        c.molec_diff_type = C.MOLEC_NONE
    elif change == "z0_above_zref":
        c.most_z0 = 0.5 * c.dz + 1.0   # above the first cell centre
        c.most_zref = 0.0
    elif change == "zref_outside":
        c.most_zref = c.nz * c.dz + 1.0
    elif change == "most_lid":
        c.zhi_bc = C.BC_MOST
    ctx = ctypes.c_void_p()
    lib.erf_b200_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_void_p]
    assert lib.erf_b200_create(ctypes.byref(ctx), ctypes.byref(c), None) == 8  # ERF_B200_ECONFIG


@pytest.mark.parametrize("moist", [False, True])
def test_create_accepts_most_config(lib, moist):
    """The supported MOST ground passes validation, dry or with Kessler
    moisture (without a GPU the create call then fails at its first CUDA
    call, ERF_B200_ECUDA)."""
    c = C.defaults()
    c.zlo_bc = C.BC_MOST
    c.les_type = C.LES_DEARDORFF
    c.most_z0, c.most_zref = 0.1, 8.0
    if moist:
        c.moisture, c.ncomp = C.MOIST_KESSLER, 8
    ctx = ctypes.c_void_p()
    lib.erf_b200_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_void_p]
    lib.erf_b200_destroy.argtypes = [ctypes.c_void_p]
    rc = lib.erf_b200_create(ctypes.byref(ctx), ctypes.byref(c), None)
    assert rc in (0, 2)
    if rc == 0:
        lib.erf_b200_destroy(ctx)


@pytest.mark.parametrize("change", ["static_flag", "moist", "les", "molec", "upwind", "buoyancy",
                                    "noslip", "wavelength", "bad_type", "unlagged_static"])
def test_create_rejects_unsupported_moving_terrain(lib, change):
    """Moving terrain is accepted as the reference's MovingTerrain problems
    run it: dry, no diffusion, Centered_2nd dycore, buoyancy type 1, slip
    walls, with or without acoustic substepping; use_lagged_delta_rt =
    false only there; the rest is refused before any
    CUDA call."""
    from erf_b200 import terrain as T
    c = T.moving_terrain(nx=8, ny=4, nz=10).cfg
    if change == "static_flag":
        c.use_terrain = 0
    elif change == "unlagged_static":
        c = C.defaults()
        c.no_lagged_delta_rt = 1
    elif change == "moist":
        c.moisture, c.ncomp = C.MOIST_KESSLER, 8
    elif change == "les":
        c.les_type = C.LES_SMAGORINSKY
    elif change == "molec":
        c.molec_diff_type = C.MOLEC_CONSTANT
    elif change == "upwind":
        c.dycore_horiz_adv = C.UPWIND_3RD
    elif change == "buoyancy":
        c.buoyancy_type = 2
    elif change == "noslip":
        c.zlo_bc = C.BC_NO_SLIP_WALL
    elif change == "wavelength":
        c.mt_wavelength = 0.0
    elif change == "bad_type":
        c.terrain_type = 2
    ctx = ctypes.c_void_p()
    lib.erf_b200_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_void_p]
    assert lib.erf_b200_create(ctypes.byref(ctx), ctypes.byref(c), None) == 8  # ERF_B200_ECONFIG


@pytest.mark.parametrize("substeps", [False, True])
def test_create_accepts_moving_terrain_config(lib, substeps):
    from erf_b200 import terrain as T
    c = T.moving_terrain(nx=8, ny=4, nz=10, substeps=substeps).cfg
    ctx = ctypes.c_void_p()
    lib.erf_b200_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_void_p]
    lib.erf_b200_destroy.argtypes = [ctypes.c_void_p]
    rc = lib.erf_b200_create(ctypes.byref(ctx), ctypes.byref(c), None)
    assert rc in (0, 2)
    if rc == 0:
        lib.erf_b200_destroy(ctx)
