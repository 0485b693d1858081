"""The C-ABI library without a GPU: it loads, exports every function that
include/*.h declares, its struct sizes match the ctypes bindings, and (when
the reference headers are present) every boundary struct has the
reference's field offsets, so callers compiled against HotSpot's headers
can use it."""
import ctypes as C
import os
import re
import subprocess

import pytest

from hotspot_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
REFERENCE_SRC = os.environ.get("HOTSPOT_REFERENCE_SRC", "/root/reference")


def _declared_functions():
    names = set()
    for h in os.listdir(INCLUDE):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_]\w*)\s*\(([^;{]*?)\)\s*;", text):
            name = m.group(1)
            if name not in ("if", "while", "for", "sizeof", "return"):
                names.add(name)
    return names


def test_library_loads_and_exports_every_declared_symbol():
    L = _abi.lib()
    missing = [n for n in sorted(_declared_functions()) if not hasattr(L, n)]
    assert not missing, missing


def test_bindings_cover_the_declared_api():
    assert _declared_functions() <= set(_abi.exported_symbols())


def test_struct_sizes_match_bindings():
    out = (C.c_longlong * 16)()
    n = _abi.lib().hsb_abi_sizes(out, 16)
    py = [C.sizeof(t) for t in (_abi.ThermalConfig, _abi.Unit, _abi.Flp, _abi.MaterialsList,
                                _abi.MicrochannelConfig, _abi.PackageRC, _abi.Layer, _abi.GridVector,
                                _abi.GridModel, _abi.Stats)]
    assert list(out)[:n] == py


OFFSETS = {
    "thermal_config_t": ["t_chip", "model_secondary", "ambient", "init_file", "init_temp", "steady_file",
                         "sampling_intvl", "model_type", "package_config_file", "grid_rows",
                         "grid_layer_file", "grid_map_mode", "grid_transient_file", "detailed_3D_used"],
    "unit_t": ["name", "width", "height", "leftx", "bottomy", "specificheat", "resistivity", "hasRes", "hasSh"],
    "flp_t": ["units", "n_units", "wire_density"],
    "microchannel_config_t": ["cell_width", "htc", "network_file", "floorplan_file", "num_rows",
                              "n_fluid_cells", "cell_types", "mapping", "A", "b", "nnz"],
    "package_RC_t": ["r_sp1_x", "r_hs", "c_hs_per", "r_amb_per", "r_sub1_x", "r_pcb", "c_pcb_per",
                     "c_amb_sec_per"],
    "layer_t": ["flp", "no", "has_power", "k", "sp", "is_microchannel", "microchannel_config", "rx", "c",
                "b2gmap", "g2bmap"],
    "grid_model_t": ["config", "layers", "n_layers", "rows", "width", "pack", "total_n_blocks", "map_mode",
                     "has_lcf", "last_steady", "last_trans", "last_temp", "base_n_units",
                     "use_microchannels", "default_microchannel_config"],
}


def _offsets_program(includes: str) -> str:
    body = []
    for st, fields in OFFSETS.items():
        body.append(f'printf("{st} %zu\\n", sizeof({st}));')
        for f in fields:
            body.append(f'printf("{st}.{f} %zu\\n", offsetof({st}, {f}));')
    return "#include <stdio.h>\n#include <stddef.h>\n" + includes + "\nint main(void){\n" + "\n".join(body) + \
        "\nreturn 0;}\n"


def _run_c(src: str, incdir: str, tmp: str, name: str) -> dict:
    c = os.path.join(tmp, name + ".c")
    exe = os.path.join(tmp, name)
    open(c, "w").write(src)
    subprocess.run(["gcc", "-std=gnu99", "-w", "-DSUPERLU=0", "-DMATHACCEL=0", f"-I{incdir}", c, "-o", exe],
                   check=True, capture_output=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return dict(l.rsplit(" ", 1) for l in out.strip().splitlines())


@pytest.mark.skipif(not os.path.isdir(REFERENCE_SRC), reason="reference headers not present")
def test_boundary_layouts_match_reference_headers(tmp_path):
    ours = _run_c(_offsets_program('#include "hotspot_b200_types.h"'), INCLUDE, str(tmp_path), "ours")
    ref = _run_c(_offsets_program('#include "temperature.h"\n#include "temperature_grid.h"'),
                 REFERENCE_SRC, str(tmp_path), "ref")
    for k, v in ref.items():
        if k == "grid_model_t":
            # our grid_model_t appends two pointers after the reference's fields
            assert int(ours[k]) == int(v) + 2 * C.sizeof(C.c_void_p), k
        else:
            assert ours[k] == v, (k, ours[k], v)
