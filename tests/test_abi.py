"""CPU checks of the drop-in boundary: the C-ABI library loads and exports exactly the
entry points include/droplet.h declares (no compute calls: no GPU here)."""
import ctypes as C
import os
import re

from mpi_2d_domain_decomp_turb_particles_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "droplet.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dl_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_the_subroutine_surface():
    names = _declared()
    for sub in ("prepare_interp", "interpolate", "part_history_fvp", "headlist", "nei_list_precomp",
                "hdi_gmres", "part_history_fdp", "part_advance", "complete_ypn", "mean_vel",
                "collision_det", "update_part_position", "relocate", "coalesce", "periodic",
                "overlap_det", "part_init"):
        assert "dl_" + sub in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_the_header():
    assert set(_declared()) == set(_lib.SIGNATURES)


def test_struct_layouts_match_the_c_header(tmp_path):
    """Compile a probe against include/droplet.h with gcc and compare sizes/offsets."""
    import subprocess
    structs = {"dl_params": _lib.Params, "dl_scalars": _lib.Scalars,
               "dl_coll_report": _lib.CollReport, "dl_gmres_report": _lib.GmresReport,
               "dl_adj_params": _lib.AdjParams}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "droplet.h"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.split("\n") if l)
    for cname, py in structs.items():
        assert int(out[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(out[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)
