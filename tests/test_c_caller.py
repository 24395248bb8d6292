"""The drop-in boundary seen from a C or Fortran (iso_c_binding) caller, on the CPU.

* include/acs.h and include/unet.h compile as strict C99 (-Wall -Wextra -pedantic -Werror);
* the BIND(C) derived types of the Fortran interface module in INTEGRATION.md have the same
  field offsets and size as the C structs (interoperable types are laid out like the C struct
  with the same members in the same order);
* every BIND(C) function of that module names an exported function of acs.h with the same
  number of arguments;
* a C program linked against libacs_b200.so calls the host-side entry points (channel mesh,
  version) and gets ACS_E_CUDA with a message from acs_create where no device exists.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
PKG = os.path.join(ROOT, "solver-cfd_b200")

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")


def _fortran_types():
    """Ordered (kind, name) members of each BIND(C) TYPE in INTEGRATION.md's module."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    types = {}
    for m in re.finditer(r"TYPE, BIND\(C\) :: (\w+)\n(.*?)END TYPE", text, re.S):
        members = []
        for line in m.group(2).splitlines():
            d = re.match(r"\s*(INTEGER\(c_int\)|REAL\(c_double\)|TYPE\(c_ptr\))\s*::\s*(.*)", line)
            if d:
                kind = {"INTEGER(c_int)": "int", "REAL(c_double)": "double", "TYPE(c_ptr)": "ptr"}[d.group(1)]
                members += [(kind, n.strip()) for n in d.group(2).split(",")]
        types[m.group(1)] = members
    return types


def _layout(members):
    size = {"int": 4, "double": 8, "ptr": 8}
    off, offs, align = 0, {}, 1
    for kind, name in members:
        a = size[kind]
        off = (off + a - 1) // a * a
        offs[name] = off
        off += a
        align = max(align, a)
    return offs, (off + align - 1) // align * align


C_PROGRAM = r"""
#include <stddef.h>
#include <stdio.h>
#include "acs.h"
#include "unet.h"
#define OFF(T, f) printf("%s %s %zu\n", #T, #f, offsetof(T, f))
int main(void) {
  double x[20], y[16], xm[21], ym[17], eps[20 * 16], liga[20 * 16];
  int flag[20 * 16];
  const double box[4] = {0.5, 1.5, 0.3, 0.7};
  acs_grid g;
  acs_params p;
  acs_handle* h = NULL;
  int code;
  %OFFSETS%
  printf("size acs_params %zu\nsize acs_grid %zu\n", sizeof(acs_params), sizeof(acs_grid));
  code = acs_mesh_channel(20, 16, 2.0, 1.0, 1.5, box, NULL, 0.4, x, y, xm, ym, flag, eps, liga);
  printf("mesh %d %d\n", code, flag[10 + 8 * 20]);
  printf("version %s\n", acs_version() ? acs_version() : "");
  g.imax = 20; g.jmax = 16; g.x = x; g.y = y; g.xm = xm; g.ym = ym; g.epsilon1 = eps; g.liga_poros = liga;
  (void)p;
  code = acs_create(&g, NULL, &h);
  printf("create_null %d\n", code);
  return 0;
}
"""


@pytest.fixture(scope="module")
def c_run(pkg, tmp_path_factory):
    types = _fortran_types()
    offsets = "\n  ".join(f"OFF({t}, {n});" for t, mem in types.items() for _, n in mem)
    d = tmp_path_factory.mktemp("ccaller")
    src = d / "caller.c"
    src.write_text(C_PROGRAM.replace("%OFFSETS%", offsets))
    exe = d / "caller"
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", INC, str(src), "-o", str(exe),
           "-L", PKG, "-lacs_b200", f"-Wl,-rpath,{PKG}"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stderr
    return types, run.stdout


def test_fortran_types_match_c_layout(c_run):
    types, out = c_run
    got = {}
    for line in out.splitlines():
        parts = line.split()
        if len(parts) == 3 and parts[0] != "size":
            got[(parts[0], parts[1])] = int(parts[2])
    sizes = {p[1]: int(p[2]) for p in (l.split() for l in out.splitlines()) if p and p[0] == "size"}
    assert set(types) == {"acs_params", "acs_grid"}
    for t, members in types.items():
        offs, size = _layout(members)
        for _, n in members:
            assert got[(t, n)] == offs[n], (t, n, got[(t, n)], offs[n])
        assert sizes[t] == size, (t, sizes[t], size)


def test_host_entry_points_from_c(c_run):
    _, out = c_run
    kv = {l.split()[0]: l.split()[1:] for l in out.splitlines() if l.split()}
    assert kv["mesh"][0] == "0"               # ACS_OK
    assert kv["mesh"][1] in {"1", "2", "3"}   # the node inside the porous block is flagged
    assert kv["create_null"][0] != "0"        # NULL params: an error code, never a crash


def test_fortran_interfaces_name_c_functions_with_same_arity():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    header = open(os.path.join(INC, "acs.h")).read()
    found = 0
    for m in re.finditer(r"FUNCTION (\w+)\(([^)]*)\)\s*(?:&\s*\n\s*)?BIND\(C, name=\"(\w+)\"\)", text):
        fargs = [a for a in m.group(2).replace("&", " ").split(",") if a.strip()]
        proto = re.search(r"\bint\s+" + m.group(3) + r"\(([^)]*)\);", header, re.S)
        assert proto, m.group(3)
        cargs = [a for a in proto.group(1).split(",") if a.strip() and a.strip() != "void"]
        assert len(fargs) == len(cargs), (m.group(3), fargs, cargs)
        found += 1
    assert found >= 10, found
