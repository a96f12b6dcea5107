"""The C-ABI library loads and exports every function declared in include/*.h (no GPU needed)."""
import ctypes
import os
import re

from conftest import REPO


def declared_functions():
    names = set()
    inc = os.path.join(REPO, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(lbm_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_core_entry_points():
    names = declared_functions()
    for n in ("lbm_create", "lbm_add_particle", "lbm_step", "lbm_get_fields", "lbm_get_distributions",
              "lbm_get_particles", "lbm_get_mask", "lbm_get_links", "lbm_destroy", "lbm_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, f"symbols declared in include/ but not exported: {missing}"


def test_python_binding_covers_every_declared_symbol():
    from lbmengine import _capi
    bound = {name for name, _, _ in _capi.PROTOTYPES}
    assert declared_functions() <= bound


def test_abi_version_and_info_without_gpu(lib):
    assert lib.lbm_abi_version() == 1
    assert b"sm_100a" in lib.lbm_build_info()


def test_struct_layouts_match_header(lib):
    """Field offsets of the ctypes mirrors agree with a C compile of the header."""
    import subprocess
    import tempfile
    from lbmengine import _capi
    src = r'''
#include <stddef.h>
#include <stdio.h>
#include "lbm_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(lbm_config), offsetof(lbm_config, store_scale),
         offsetof(lbm_config, force_field), offsetof(lbm_config, rho_ref), offsetof(lbm_config, storage));
  printf("%zu %zu %zu\n", sizeof(lbm_particle_params), offsetof(lbm_particle_params, B1),
         offsetof(lbm_particle_params, swimming_direction));
  printf("%zu %zu %zu\n", sizeof(lbm_particle_state), offsetof(lbm_particle_state, last_torque),
         offsetof(lbm_particle_state, position));
  printf("%zu %zu\n", sizeof(lbm_info), offsetof(lbm_info, device_bytes));
  printf("%zu %zu %zu %zu\n", offsetof(lbm_config, particle_rules), offsetof(lbm_info, tick),
         offsetof(lbm_info, time), offsetof(lbm_info, bulk_kernel));
  printf("%zu %zu\n", sizeof(lbm_profile), offsetof(lbm_profile, profiled_steps));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "l.c")
        exe = os.path.join(td, "l")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    got = list(map(int, out))
    C = _capi
    exp = [ctypes.sizeof(C.LbmConfig), C.LbmConfig.store_scale.offset, C.LbmConfig.force_field.offset,
           C.LbmConfig.rho_ref.offset, C.LbmConfig.storage.offset,
           ctypes.sizeof(C.LbmParticleParams), C.LbmParticleParams.B1.offset,
           C.LbmParticleParams.swimming_direction.offset,
           ctypes.sizeof(C.LbmParticleState), C.LbmParticleState.last_torque.offset,
           C.LbmParticleState.position.offset,
           ctypes.sizeof(C.LbmInfo), C.LbmInfo.device_bytes.offset,
           C.LbmConfig.particle_rules.offset, C.LbmInfo.tick.offset, C.LbmInfo.time.offset,
           C.LbmInfo.bulk_kernel.offset,
           ctypes.sizeof(C.LbmProfile), C.LbmProfile.profiled_steps.offset]
    assert got == exp


def _c_fields(header, name):
    """Field names of `typedef struct name {...} name;` in declaration order."""
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), header, flags=re.S)
    body = re.sub(r"/\*.*?\*/", "", m.group(1), flags=re.S)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        first, *rest = decl.split(",")  # "double B1, B2" declares two fields
        for d in [first] + rest:
            m2 = re.search(r"(\w+)\s*(\[\s*\d+\s*\])?$", d.strip())
            out.append(m2.group(1))
    return out


def _julia_fields(src, name):
    m = re.search(r"struct %s\n(.*?)\nend" % name, src, flags=re.S)
    return [f.split("::")[0].strip() for line in m.group(1).splitlines() for f in line.split(";") if "::" in f]


def test_julia_struct_mirrors_follow_the_header():
    """The Julia shim's ccall structs list the C fields in the header's order
    (Julia is not installed here; this is a check of the source text)."""
    header = open(os.path.join(REPO, "include", "lbm_b200.h")).read()
    jl = open(os.path.join(REPO, "lbmengine.jl_b200", "julia", "LBMengineB200.jl")).read()
    for c_name, j_name in (("lbm_config", "LbmConfig"), ("lbm_particle_params", "LbmParticleParams"),
                           ("lbm_particle_state", "LbmParticleState"), ("lbm_info", "LbmInfo")):
        assert _julia_fields(jl, j_name) == _c_fields(header, c_name), c_name
